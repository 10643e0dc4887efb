"""Request loop (pppm_server_*): each result equals the result the same
request gets alone, while other requests run concurrently; scenes evicted
under a small HBM budget continue from their saved positions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def srvmod():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pppm_vortex_bouyant_flow_sample_b200 import server
    return server


def _scenes():
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    specs = [(32, "cloud", 8000, 41), (48, "ring", 30000, 42), (64, "cloud", 20000, 43), (32, "ring", 12000, 44)]
    return [(n,) + W.make_scene(kind, N, seed) for n, kind, N, seed in specs]


def test_result_same_alone_and_in_the_mix(srvmod):
    srv = srvmod.Server(hbm_budget_bytes=8 << 30, slots=4)
    try:
        ids = [srv.add_scene(n, pos, al) for n, pos, al in _scenes()]
        _, alone = srv.wait(srv.submit_eval(ids[1]))
        tickets = []
        for rep in range(3):
            for sid in ids:
                tickets.append(srv.submit_eval(sid))
            tickets.append(srv.submit_advance(ids[3], 2, 1e-3))
        mixed = []
        for t in tickets:
            info, v = srv.wait(t)
            assert info["end_s"] >= info["start_s"] >= info["submit_s"]
            if t[1] == ids[1]:
                mixed.append(v.copy())
        assert len(mixed) == 3
        for v in mixed:
            assert np.array_equal(v, alone)
    finally:
        srv.close()


def test_eviction_keeps_advanced_positions(srvmod):
    import torch
    import pppm_vortex_bouyant_flow_sample_b200 as pb
    sc = _scenes()
    # a 60 MB budget holds one or two of these scenes: later requests evict
    # the advanced scene, whose positions must survive the round trip
    srv = srvmod.Server(hbm_budget_bytes=60 << 20, slots=2)
    try:
        ids = [srv.add_scene(n, pos, al) for n, pos, al in sc]
        srv.wait(srv.submit_advance(ids[0], 3, 2e-3))
        for sid in ids[1:]:
            srv.wait(srv.submit_eval(sid))
        got = srv.positions(ids[0])
    finally:
        srv.close()
    n, pos, al = sc[0]
    scene = pb.Scene(n, cap_vort=len(pos), cap_eval=len(pos))
    dpos = torch.from_numpy(pos.copy()).cuda()
    dal = torch.from_numpy(np.ascontiguousarray(al)).cuda()
    for _ in range(3):
        scene.advect(dpos, dal, 2e-3, method="rk2")
    assert np.array_equal(got, dpos.cpu().numpy())
    scene.close()


def test_admission_near_the_budget_under_concurrent_requests(srvmod):
    """Six scenes whose footprints together exceed the HBM budget about
    threefold, requested from three threads at once over four slots: every
    request completes, each EVAL equals the scene's result alone, and the
    resident footprint never exceeds the budget (the loop evicts idle scenes,
    least recently used first, to admit the next)."""
    import threading
    import time
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    specs = [(32, "cloud", 9000, 51), (48, "ring", 25000, 52), (64, "cloud", 18000, 53), (32, "ring", 12000, 54),
             (48, "cloud", 15000, 55), (64, "ring", 22000, 56)]
    scenes = [(n,) + W.make_scene(kind, N, seed) for n, kind, N, seed in specs]
    # alone: each scene's EVAL with a budget that holds everything
    ref = {}
    srv = srvmod.Server(hbm_budget_bytes=8 << 30, slots=1)
    try:
        for q, (n, pos, al) in enumerate(scenes):
            _, v = srv.wait(srv.submit_eval(srv.add_scene(n, pos, al)))
            ref[q] = v.copy()
    finally:
        srv.close()
    budget = 110 << 20
    srv = srvmod.Server(hbm_budget_bytes=budget, slots=4)
    try:
        ids = [srv.add_scene(n, pos, al) for n, pos, al in scenes]
        results, errors, peak = [], [], [0]
        lock = threading.Lock()
        stop = threading.Event()

        def sampler():
            while not stop.is_set():
                peak[0] = max(peak[0], srv.stats()["resident_bytes"])
                time.sleep(0.001)

        def client(offset):
            try:
                for rep in range(4):
                    for k in range(len(ids)):
                        q = (k + offset + rep) % len(ids)
                        info, v = srv.wait(srv.submit_eval(ids[q]))
                        with lock:
                            results.append((q, v.copy()))
            except Exception as exc:  # reported below
                errors.append(exc)

        th = [threading.Thread(target=client, args=(o,)) for o in range(3)]
        sm = threading.Thread(target=sampler)
        sm.start()
        for t in th:
            t.start()
        for t in th:
            t.join()
        stop.set()
        sm.join()
        assert not errors, errors
        assert len(results) == 3 * 4 * len(ids)
        for q, v in results:
            assert np.array_equal(v, ref[q]), q
        assert 0 < peak[0] <= budget
        assert srv.stats()["completed"] == len(results)
    finally:
        srv.close()
