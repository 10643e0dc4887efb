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
