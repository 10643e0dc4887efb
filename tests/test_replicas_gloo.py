"""The multi-GPU plumbing on CPU: two gloo ranks (spawned processes) agree on
the scene partition, cover every scene exactly once, and reduce their times
to the maximum.  No GPU is touched."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from pppm_vortex_bouyant_flow_sample_b200 import replicas as R


def test_partition_is_complete_and_balanced():
    costs = [R.scene_cost(n, N) for n, N in [(32, 10000), (128, 1000000), (64, 200000), (96, 50000), (48, 900000),
                                             (32, 30000), (128, 20000), (64, 600000)]]
    for world in (1, 2, 3, 8):
        parts = R.partition_scenes(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT: no rank exceeds the mean by more than the largest single scene
        assert max(loads) <= sum(costs) / world + max(costs)
    assert R.partition_scenes(costs, 2) == R.partition_scenes(list(costs), 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    w, r, _ = R.env_ranks()
    R.init(w, r, "gloo", timeout_s=60)
    costs = [float(c) for c in (5, 3, 8, 1, 9, 2, 7)]
    mine = R.partition_scenes(costs, w)[r]
    R.barrier()
    t = R.max_over_ranks(10.0 * (r + 1))
    total = R.sum_over_ranks(len(mine))
    q.put((r, mine, t, total))
    R.finish()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert sorted(out[0][1] + out[1][1]) == list(range(7))
    assert not set(out[0][1]) & set(out[1][1])
    assert all(t == 20.0 for _, _, t, _ in out)
    assert all(total == 7 for _, _, _, total in out)
