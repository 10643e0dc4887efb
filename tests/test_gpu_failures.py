"""Failure paths, made on the host: every device and pinned allocation of a
call sequence is made to fail in turn (pppm_debug_fail_allocation), with no
real memory pressure and no device fault.

Each failure must come back as PPPM_ERR_OOM from the call that allocated,
leave the objects destroyable, leak no device memory over the walk, and leave
the device serving a normal scene with the oracle's answer afterwards.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pppm_vortex_bouyant_flow_sample_b200 as pb
    pb.load()
    return pb


def _sequence(pb, keep):
    """Scene with growth, far field, evaluation, pair count, sorted copies, a
    vortex step, the buoyancy source, the scalar PPPM, the hasher and the
    renderer; every object created goes into keep."""
    import torch
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    from pppm_vortex_bouyant_flow_sample_b200.potential import PotentialFieldSolver
    from pppm_vortex_bouyant_flow_sample_b200.render import Renderer
    pos, al = W.uniform_cloud(3000, seed=1)
    dpos = torch.from_numpy(pos).cuda()
    dal = torch.from_numpy(np.ascontiguousarray(al)).cuda()
    scene = pb.Scene(16, cap_vort=100, cap_eval=100)     # small capacities: growth allocates
    keep.append(scene)
    scene.set_vortices(dpos, dal)
    scene.build_far_field()
    scene.eval(dpos, dpos, 1)
    scene.count_pairs(dpos)
    scene.sorted_vortices()
    p2, a2 = dpos.clone(), dal.clone()
    scene.vortex_step(p2, a2, 0.01)
    heat = torch.ones(len(pos), dtype=torch.float32, device="cuda")
    scene.baroclinic(dpos, heat, dpos, dal.clone(), 0.002)
    solver = PotentialFieldSolver()
    keep.append(solver)
    solver.initializeSolver(16, 16, 16, 1, 500, len(pos))
    solver.setMassParameter(len(pos), dpos, dal[:, 0].contiguous())
    solver.setEvalParameter(500, dpos[:500])
    solver.computeFarFieldBuffer()
    solver.evaluateGradient(True)
    pm = pb.ParticleManager()
    keep.append(pm)
    pm.initSpatialHash(len(pos), 16, 16, 16)
    pm.setSpatialHashGrid(16, 1.0 / 16, (0.0, 0.0, 0.0), len(pos))
    pm.doSpatialHash(dpos, len(pos))
    rnd = Renderer()
    keep.append(rnd)
    dens = torch.ones(len(pos), dtype=torch.float32, device="cuda")
    illum, _ = rnd.shadows(dpos, dens, 0.01, 0.05, (0.5, 4.0, -2.0), 1.0)
    col = torch.full((len(pos), 4), 0.5, dtype=torch.float32, device="cuda")
    rnd.smoke(dpos, illum, col[:, :3].contiguous(), col[:, :3].contiguous(), 0.01, 0.05, dens, (0.0, 0.0, 0.0),
              (0.5, 0.5, -2.0), (0.5, 0.5, 0.5), 2.0, 64, 48)


def _close(obj):
    for name in ("close", "shutdown", "endSpatialHash"):
        if hasattr(obj, name):
            getattr(obj, name)()
            return


def test_every_allocation_failure_is_reported(pb, oracle):
    import torch
    from pppm_vortex_bouyant_flow_sample_b200._lib import PppmError, load
    lib = load()
    # one complete pass first, so that every kernel module is loaded and every
    # lazily created resource exists before free memory is recorded
    keep = []
    try:
        _sequence(pb, keep)
    finally:
        for obj in keep:
            _close(obj)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free0 = torch.cuda.mem_get_info()[0]
    free_at = []
    failures = 0
    completed = False
    for k in range(400):
        lib.pppm_debug_fail_allocation(k)
        keep = []
        try:
            _sequence(pb, keep)
            completed = True          # k is past the last allocation: nothing failed
        except PppmError as exc:
            assert exc.status == 3, str(exc)
            failures += 1
        finally:
            lib.pppm_debug_fail_allocation(-1)
            for obj in keep:
                _close(obj)
            torch.cuda.synchronize()
        torch.cuda.empty_cache()
        free_at.append(torch.cuda.mem_get_info()[0])
        if completed:
            break
    assert completed and failures > 20
    # no device memory held after the walk (beyond allocator noise)
    assert free_at[-1] >= free0 - (16 << 20), (free0, free_at[-1])
    assert min(free_at) >= free0 - (16 << 20), (free0, min(free_at))
    # the device still serves a scene correctly
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(6000, seed=5)
    scene = pb.Scene(32, cap_vort=len(pos), cap_eval=len(pos))
    dpos = torch.from_numpy(pos).cuda()
    scene.set_vortices(dpos, torch.from_numpy(np.ascontiguousarray(al)).cuda())
    scene.build_far_field()
    u = scene.eval(dpos, dpos, 1).cpu().numpy()
    scene.close()
    ref, _ = oracle.pppm(oracle.params(32), pos, al, pos, pos, 1, dump=True)
    assert rel_l2(u, ref) <= 1e-5
