"""Edge cases of the velocity path (through the C ABI) against the CPU oracle.

Degenerate domains (one vortex, all vortices coincident), the smallest
non-degenerate scene, empty evaluation sets, grid edges the multigrid cannot
take, capacity growth, evaluation points outside the grid, and grid edges
other than the headline's (96: four even levels above a 6^3 coarsest grid;
256: six levels, the largest grid the reference's scenes use).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

VEL_TOL = 1e-5


@pytest.fixture(scope="module")
def pb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pppm_vortex_bouyant_flow_sample_b200 as pb
    pb.load()
    return pb


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _velocity(pb, n, pos, al, ev_a, ev_b=None, is_segment=0, cap_vort=None, cap_eval=None, **kw):
    scene = pb.Scene(n, cap_vort=cap_vort or len(pos), cap_eval=cap_eval or len(ev_a), **kw)
    scene.set_vortices(_dev(pos), _dev(al))
    scene.build_far_field()
    da = _dev(ev_a)
    db = _dev(ev_b) if ev_b is not None else None
    return scene, scene.eval(da, db, is_segment).cpu().numpy()


def _check_healthy(pb, oracle):
    """The context still serves an ordinary scene correctly."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(6000, seed=21)
    scene, u = _velocity(pb, 32, pos, al, pos, pos, 1)
    ref, _ = oracle.pppm(oracle.params(32), pos, al, pos, pos, 1, dump=True)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


@pytest.mark.parametrize("N", [1, 64])
def test_degenerate_domain_reports_and_returns_zero(pb, oracle, N):
    """One vortex, or N coincident ones: the bbox3x domain edge is 0.  The
    build succeeds, the velocity is zero everywhere (the oracle's answer),
    pppm_get_domain reports PPPM_ERR_DOMAIN, and the device stays usable."""
    from pppm_vortex_bouyant_flow_sample_b200._lib import PppmError
    rng = np.random.default_rng(40 + N)
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = (0.3, 0.2, 0.1)
    al = rng.normal(size=(N, 3))
    ev = np.zeros((7, 4), np.float32)
    ev[:, :3] = pos[0, :3] + rng.normal(0, 0.1, (7, 3))
    ev[0, :3] = pos[0, :3]
    for K in (0, 1, 2):
        scene, u = _velocity(pb, 16, pos, al, ev, K=K)
        ref, _ = oracle.pppm(oracle.params(16, K=K), pos, al, ev, None, 0, dump=True)
        assert np.array_equal(u, ref) and not np.any(u)
        with pytest.raises(PppmError) as ei:
            scene.domain()
        assert ei.value.status == 5
        scene.close()
    _check_healthy(pb, oracle)


def test_two_vortices(pb, oracle):
    """The smallest scene with a finite domain."""
    pos = np.zeros((2, 4), np.float32)
    pos[0, :3] = (0.1, 0.2, 0.3)
    pos[1, :3] = (0.13, 0.21, 0.28)
    al = np.array([[0.5, -0.2, 0.1], [0.3, 0.4, -0.6]])
    ev = np.zeros((6, 4), np.float32)
    ev[:2] = pos
    ev[2:, :3] = np.random.default_rng(3).uniform(0.05, 0.35, (4, 3))
    for n in (4, 16):
        scene, u = _velocity(pb, n, pos, al, ev)
        ref, _ = oracle.pppm(oracle.params(n), pos, al, ev, None, 0, dump=True)
        assert rel_l2(u, ref) <= VEL_TOL
        scene.close()


def test_empty_eval_is_noop(pb):
    import torch
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(3000, seed=8)
    scene = pb.Scene(16, cap_vort=len(pos), cap_eval=16)
    scene.set_vortices(_dev(pos), _dev(al))
    scene.build_far_field()
    empty = torch.empty((0, 4), dtype=torch.float32, device="cuda")
    assert tuple(scene.eval(empty).shape) == (0, 3)
    assert tuple(scene.eval(empty, empty, 1).shape) == (0, 3)
    assert tuple(scene.eval_f32(empty).shape) == (0, 3)
    scene.close()


@pytest.mark.parametrize("n", [3, 100, 513])
def test_grid_edges_the_multigrid_cannot_take(pb, n):
    """Edges outside [4, 512], or with an odd level above the coarsest
    (100 -> 50 -> 25), are refused before anything is allocated."""
    from pppm_vortex_bouyant_flow_sample_b200._lib import PppmError
    with pytest.raises(PppmError) as ei:
        pb.Scene(n, cap_vort=16, cap_eval=16)
    assert ei.value.status == 1


def test_capacity_growth(pb, oracle):
    """Scenes created small grow their vortex and evaluation buffers."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(12000, seed=17)
    ev, _ = W.uniform_cloud(9000, seed=18)
    scene, u = _velocity(pb, 32, pos, al, ev, cap_vort=100, cap_eval=10)
    ref, _ = oracle.pppm(oracle.params(32), pos, al, ev, None, 0, dump=True)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_eval_points_outside_the_grid(pb, oracle):
    """Points beyond the domain box: no far field there; the near field of
    vortices within (K+0.5)h still counts, as in the oracle."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(8000, seed=23)
    rng = np.random.default_rng(24)
    ev = np.zeros((3000, 4), np.float32)
    ev[:, :3] = rng.uniform(-1.6, 2.6, (3000, 3))   # domain is [-1, 2]^3
    scene, u = _velocity(pb, 32, pos, al, ev)
    ref, _ = oracle.pppm(oracle.params(32), pos, al, ev, None, 0, dump=True)
    assert rel_l2(u, ref) <= VEL_TOL
    origin, L, _ = scene.domain()
    outside = np.any((ev[:, :3] < np.array(origin) - 0.2) | (ev[:, :3] > np.array(origin) + L + 0.2), axis=1)
    assert outside.sum() > 100 and not np.any(u[outside])
    scene.close()


def test_far_vortex_sends_every_lane_on_its_own_walk(pb, oracle):
    """The warp-uniform walk drops a lane's hash-cell range test, which is
    sound while the hash cells and the coordinates differ by far less than half
    a cell (the build's rounding bound prune_cells < 1/4).  One vortex 20,000
    units out in a fixed unit-cube domain on 32^3 lifts that bound to about
    0.6, and every lane then walks its own cells; the result is the oracle's."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(12000, seed=31)
    pos[:, :3] = 0.1 + 0.8 * (pos[:, :3] - pos[:, :3].min(0)) / np.ptp(pos[:, :3], axis=0)
    pos[0, :3] = (20000.0, 0.5, 0.5)
    box = dict(domain_mode=1, fixed_origin=(0.0, 0.0, 0.0), fixed_length=1.0)
    ev = np.ascontiguousarray(pos[1:])
    scene, u = _velocity(pb, 32, pos, al, ev, ev, 1, domain="fixed", fixed_origin=(0.0, 0.0, 0.0),
                         fixed_length=1.0)
    ref, _ = oracle.pppm(oracle.params(32, **box), pos, al, ev, ev, 1, dump=True)
    assert np.linalg.norm(ref) > 0
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_grid_96(pb, oracle):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(40000, seed=3)
    scene, u = _velocity(pb, 96, pos, al, pos, pos, 1)
    ref, _ = oracle.pppm(oracle.params(96), pos, al, pos, pos, 1, dump=True)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_grid_256_ring_subsample(pb, oracle):
    """256^3 (six multigrid levels) with 262,144 vortices: every 97th
    vortex checked, the near-field pair count exactly."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(1 << 18, seed=3)
    n = 256
    scene = pb.Scene(n, cap_vort=len(pos), cap_eval=len(pos))
    scene.set_vortices(_dev(pos), _dev(al))
    scene.build_far_field()
    sub = np.ascontiguousarray(pos[::97])
    dsub = _dev(sub)
    u = scene.eval(dsub, dsub, 1).cpu().numpy()
    pairs = scene.count_pairs(dsub)
    ref, d = oracle.pppm(oracle.params(n), pos, al, sub, sub, 1, dump=True)
    assert pairs == int(d["pairs"][0])
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_profile_environment_switch(pb, monkeypatch):
    """PPPM_PROFILE=1 turns stage timing on at scene creation; unset (or "0")
    it stays off until set_profiling."""
    import torch
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(4000, seed=6)
    dpos = torch.from_numpy(pos).cuda()
    dal = torch.from_numpy(np.ascontiguousarray(al)).cuda()
    for env, timed in (("1", True), ("0", False), (None, False)):
        if env is None:
            monkeypatch.delenv("PPPM_PROFILE", raising=False)
        else:
            monkeypatch.setenv("PPPM_PROFILE", env)
        scene = pb.Scene(16, cap_vort=len(pos), cap_eval=len(pos))
        scene.set_vortices(dpos, dal)
        scene.build_far_field()
        scene.eval(dpos, dpos, 1)
        st = scene.stage_times()
        scene.close()
        assert (st["eval"] > 0 and st["multigrid"] > 0) == timed, (env, st)
        assert (min(st[k] for k in ("domain", "p2m", "farfield", "eval")) >= 0) == timed
