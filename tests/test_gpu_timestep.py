"""Parity of pppm_vortex_step (the reference's solveTimeStep without boundary,
buoyancy or heat) against the oracle's restatement.

Two checks per case:
  * the moved segment ends and centres against orc_vortex_step: the end
    velocities differ from the oracle's only by the FP32 evaluation, so the
    displacements agree to the velocity tolerance;
  * the smoothed strengths against orc_gaussian_smooth run on the GPU's own
    moved centres and the strengths rebuilt from the GPU's own ends, so that a
    one-ulp difference in a centre cannot move a vortex to another hash cell
    between the two sides.  The GPU evaluates the Gaussian weights in FP32 and
    sums them in FP32 per staged chunk of 32 and in FP64 across chunks: error
    <= 2e-6 of the largest strength averaged.
The whole step is also compared end to end (relative L2 of the strengths).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

DISP_TOL = 1e-4      # relative L2 of the end displacements (velocity tolerance)
SMOOTH_TOL = 2e-6    # max error of a smoothed strength, relative to the largest input


@pytest.fixture(scope="module")
def pb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pppm_vortex_bouyant_flow_sample_b200 as pb
    pb.load()
    return pb


def _step_gpu(pb, n, pos, al, dt, h_seg, nu, K=1, **kw):
    import torch
    scene = pb.Scene(n, K=K, cap_vort=len(pos), cap_eval=2 * len(pos), **kw)
    dpos = torch.from_numpy(pos.copy()).cuda()
    dal = torch.from_numpy(np.ascontiguousarray(al, dtype=np.float64)).cuda()
    _, _, ea, eb = scene.vortex_step(dpos, dal, dt, h_seg=h_seg, nu=nu, return_ends=True)
    out = (dpos.cpu().numpy(), dal.cpu().numpy(), ea.cpu().numpy(), eb.cpu().numpy())
    scene.close()
    return out


def _rebuilt_strengths(al, h_seg, ea, eb):
    """alpha + (kappa (endb - enda) - alpha) from the GPU's ends (ComputeVortex + VectorAdd)."""
    l = np.sqrt((al * al).sum(axis=1))
    kappa = np.where(l < h_seg, 1.0, l / h_seg)
    seg = (eb[:, :3] - ea[:, :3]).astype(np.float64)   # float subtraction, as the reference
    return 1.0 * al + 1.0 * (kappa[:, None] * seg - al)


def _check(pb, oracle, n, pos, al, dt, h_seg, nu=0.1, K=1, orc_kw=None, **kw):
    cent, anew, ea, eb = _step_gpu(pb, n, pos, al, dt, h_seg, nu, K=K, **kw)
    prm = oracle.params(n, K=K, **(orc_kw or {}))
    rc, ra, rea, reb = oracle.vortex_step(prm, pos, al, dt, h_seg=h_seg, nu=nu)
    # unmoved ends (dt = 0 in the oracle) give the displacement baseline
    _, _, ea0, eb0 = oracle.vortex_step(prm, pos, al, 0.0, h_seg=h_seg, nu=nu)
    for got, ref, base in ((ea, rea, ea0), (eb, reb, eb0)):
        dg = got[:, :3].astype(np.float64) - base[:, :3]
        dr = ref[:, :3].astype(np.float64) - base[:, :3]
        assert rel_l2(dg, dr) <= DISP_TOL
    assert np.all(ea[:, 3] == 0.0) and np.all(eb[:, 3] == 0.0)
    mid = (0.5 * (eb[:, :3] + ea[:, :3]).astype(np.float64)).astype(np.float32)
    assert np.array_equal(cent[:, :3], mid)
    assert np.array_equal(cent[:, 3], pos[:, 3])        # ComputePosa leaves w alone
    dv = _rebuilt_strengths(al, h_seg, ea, eb)
    smooth_ref = oracle.gaussian_smooth(prm, cent, dv, nu)
    # a weighted mean's error is bounded by the weights' relative error times
    # the largest input it averages
    assert np.max(np.abs(anew - smooth_ref)) <= SMOOTH_TOL * np.abs(dv).max()
    assert rel_l2(anew, ra) <= 1e-4
    return anew, ra


@pytest.mark.parametrize("h_seg", [0.1, 7.852e-5])
def test_ring_step(pb, oracle, h_seg):
    """Ring of 20,000 blobs at 64^3: all segments uncapped (h_seg = 0.1, the
    reference's d_h) or about 60 % of them capped (h_seg = 7.852e-5, inside
    the spread of |alpha| = 7.82e-5 .. 7.88e-5)."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(20000, seed=41)
    if h_seg < 0.1:
        capped = (np.linalg.norm(al, axis=1) >= h_seg).mean()
        assert 0.2 < capped < 0.8
    _check(pb, oracle, 64, pos, al, 0.01, h_seg)


def test_cloud_step_k2(pb, oracle):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(12000, seed=42)
    _check(pb, oracle, 32, pos, al, 0.005, 0.1, K=2)


def test_sparse_step_wide_warps(pb, oracle):
    """Few vortices per cell: warps span many cells and each lane walks its own box."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(3000, seed=43)
    _check(pb, oracle, 64, pos, al, 0.005, 0.1)


def test_fixed_domain_with_outside_vortices(pb, oracle):
    """Fixed unit box; a few vortices start outside it.  Their smoothed strength
    is zero (no in-grid cell around them), as in the reference."""
    rng = np.random.default_rng(44)
    N = 4000
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.uniform(0.3, 0.7, (N, 3))
    pos[:5, 0] = 2.5
    al = rng.normal(0, 1e-3, (N, 3))
    box = dict(domain_mode=1, fixed_origin=(0.0, 0.0, 0.0), fixed_length=1.0)
    anew, _ = _check(pb, oracle, 32, pos, al, 0.005, 0.1, orc_kw=box, domain="fixed",
                     fixed_origin=(0.0, 0.0, 0.0), fixed_length=1.0)
    assert np.array_equal(anew[:5], np.zeros((5, 3)))


def test_two_steps_in_a_row(pb, oracle):
    """The step reuses the scene: a second step on the outputs of the first
    matches the oracle run twice."""
    import torch
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(8000, seed=45)
    scene = pb.Scene(32, cap_vort=len(pos), cap_eval=2 * len(pos))
    dpos = torch.from_numpy(pos.copy()).cuda()
    dal = torch.from_numpy(al.copy()).cuda()
    prm = oracle.params(32)
    rp, ra = pos.copy(), al.copy()
    for _ in range(2):
        scene.vortex_step(dpos, dal, 0.01)
        rp, ra, _, _ = oracle.vortex_step(prm, rp, ra, 0.01)
    assert rel_l2(dal.cpu().numpy(), ra) <= 1e-4
    disp_g = dpos.cpu().numpy()[:, :3].astype(np.float64) - pos[:, :3]
    disp_r = rp[:, :3].astype(np.float64) - pos[:, :3]
    assert rel_l2(disp_g, disp_r) <= DISP_TOL
    scene.close()


def test_passive_points_move_with_the_same_far_field(pb, oracle):
    """Tracers / heat particles in the step: plain evaluation (is_segment 0) with
    the step's far field, then move_particle."""
    import torch
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(8000, seed=46)
    rng = np.random.default_rng(47)
    P = 3000
    tr = np.zeros((P, 4), np.float32)
    tr[:, :3] = pos[rng.integers(0, len(pos), P), :3] + rng.normal(0, 0.05, (P, 3)).astype(np.float32)
    tr[:, 3] = 1.0
    scene = pb.Scene(32, cap_vort=len(pos), cap_eval=2 * len(pos))
    dpos = torch.from_numpy(pos.copy()).cuda()
    dal = torch.from_numpy(al.copy()).cuda()
    dtr = torch.from_numpy(tr.copy()).cuda()
    _, _, vel = scene.vortex_step(dpos, dal, 0.01, passive=dtr)
    prm = oracle.params(32)
    _, ra, _, _, rtr, rvel = oracle.vortex_step(prm, pos, al, 0.01, passive4=tr)
    assert rel_l2(vel.cpu().numpy(), rvel) <= 1e-5
    got = dtr.cpu().numpy()
    assert np.all(got[:, 3] == 0.0)
    assert rel_l2(got[:, :3].astype(np.float64) - tr[:, :3], rtr[:, :3].astype(np.float64) - tr[:, :3]) <= DISP_TOL
    assert rel_l2(dal.cpu().numpy(), ra) <= 1e-4
    scene.close()


def _heat_sphere(H, radius, centre, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(0, 1, (H, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    r = radius * rng.uniform(0, 1, H) ** (1.0 / 3.0)
    pos = np.zeros((H, 4), np.float32)
    pos[:, :3] = np.asarray(centre) + v * r[:, None]
    heat = rng.normal(1.0, 0.05, H).astype(np.float32)
    return pos, heat


@pytest.mark.parametrize("H,radius,N", [
    (200000, 0.1, 30000),     # compact plume: a 2^3 grid, whose periodic gradient is zero
    (200000, 0.35, 30000),    # 5^3 grid: each cell's particles split over many warps
    (60000, 1.0, 20000),      # 12^3 grid
    (100000, 17.0, 20000),    # L > 39.8: the grid edge is capped at 200 (8M cells)
])
def test_baroclinic_matches_oracle(pb, oracle, H, radius, N):
    import torch
    heat4, heat = _heat_sphere(H, radius, (0.5, 0.15, 0.5), seed=48)
    rng = np.random.default_rng(49)
    cent = np.zeros((N, 4), np.float32)
    cent[:, :3] = heat4[rng.integers(0, H, N), :3] + rng.normal(0, 0.02 * radius, (N, 3)).astype(np.float32)
    al = rng.normal(0, 1e-4, (N, 3))
    dt = 0.002
    cap = 201 ** 3
    ra, dim, origin, h, rrho, rgrad = oracle.baroclinic(heat4, heat, cent, al, dt, cap=cap)
    scene = pb.Scene(32, cap_vort=N, cap_eval=N)
    dal = torch.from_numpy(al.copy()).cuda()
    scene.baroclinic(torch.from_numpy(heat4).cuda(), torch.from_numpy(heat).cuda(),
                     torch.from_numpy(cent).cuda(), dal, dt)
    gdim, gorg, gh, grho, ggrad = scene.density()
    assert gdim == dim and tuple(gorg) == tuple(origin) and gh == h
    grho = grho.numpy()
    # FP64 sums in another order: the float densities agree to an ulp or two
    scale = np.abs(rrho).max()
    assert np.max(np.abs(grho - rrho)) <= 4 * np.finfo(np.float32).eps * scale
    gscale = 4 * np.finfo(np.float32).eps * scale / h
    assert np.max(np.abs(ggrad.numpy().T - rgrad)) <= gscale
    d_gpu = dal.cpu().numpy() - al
    d_ref = ra - al
    if dim <= 2:
        # with two cells per axis the periodic central difference of any field
        # is zero, so the reference adds nothing
        assert not d_ref.any() and not d_gpu.any()
    else:
        assert np.linalg.norm(d_ref) > 0
        assert rel_l2(d_gpu, d_ref) <= 1e-5
    scene.close()


def test_baroclinic_no_heat_is_a_no_op(pb):
    import torch
    scene = pb.Scene(32, cap_vort=10, cap_eval=10)
    al = torch.ones((10, 3), dtype=torch.float64, device="cuda")
    cent = torch.zeros((10, 4), dtype=torch.float32, device="cuda")
    heat4 = torch.zeros((1, 4), dtype=torch.float32, device="cuda")   # one point: zero-size box
    scene.baroclinic(heat4, torch.ones(1, dtype=torch.float32, device="cuda"), cent, al, 0.01)
    assert torch.equal(al, torch.ones_like(al))
    scene.close()
