"""Parity of the sm_100a path (through the C ABI) against the CPU oracle.

Integer / index work (domain, cell keys, sorted order, cell tables) must be
bit-exact.  Floating point is held to relative L2 <= 1e-5 on velocities (the
north-star tolerance) and tighter on intermediate grids where FP32 storage
is the only difference.
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


def _run(pb, n, pos, al, eval_a=None, eval_b=None, is_segment=1, **kw):
    scene = pb.Scene(n, cap_vort=len(pos), cap_eval=len(pos) if eval_a is None else len(eval_a), **kw)
    dpos, dal = _dev(pos), _dev(al)
    scene.set_vortices(dpos, dal)
    scene.build_far_field()
    ea = dpos if eval_a is None else _dev(eval_a)
    eb = None
    if is_segment == 1:
        eb = dpos if eval_b is None else _dev(eval_b)
    u = scene.eval(ea, eb, is_segment).cpu().numpy()
    return scene, u


def _orc(oracle, n, pos, al, eval_a=None, eval_b=None, is_segment=1, **kw):
    prm = oracle.params(n, **kw)
    ea = pos if eval_a is None else eval_a
    eb = (pos if eval_b is None else eval_b) if is_segment == 1 else None
    return oracle.pppm(prm, pos, al, ea, eb, is_segment, dump=True)


def test_domain_and_hash_bit_exact(pb, oracle):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(20000, seed=11)
    scene, _ = _run(pb, 32, pos, al)
    ref, d = _orc(oracle, 32, pos, al)
    origin, L, h = scene.domain()
    assert tuple(origin) == tuple(d["origin"]) and L == d["length"][0]
    assert h == float(d["h_f"][0])
    key, idx = scene.sorted_index()
    assert np.array_equal(key.numpy(), d["vort_key"].astype(np.int64))
    assert np.array_equal(idx.numpy(), d["vort_idx"].astype(np.int64))
    start, end = scene.cell_tables()
    assert np.array_equal(start.numpy(), d["cell_start"].astype(np.int64))
    assert np.array_equal(end.numpy(), d["cell_end"].astype(np.int64))
    scene.close()


def test_sorted_vortices_match_gather(pb, oracle):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(5000, seed=12)
    scene, _ = _run(pb, 16, pos, al)
    _, d = _orc(oracle, 16, pos, al)
    spos, sal = scene.sorted_vortices()
    idx = d["vort_idx"]
    assert np.array_equal(spos.cpu().numpy(), pos[idx])
    assert np.array_equal(sal.cpu().numpy(), al[idx].T)
    scene.close()


def test_grids_match_oracle(pb, oracle):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(16384, seed=0)
    scene, _ = _run(pb, 32, pos, al)
    _, d = _orc(oracle, 32, pos, al)
    vort = scene.grid(pb.GRID_VORT if hasattr(pb, "GRID_VORT") else 0).numpy()
    assert rel_l2(vort, d["grid_vort"]) <= 1e-6
    psi = scene.grid(1).numpy()
    assert rel_l2(psi, d["psi"]) <= 1e-5
    far = scene.grid(2).numpy()
    assert rel_l2(far, d["far_u"]) <= 1e-5
    scene.close()


@pytest.mark.parametrize("n,N,seed", [(32, 16384, 0), (16, 3000, 5), (48, 30000, 6)])
def test_velocity_uniform_cloud(pb, oracle, n, N, seed):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(N, seed=seed)
    scene, u = _run(pb, n, pos, al)
    ref, _ = _orc(oracle, n, pos, al)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_velocity_ring(pb, oracle):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(65536, seed=1)
    scene, u = _run(pb, 64, pos, al)
    ref, _ = _orc(oracle, 64, pos, al)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_velocity_separate_eval_points(pb, oracle):
    """Tracer-style evaluation (is_segment = 0) at points that are not vortices,
    some outside the grid (no far field there, near field still applies)."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(8000, seed=3)
    ev, _ = W.uniform_cloud(5000, seed=4)
    ev[:, :3] = ev[:, :3] * 5.0 - 2.0  # spans well beyond the 3x box
    scene, u = _run(pb, 32, pos, al, eval_a=ev, is_segment=0)
    ref, _ = _orc(oracle, 32, pos, al, eval_a=ev, is_segment=0)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_velocity_segments(pb, oracle):
    """Segment ends (is_segment = 1) with the other end at the vortex centre,
    as computeURotation drives it."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(8000, seed=7)
    endb = pos.copy()
    endb[:, :3] += np.float32(0.01)
    scene, u = _run(pb, 32, pos, al, eval_a=endb, eval_b=pos, is_segment=1)
    ref, _ = _orc(oracle, 32, pos, al, eval_a=endb, eval_b=pos, is_segment=1)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


@pytest.mark.parametrize("K", [-1, 0, 2])
def test_velocity_other_K(pb, oracle, K):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(6000, seed=8)
    scene, u = _run(pb, 32, pos, al, K=K)
    ref, _ = _orc(oracle, 32, pos, al, K=K)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_fixed_domain_with_outside_particles(pb, oracle):
    """DOMAIN_FIXED: some vortices fall outside the box; the hash wraps them
    (int % uint), NGP deposit ignores them, the near field follows the cells."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(6000, seed=9)
    kw = dict(domain_mode=1, fixed_origin=(-0.5, -0.5, -0.5), fixed_length=1.8)
    scene, u = _run(pb, 32, pos * np.float32([1.3, 1.0, 1.0, 1.0]), al, domain="fixed",
                    fixed_origin=(-0.5, -0.5, -0.5), fixed_length=1.8)
    ref, _ = _orc(oracle, 32, pos * np.float32([1.3, 1.0, 1.0, 1.0]), al, **kw)
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_mg_standalone_reference_and_converged(pb, oracle):
    import torch
    n = 32
    rng = np.random.default_rng(3)
    b = rng.standard_normal(n ** 3)
    mg = pb.MultiGridSolver3DPeriod_double()
    mg.m_InitialSystem(n, n, n)
    x = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    mg.m_FullMultiGrid(x, _dev(b), mode=pb.MG_REFERENCE)
    xr, _, _ = oracle.mg_solve(b, n, mg_mode=0)
    assert rel_l2(x.cpu().numpy(), xr) <= 1e-6
    x.zero_()
    rr = mg.m_FullMultiGrid(x, _dev(b), tol=1e-10, mode=pb.MG_CONVERGED)
    assert 0 <= rr <= 1e-10
    xc, _, rc = oracle.mg_solve(b, n, mg_mode=1, tol=1e-12)
    assert rel_l2(x.cpu().numpy(), xc) <= 1e-9
    # repeated calls continue from the x they are given (the scalar PPPM
    # calls the full multigrid three times in a row)
    x.zero_()
    for _ in range(3):
        mg.m_FullMultiGrid(x, _dev(b), mode=pb.MG_REFERENCE)
    x3 = oracle.mg_fmg(np.zeros(n ** 3), b, n, repeats=3)
    assert rel_l2(x.cpu().numpy(), x3) <= 1e-6
    mg.m_FinalMemoryEachLevel()


@pytest.mark.parametrize("n", [32, 64, 96])
def test_mg_vcycle_each_level(pb, oracle, n):
    """m_Vcycle(x, b, tol, res, level) (MG/MultiGrid.cpp:128-201): one V(4,4)
    cycle on level `level`'s arrays.  The hierarchy below level l is the one a
    grid of that level's edge has, so the oracle's cycle on that edge is the
    check, starting from a nonzero x.  The cycle's correction is computed in
    FP32 (r = b - A x in FP64, e = V32(0, r), x += e), so a random b and x hold
    it to 2e-6."""
    import torch
    mg = pb.MultiGridSolver3DPeriod_double()
    mg.m_InitialSystem(n, n, n)
    edges = mg.levels()
    assert edges[0] == n and len(edges) == oracle.mg_levels(n)
    rng = np.random.default_rng(n)
    for level, d in enumerate(edges):
        b = rng.standard_normal(d ** 3)
        x0 = 0.1 * rng.standard_normal(d ** 3)
        x = _dev(x0)
        mg.m_Vcycle(x, _dev(b), 1e-10, None, level)
        want = oracle.mg_vcycle(x0, b, d)
        assert rel_l2(x.cpu().numpy(), want) <= 2e-6, (level, d)
    with pytest.raises(pb.PppmError):
        mg.m_Vcycle(torch.zeros(8, dtype=torch.float64, device="cuda"), torch.zeros(8, dtype=torch.float64,
                                                                                   device="cuda"), 0, None, len(edges))
    mg.m_FinalMemoryEachLevel()


def test_direct_sum_gpu_matches_oracle(pb, oracle):
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(3000, seed=10)
    u = pb.direct_sum_fp64(_dev(pos), _dev(al), _dev(pos), 0.08, _dev(pos), 1).cpu().numpy()
    ref = oracle.direct_sum(pos, al, pos, 0.08, pos, 1)
    assert rel_l2(u, ref) <= 1e-12


def _orc_move(pos, u, dt):
    """move_particle (HFS/GPU_kernel.cu:3118-3140): float(double(p) + u dt), w = 0."""
    out = np.zeros_like(pos)
    out[:, :3] = (pos[:, :3].astype(np.float64) + u * dt).astype(np.float32)
    return out


@pytest.mark.parametrize("method", ["euler", "rk2"])
def test_advection_step(pb, oracle, method):
    import torch
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(40000, seed=13)
    n, dt = 64, 0.002
    scene = pb.Scene(n, cap_vort=len(pos), cap_eval=len(pos))
    dpos = torch.from_numpy(pos.copy()).cuda()
    scene.advect(dpos, _dev(al), dt, method=method)
    got = dpos.cpu().numpy()
    prm = oracle.params(n)
    u1, _ = oracle.pppm(prm, pos, al, pos, pos, 1)
    if method == "rk2":
        mid = _orc_move(pos, u1, 0.5 * dt)
        u2, _ = oracle.pppm(prm, mid, al, mid, mid, 1)
        ref = _orc_move(pos, u2, dt)
    else:
        ref = _orc_move(pos, u1, dt)
    disp_got = got[:, :3].astype(np.float64) - pos[:, :3]
    disp_ref = ref[:, :3].astype(np.float64) - pos[:, :3]
    assert rel_l2(disp_got, disp_ref) <= 1e-4
    assert np.all(got[:, 3] == 0.0)
    scene.close()


def test_batch_results_equal_alone(pb, oracle):
    """Several scenes of different sizes in one pppm_batch_run give exactly
    the velocities each scene gives alone (no cross-scene reduction), and
    every one of them matches the oracle.  The scenes mix the reference's
    absolute radius with a radius of one cell, so the batch's evaluation runs
    as two launches (two smoothing series), each over its scenes' work list."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    specs = [(32, "cloud", 9000, 31, {}), (48, "ring", 20000, 32, {"a_cells": 1.0}), (64, "cloud", 15000, 33, {}),
             (32, "ring", 5000, 34, {"a_cells": 1.0}), (16, "cloud", 40000, 35, {"a_cells": 1.0})]
    alone, jobs, scenes, inputs = [], [], [], []
    for n, kind, N, seed, kw in specs:
        pos, al = W.make_scene(kind, N, seed)
        inputs.append((pos, al))
        sc, u = _run(pb, n, pos, al, **kw)
        a = sc.smoothing()
        alone.append((u, a))
        sc.close()
        s2 = pb.Scene(n, cap_vort=N, cap_eval=N, **kw)
        scenes.append(s2)
        jobs.append((s2, _dev(pos), _dev(al), None, None, 1))
    together = pb.batch_run(jobs)
    for (u_alone, a), u_mix, (n, kind, N, seed, kw), (pos, al) in zip(alone, together, specs, inputs):
        assert np.array_equal(u_alone, u_mix.cpu().numpy()), (n, kind, N)
        ref, _ = _orc(oracle, n, pos, al, a=a)
        assert rel_l2(u_mix.cpu().numpy(), ref) <= VEL_TOL, (n, kind, N)
    for s2 in scenes:
        s2.close()


def test_full_scale_ring_subsample(pb, oracle):
    """The at-scale workload (1,048,576-particle ring, 128^3): every 100th
    particle checked against the oracle — the near-field pair count exactly
    and the velocity to 1e-5."""
    import torch
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(1 << 20, seed=1)
    n = 128
    scene = pb.Scene(n, cap_vort=len(pos), cap_eval=len(pos))
    dpos, dal = _dev(pos), _dev(al)
    scene.set_vortices(dpos, dal)
    scene.build_far_field()
    sub = np.ascontiguousarray(pos[::100])
    dsub = _dev(sub)
    u = scene.eval(dsub, dsub, 1).cpu().numpy()
    pairs = scene.count_pairs(dsub)
    ref, d = oracle.pppm(oracle.params(n), pos, al, sub, sub, 1, dump=True)
    assert pairs == int(d["pairs"][0])
    assert rel_l2(u, ref) <= VEL_TOL
    scene.close()


def test_solve_host_equals_the_device_path(pb, oracle):
    """pppm_solve_host, the end-to-end entry point on (pinned) host buffers
    (copies in, build, evaluation, copies out), gives bit for bit the device
    path's velocities on the same inputs, both for the vortices themselves and
    for separate points, and the oracle's within the velocity tolerance."""
    import torch
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(20000, seed=61)
    ev, _ = W.uniform_cloud(5000, seed=62)
    n = 32
    scene = pb.Scene(n, cap_vort=len(pos), cap_eval=len(pos), a_cells=1.0)
    try:
        dpos, dal = _dev(pos), _dev(al)
        scene.set_vortices(dpos, dal)
        scene.build_far_field()
        u_self = scene.eval(dpos, dpos, 1).cpu().numpy()
        u_pts = scene.eval(_dev(ev)).cpu().numpy()
        a = scene.smoothing()
        hpos = torch.from_numpy(np.ascontiguousarray(pos)).pin_memory()
        hal = torch.from_numpy(np.ascontiguousarray(np.asarray(al).T)).pin_memory()
        h_self = scene.solve_host(hpos, hal).numpy().T.copy()
        hev = torch.from_numpy(np.ascontiguousarray(ev)).pin_memory()
        h_pts = scene.solve_host(hpos, hal, hev, None, 0).numpy().T.copy()
    finally:
        scene.close()
    assert np.array_equal(h_self, u_self)
    assert np.array_equal(h_pts, u_pts)
    ref = oracle.pppm(oracle.params(n, a=a), pos, al, pos, pos, 1)[0]
    assert rel_l2(h_self, ref) <= VEL_TOL
