"""Known-answer checks of the oracle's vortex-segment time step (CPU only).

The oracle's orc_vortex_step / orc_gaussian_smooth restate the reference's
solveTimeStep sub-steps (HFS/VortexSimulationSystemImp.cpp:90-125,
HFS/GPU_kernel.cu:3118-3254, 3327-3459).  These tests pin them to an
independent numpy statement of the same rules and to closed-form answers.
"""
import numpy as np

from conftest import rel_l2


def _np_domain(pos):
    lo = pos[:, :3].astype(np.float64).min(axis=0)
    hi = pos[:, :3].astype(np.float64).max(axis=0)
    L = float((hi - lo).max())
    cen = 0.5 * (lo + hi)
    return cen - 1.5 * L, 3.0 * L


def _np_smooth(pos, d, n, nu, origin, L):
    """Brute-force restatement: every vortex whose hash cell lies in the 5^3
    block around the centre's FP64-origin cell contributes."""
    h_f = np.float32(L / n)
    of = origin.astype(np.float32)
    invh = 1.0 / float(h_f)
    rel_hash = (pos[:, :3] - of).astype(np.float32)
    hk = np.floor(rel_hash / h_f).astype(np.int64)          # hash cell (float arithmetic)
    rel = (pos[:, :3].astype(np.float64) - origin).astype(np.float32)
    ck = np.floor(rel.astype(np.float64) * invh).astype(np.int64)
    out = np.zeros_like(d)
    inside = np.all((hk >= 0) & (hk < n), axis=1)
    for t in range(len(pos)):
        lo, hi = np.maximum(ck[t] - 2, 0), np.minimum(ck[t] + 2, n - 1)
        sel = inside & np.all((hk >= lo) & (hk <= hi), axis=1)
        diff = (rel[sel] - rel[t]).astype(np.float32).astype(np.float64)
        w = np.exp(-(diff ** 2).sum(axis=1) / (2 * nu * nu))
        tw = w.sum()
        if tw < 1e-12:
            tw = 1e24
        out[t] = (w[:, None] * d[sel]).sum(axis=0) / tw
    return out


def test_smoothing_matches_numpy(oracle):
    rng = np.random.default_rng(5)
    N, n, nu = 600, 16, 0.1
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.normal(0, 0.3, (N, 3))
    d = rng.normal(0, 1, (N, 3))
    got = oracle.gaussian_smooth(oracle.params(n), pos, d, nu)
    origin, L = _np_domain(pos)
    ref = _np_smooth(pos, d, n, nu, origin, L)
    assert rel_l2(got, ref) <= 1e-13


def test_smoothing_keeps_constant_and_isolated(oracle):
    rng = np.random.default_rng(6)
    N = 300
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.uniform(-0.2, 0.2, (N, 3))
    pos[-1, :3] = (3.0, 3.0, 3.0)          # far from the cluster: sees only itself
    d = np.tile(np.array([[1.5, -2.0, 0.25]]), (N, 1))
    d[-1] = (7.0, 8.0, 9.0)
    got = oracle.gaussian_smooth(oracle.params(32), pos, d, 0.1)
    assert np.allclose(got[:-1], d[:-1], rtol=0, atol=1e-12)
    assert np.array_equal(got[-1], d[-1])


def test_smoothing_outside_fixed_domain_is_zero(oracle):
    pos = np.zeros((3, 4), np.float32)
    pos[0, :3] = (0.5, 0.5, 0.5)
    pos[1, :3] = (0.52, 0.5, 0.5)
    pos[2, :3] = (5.0, 0.5, 0.5)           # outside the unit box: no in-grid cell near it
    d = np.ones((3, 3))
    prm = oracle.params(16, domain_mode=1, fixed_origin=(0.0, 0.0, 0.0), fixed_length=1.0)
    got = oracle.gaussian_smooth(prm, pos, d, 0.1)
    assert np.allclose(got[:2], 1.0) and np.array_equal(got[2], np.zeros(3))


def test_segments_at_zero_dt(oracle):
    """dt = 0: the ends are c -/+ s/2 and the new strength is kappa * (endb - enda)
    smoothed, for both the uncapped (|alpha| < h) and the capped branch."""
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.uniform_cloud(400, seed=9)
    al = al * 0.02 / np.abs(al).max()
    h = 0.012
    cap = np.linalg.norm(al, axis=1) >= h
    assert 0 < cap.sum() < len(al)
    prm = oracle.params(16)
    cent, anew, ea, eb = oracle.vortex_step(prm, pos, al, 0.0, h_seg=h, nu=0.1)
    l = np.linalg.norm(al, axis=1)
    s = np.where(cap[:, None], 0.5 * al / l[:, None] * h, 0.5 * al)
    c = pos[:, :3].astype(np.float64)
    assert np.array_equal(eb[:, :3], (c + s).astype(np.float32))
    assert np.array_equal(ea[:, :3], (c - s).astype(np.float32))
    mid = (0.5 * (eb[:, :3] + ea[:, :3]).astype(np.float64)).astype(np.float32)
    assert np.array_equal(cent[:, :3], mid)
    kappa = np.where(cap, l / h, 1.0)
    seg = (eb[:, :3] - ea[:, :3]).astype(np.float64)
    dv = al + (kappa[:, None] * seg - al)
    ref = oracle.gaussian_smooth(prm, cent, dv, 0.1)
    assert rel_l2(anew, ref) <= 1e-15


def _np_baroclinic(heat4, heat, cent, al, dt):
    """Independent numpy statement of addBaroclinicForce for small inputs."""
    p = heat4[:, :3].astype(np.float64)
    lo, hi = p.min(axis=0), p.max(axis=0)
    L = 1.2 * float((hi - lo).max())
    origin = (lo + 0.5 * (hi - lo)) - 0.5 * L
    dim = min(int(np.floor(L / 0.2) + 1), 200)
    h = L / dim
    h_f = np.float32(L / dim)
    of = origin.astype(np.float32)
    hk = np.floor((heat4[:, :3] - of).astype(np.float32) / h_f).astype(np.int64)   # hash cells
    rel = (p - origin).astype(np.float32).astype(np.float64) / h                   # particle, in cells
    occupied = set(map(tuple, hk))
    rho = np.zeros((dim, dim, dim), np.float32)                                    # [k, j, i]
    for k in range(dim):
        for j in range(dim):
            for i in range(dim):
                g = np.array([i + 0.5, j + 0.5, k + 0.5])
                sel = np.all(np.abs(hk - np.array([i, j, k])) <= 2, axis=1)
                r = ((rel[sel] - g) ** 2).sum(axis=1)
                w = np.where(r < 1, (1 - r) ** 4, 0.0)
                tw = w.sum() + (0.0 if (i, j, k) in occupied else 1.0)
                rho[k, j, i] = np.float32((w * heat[sel]).sum() / (tw if tw >= 1e-12 else 1e24))
    r64 = rho.astype(np.float64)
    gx = ((np.roll(r64, -1, 2) - np.roll(r64, 1, 2)) * 0.5 / h).astype(np.float32)
    gy = ((np.roll(r64, -1, 1) - np.roll(r64, 1, 1)) * 0.5 / h).astype(np.float32)
    gz = ((np.roll(r64, -1, 0) - np.roll(r64, 1, 0)) * 0.5 / h).astype(np.float32)
    inv_hf = 1.0 / float(h_f)
    q = (cent[:, :3].astype(np.float64) - origin).astype(np.float32).astype(np.float64) * inv_hf
    out = al.copy()
    for t in range(len(cent)):
        s = np.zeros(3)
        base = np.floor(q[t]).astype(int)
        for k in range(base[2] - 2, base[2] + 3):
            for j in range(base[1] - 2, base[1] + 3):
                for i in range(base[0] - 2, base[0] + 3):
                    if not (0 <= i < dim and 0 <= j < dim and 0 <= k < dim):
                        continue
                    wv = np.clip(1 - np.abs(np.array([i, j, k]) + 0.5 - q[t]), 0, None).prod()
                    s += np.array([gx[k, j, i], gy[k, j, i], gz[k, j, i]], np.float64) * wv
        b = np.cross(s, [0.0, 10.0, 0.0])
        out[t] += dt * 5.0 * 0.1 * b
    return out, dim, rho.reshape(-1), np.stack([gx.reshape(-1), gy.reshape(-1), gz.reshape(-1)], axis=1)


def test_baroclinic_matches_numpy(oracle):
    rng = np.random.default_rng(12)
    H, N = 400, 60
    heat4 = np.zeros((H, 4), np.float32)
    heat4[:, :3] = rng.uniform(-0.6, 0.6, (H, 3))
    heat = rng.normal(1.0, 0.05, H).astype(np.float32)
    cent = np.zeros((N, 4), np.float32)
    cent[:, :3] = rng.uniform(-0.6, 0.6, (N, 3))
    al = rng.normal(0, 1e-3, (N, 3))
    got, dim, _, _, rho, grad = oracle.baroclinic(heat4, heat, cent, al, 0.002, cap=4096)
    ref, rdim, rrho, rgrad = _np_baroclinic(heat4, heat, cent, al, 0.002)
    assert dim == rdim == 8
    assert np.max(np.abs(rho - rrho)) <= 2 * np.finfo(np.float32).eps
    assert np.max(np.abs(grad - rgrad)) <= 1e-5 * np.abs(rgrad).max()
    assert rel_l2(got - al, ref - al) <= 1e-5
