"""Known-answer checks of the oracle's scalar PPPM (orc_potential, the
reference's PotentialFieldSolver restated; CPU only)."""
import numpy as np

from conftest import rel_l2


def _masses(N, seed):
    rng = np.random.default_rng(seed)
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.normal(0.2, 0.1, (N, 3))
    return pos, rng.uniform(0.5, 1.5, N)


def test_domain_density_and_dirichlet_data(oracle):
    """2 x bounding box, NGP density conserving mass, and the right-hand side
    -h^2 rho minus the monopole's ghost values on every boundary face."""
    n = 8
    pos, m = _masses(500, 1)
    ev = pos[:4].copy()
    _, d = oracle.potential(n, 1, pos, m, ev, dump=True)
    p = pos[:, :3].astype(np.float64)
    lo, hi = p.min(0), p.max(0)
    L = 2.0 * (hi - lo).max()
    origin = (lo + 0.5 * (hi - lo)) - 0.5 * L
    assert np.array_equal(d["origin"][:3], origin) and d["origin"][3] == L
    h_f = np.float32(L / n)
    h = float(h_f)
    assert abs(d["density"].sum() * h ** 3 - m.sum()) <= 1e-12 * m.sum()
    cx = (p * m[:, None]).sum(0) / m.sum()
    assert np.allclose(d["monopole"][:3], cx, rtol=1e-12) and abs(d["monopole"][3] - m.sum()) < 1e-12
    rhs = -d["density"] * float(h_f * h_f)
    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    ii, jj, kk = ii.T.reshape(-1), jj.T.reshape(-1), kk.T.reshape(-1)    # x fastest
    for axis, idx in ((0, ii), (1, jj), (2, kk)):
        for side, face in ((-1, 0), (1, n - 1)):
            sel = idx == face
            g = np.stack([ii, jj, kk], axis=1)[sel].astype(np.float64) + 0.5
            g[:, axis] += side
            world = g * h + origin
            r = np.linalg.norm(world - d["monopole"][:3], axis=1)
            rhs[sel] -= m.sum() / (4 * np.pi * r * (12.5663706144 / (4 * np.pi)))
    assert rel_l2(d["rhs"], rhs) <= 1e-13


def test_far_field_is_the_monopole(oracle):
    pos, m = _masses(4000, 2)
    m = m / m.sum()
    rng = np.random.default_rng(3)
    dirs = rng.normal(0, 1, (300, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    centre = (pos[:, :3].astype(np.float64) * m[:, None]).sum(0)
    ev = np.zeros((300, 4), np.float32)
    ev[:, :3] = centre + dirs * 0.35
    r = np.linalg.norm(ev[:, :3].astype(np.float64) - centre, axis=1)
    phi = oracle.potential(64, 1, pos, m, ev, scalar=True)
    assert rel_l2(phi, 1.0 / (4 * np.pi * r)) <= 0.05
    g = oracle.potential(64, 1, pos, m, ev)
    want = -(ev[:, :3].astype(np.float64) - centre) / (4 * np.pi * r[:, None] ** 3)
    assert rel_l2(g, want) <= 0.05


def test_repeated_full_multigrid_continues_from_x(oracle):
    """Three m_FullMultiGrid calls from x = 0 equal one call from the result
    of two (the calls chain through x)."""
    n = 16
    b = np.random.default_rng(4).standard_normal(n ** 3)
    x3 = oracle.mg_fmg(np.zeros(n ** 3), b, n, repeats=3)
    x2 = oracle.mg_fmg(np.zeros(n ** 3), b, n, repeats=2)
    assert np.array_equal(oracle.mg_fmg(x2, b, n, repeats=1), x3)
    x1 = oracle.mg_fmg(np.zeros(n ** 3), b, n, repeats=1)
    assert not np.array_equal(x1, x3)
