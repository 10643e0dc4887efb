"""Parity of the scalar PPPM (csrc/potential.cu, the reference's
PotentialFieldSolver) against the oracle's restatement (orc_potential).

Grids: density and right-hand side (with the monopole Dirichlet data) to FP64
round-off (different summation order); the potential after the three
full-multigrid calls to 1e-6 (FP32 multigrid with FP64 defect correction, as
the vector path); gradients and potentials at the evaluation points to 1e-5
relative L2.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pf():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pppm_vortex_bouyant_flow_sample_b200 as pb
    pb.load()
    from pppm_vortex_bouyant_flow_sample_b200.potential import PotentialFieldSolver
    return PotentialFieldSolver


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _case(N, M, seed, spread=0.2, signed=True):
    rng = np.random.default_rng(seed)
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.normal(0.3, spread, (N, 3))
    mass = rng.normal(0.5, 1.0, N) if signed else rng.uniform(0.5, 1.5, N)
    ev = np.zeros((M, 4), np.float32)
    ev[:, :3] = rng.normal(0.3, 2.5 * spread, (M, 3))      # some outside the 2x box
    ev[: M // 4] = pos[rng.integers(0, N, M // 4)]          # some on the masses themselves
    return pos, mass, ev


@pytest.mark.parametrize("n,K", [(32, 1), (64, 1), (32, 2), (32, -1)])
def test_gradient_matches_oracle(pf, oracle, n, K):
    pos, mass, ev = _case(20000, 8000, seed=n + K)
    s = pf()
    s.initializeSolver(n, n, n, K, len(ev), len(pos))
    s.setMassParameter(len(pos), _dev(pos), _dev(mass))
    s.setEvalParameter(len(ev), _dev(ev))
    s.computeFarFieldBuffer()
    s.evaluateGradient(True)
    g = s.getGradPhi().cpu().numpy()
    ref, d = oracle.potential(n, K, pos, mass, ev, dump=True)
    grids = s.grids()
    assert grids["origin"] == tuple(d["origin"][:3]) and grids["length"] == d["origin"][3]
    assert rel_l2(grids["density"].numpy(), d["density"]) <= 1e-13
    assert np.allclose(grids["monopole"], d["monopole"], rtol=1e-12, atol=1e-15)
    assert rel_l2(grids["rhs"].numpy(), d["rhs"]) <= 1e-13
    assert rel_l2(grids["phi"].numpy(), d["phi"]) <= 1e-6
    assert rel_l2(grids["far"].numpy(), d["far"]) <= 1e-6
    assert rel_l2(g, ref) <= 1e-5
    # outside the grid box the gradient is zero on both sides
    out = np.all(ref == 0.0, axis=1)
    assert out.any() and np.array_equal(g[out], ref[out])
    s.shutdown()


@pytest.mark.parametrize("n,K", [(32, 1), (48, 2)])
def test_scalar_potential_matches_oracle(pf, oracle, n, K):
    pos, mass, ev = _case(15000, 6000, seed=7 * n + K, signed=False)
    s = pf()
    s.initializeSolver(n, n, n, K, len(ev), len(pos))
    s.setMassParameter(len(pos), _dev(pos), _dev(mass))
    s.setEvalParameter(len(ev), _dev(ev))
    s.computeFarFieldPotentialBuffer()
    s.evaluateScalarPotential()
    phi = s.getScalarPhi().cpu().numpy()
    ref, d = oracle.potential(n, K, pos, mass, ev, scalar=True, dump=True)
    assert rel_l2(s.grids()["far"].numpy()[: n ** 3], d["far"]) <= 1e-6
    assert rel_l2(phi, ref) <= 1e-5
    s.shutdown()


def test_far_from_the_masses_the_potential_is_the_monopole(pf):
    """Beyond the masses the computed potential and gradient approach
    M / (4 pi r) and its gradient (a physics check on the whole chain)."""
    import torch
    rng = np.random.default_rng(11)
    N = 5000
    pos = np.zeros((N, 4), np.float32)
    pos[:, :3] = rng.normal(0.0, 0.05, (N, 3))
    mass = np.full(N, 1.0 / N)
    d = rng.normal(0, 1, (400, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ev = np.zeros((400, 4), np.float32)
    ev[:, :3] = d * 0.18
    s = pf()
    s.initializeSolver(64, 64, 64, 1, 400, N)
    s.setMassParameter(N, _dev(pos), _dev(mass))
    s.setEvalParameter(400, _dev(ev))
    s.computeFarFieldPotentialBuffer()
    s.evaluateScalarPotential()
    r = np.linalg.norm(ev[:, :3].astype(np.float64) - pos[:, :3].mean(0), axis=1)
    assert rel_l2(s.getScalarPhi().cpu().numpy(), 1.0 / (4 * np.pi * r)) <= 0.05
    s.computeFarFieldBuffer()
    s.evaluateGradient(True)
    rv = ev[:, :3].astype(np.float64) - pos[:, :3].mean(0)
    grad = -rv / (4 * np.pi * r[:, None] ** 3)
    assert rel_l2(s.getGradPhi().cpu().numpy(), grad) <= 0.05
    # dphi/dn on the sphere: -0.5 m / area + n . grad
    normals = torch.from_numpy(d).cuda()
    areas = torch.full((400,), 4 * np.pi * 0.18 ** 2 / 400, dtype=torch.float64, device="cuda")
    s.setEvalNormals(400, normals)
    s.setEvalAreas(400, areas)
    s._mass = torch.full((400,), 1.0 / 400, dtype=torch.float64, device="cuda")
    s.computeDphiDn()
    g = s.getGradPhi().cpu().numpy()
    want = -0.5 * (1.0 / 400) / areas.cpu().numpy() + (d * g).sum(axis=1)
    assert np.allclose(s.getDpDn().cpu().numpy(), want, rtol=1e-12, atol=1e-15)
    s.shutdown()
