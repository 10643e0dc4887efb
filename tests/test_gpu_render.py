"""Parity of the CUDA splatting renderer (csrc/render.cu) with the reference's
own CPU renderer (Particle_renderer/.../shadow.cpp compute_shadows,
render.cpp render_smoke), compiled from its sources into oracle/_ref.

The projection, distances and disc tests use the reference's float operation
order without contraction, so both sides sort the particles the same way and
cover the same pixels; only expf differs in the last place from the host's.
Illumination and shadow-map values are products of up to a few hundred such
factors: they agree to 2e-5 absolute (values in [0, 1]); image channels, a
chain of over-blends, to 5e-5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ILLUM_TOL = 2e-5
IMAGE_TOL = 5e-5


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import pyrender_ref as R
    if not R.available():
        pytest.skip("reference renderer not built (make -C oracle ref)")
    from pppm_vortex_bouyant_flow_sample_b200.render import Renderer
    return Renderer(), R


def _plume(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(0, 1, (n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    r = 0.4 * rng.uniform(0, 1, n) ** (1 / 3)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = np.array([0.0, 1.0, 0.0]) + v * r[:, None] * np.array([1.0, 2.0, 1.0])
    pos[:, 3] = 1.0
    return pos


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n,quality", [(20000, 1.0), (150000, 4.0)])
def test_shadows_match_reference(env, n, quality):
    rnd, R = env
    pos = _plume(n, seed=n)
    dens = (pos[:, 3] * 2.0).astype(np.float32)
    light = (0.3, 6.0, -4.0)
    ok, ref_illum, ref_map = R.compute_shadows(pos, 0.01, 0.05, dens, light, quality)
    assert ok
    illum, smap = rnd.shadows(_dev(pos), _dev(dens), 0.01, 0.05, light, quality)
    smap = smap.cpu().numpy()
    assert smap.shape == ref_map.shape
    assert np.max(np.abs(smap - ref_map)) <= ILLUM_TOL
    assert np.max(np.abs(illum.cpu().numpy() - ref_illum)) <= ILLUM_TOL
    assert ref_illum.min() < 0.9          # the case has real shadowing


def test_light_too_close_is_refused(env):
    rnd, R = env
    import pppm_vortex_bouyant_flow_sample_b200 as pb
    pos = _plume(1000, seed=1)
    dens = np.ones(1000, np.float32)
    ok, _, _ = R.compute_shadows(pos, 0.01, 0.05, dens, (0.0, 1.0, 0.0), 1.0)
    assert not ok
    with pytest.raises(pb.PppmError):
        rnd.shadows(_dev(pos), _dev(dens), 0.01, 0.05, (0.0, 1.0, 0.0), 1.0)


@pytest.mark.parametrize("n,size", [(20000, (240, 160)), (150000, (480, 320))])
def test_smoke_matches_reference(env, n, size):
    rnd, R = env
    pos = _plume(n, seed=n + 1)
    dens = (pos[:, 3] * 2.0).astype(np.float32)
    light = (0.3, 6.0, -4.0)
    _, ref_illum, _ = R.compute_shadows(pos, 0.01, 0.05, dens, light, 2.0)
    base = np.tile(np.array([[0.5, 0.7, 0.9]], np.float32), (n, 1))
    lit = np.tile(np.array([[0.9, 0.9, 0.99]], np.float32), (n, 1))
    cam, tgt, bg = (0.0, 1.3, -2.5), (0.0, 1.1, 0.0), (0.0, 0.0, 0.0)
    w, h = size
    ref = R.render_smoke(pos, ref_illum, base, lit, 0.01, 0.05, dens, light, bg, cam, tgt, 2.0, w, h)
    got = rnd.smoke(_dev(pos), _dev(ref_illum), _dev(base), _dev(lit), 0.01, 0.05, _dev(dens), bg, cam, tgt,
                    2.0, w, h).cpu().numpy()
    assert np.max(np.abs(got - ref)) <= IMAGE_TOL
    assert ref.max() > 0.05               # something was drawn


def test_smoke_behind_camera_and_empty(env):
    rnd, R = env
    pos = _plume(5000, seed=7)
    dens = np.ones(5000, np.float32)
    base = np.full((5000, 3), 0.5, np.float32)
    lit = np.full((5000, 3), 0.9, np.float32)
    il = np.full(5000, 0.7, np.float32)
    cam, tgt, bg = (0.0, 1.0, 0.5), (0.0, 1.0, 3.0), (0.1, 0.2, 0.3)   # half the particles behind
    ref = R.render_smoke(pos, il, base, lit, 0.02, 0.1, dens, (0, 9, 0), bg, cam, tgt, 1.5, 128, 96)
    got = rnd.smoke(_dev(pos), _dev(il), _dev(base), _dev(lit), 0.02, 0.1, _dev(dens), bg, cam, tgt, 1.5,
                    128, 96).cpu().numpy()
    assert np.max(np.abs(got - ref)) <= IMAGE_TOL
    import torch
    empty = rnd.smoke(torch.zeros((0, 4), dtype=torch.float32, device="cuda"),
                      torch.zeros(0, dtype=torch.float32, device="cuda"),
                      torch.zeros((0, 3), dtype=torch.float32, device="cuda"),
                      torch.zeros((0, 3), dtype=torch.float32, device="cuda"), 0.02, 0.1,
                      torch.zeros(0, dtype=torch.float32, device="cuda"), bg, cam, tgt, 1.5, 64, 48).cpu().numpy()
    assert np.allclose(empty, np.array(bg, np.float32)[None, None, :])
