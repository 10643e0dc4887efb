"""Seeded synthetic scenes for the PPPM vortex-particle evaluation.

The generator is SplitMix64 (Steele, Lea & Flood 2014) mapped to U[0,1) with 53
random bits, and Box-Muller for normals, so the same seed gives the same scene
on every host.  The reference draws its emitters with the C library's rand()
(hybridFastSummation/VortexSimulationSystemImp.cpp:2-5), which is not portable;
these scenes follow the workload descriptions instead:

* ``uniform_cloud``: positions U[0,1)^3, strengths i.i.d. N(0,1) per component.
* ``vortex_ring``: ring of major radius R centred at (0.5,0.5,0.5) with axis +z;
  azimuth U[0,2pi), radial and axial core offsets N(0, sigma^2); strength
  (Gamma * 2 pi R / N) * (t_hat + noise), noise i.i.d. N(0, rel_noise^2) per
  component (the ring's circulation stays Gamma).
* ``plume_sphere``: positions uniform in a sphere (radius 0.1 at
  (0.5, 0.15, 0.5)), zero strength, temperature N(1, 0.05^2).
* ``sphere_panels`` / ``shell_points``: sources of the scalar PPPM on a sphere
  (mass = area x cos of the polar angle) and evaluation points in a shell
  around it.
* ``scene_mix``: the batched mix (grid edge from {32,48,64,96,128}, particle
  count log-uniform in [1e4, 1e6], even scenes clouds, odd scenes rings).
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


class SplitMix64:
    """Counter-based SplitMix64 stream; draws are vectorised."""

    def __init__(self, seed: int):
        self.state = np.uint64(seed & 0xFFFFFFFFFFFFFFFF)

    def next_u64(self, count: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            steps = np.arange(1, count + 1, dtype=np.uint64)
            z = self.state + steps * _GOLDEN
            self.state = self.state + np.uint64(count) * _GOLDEN
            z = (z ^ (z >> np.uint64(30))) * _M1
            z = (z ^ (z >> np.uint64(27))) * _M2
            z = z ^ (z >> np.uint64(31))
        return z

    def uniform(self, count: int) -> np.ndarray:
        """U[0,1) doubles from the top 53 bits."""
        return (self.next_u64(count) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)

    def normal(self, count: int) -> np.ndarray:
        """N(0,1) by Box-Muller on pairs of uniforms."""
        m = (count + 1) // 2
        u1 = self.uniform(m)
        u2 = self.uniform(m)
        r = np.sqrt(-2.0 * np.log1p(-u1))  # 1-u1 in (0,1]
        t = 2.0 * np.pi * u2
        out = np.empty(2 * m)
        out[0::2] = r * np.cos(t)
        out[1::2] = r * np.sin(t)
        return out[:count]


def _pack_pos(x, y, z) -> np.ndarray:
    pos = np.zeros((x.shape[0], 4), dtype=np.float32)
    pos[:, 0], pos[:, 1], pos[:, 2] = x, y, z
    return pos


def uniform_cloud(N: int, seed: int = 0):
    """N positions U[0,1)^3 (float4, w=0) and N(0,1) strengths (N,3) float64."""
    g = SplitMix64(seed)
    u = g.uniform(3 * N).reshape(N, 3)
    pos = _pack_pos(u[:, 0], u[:, 1], u[:, 2])
    alpha = g.normal(3 * N).reshape(N, 3)
    return pos, alpha


def vortex_ring(N: int, seed: int = 1, R: float = 0.25, sigma: float = 0.03,
                gamma: float = 1.0, rel_noise: float = 1e-3, centre=(0.5, 0.5, 0.5)):
    g = SplitMix64(seed)
    phi = 2.0 * np.pi * g.uniform(N)
    dr = sigma * g.normal(N)
    dz = sigma * g.normal(N)
    rad = R + dr
    x = centre[0] + rad * np.cos(phi)
    y = centre[1] + rad * np.sin(phi)
    z = centre[2] + dz
    pos = _pack_pos(x, y, z)
    t = np.stack([-np.sin(phi), np.cos(phi), np.zeros(N)], axis=1)
    noise = rel_noise * g.normal(3 * N).reshape(N, 3)
    alpha = (gamma * 2.0 * np.pi * R / N) * (t + noise)
    return pos, alpha


def plume_sphere(N: int, seed: int = 3, radius: float = 0.1, centre=(0.5, 0.15, 0.5)):
    """Positions uniform in a sphere, zero strength, temperature N(1, 0.05^2)."""
    g = SplitMix64(seed)
    d = g.normal(3 * N).reshape(N, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * np.cbrt(g.uniform(N))
    p = np.asarray(centre)[None, :] + d * r[:, None]
    pos = _pack_pos(p[:, 0], p[:, 1], p[:, 2])
    alpha = np.zeros((N, 3))
    temp = 1.0 + 0.05 * g.normal(N)
    return pos, alpha, temp


def sphere_panels(N: int, radius: float = 0.15, centre=(0.5, 0.5, 0.5)):
    """Boundary-element sources: N points of a Fibonacci lattice on a sphere,
    mass = panel area x cos(polar angle) (the source layer of a sphere in a
    uniform stream along +y), as float4 positions and float64 masses."""
    k = np.arange(N, dtype=np.float64) + 0.5
    y = 1.0 - 2.0 * k / N
    r = np.sqrt(np.maximum(0.0, 1.0 - y * y))
    phi = np.pi * (3.0 - np.sqrt(5.0)) * k
    p = np.stack([r * np.cos(phi), y, r * np.sin(phi)], axis=1)
    pos = _pack_pos(*(centre[c] + radius * p[:, c] for c in range(3)))
    mass = (4.0 * np.pi * radius * radius / N) * y
    return pos, mass


def shell_points(N: int, seed: int = 4, r0: float = 0.16, r1: float = 0.29, centre=(0.5, 0.5, 0.5)):
    """N points uniform in the spherical shell r0 <= |x - centre| <= r1."""
    g = SplitMix64(seed)
    d = g.normal(3 * N).reshape(N, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.cbrt(r0 ** 3 + (r1 ** 3 - r0 ** 3) * g.uniform(N))
    p = np.asarray(centre)[None, :] + d * r[:, None]
    return _pack_pos(p[:, 0], p[:, 1], p[:, 2])


def scene_mix(count: int = 64, seed: int = 2, grids=(32, 48, 64, 96, 128),
              n_min: float = 1e4, n_max: float = 1e6):
    """List of (grid_edge, N, kind, scene_seed) for the batched-scene mix."""
    g = SplitMix64(seed)
    ug = g.uniform(count)
    un = g.uniform(count)
    out = []
    for s in range(count):
        n = grids[min(int(ug[s] * len(grids)), len(grids) - 1)]
        N = int(round(np.exp(np.log(n_min) + un[s] * (np.log(n_max) - np.log(n_min)))))
        kind = "cloud" if s % 2 == 0 else "ring"
        out.append((n, N, kind, 1000 + s))
    return out


def make_scene(kind: str, N: int, seed: int):
    if kind == "cloud":
        return uniform_cloud(N, seed)
    if kind == "ring":
        return vortex_ring(N, seed)
    raise ValueError(kind)
