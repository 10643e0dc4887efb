"""Generates the known-answer fixtures in tests/golden/ (committed).

The reference ships no golden vectors and cannot run here, so these fixtures
are closed-form answers computed independently of the oracle with numpy:

hash_kat.npz
    Particles placed exactly on cell faces and one float ulp either side,
    plus negative and beyond-the-box coordinates.  Expected cell keys follow
    PH/particle_hash_kernel.cu:32-70 evaluated in numpy float32 arithmetic:
    floor((p - o) / h) per axis with IEEE single-precision subtraction and
    division, int % uint wrap, key = (z*n + y)*n + x.

fd_table.npz
    The far-field Green's-gradient table of HFS/GPU_kernel.cu:2646-2677 for
    K = 1, 2 at two cell sizes, written out from the closed form
    D[off] = (G(-off*h + h e) - G(-off*h - h e)) / (2h), G(r) = 1/(4 pi |r|)
    (G(0) taken as 1e-24 as the reference does).

Run: python tests/golden/make_golden.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FOUR_PI = 12.5663706144


def hash_kat():
    n = 16
    h = np.float32(1.0) / np.float32(16.0)  # 0.0625, exact
    o = np.float32(-0.3)
    pts = []
    for k in range(-2, n + 2):
        face = np.float32(o + np.float32(k) * h)
        for v in (face, np.nextafter(face, np.float32(-1e30)), np.nextafter(face, np.float32(1e30))):
            pts.append(v)
    pts = np.array(pts, dtype=np.float32)
    rng = np.random.default_rng(20240601)
    N = len(pts)
    pos = np.zeros((N, 4), dtype=np.float32)
    pos[:, 0] = pts
    pos[:, 1] = rng.permutation(pts)
    pos[:, 2] = rng.permutation(pts)
    origin = np.array([o, o, o], dtype=np.float32)

    def axis(p, oo):
        q = np.float32(p - oo) / h  # float32 ops
        g = np.floor(q).astype(np.int64)
        return (g.astype(np.int64) & 0xFFFFFFFF) % n  # (unsigned) int % uint

    kx = axis(pos[:, 0], origin[0])
    ky = axis(pos[:, 1], origin[1])
    kz = axis(pos[:, 2], origin[2])
    keys = ((kz * n + ky) * n + kx).astype(np.uint32)
    np.savez(os.path.join(HERE, "hash_kat.npz"), pos=pos, origin=origin, h=np.float32(h), n=np.int64(n),
             keys=keys)


def fd_table():
    out = {}
    for K in (1, 2):
        for h in (0.09375, 0.0125):
            W = 2 * K + 1
            t = np.zeros((W, W, W, 3))
            for kk in range(-K, K + 1):
                for jj in range(-K, K + 1):
                    for ii in range(-K, K + 1):
                        if ii == 0 and jj == 0 and kk == 0:
                            continue
                        r = -np.array([ii, jj, kk], dtype=np.float64) * h

                        def G(v):
                            d = np.sqrt(np.dot(v, v))
                            return 1e-24 if d * d <= 1e-12 else 1.0 / (FOUR_PI * d)

                        for a in range(3):
                            e = np.zeros(3)
                            e[a] = h
                            t[kk + K, jj + K, ii + K, a] = 0.5 * (G(r + e) - G(r - e)) / h
            out[f"K{K}_h{h}"] = t
    np.savez(os.path.join(HERE, "fd_table.npz"), **out)


if __name__ == "__main__":
    hash_kat()
    fd_table()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))
