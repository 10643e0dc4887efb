"""ctypes bindings of oracle/_ref/librefgpu.so: the reference's own GPU kernels
(hybridFastSummation/GPU_kernel.cu, particle_hash/particle_hash_kernel.cu,
multigrid/MultiGrid_kernel.cu) behind ref_gpu/ref_gpu_shim.cu,
ref_gpu/ref_hash_shim.cu and ref_gpu/ref_mg_shim.cu, built by
`make -C oracle refgpu` where the reference's sources are present.  TEST
INFRASTRUCTURE ONLY: the parity tests run it on the GPU as a checker of the
oracle and of the product; the product never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "librefgpu.so")
_lib = None
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


def available() -> bool:
    return os.path.exists(_LIB_PATH)


def build() -> bool:
    """Compile the reference's kernels when its sources are present; True if the library exists."""
    from oracle.refroot import reference_root
    src = reference_root()
    if src:
        subprocess.run(["make", "-s", "-C", _HERE, "refgpu", f"REF_ROOT={src}"], check=True)
    return available()


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/librefgpu.so is missing (make -C oracle refgpu)")
        L = C.CDLL(_LIB_PATH)
        L.refgpu_farfield_eval.argtypes = [C.c_uint32, C.c_int, C.c_uint32, f32p, f64p, u32p, u32p, f64p, f64p,
                                           C.c_double, C.c_uint32, f32p, f32p, C.c_int, f64p, f64p, f64p, f64p,
                                           f64p, f32p]
        L.refgpu_farfield_eval.restype = C.c_int
        L.refgpu_hash.argtypes = [C.c_uint32, C.c_float, f32p, C.c_uint32, f32p, u32p, u32p, u32p, u32p, f32p]
        L.refgpu_hash.restype = C.c_int
        L.refgpu_segments.argtypes = [C.c_uint32, f32p, f64p, C.c_double, f32p, f32p, f64p]
        L.refgpu_segment_update.argtypes = [C.c_uint32, f32p, f32p, f64p, f64p, f64p, f64p, C.c_double, f32p, f64p]
        L.refgpu_gaussian_smooth.argtypes = [C.c_uint32, C.c_double, f64p, C.c_uint32, f32p, f32p, u32p, u32p, f64p,
                                             C.c_double, C.c_double, f64p, f32p]
        L.refgpu_baroclinic.argtypes = [C.c_uint32, C.c_double, C.c_float, f64p, C.c_uint32, f32p, f32p, u32p, u32p,
                                        C.c_uint32, f32p, f64p, C.c_double, f32p, f32p, f32p]
        L.refgpu_potential.argtypes = [C.c_uint32, C.c_int, C.c_uint32, f32p, f64p, f64p, u32p, u32p, f64p, f64p,
                                       C.c_float, C.c_double, C.c_uint32, f32p, C.c_int, C.c_void_p, C.c_void_p,
                                       f64p, f64p, f64p, f64p, C.c_void_p, f32p]
        L.refgpu_mg_fmg.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, f64p, f64p, C.c_void_p]
        for name in ("refgpu_segments", "refgpu_segment_update", "refgpu_gaussian_smooth", "refgpu_baroclinic",
                     "refgpu_potential", "refgpu_mg_fmg"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def farfield_eval(n, K, sorted_pos4, sorted_alpha, start, end, psi, origin, cell_h, eval_a4, eval_b4=None,
                  is_segment=0):
    """The reference's P2M, curl, far-field correction, interpolation and
    near-field correction on the given sorted vortices, cell tables and psi.
    Returns a dict of FP64 arrays: vort, curl, far (3, n^3), far_at, uvw (3, M),
    and stage_ms: device milliseconds of P2M, curl, far field, interpolation and
    near field."""
    N = len(sorted_pos4)
    M = len(eval_a4)
    Cn = n ** 3
    pos = np.ascontiguousarray(sorted_pos4, dtype=np.float32)
    al = np.ascontiguousarray(np.asarray(sorted_alpha, dtype=np.float64).reshape(N, 3).T)
    ea = np.ascontiguousarray(eval_a4, dtype=np.float32)
    eb = np.ascontiguousarray(eval_b4 if eval_b4 is not None else np.zeros_like(ea), dtype=np.float32)
    out = {k: np.zeros(3 * Cn) for k in ("vort", "curl", "far")}
    out.update({k: np.zeros(3 * M) for k in ("far_at", "uvw")})
    ms = np.zeros(5, np.float32)
    rc = lib().refgpu_farfield_eval(n, K, N, pos, al, np.ascontiguousarray(start, dtype=np.uint32),
                                    np.ascontiguousarray(end, dtype=np.uint32),
                                    np.ascontiguousarray(psi, dtype=np.float64).reshape(-1),
                                    np.ascontiguousarray(origin, dtype=np.float64), float(cell_h), M, ea, eb,
                                    int(is_segment), out["vort"], out["curl"], out["far"], out["far_at"],
                                    out["uvw"], ms)
    if rc != 0:
        raise RuntimeError(f"refgpu_farfield_eval: CUDA error {rc}")
    res = {k: v.reshape(3, -1) for k, v in out.items()}
    res["stage_ms"] = dict(zip(("p2m", "curl", "farfield", "interp", "near_field"), ms.tolist()))
    return res


def hash_particles(n, h, origin, pos4, end_fill=0xFFFFFFFF):
    """The reference's calcHashD, stable key sort and FindCellStartD for float
    cell size h and float origin.  Returns (sorted keys, sorted indices,
    cellStart, cellEnd, milliseconds); cellEnd holds end_fill where the
    reference leaves it unwritten (empty cells)."""
    pos = np.ascontiguousarray(pos4, dtype=np.float32)
    N = len(pos)
    Cn = n ** 3
    keys = np.zeros(N, np.uint32)
    idx = np.zeros(N, np.uint32)
    start = np.zeros(Cn, np.uint32)
    end = np.full(Cn, end_fill, np.uint32)
    ms = np.zeros(1, np.float32)
    rc = lib().refgpu_hash(n, C.c_float(h), np.ascontiguousarray(origin, dtype=np.float32), N, pos, keys, idx,
                           start, end, ms)
    if rc != 0:
        raise RuntimeError(f"refgpu_hash: CUDA error {rc}")
    return keys, idx, start, end, float(ms[0])


def _check(rc, name):
    if rc != 0:
        raise RuntimeError(f"{name}: error {rc}")


def _soa(a, N):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(N, 3).T)


def segments(cent4, alpha3, h_seg):
    """ComputePosb: (enda4, endb4, kappa)."""
    cent = np.ascontiguousarray(cent4, dtype=np.float32)
    N = len(cent)
    ea = np.zeros((N, 4), np.float32)
    eb = np.zeros((N, 4), np.float32)
    k = np.zeros(N)
    _check(lib().refgpu_segments(N, cent, _soa(alpha3, N), float(h_seg), ea, eb, k), "refgpu_segments")
    return ea, eb, k


def segment_update(enda4, endb4, alpha3, kappa, ua3, ub3, dt):
    """move_particle on both ends, ComputePosa, ComputeVortex, VectorAdd:
    (moved enda4, moved endb4, centres4, strengths to smooth (N, 3))."""
    ea = np.array(enda4, dtype=np.float32, order="C", copy=True)
    eb = np.array(endb4, dtype=np.float32, order="C", copy=True)
    N = len(ea)
    cent = np.zeros((N, 4), np.float32)
    dv = np.zeros(3 * N)
    _check(lib().refgpu_segment_update(N, ea, eb, _soa(alpha3, N), np.ascontiguousarray(kappa, dtype=np.float64),
                                       _soa(ua3, N), _soa(ub3, N), float(dt), cent, dv), "refgpu_segment_update")
    return ea, eb, cent, dv.reshape(3, N).T.copy()


def gaussian_smooth(n, cell_h, origin, cent4, sorted_cent4, start, end, sorted_d3, nu, dt, timing=None):
    """ParticleGaussianSmooth: smoothed strengths (N, 3) in caller order (the
    kernel's milliseconds appended to the list timing when given)."""
    cent = np.ascontiguousarray(cent4, dtype=np.float32)
    N = len(cent)
    out = np.zeros(3 * N)
    ms = np.zeros(1, np.float32)
    _check(lib().refgpu_gaussian_smooth(n, float(cell_h), np.ascontiguousarray(origin, dtype=np.float64), N, cent,
                                        np.ascontiguousarray(sorted_cent4, dtype=np.float32),
                                        np.ascontiguousarray(start, dtype=np.uint32),
                                        np.ascontiguousarray(end, dtype=np.uint32), _soa(sorted_d3, N), float(nu),
                                        float(dt), out, ms), "refgpu_gaussian_smooth")
    if timing is not None:
        timing.append(float(ms[0]))
    return out.reshape(3, N).T.copy()


def baroclinic(dim, h, h_f, origin, sorted_heat4, sorted_heat, start, end, cent4, alpha3, dt, timing=None):
    """AssignDensity, GradDensity, ParticleGetBaroclinic: (alpha (N, 3),
    rho (dim^3,), grad (dim^3, 3)); the kernels' milliseconds appended to the
    list timing when given."""
    cent = np.ascontiguousarray(cent4, dtype=np.float32)
    N = len(cent)
    al = _soa(alpha3, N)
    c = dim ** 3
    rho = np.zeros(c, np.float32)
    grad = np.zeros(3 * c, np.float32)
    hp = np.ascontiguousarray(sorted_heat4, dtype=np.float32)
    ms = np.zeros(1, np.float32)
    _check(lib().refgpu_baroclinic(dim, float(h), C.c_float(h_f), np.ascontiguousarray(origin, dtype=np.float64),
                                   len(hp), hp, np.ascontiguousarray(sorted_heat, dtype=np.float32),
                                   np.ascontiguousarray(start, dtype=np.uint32),
                                   np.ascontiguousarray(end, dtype=np.uint32), N, cent, al, float(dt), rho, grad, ms),
           "refgpu_baroclinic")
    if timing is not None:
        timing.append(float(ms[0]))
    return al.T.copy(), rho, grad.reshape(3, c).T.copy()


def potential(n, K, sorted_pos4, sorted_mass, mass, start, end, phi, origin, h_f, L, eval4, scalar=False,
              normals=None, areas=None):
    """PotentialFieldSolver's stages with the reference's kernels and the
    given phi: dict of density, rhs (n^3), far (n^3 or (n^3, 3)), out (M or
    (M, 3)), stage_ms (density + RHS, far-field buffer, evaluation) and, with
    normals and areas, dphidn (M)."""
    pos = np.ascontiguousarray(sorted_pos4, dtype=np.float32)
    ev = np.ascontiguousarray(eval4, dtype=np.float32)
    N, M, Cn = len(pos), len(ev), n ** 3
    out = {"density": np.zeros(Cn), "rhs": np.zeros(Cn), "far": np.zeros(3 * Cn), "out": np.zeros(3 * M)}
    nrm = ar = dp = None
    if normals is not None:
        nrm = np.ascontiguousarray(np.asarray(normals, dtype=np.float64).reshape(M, 3))
        ar = np.ascontiguousarray(areas, dtype=np.float64)
        dp = np.zeros(M)
    ptr = lambda a: None if a is None else a.ctypes.data
    ms = np.zeros(3, np.float32)
    _check(lib().refgpu_potential(n, K, N, pos, np.ascontiguousarray(sorted_mass, dtype=np.float64),
                                  np.ascontiguousarray(mass, dtype=np.float64),
                                  np.ascontiguousarray(start, dtype=np.uint32),
                                  np.ascontiguousarray(end, dtype=np.uint32),
                                  np.ascontiguousarray(phi, dtype=np.float64),
                                  np.ascontiguousarray(origin, dtype=np.float64), C.c_float(h_f), float(L), M, ev,
                                  int(bool(scalar)), ptr(nrm), ptr(ar), out["density"], out["rhs"], out["far"],
                                  out["out"], ptr(dp), ms), "refgpu_potential")
    out["stage_ms"] = dict(zip(("density", "far_field", "evaluation"), ms.tolist()))
    if scalar:
        out["far"] = out["far"][:Cn]
        out["out"] = out["out"][:M]
    else:
        out["far"] = out["far"].reshape(3, Cn).T.copy()
        out["out"] = out["out"].reshape(3, M).T.copy()
    if dp is not None:
        out["dphidn"] = dp
    return out


def mg_fmg(n, b, timing=None, repeats=1):
    """The reference's FP64 full multigrid (its own kernels, its V(4,4) / FMG
    schedule and its racing coarsest solve) from x = 0 for each right-hand side
    b[c] (shape (comps, n^3), FP64), repeated `repeats` times from the x the
    previous call left; returns x of the same shape.  timing (a dict, optional)
    receives "ms": the summed device time of its launches."""
    b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, n ** 3)
    x = np.zeros_like(b)
    ms = np.zeros(1, np.float32)
    _check(lib().refgpu_mg_fmg(n, b.shape[0], repeats, b, x, ms.ctypes.data if timing is not None else None),
           "refgpu_mg_fmg")
    if timing is not None:
        timing["ms"] = float(ms[0])
    return x
