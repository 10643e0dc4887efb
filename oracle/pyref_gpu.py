"""ctypes bindings of oracle/_ref/librefgpu.so: the reference's own GPU kernels
(hybridFastSummation/GPU_kernel.cu, particle_hash/particle_hash_kernel.cu)
behind ref_gpu/ref_gpu_shim.cu and ref_gpu/ref_hash_shim.cu, built by
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
    src = os.environ.get("PPPM_REFERENCE_ROOT", "/root/reference")
    if os.path.isdir(src):
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


def hash_particles(n, h, origin, pos4):
    """The reference's calcHashD, stable key sort and FindCellStartD for float
    cell size h and float origin.  Returns (sorted keys, sorted indices,
    cellStart, cellEnd, milliseconds); cellEnd holds 0xFFFFFFFF where the
    reference leaves it unwritten (empty cells)."""
    pos = np.ascontiguousarray(pos4, dtype=np.float32)
    N = len(pos)
    Cn = n ** 3
    keys = np.zeros(N, np.uint32)
    idx = np.zeros(N, np.uint32)
    start = np.zeros(Cn, np.uint32)
    end = np.full(Cn, 0xFFFFFFFF, np.uint32)
    ms = np.zeros(1, np.float32)
    rc = lib().refgpu_hash(n, C.c_float(h), np.ascontiguousarray(origin, dtype=np.float32), N, pos, keys, idx,
                           start, end, ms)
    if rc != 0:
        raise RuntimeError(f"refgpu_hash: CUDA error {rc}")
    return keys, idx, start, end, float(ms[0])
