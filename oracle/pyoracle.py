"""ctypes binding of the CPU oracle (oracle/pppm_oracle.cpp) — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
legs load this module; the product path never does.  Arrays are numpy; float4
positions are (N, 4) float32, strengths and velocities are float64.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libpppm_oracle.so")
_lib = None

u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


class OrcParams(C.Structure):
    _fields_ = [
        ("n", C.c_uint32),
        ("K", C.c_int32),
        ("a", C.c_double),
        ("domain_mode", C.c_int32),
        ("fixed_origin", C.c_double * 3),
        ("fixed_length", C.c_double),
        ("mg_mode", C.c_int32),
        ("coarse_mode", C.c_int32),
        ("mg_tol", C.c_double),
        ("mg_max_cycles", C.c_int32),
    ]


class OrcDump(C.Structure):
    _fields_ = [(name, C.c_void_p) for name in (
        "origin", "length", "h_f", "vort_key", "vort_idx", "cell_start", "cell_end",
        "grid_vort", "psi", "grid_u", "far_u", "u_far_only", "pairs", "mg_cycles",
        "mg_relres")]


def build() -> str:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_set_domain.argtypes = [f32p, C.c_uint32, f64p, f64p]
        L.orc_calc_hash.argtypes = [f32p, C.c_uint32, C.c_uint32, C.c_float, f32p, u32p, u32p]
        L.orc_sort_by_key.argtypes = [u32p, u32p, C.c_uint32]
        L.orc_find_cell_start.argtypes = [u32p, C.c_uint32, C.c_uint32, u32p, u32p]
        L.orc_p2m.argtypes = [u32p, u32p, f32p, f64p, C.c_double, C.c_uint32, C.c_uint32, f64p, f64p]
        L.orc_mg_levels.argtypes = [C.c_uint32]
        L.orc_mg_levels.restype = C.c_int
        L.orc_mg_solve.argtypes = [f64p, f64p, C.c_uint32, C.c_int, C.c_int, C.c_double, C.c_int,
                                   i32p, f64p]
        L.orc_mg_vcycle.argtypes = [f64p, f64p, C.c_uint32, C.c_int]
        L.orc_residual_norm.argtypes = [f64p, f64p, C.c_uint32]
        L.orc_residual_norm.restype = C.c_double
        L.orc_apply_laplacian.argtypes = [f64p, f64p, C.c_uint32]
        L.orc_curl.argtypes = [f64p, f64p, C.c_uint32, C.c_double]
        L.orc_farfield_table.argtypes = [C.c_int, C.c_double, f64p]
        L.orc_farfield.argtypes = [f64p, f64p, f64p, C.c_uint32, C.c_int, C.c_double]
        L.orc_interp.argtypes = [f32p, C.c_uint32, f64p, C.c_uint32, C.c_double, f64p, f64p]
        L.orc_pp.argtypes = [u32p, u32p, f32p, f32p, C.c_int, f32p, f64p, f64p, C.c_uint32,
                             C.c_double, C.c_int, C.c_uint32, C.c_uint32, f64p, C.c_double]
        L.orc_pp.restype = C.c_uint64
        L.orc_pppm.argtypes = [C.POINTER(OrcParams), C.c_uint32, f32p, f64p, f64p, f64p,
                               C.c_uint32, f32p, f32p, C.c_int, f64p, f64p, f64p,
                               C.POINTER(OrcDump)]
        L.orc_pppm.restype = C.c_int
        L.orc_direct_sum.argtypes = [C.c_uint32, f32p, f64p, f64p, f64p, C.c_uint32, f32p, f32p,
                                     C.c_int, C.c_double, f64p, f64p, f64p]
        L.orc_num_threads.restype = C.c_int
        L.orc_vortex_step.argtypes = [C.POINTER(OrcParams), C.c_uint32, f32p, f64p, f64p, f64p, C.c_double,
                                      C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_vortex_step.restype = C.c_int
        L.orc_gaussian_smooth.argtypes = [C.POINTER(OrcParams), C.c_uint32, f32p, f64p, f64p, f64p, C.c_double,
                                          f64p, f64p, f64p]
        L.orc_gaussian_smooth.restype = None
        L.orc_baroclinic.argtypes = [C.c_uint32, f32p, f32p, C.c_uint32, f32p, f64p, f64p, f64p, C.c_double,
                                     f64p, f64p, C.c_void_p, C.c_void_p, C.c_size_t]
        L.orc_baroclinic.restype = C.c_uint32
        L.orc_potential.argtypes = [C.c_uint32, C.c_int, C.c_int, C.c_uint32, f32p, f64p, C.c_uint32, f32p, f64p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_potential.restype = C.c_int
        L.orc_mg_fmg.argtypes = [f64p, f64p, C.c_uint32, C.c_int, C.c_int]
        L.orc_mg_fmg.restype = None
        L.orc_density_domain.argtypes = [f32p, C.c_uint32, f64p, f64p]
        L.orc_density_domain.restype = None
        _lib = L
    return _lib


def params(n, K=1, a=0.08, domain_mode=0, fixed_origin=(0.0, 0.0, 0.0), fixed_length=1.0,
           mg_mode=0, coarse_mode=1, mg_tol=1e-10, mg_max_cycles=50) -> OrcParams:
    p = OrcParams()
    p.n, p.K, p.a, p.domain_mode = n, K, a, domain_mode
    p.fixed_origin[:] = list(fixed_origin)
    p.fixed_length = fixed_length
    p.mg_mode, p.coarse_mode, p.mg_tol, p.mg_max_cycles = mg_mode, coarse_mode, mg_tol, mg_max_cycles
    return p


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def set_domain(pos4):
    pos4 = _c(pos4, np.float32)
    o = np.zeros(3); L = np.zeros(1)
    lib().orc_set_domain(pos4, pos4.shape[0], o, L)
    return o, float(L[0])


def hash_params(origin, length, n):
    """(h_f, origin_f) exactly as PH/SpaceHashClass.h:46-54 stores them."""
    h_f = np.float32(length / float(n))
    return h_f, np.asarray(origin, dtype=np.float64).astype(np.float32)


def calc_hash(pos4, n, h_f, origin_f):
    pos4 = _c(pos4, np.float32)
    N = pos4.shape[0]
    key = np.zeros(N, np.uint32); idx = np.zeros(N, np.uint32)
    lib().orc_calc_hash(pos4, N, n, float(h_f), _c(origin_f, np.float32), key, idx)
    return key, idx


def sort_by_key(key, idx):
    key = key.copy(); idx = idx.copy()
    lib().orc_sort_by_key(key, idx, key.shape[0])
    return key, idx


def find_cell_start(skey, ncells):
    skey = _c(skey, np.uint32)
    s = np.zeros(ncells, np.uint32); e = np.zeros(ncells, np.uint32)
    lib().orc_find_cell_start(skey, skey.shape[0], ncells, s, e)
    return s, e


def mg_levels(n):
    return lib().orc_mg_levels(n)


def mg_solve(b, n, mg_mode=0, coarse_mode=1, tol=1e-10, max_cycles=50):
    b = _c(b, np.float64).ravel()
    x = np.zeros_like(b)
    cyc = np.zeros(1, np.int32); rr = np.zeros(1)
    lib().orc_mg_solve(x, b, n, mg_mode, coarse_mode, tol, max_cycles, cyc, rr)
    return x, int(cyc[0]), float(rr[0])


def mg_vcycle(x, b, n, coarse_mode=1):
    x = _c(x, np.float64).ravel().copy()
    lib().orc_mg_vcycle(x, _c(b, np.float64).ravel(), n, coarse_mode)
    return x


def apply_laplacian(x, n):
    x = _c(x, np.float64).ravel()
    y = np.zeros_like(x)
    lib().orc_apply_laplacian(x, y, n)
    return y


def residual_norm(x, b, n):
    return lib().orc_residual_norm(_c(x, np.float64).ravel(), _c(b, np.float64).ravel(), n)


def curl(psi3, n, h):
    psi3 = _c(psi3, np.float64).ravel()
    u = np.zeros_like(psi3)
    lib().orc_curl(psi3, u, n, h)
    return u.reshape(3, -1)


def farfield_table(K, h):
    W = 2 * K + 1
    t = np.zeros(W * W * W * 3)
    lib().orc_farfield_table(K, h, t)
    return t.reshape(W, W, W, 3)


def farfield(vort3, u3, n, K, h):
    vort3 = _c(vort3, np.float64).ravel(); u3 = _c(u3, np.float64).ravel()
    far = np.zeros_like(u3)
    lib().orc_farfield(vort3, u3, far, n, K, h)
    return far.reshape(3, -1)


def pppm(prm: OrcParams, vort_pos4, alpha3, eval_a4, eval_b4=None, is_segment=0, dump=False):
    """Whole path.  Returns (u (M,3) float64, dump dict or None)."""
    vp = _c(vort_pos4, np.float32)
    al = _c(alpha3, np.float64)
    N = vp.shape[0]
    ea = _c(eval_a4, np.float32)
    M = ea.shape[0]
    eb = _c(eval_b4 if eval_b4 is not None else np.zeros_like(ea), np.float32)
    u = np.zeros(M); v = np.zeros(M); w = np.zeros(M)
    d = None
    D = OrcDump()
    if dump:
        n = prm.n; Cn = n ** 3
        d = dict(origin=np.zeros(3), length=np.zeros(1), h_f=np.zeros(1, np.float32),
                 vort_key=np.zeros(N, np.uint32), vort_idx=np.zeros(N, np.uint32),
                 cell_start=np.zeros(Cn, np.uint32), cell_end=np.zeros(Cn, np.uint32),
                 grid_vort=np.zeros(3 * Cn), psi=np.zeros(3 * Cn), grid_u=np.zeros(3 * Cn),
                 far_u=np.zeros(3 * Cn), u_far_only=np.zeros(3 * M),
                 pairs=np.zeros(1, np.uint64), mg_cycles=np.zeros(3, np.int32),
                 mg_relres=np.zeros(3))
        for k, arr in d.items():
            setattr(D, k, arr.ctypes.data)
    rc = lib().orc_pppm(C.byref(prm), N, vp, _c(al[:, 0], np.float64), _c(al[:, 1], np.float64),
                        _c(al[:, 2], np.float64), M, ea, eb, int(is_segment), u, v, w,
                        C.byref(D) if dump else None)
    if rc != 0:
        raise RuntimeError(f"orc_pppm failed ({rc})")
    if d is not None:
        for k in ("grid_vort", "psi", "grid_u", "far_u", "u_far_only"):
            d[k] = d[k].reshape(3, -1)
    return np.stack([u, v, w], axis=1), d


def direct_sum(vort_pos4, alpha3, eval_a4, a, eval_b4=None, is_segment=0):
    vp = _c(vort_pos4, np.float32)
    al = _c(alpha3, np.float64)
    ea = _c(eval_a4, np.float32)
    eb = _c(eval_b4 if eval_b4 is not None else np.zeros_like(ea), np.float32)
    M = ea.shape[0]
    u = np.zeros(M); v = np.zeros(M); w = np.zeros(M)
    lib().orc_direct_sum(vp.shape[0], vp, _c(al[:, 0], np.float64), _c(al[:, 1], np.float64),
                         _c(al[:, 2], np.float64), M, ea, eb, int(is_segment), float(a), u, v, w)
    return np.stack([u, v, w], axis=1)


def vortex_step(prm: OrcParams, cent4, alpha3, dt, h_seg=0.1, nu=0.1, passive4=None):
    """One reference time step; returns (cent4, alpha (N,3), enda4, endb4), plus
    (passive4 moved, passive velocity (P,3)) when passive points are given."""
    cent = np.array(cent4, dtype=np.float32, order="C", copy=True)
    al = np.ascontiguousarray(alpha3, dtype=np.float64)
    vx, vy, vz = (np.ascontiguousarray(al[:, c]) for c in range(3))
    N = cent.shape[0]
    ea = np.zeros((N, 4), np.float32)
    eb = np.zeros((N, 4), np.float32)
    P = 0 if passive4 is None else len(passive4)
    pas = np.array(passive4, dtype=np.float32, order="C", copy=True) if P else np.zeros((1, 4), np.float32)
    pvel = [np.zeros(max(P, 1)) for _ in range(3)]
    rc = lib().orc_vortex_step(C.byref(prm), N, cent, vx, vy, vz, float(dt), float(h_seg), float(nu),
                               ea.ctypes.data, eb.ctypes.data, P, pas.ctypes.data,
                               *(v.ctypes.data for v in pvel))
    if rc != 0:
        raise RuntimeError("orc_vortex_step failed")
    out = (cent, np.stack([vx, vy, vz], axis=1), ea, eb)
    if P:
        out = out + (pas, np.stack(pvel, axis=1))
    return out


def baroclinic(heat4, life, cent4, alpha3, dt, cap=0):
    """addBaroclinicForce; returns (alpha (N,3), dim, origin, h, rho, grad) (grids when dim^3 <= cap)."""
    heat = np.ascontiguousarray(heat4, dtype=np.float32)
    lf = np.ascontiguousarray(life, dtype=np.float32)
    cent = np.ascontiguousarray(cent4, dtype=np.float32)
    al = np.ascontiguousarray(alpha3, dtype=np.float64)
    vx, vy, vz = (np.ascontiguousarray(al[:, c]) for c in range(3))
    o = np.zeros(3); h = np.zeros(1)
    rho = np.zeros(max(cap, 1), np.float32)
    grad = np.zeros(3 * max(cap, 1), np.float32)
    dim = lib().orc_baroclinic(len(heat), heat, lf, len(cent), cent, vx, vy, vz, float(dt), o, h,
                               rho.ctypes.data, grad.ctypes.data, cap)
    c = dim ** 3
    g = (rho[:c].copy(), grad[:3 * c].reshape(c, 3).copy()) if dim and c <= cap else (None, None)
    return np.stack([vx, vy, vz], axis=1), dim, o, float(h[0]), g[0], g[1]


def gaussian_smooth(prm: OrcParams, cent4, d3, nu=0.1):
    """Hash of cent4 + Gaussian-weighted mean of d3 (N, 3) over 5^3 cells; returns (N, 3)."""
    cent = np.ascontiguousarray(cent4, dtype=np.float32)
    d = np.ascontiguousarray(d3, dtype=np.float64)
    dx, dy, dz = (np.ascontiguousarray(d[:, c]) for c in range(3))
    N = cent.shape[0]
    out = [np.zeros(N) for _ in range(3)]
    lib().orc_gaussian_smooth(C.byref(prm), N, cent, dx, dy, dz, float(nu), *out)
    return np.stack(out, axis=1)


def mg_fmg(x0, b, n, repeats=1, coarse_mode=1):
    """m_FullMultiGrid called `repeats` times from x0."""
    x = np.array(x0, dtype=np.float64, copy=True)
    lib().orc_mg_fmg(x, np.ascontiguousarray(b, dtype=np.float64), n, repeats, coarse_mode)
    return x


def potential(n, K, pos4, mass, eval4, scalar=False, dump=False):
    """PotentialFieldSolver: gradient (M, 3) or scalar potential (M,) at eval4;
    with dump, also a dict of the intermediate grids."""
    pos = np.ascontiguousarray(pos4, dtype=np.float32)
    m = np.ascontiguousarray(mass, dtype=np.float64)
    ev = np.ascontiguousarray(eval4, dtype=np.float32)
    M = len(ev)
    C3 = n ** 3
    out = np.zeros(M if scalar else 3 * M)
    d = {}
    if dump:
        d = {"origin": np.zeros(4), "density": np.zeros(C3), "rhs": np.zeros(C3), "phi": np.zeros(C3),
             "far": np.zeros(C3 if scalar else 3 * C3), "monopole": np.zeros(4)}
    ptr = (lambda k: d[k].ctypes.data) if dump else (lambda k: None)
    rc = lib().orc_potential(n, K, int(scalar), len(pos), pos, m, M, ev, out, ptr("origin"), ptr("density"),
                             ptr("rhs"), ptr("phi"), ptr("far"), ptr("monopole"))
    if rc != 0:
        raise RuntimeError("orc_potential failed")
    res = out if scalar else out.reshape(3, M).T.copy()
    return (res, d) if dump else res


def num_threads():
    return lib().orc_num_threads()
