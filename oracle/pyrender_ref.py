"""ctypes bindings of oracle/_ref/librender_ref.so: the reference's own CPU
renderer (Particle_renderer/.../shadow.cpp, render.cpp, write_sgi.cpp),
compiled from its sources by `make -C oracle ref`.  TEST INFRASTRUCTURE ONLY:
tests and the bench's CPU baseline call it as the checker; the product never
does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "librender_ref.so")
_lib = None
f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


def available() -> bool:
    return os.path.exists(_LIB_PATH)


def build() -> bool:
    """Compile the reference renderer when its sources are present; True if the library exists."""
    from oracle.refroot import reference_root
    src = reference_root()
    if src:
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF_ROOT={src}"], check=True)
    return available()


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/librender_ref.so is missing (make -C oracle ref)")
        L = C.CDLL(_LIB_PATH)
        L.ref_compute_shadows.argtypes = [C.c_int, f32p, C.c_float, C.c_float, f32p, f32p, C.c_float, f32p,
                                          C.POINTER(C.c_int), f32p, C.c_long]
        L.ref_compute_shadows.restype = C.c_int
        L.ref_render_smoke.argtypes = [C.c_int, f32p, f32p, f32p, f32p, C.c_float, C.c_float, f32p, f32p, f32p,
                                       f32p, f32p, C.c_float, C.c_int, C.c_int, f32p]
        L.ref_render_smoke.restype = None
        L.ref_write_sgi.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, f32p, C.c_int]
        L.ref_write_sgi.restype = C.c_int
        _lib = L
    return _lib


class _quiet_stdout:
    """The reference renderer prints progress with printf; send the process's
    fd 1 to /dev/null around its calls so callers' stdout stays clean."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        C.CDLL(None).fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False


def _v3(v):
    return np.asarray(v, dtype=np.float32).reshape(3).copy()


def compute_shadows(xyz, radius, opacity, dens, light, quality=1.0, cap=4096 * 4096):
    """Returns (ok, illum (n,), shadow map (npix, npix) [j, i])."""
    x = np.ascontiguousarray(np.asarray(xyz, dtype=np.float32)[:, :3])
    n = len(x)
    d = np.ascontiguousarray(dens, dtype=np.float32)
    illum = np.zeros(max(n, 1), np.float32)
    npix = C.c_int(0)
    sm = np.zeros(cap, np.float32)
    with _quiet_stdout():
        ok = lib().ref_compute_shadows(n, x, float(radius), float(opacity), d, _v3(light), float(quality), illum,
                                       C.byref(npix), sm, cap)
    k = npix.value
    return bool(ok), illum[:n], sm[:k * k].reshape(k, k)


def render_smoke(xyz, illum, base_rgb, lit_rgb, radius, opacity, den, light, background, camera, target,
                 perspective, width, height):
    """Returns the image as (height, width, 3) float32."""
    x = np.ascontiguousarray(np.asarray(xyz, dtype=np.float32)[:, :3])
    img = np.zeros((height, width, 3), np.float32)
    with _quiet_stdout():
        lib().ref_render_smoke(len(x), x, np.ascontiguousarray(illum, dtype=np.float32),
                               np.ascontiguousarray(base_rgb, dtype=np.float32),
                               np.ascontiguousarray(lit_rgb, dtype=np.float32), float(radius), float(opacity),
                               np.ascontiguousarray(den, dtype=np.float32), _v3(light), _v3(background),
                               _v3(camera), _v3(target), float(perspective), int(width), int(height), img)
    return img


def write_sgi(path, image, high_precision=False) -> bool:
    a = np.ascontiguousarray(np.asarray(image, dtype=np.float32))
    ch = 1 if a.ndim == 2 else 3
    h, w = a.shape[:2]
    return bool(lib().ref_write_sgi(path.encode(), w, h, ch, a.reshape(-1), int(high_precision)))
