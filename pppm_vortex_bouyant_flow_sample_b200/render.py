"""Headless particle splatting renderer (pppm_renderer_* in include/pppm.h).

Mirror of the reference's CPU renderer (Particle_renderer/particle_renderer/
particle_renderer/shadow.cpp compute_shadows, render.cpp render_smoke,
write_sgi.cpp) on the CUDA kernels of csrc/render.cu.  Tensors are device
buffers; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from ._lib import check, load


def _f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


def _dev_f32(t: torch.Tensor, shape_tail, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float32:
        raise ValueError(f"{name} must be a CUDA float32 tensor")
    if tuple(t.shape[1:]) != tuple(shape_tail):
        raise ValueError(f"{name} must have shape (n, {', '.join(map(str, shape_tail))})")
    return t.contiguous()


class Renderer:
    """Shadow pass + smoke pass over particles, on one stream."""

    def __init__(self, stream: torch.cuda.Stream | None = None):
        if not torch.cuda.is_available():
            raise RuntimeError("the renderer needs a CUDA device (sm_100a); there is no CPU path")
        self._lib = load()
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        h = C.c_void_p()
        check(self._lib.pppm_renderer_create(C.c_void_p(self.stream.cuda_stream), C.byref(h)),
              "pppm_renderer_create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pppm_renderer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shadows(self, pos4: torch.Tensor, dens: torch.Tensor, radius: float, opacity: float, light,
                quality: float = 1.0):
        """compute_shadows: returns (illum (n,) float32, shadow map (npix, npix) float32, [j, i])."""
        pos4 = _dev_f32(pos4, (4,), "pos4")
        n = pos4.shape[0]
        dens = dens.contiguous()
        illum = torch.empty(max(n, 1), dtype=torch.float32, device=pos4.device)
        npix = C.c_uint32()
        with torch.cuda.stream(self.stream):
            check(self._lib.pppm_render_shadows(self._h, n, C.c_void_p(pos4.data_ptr()),
                                                C.c_void_p(dens.data_ptr()), float(radius), float(opacity),
                                                _f3(light), float(quality), C.c_void_p(illum.data_ptr()),
                                                C.byref(npix)), "pppm_render_shadows")
            p = C.c_void_p()
            m = C.c_uint32()
            check(self._lib.pppm_render_shadow_map(self._h, C.byref(p), C.byref(m)), "pppm_render_shadow_map")
            k = m.value
            flat = torch.empty(k * k, dtype=torch.float32, device=pos4.device)
            # copy out of the renderer's buffer (it is reused by the next call)
            src = torch.as_tensor(_Dev(p.value, k * k), device=pos4.device)
            flat.copy_(src)
        return illum[:n], flat.reshape(k, k)

    def smoke(self, pos4: torch.Tensor, illum: torch.Tensor, base_rgb: torch.Tensor, lit_rgb: torch.Tensor,
              radius: float, opacity: float, den: torch.Tensor, background, camera, target,
              perspective: float, width: int, height: int) -> torch.Tensor:
        """render_smoke: returns the image as (height, width, 3) float32."""
        pos4 = _dev_f32(pos4, (4,), "pos4")
        n = pos4.shape[0]
        base_rgb = _dev_f32(base_rgb, (3,), "base_rgb")
        lit_rgb = _dev_f32(lit_rgb, (3,), "lit_rgb")
        illum = illum.contiguous()
        den = den.contiguous()
        img = torch.empty((height, width, 3), dtype=torch.float32, device=pos4.device)
        with torch.cuda.stream(self.stream):
            check(self._lib.pppm_render_smoke(self._h, n, C.c_void_p(pos4.data_ptr()),
                                              C.c_void_p(illum.data_ptr()), C.c_void_p(base_rgb.data_ptr()),
                                              C.c_void_p(lit_rgb.data_ptr()), float(radius), float(opacity),
                                              C.c_void_p(den.data_ptr()), _f3(background), _f3(camera),
                                              _f3(target), float(perspective), int(width), int(height),
                                              C.c_void_p(img.data_ptr())), "pppm_render_smoke")
        return img


class _Dev:
    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f4", "data": (ptr, False), "version": 3}


def write_sgi(path: str, image, high_precision: bool = False) -> None:
    """Write an (h, w) or (h, w, 3) float image as an SGI file (write_sgi.cpp)."""
    a = np.ascontiguousarray(np.asarray(image, dtype=np.float32))
    if a.ndim == 2:
        ch = 1
    elif a.ndim == 3 and a.shape[2] == 3:
        ch = 3
    else:
        raise ValueError("image must be (h, w) or (h, w, 3)")
    h, w = a.shape[:2]
    lib = load()
    check(lib.pppm_write_sgi(path.encode(), w, h, ch, a.ctypes.data, int(high_precision)), "pppm_write_sgi")
