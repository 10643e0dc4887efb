"""Frame files of the demo driver (Particle_data%04d.bin, float4 with w = 1),
through the library's native writer and reader (pppm_write_frame /
pppm_read_frame)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import check, load


def frame_path(directory: str, frame: int) -> str:
    buf = C.create_string_buffer(4096)
    check(load().pppm_frame_path(directory.encode(), int(frame), buf, len(buf)), "pppm_frame_path")
    return buf.value.decode()


def write_frame(directory: str, frame: int, pos4) -> str:
    """pos4: (N, 4) float32 numpy array or CUDA tensor."""
    L = load()
    on_dev = hasattr(pos4, "is_cuda") and pos4.is_cuda
    if on_dev:
        ptr, N = pos4.data_ptr(), pos4.shape[0]
    else:
        pos4 = np.ascontiguousarray(pos4, dtype=np.float32)
        ptr, N = pos4.ctypes.data, pos4.shape[0]
    os.makedirs(directory, exist_ok=True)
    check(L.pppm_write_frame(directory.encode(), int(frame), N, C.c_void_p(ptr), int(on_dev)), "pppm_write_frame")
    return frame_path(directory, frame)


def read_frame(path: str) -> np.ndarray:
    L = load()
    n = C.c_uint32()
    check(L.pppm_read_frame(path.encode(), None, 0, C.byref(n)), "pppm_read_frame")
    out = np.empty((n.value, 4), dtype=np.float32)
    check(L.pppm_read_frame(path.encode(), C.c_void_p(out.ctypes.data), n.value, C.byref(n)), "pppm_read_frame")
    return out
