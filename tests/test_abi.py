"""The C-ABI library loads and exports every symbol include/pppm.h declares;
the host mirror refuses to run without a GPU (no CPU fallback).  CPU only."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(pppm_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    from pppm_vortex_bouyant_flow_sample_b200 import _build, _lib
    _build.build()
    lib = ctypes.CDLL(_build.LIB)
    declared = _declared()
    assert declared, "no declarations found"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, f"missing exports: {missing}"
    assert set(_lib.EXPORTED) == declared


def test_params_default_and_validation_without_gpu():
    import pppm_vortex_bouyant_flow_sample_b200._lib as L
    lib = L.load()
    p = L.default_params(32)
    assert p.K == 1 and abs(p.a - 0.08) < 1e-15 and p.mg_mode == L.MG_REFERENCE
    h = ctypes.c_void_p()
    bad = L.default_params(36)  # 36 -> 18 -> 9 -> 4: odd level above the coarsest
    assert lib.pppm_scene_create(ctypes.byref(bad), 10, 10, None, ctypes.byref(h)) == 1
    assert b"odd edge" in lib.pppm_last_error()
    bad = L.default_params(32, K=9)
    assert lib.pppm_scene_create(ctypes.byref(bad), 10, 10, None, ctypes.byref(h)) == 1


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import pppm_vortex_bouyant_flow_sample_b200 as pb
    with pytest.raises(RuntimeError):
        pb.Scene(32)


def test_version_string():
    import pppm_vortex_bouyant_flow_sample_b200._lib as L
    assert b"sm_100a" in L.load().pppm_version()


def test_every_package_module_imports_without_gpu():
    """Every module of the package imports on a machine without a GPU (the
    GPU is needed only when a solver is created)."""
    import importlib
    for m in ("potential", "render", "replicas", "server", "frames", "workloads", "_lib"):
        importlib.import_module("pppm_vortex_bouyant_flow_sample_b200." + m)


def test_reference_gpu_checker_exports():
    """The reference's own kernels, built as a checker (oracle/_ref), load on
    the host and export the two shim entry points the GPU tests call."""
    import ctypes
    from oracle import pyref_gpu
    if not pyref_gpu.available():
        import pytest
        pytest.skip("oracle/_ref/librefgpu.so not built (the reference's sources were absent)")
    lib = ctypes.CDLL(pyref_gpu._LIB_PATH)
    assert hasattr(lib, "refgpu_farfield_eval") and hasattr(lib, "refgpu_hash")
