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


@pytest.mark.parametrize("kw,why", [
    (dict(n=3), b"outside [4, 512]"),
    (dict(n=513), b"outside [4, 512]"),
    (dict(n=100), b"odd edge"),              # 100 -> 50 -> 25: odd level above the coarsest
    (dict(n=32, K=-2), b"K=-2"),
    (dict(n=32, K=5), b"K=5"),
    (dict(n=32, a=0.0), b"smoothing radius"),
    (dict(n=32, a=float("nan")), b"smoothing radius"),
    (dict(n=32, domain_mode=7), b"domain_mode"),
    (dict(n=32, domain_mode=1, fixed_length=0.0), b"fixed_length"),
    (dict(n=32, domain_mode=1, fixed_length=float("inf")), b"fixed_length"),
    (dict(n=32, mg_mode=9), b"mg_mode"),
    (dict(n=32, mg_mode=1, mg_max_cycles=0), b"CONVERGED"),
    (dict(n=32, mg_mode=1, mg_tol=0.0), b"CONVERGED"),
])
def test_scene_parameters_refused_before_any_allocation(kw, why):
    """Every invalid parameter set is refused with PPPM_ERR_INVALID and a
    message, before the library touches a device (so it runs on CPU)."""
    import pppm_vortex_bouyant_flow_sample_b200._lib as L
    lib = L.load()
    n = kw.pop("n")
    p = L.default_params(n, **kw)
    h = ctypes.c_void_p()
    assert lib.pppm_scene_create(ctypes.byref(p), 10, 10, None, ctypes.byref(h)) == 1
    assert h.value is None
    assert why in lib.pppm_last_error()


def test_null_handles_and_arguments_refused():
    """NULL scenes and output pointers give PPPM_ERR_INVALID, not a crash."""
    import pppm_vortex_bouyant_flow_sample_b200._lib as L
    lib = L.load()
    vp = ctypes.c_void_p
    assert lib.pppm_scene_create(ctypes.byref(L.default_params(32)), 10, 10, None, None) == 1
    assert lib.pppm_set_vortices(None, 1, vp(8), vp(8), vp(8), vp(8)) == 1
    assert lib.pppm_build_far_field(None) == 1
    assert lib.pppm_eval(None, 1, vp(8), None, 0, vp(8), vp(8), vp(8)) == 1
    assert lib.pppm_get_domain(None, None, None, None) == 1
    h = ctypes.c_void_p()
    assert lib.pppm_potential_create(3, 1, 10, 10, None, ctypes.byref(h)) == 1
    assert lib.pppm_potential_create(32, 9, 10, 10, None, ctypes.byref(h)) == 1
    assert lib.pppm_hasher_create(0, 32, None, ctypes.byref(h)) == 1
    assert lib.pppm_hasher_create(16, 1, None, ctypes.byref(h)) == 1
    assert lib.pppm_mg_create(100, None, ctypes.byref(h)) == 1
    assert lib.pppm_renderer_create(None, None) == 1
    assert lib.pppm_scene_destroy(None) == 0


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
