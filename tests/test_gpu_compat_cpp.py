"""The C++ classes of include/pppm_compat.hpp (BiotSavartSolver,
ParticleManager, MultiGridSolver3DPeriod_double, PotentialFieldSolver) compiled with g++ into a
driver that calls them with the reference's own call expressions
(getU(c)->getDevicePtr(), getSortPos()->getDevicePtr(), ParticleManager(N),
setSpatialHashGrid(n, h, float3, N), m_Vcycle(x, b, tol, res, 0)), checked
against the oracle: velocities <= 1e-5, hash keys, sorted indices, sorted
positions and strengths and the cell start table bit-exact, and the multigrid
solution (full multigrid, then one more V-cycle) against the oracle's FP64
reference schedule."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _build_driver(tmp):
    from pppm_vortex_bouyant_flow_sample_b200 import _build
    _build.build()
    cuda = os.path.dirname(os.path.dirname(shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"))
    exe = os.path.join(tmp, "compat_driver")
    libdir = os.path.dirname(_build.LIB)
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
           os.path.join(HERE, "compat_driver.cpp"), "-o", exe, "-L", libdir, "-lpppm_b200",
           "-L", os.path.join(cuda, "lib64"), "-lcudart", f"-Wl,-rpath,{libdir}",
           f"-Wl,-rpath,{os.path.join(cuda, 'lib64')}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_compat_classes_match_oracle(tmp_path, oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    n, N = 32, 12000
    pos, al = W.uniform_cloud(N, seed=21)
    exe = _build_driver(str(tmp_path))
    fin, fout = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(fin, "wb") as f:
        np.array([N], np.uint32).tofile(f)
        pos.astype(np.float32).tofile(f)
        np.ascontiguousarray(al.T).tofile(f)
    r = subprocess.run([exe, str(fin), str(fout), str(n)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = open(fout, "rb").read()
    off = 0
    u = np.frombuffer(raw, np.float64, 3 * N, off).reshape(3, N).T; off += 24 * N
    keys = np.frombuffer(raw, np.uint32, N, off); off += 4 * N
    idx = np.frombuffer(raw, np.uint32, N, off); off += 4 * N
    h, ox, oy, oz = np.frombuffer(raw, np.float64, 4, off); off += 32
    x = np.frombuffer(raw, np.float64, n ** 3, off); off += 8 * n ** 3
    grad = np.frombuffer(raw, np.float64, 3 * N, off).reshape(N, 3); off += 24 * N
    xv = np.frombuffer(raw, np.float64, n ** 3, off); off += 8 * n ** 3
    spos = np.frombuffer(raw, np.float32, 4 * N, off).reshape(N, 4); off += 16 * N
    svort = np.frombuffer(raw, np.float64, 3 * N, off).reshape(3, N).T; off += 24 * N
    cstart = np.frombuffer(raw, np.uint32, n ** 3, off); off += 4 * n ** 3
    gsize = np.frombuffer(raw, np.uint32, 3, off)

    ref, d = oracle.pppm(oracle.params(n), pos, al, pos, pos, 1, dump=True)
    assert rel_l2(u, ref) <= 1e-5
    assert h == float(d["h_f"][0]) and (ox, oy, oz) == tuple(d["origin"])
    assert np.array_equal(keys, d["vort_key"]) and np.array_equal(idx, d["vort_idx"])
    q = np.arange(n ** 3, dtype=np.float64)
    bq = np.sin(0.001 * q) - 0.5
    xr, _, _ = oracle.mg_solve(bq, n, mg_mode=0)
    assert rel_l2(x, xr) <= 1e-6
    # one more V(4,4) cycle from the solver's own x: the oracle's cycle from the same x
    assert rel_l2(xv, oracle.mg_vcycle(x, bq, n)) <= 1e-6
    assert rel_l2(xv, xr) > 0.0  # the cycle changed x
    # computeStretching's inputs: sorted positions / strengths and the start table
    order = d["vort_idx"]
    assert np.array_equal(spos[:, :3], pos[order][:, :3])
    assert np.array_equal(svort, al[order])
    assert np.array_equal(cstart, d["cell_start"])
    assert tuple(gsize) == (n, n, n)
    gref = oracle.potential(n, 1, pos, al[:, 0], pos)
    assert rel_l2(grad, gref) <= 1e-5
