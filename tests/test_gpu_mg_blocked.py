"""The temporally blocked smoother (csrc/mg_tb.cu) runs the reference's
red-black half sweeps (MG/Multigrid.cu:202-239) T at a time; every variant
must give the plain half sweeps' multigrid result bit for bit.  The blocked
path serves levels of edge >= 256, so the scene is 256^3.  PPPM_MG_TB forces a
variant (-1: the plain half sweeps, the default) and "auto" runs the
autotuner when a scene is created."""
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _psi(pb, n, pos, al, variant, monkeypatch):
    import torch
    if variant is None:
        monkeypatch.delenv("PPPM_MG_TB", raising=False)
    else:
        monkeypatch.setenv("PPPM_MG_TB", str(variant))
    scene = pb.Scene(n, cap_vort=len(pos), cap_eval=len(pos), a_cells=1.0)
    try:
        scene.set_vortices(torch.from_numpy(pos).cuda(), torch.from_numpy(np.ascontiguousarray(al)).cuda())
        scene.build_far_field()
        return scene.grid(pb.GRID_PSI).cpu().numpy()
    finally:
        scene.close()


def test_every_blocked_variant_matches_the_plain_half_sweeps(monkeypatch):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import pppm_vortex_bouyant_flow_sample_b200 as pb
    from pppm_vortex_bouyant_flow_sample_b200 import workloads as W
    pos, al = W.vortex_ring(1 << 16, seed=7)
    n = 256
    # a scene with the autotuner: its report lists every variant it timed
    _psi(pb, n, pos, al, "auto", monkeypatch)
    report = pb.tuning_report()
    variants = sorted({int(v) for v in re.findall(r"v(\d+)\(", report)})
    assert variants == list(range(len(variants))) and len(variants) >= 4, report
    plain = _psi(pb, n, pos, al, -1, monkeypatch)
    assert np.isfinite(plain).all()
    assert np.array_equal(_psi(pb, n, pos, al, None, monkeypatch), plain)  # the default
    for v in variants:
        got = _psi(pb, n, pos, al, v, monkeypatch)
        assert np.array_equal(got, plain), (v, float(np.abs(got - plain).max()))
