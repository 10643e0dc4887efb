"""SGI image writer (CPU): byte-for-byte against the reference's own
write_sgi (Particle_renderer/.../write_sgi.cpp, built into oracle/_ref)."""
import os

import numpy as np
import pytest


def _ours(tmp_path, img, hp):
    from pppm_vortex_bouyant_flow_sample_b200.render import write_sgi
    p = os.path.join(tmp_path, f"ours_{img.ndim}_{int(hp)}.sgi")
    write_sgi(p, img, high_precision=hp)
    return open(p, "rb").read()


def test_sgi_header_layout(tmp_path):
    img = np.zeros((3, 5), np.float32)
    b = _ours(str(tmp_path), img, False)
    assert len(b) == 512 + 15
    assert b[:2] == (474).to_bytes(2, "big") and b[2] == 0 and b[3] == 1
    assert int.from_bytes(b[4:6], "big") == 2                                  # dimension
    assert [int.from_bytes(b[k:k + 2], "big") for k in (6, 8, 10)] == [5, 3, 1]
    assert int.from_bytes(b[16:20], "big") == 255 and not any(b[20:512])


@pytest.mark.parametrize("rgb", [False, True])
@pytest.mark.parametrize("hp", [False, True])
def test_sgi_matches_reference_writer(tmp_path, rgb, hp):
    from oracle import pyrender_ref as R
    if not R.available():
        pytest.skip("reference renderer not built (make -C oracle ref)")
    rng = np.random.default_rng(3)
    shape = (37, 53, 3) if rgb else (37, 53)
    img = rng.uniform(-0.2, 1.3, shape).astype(np.float32)   # exercises both clamps
    ours = _ours(str(tmp_path), img, hp)
    p = os.path.join(str(tmp_path), "ref.sgi")
    assert R.write_sgi(p, img, hp)
    assert ours == open(p, "rb").read()
