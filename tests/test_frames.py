"""Frame files (Particle_data%04d.bin, hybridFastSummation/newTest.cpp:23-36):
raw float4 records with w forced to 1, round trip through the native writer
and reader.  CPU only (host arrays)."""
import os

import numpy as np


def test_frame_round_trip_and_format(tmp_path):
    from pppm_vortex_bouyant_flow_sample_b200 import frames, workloads as W
    pos, _ = W.vortex_ring(1000, seed=5)
    pos[:, 3] = 7.0
    path = frames.write_frame(str(tmp_path), 12, pos)
    assert os.path.basename(path) == "Particle_data0012.bin"
    raw = np.fromfile(path, dtype=np.float32).reshape(-1, 4)
    assert raw.shape == (1000, 4) and np.all(raw[:, 3] == 1.0)
    assert np.array_equal(raw[:, :3], pos[:, :3])
    back = frames.read_frame(path)
    assert np.array_equal(back, raw)


def test_frame_rejects_truncated_file(tmp_path):
    import pytest
    from pppm_vortex_bouyant_flow_sample_b200 import frames
    from pppm_vortex_bouyant_flow_sample_b200._lib import PppmError
    p = tmp_path / "Particle_data0000.bin"
    p.write_bytes(b"\0" * 20)
    with pytest.raises(PppmError):
        frames.read_frame(str(p))
