"""Recorded sequences in the reference's on-disk format (CPU): Parameters.txt
as Source/data/ParametersFileFormat.txt lays it out and WriteToFile writes it
(Source/src/CameraSupport/WriteToFile.cpp:32-58), raw `recorded<N>` frames of
W x H native-order uint16, round trips, and the error codes."""
import numpy as np
import pytest

# The layout of ParametersFileFormat.txt:1-11, one item per line, with the
# values of a 640x480 recording.
PARAMETERS_TXT = """640
480
525 525
319.5 239.5
0
300
5000
3
Video/room
2026-12-03-10-00-00
PrimeSense
"""


def test_parameters_file_fields(of, tmp_path):
    (tmp_path / "Parameters.txt").write_text(PARAMETERS_TXT)
    info = of.read_recording_info(tmp_path)
    c = info.camera
    assert (c.width, c.height, c.fx, c.fy, c.cx, c.cy) == (640, 480, 525.0, 525.0, 319.5, 239.5)
    assert (info.z_offset_mm, c.min_depth_mm, c.max_depth_mm, info.frames) == (0.0, 300.0, 5000.0, 3)
    assert (info.name, info.date, info.camera_type) == (b"Video/room", b"2026-12-03-10-00-00",
                                                        b"PrimeSense")


def test_reader_fields_only(of, tmp_path):
    """CameraFromFile reads only the first nine numbers (CameraFromFile.cpp:33-37)."""
    (tmp_path / "Parameters.txt").write_text("320 240\n262.5 262.5\n160 120\n0\n300\n5000\n")
    info = of.read_recording_info(tmp_path)
    assert (info.camera.width, info.camera.height, info.frames) == (320, 240, 0)
    assert info.name == b""


def test_write_read_round_trip(of, tmp_path):
    import dataclasses
    cfg = dataclasses.replace(of.CONFIGS["c1"], width=64, height=48, cx=31.5, cy=23.5)
    rng = np.random.default_rng(5)
    frames = rng.integers(0, 6000, (3, 48, 64)).astype(np.uint16)
    of.write_recording(tmp_path, cfg, frames, name="Video/t", date="2026-12-03", camera_type="Synthetic")
    text = (tmp_path / "Parameters.txt").read_text().splitlines()
    assert text[:8] == ["64", "48", "262.5 262.5", "31.5 23.5", "0", "300", "5000", "3"]
    assert text[8:] == ["Video/t", "2026-12-03", "Synthetic"]
    info = of.read_recording_info(tmp_path)
    assert (info.camera.width, info.camera.height, info.frames) == (64, 48, 3)
    for k in range(3):
        raw = (tmp_path / f"recorded{k + 1}").read_bytes()
        assert raw == frames[k].tobytes()  # W x H uint16, row major, native order
        assert np.array_equal(of.read_recording_frame(tmp_path, k + 1, 64, 48), frames[k])


def test_missing_files_report_io_error(of, tmp_path):
    from openfusion_b200._native import OpenFusionError
    with pytest.raises(OpenFusionError) as e:
        of.read_recording_info(tmp_path / "absent")
    assert e.value.status == 6
    (tmp_path / "Parameters.txt").write_text(PARAMETERS_TXT)
    with pytest.raises(OpenFusionError) as e:
        of.read_recording_frame(tmp_path, 1, 640, 480)
    assert e.value.status == 6
    # a short frame file is an error too
    (tmp_path / "recorded1").write_bytes(b"\\0" * 100)
    with pytest.raises(OpenFusionError):
        of.read_recording_frame(tmp_path, 1, 640, 480)
