"""Recorded frames in the reference's file format (NuiFileIOUtilities.cpp, NuiFrameLoader.cpp),
read and written by the library and checked against a restatement of the format
(oracle/frame_format.py)."""
import os

import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import frame_format as F

from _util import frames


@pytest.fixture(scope="module")
def seq():
    return frames(3, W=320, H=240, seed=21, color=True)


@pytest.mark.parametrize("compressed", [False, True])
def test_library_writer_matches_the_format(tmp_path, seq, compressed):
    d, c, _, _ = seq[0]
    p = str(tmp_path / "0.depth").encode()
    L.check(L.lib().nui_frame_file_write(p, int(compressed), 123456789, 320, 240, L.ptr(d), 2))
    ts, got, stored = F.read_frame(p.decode(), np.uint16)
    assert ts == 123456789 and np.array_equal(got, d)
    assert (stored < d.nbytes) if compressed else (stored == d.nbytes)
    pc = str(tmp_path / "0.color").encode()
    cc = np.ascontiguousarray(c)
    L.check(L.lib().nui_frame_file_write(pc, int(compressed), 7, 320, 240, L.ptr(cc), 4))
    ts, got, _ = F.read_frame(pc.decode(), np.uint8, 4)
    assert ts == 7 and np.array_equal(got, cc)


@pytest.mark.parametrize("compressed", [False, True])
def test_library_reads_format_files(tmp_path, seq, compressed):
    d, c, _, _ = seq[1]
    p = str(tmp_path / "x.depth")
    F.write_frame(p, d, -5, compressed)
    import ctypes as C
    ts, w, h = C.c_int64(), C.c_uint32(), C.c_uint32()
    L.check(L.lib().nui_frame_file_header(p.encode(), C.byref(ts), C.byref(w), C.byref(h)))
    assert (ts.value, w.value, h.value) == (-5, 320, 240)
    out = np.zeros_like(d)
    L.check(L.lib().nui_frame_file_read(p.encode(), L.ptr(out), d.nbytes))
    assert np.array_equal(out, d)
    F.write_camera(str(tmp_path / "c.camIntri"), 262.5, 262.5, 159.5, 119.5)
    cam = np.zeros(4, np.float32)
    L.check(L.lib().nui_camera_file_read(str(tmp_path / "c.camIntri").encode(), L.ptr(cam)))
    assert np.array_equal(cam, np.float32([262.5, 262.5, 159.5, 119.5]))


def test_recording_round_trip_and_end(tmp_path, seq):
    rec = str(tmp_path / "rec")
    L.write_recording(rec, [(d, c) for d, c, _, _ in seq], (262.5, 262.5, 159.5, 119.5), compressed=True)
    assert sorted(os.listdir(rec))[:3] == ["0.camIntri", "0.color", "0.depth"]
    got = L.read_recording(rec, 320, 240)
    assert len(got) == len(seq)
    for (d, c, _, _), (gd, gc, cam, ts) in zip(seq, got):
        assert np.array_equal(gd, d) and np.array_equal(gc, c)
        assert np.array_equal(cam, np.float32([262.5, 262.5, 159.5, 119.5]))
    # the reference's loader reads the same files
    ts, d0, _ = F.read_frame(os.path.join(rec, "1.depth"), np.uint16)
    assert np.array_equal(d0, seq[1][0]) and ts == 33333
    # a frame of another size is refused
    bad = np.zeros((10, 10), np.uint16)
    F.write_frame(os.path.join(rec, "3.depth"), bad, 0, False)
    d = np.zeros((240, 320), np.uint16)
    assert L.lib().nui_recording_frame(rec.encode(), 3, L.ptr(d), None, None, None, 320, 240) == L.NUI_ERR_INVALID_ARG
    assert L.lib().nui_recording_frame(rec.encode(), 9, L.ptr(d), None, None, None, 320, 240) == L.NUI_ERR_INVALID_ARG


@pytest.mark.gpu
def test_recorded_session_tracks_like_the_live_one(gpu_ctx, tmp_path, seq):
    from _util import cfg_for
    rec = str(tmp_path / "rec")
    L.write_recording(rec, [(d, c) for d, c, _, _ in seq], (262.5, 262.5, 159.5, 119.5))
    cfg = cfg_for(W=320, H=240, res=(96, 96, 96))
    a, b = L.Session(gpu_ctx, cfg), L.Session(gpu_ctx, cfg)
    for (d, _, _, _), (rd, _, _, _) in zip(seq, L.read_recording(rec, 320, 240, color=False)):
        assert np.array_equal(a.process(d)[1], b.process(rd)[1])
