"""Frames that lose tracking.  A first frame of a flat wall facing the camera gives reference
normals that are exactly (0, 0, -1), so the next frames' ICP systems have zero rows (no
rotation about the optical axis or translation across it is observable) and every later
frame is lost, as the oracle's (NuiKinfuOpenCLDepthTracker.cpp:324-496: the determinant
test) says.  A lost frame leaves the session on the frame before it
(NuiKinfuTrackingEngine.cpp:68-142: no integration, no raycast), the session's frame count
stays, a reset starts it over, and the serving loop -- which launches a batch before it
reads the previous batch's results -- returns what the per-session calls return, for lost
and tracking streams in the same batches."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import cfg_for, cfg_hash, frames

pytestmark = pytest.mark.gpu

W, H = 320, 240


def _wall():
    return np.full((H, W), 1500, np.uint16)


def test_lost_frames_leave_the_session_on_the_frame_before(gpu_ctx):
    cfg = cfg_for(W=W, H=H, res=(64, 64, 64))
    wall = _wall()
    eng = O.Engine(cfg)
    s = L.Session(gpu_ctx, cfg)
    first = L.Session(gpu_ctx, cfg)
    ok0, _ = first.process(wall)
    assert ok0
    got = []
    for k in range(4):
        ok, pose = s.process(wall)
        got.append(ok)
        assert ok == eng.frame(wall), k
        R, t = eng.pose()
        assert np.array_equal(pose[:9].reshape(3, 3), R) and np.array_equal(pose[9:], t), k
    assert got == [True, False, False, False]
    # the lost frames changed neither the volume nor the frame count: a frame-0 volume
    assert np.array_equal(s.volume_ref_layout(), first.volume_ref_layout())
    assert np.array_equal(s.volume_ref_layout().reshape(-1), eng.volume().reshape(-1))
    # a reset starts the session over: a scene then tracks as in a new session
    s.reset()
    fresh = L.Session(gpu_ctx, cfg)
    for d, _, _, _ in frames(4, W=W, H=H, seed=3):
        a, pa = s.process(d)
        b, pb = fresh.process(d)
        assert a and b and np.array_equal(pa, pb)
    for x in (s, first, fresh):
        x.close()


def test_served_batches_with_lost_streams_match_the_session_calls(gpu_ctx):
    wall = _wall()
    scene = [d for d, _, _, _ in frames(5, W=W, H=H, seed=3)]
    streams = [
        (cfg_for(W=W, H=H, res=(64, 64, 64)), [wall] * 5),                       # lost from frame 1
        (cfg_for(W=W, H=H, res=(96, 96, 96), fmt=L.TSDF_F16_U8), scene),        # tracks
        (cfg_hash(W=W, H=H), [wall] * 5),                                       # lost from frame 1
        (cfg_hash(W=W, H=H), scene),                                            # tracks
    ]
    alone = []
    for cfg, seq in streams:
        s = L.Session(gpu_ctx, cfg)
        alone.append([s.process(d) for d in seq])
        s.close()
    assert [ok for ok, _ in alone[0]] == [True] + [False] * 4
    assert [ok for ok, _ in alone[2]] == [True] + [False] * 4
    assert all(ok for ok, _ in alone[1]) and all(ok for ok, _ in alone[3])
    srv = L.Server(gpu_ctx, 60 << 30, max_streams=4)
    slots = [srv.admit(cfg) for cfg, _ in streams]
    assert all(sl is not None for sl in slots)
    got = {k: {} for k in range(len(streams))}
    for f in range(5):  # one frame of every stream a step: each batch holds all four
        for k, (cfg, seq) in enumerate(streams):
            srv.submit(slots[k], seq[f], None, tag=f)
        srv.step()
        for r in srv.poll():
            got[slots.index(r.slot)][r.tag] = r
    srv.drain()
    for r in srv.poll():
        got[slots.index(r.slot)][r.tag] = r
    for k in range(len(streams)):
        for f, (ok, pose) in enumerate(alone[k]):
            r = got[k][f]
            assert r.status == (L.NUI_OK if ok else L.NUI_ERR_TRACKING_LOST), (k, f)
            assert np.array_equal(np.array(r.pose, np.float32), pose), (k, f)
    srv.close()
