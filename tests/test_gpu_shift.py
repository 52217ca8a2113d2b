"""GPU parity of the shifting dense volume (the reference's eScene_ShiftingVolume,
NuiKinfuOpenCLShiftScene) against the oracle, which restates it through the reference's
voxel wrap (and is pinned to the reference's kernels).  The CUDA path keeps the volume
unwrapped and rolls it in memory on a shift; exported in the reference's layout through the
wrap, it must hold the oracle's voxels bit for bit.

At given poses (the step-wise path): after every frame the same offsets, the same shifted
local pose, the same volume and colour volume, the same raycast maps, and in the end the
same set of points fetched from the slabs that left.  Tracked (the batched path, a shifting
session beside a fixed one): the same offsets and poses within 1e-4 rad / 0.1 mm.  The
point cloud of the whole volume equals the oracle's fetch as a set."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import cfg_for, frames, relative_gt, rot_angle, same_bits

pytestmark = pytest.mark.gpu


def _shift_cfg(W=320, H=240, res=(96, 80, 112), fmt=L.TSDF_I16, vs=3, color=True):
    cfg = cfg_for(W=W, H=H, res=res, dim=3.0, fmt=fmt, color=color)
    cfg.voxel_shift = vs
    cfg.shift_point_cap = 1 << 20
    return cfg


def _point_set(xyz, rgba):
    return np.unique(np.concatenate([xyz, rgba], axis=1), axis=0)


@pytest.mark.parametrize("fmt", [L.TSDF_I16, L.TSDF_F16_U8])
def test_shifts_at_given_poses_bit_exact(gpu_ctx, fmt):
    # a room: its walls face the camera, so the slabs that leave hold surface
    seq = frames(10, W=320, H=240, seed=5, deg=1.0, color=True, kind=L.SYNTH_ROOM)
    gt = relative_gt(seq)
    cfg = _shift_cfg(fmt=fmt)
    s = L.Session(gpu_ctx, cfg)
    eng = O.Engine(_shift_cfg())
    cell = np.array([np.float32(3.0) / np.float32(r) for r in cfg.res], np.float32)
    shifted = 0
    for i, (d, c, _, _) in enumerate(seq):
        c = np.ascontiguousarray(c)
        voff, off_m, _ = s.shift_state()
        assert np.array_equal(voff, eng.shift_state()), i
        R, tg = gt[i]
        t = (np.asarray(tg, np.float32) - off_m).astype(np.float32)  # the volume-local pose
        eng.integrate_at(d, R, t, c)
        s.upload(d, c)
        s.set_pose(R, t)
        s.integrate()
        s.raycast()
        voff2 = s.shift_state()[0]
        assert np.array_equal(voff2, eng.shift_state()), i
        shifted += int(np.any(voff2 != voff))
        Rg, tgpu = s.get_pose()
        Ro, to = eng.pose()
        assert np.array_equal(tgpu, to) and np.array_equal(Rg, Ro), i
        vg, vo = s.volume_ref_layout(), eng.volume()
        if fmt == L.TSDF_I16:
            assert np.array_equal(vg, vo), i
            assert np.array_equal(s.download(9), eng.color_volume()), i
        else:  # tolerance-mode integration: the same voxels updated, all but a few
            assert np.mean(vg[:, 1] != vo[:, 1]) <= 1e-4, i
            assert np.mean(np.any(s.download(9) != eng.color_volume(), axis=-1)) <= 1e-4, i
        if fmt == L.TSDF_I16:
            assert same_bits(s.download(3)[..., :3], eng.refmap(0)), i
            assert same_bits(s.download(4)[..., :3], eng.refmap(1)), i
        else:  # the tolerance-mode march over the shifted volume's re-classified bricks
            gv = s.download(3)[..., :3].reshape(-1, 3).astype(np.float64)
            ov = eng.refmap(0).reshape(-1, 3).astype(np.float64)
            hg, ho = ~np.isnan(gv[:, 0]), ~np.isnan(ov[:, 0])
            assert ho.mean() > 0.1 and np.mean(hg != ho) <= 0.02, (i, float(np.mean(hg != ho)))
            dist = np.linalg.norm(gv[hg & ho] - ov[hg & ho], axis=1)
            assert np.quantile(dist, 0.98) <= 5e-4, (i, float(np.quantile(dist, 0.98)))
    assert shifted >= 2
    xg, rg = s.shift_points()
    xo, ro, n = eng.points()
    assert len(xg) > 0 and n > 0
    if fmt == L.TSDF_I16:  # FP16 voxels hold other values: their points differ
        assert len(xg) == n
        assert np.array_equal(_point_set(xg, rg), _point_set(xo, ro))
    s.close()


def test_shifting_session_tracks_like_the_oracle_beside_a_fixed_one(gpu_ctx):
    seq = frames(10, W=320, H=240, seed=5, deg=0.5)
    cfg_s = _shift_cfg(res=(128, 128, 128), color=False)
    cfg_f = cfg_for(W=320, H=240, res=(128, 128, 128), dim=3.0)
    a, b = L.Session(gpu_ctx, cfg_s), L.Session(gpu_ctx, cfg_f)
    ea, eb = O.Engine(cfg_s), O.Engine(cfg_f)
    for i, (d, _, _, _) in enumerate(seq):
        st, poses = gpu_ctx.batch_tick([a, b], [d, d])
        assert np.all(st == L.NUI_OK), i
        assert ea.frame(d) and eb.frame(d), i
        for pose, e in ((poses[0], ea), (poses[1], eb)):
            Ro, to = e.pose()
            assert rot_angle(pose[:9].reshape(3, 3), Ro) < 1e-4, i
            assert np.max(np.abs(pose[9:] - to)) < 1e-4, i
        assert np.array_equal(a.shift_state()[0], ea.shift_state()), i
    assert np.any(ea.shift_state() != 0)
    assert np.all(b.shift_state()[0] == 0)
    a.close()
    b.close()


def test_point_cloud_matches_the_oracle_fetch(gpu_ctx):
    seq = frames(8, W=320, H=240, seed=5, deg=1.0, color=True, kind=L.SYNTH_ROOM)
    gt = relative_gt(seq)
    for vs in (0, 3):
        cfg = _shift_cfg(vs=vs)
        s = L.Session(gpu_ctx, cfg)
        eng = O.Engine(cfg)
        for i, (d, c, _, _) in enumerate(seq):
            c = np.ascontiguousarray(c)
            off_m = s.shift_state()[1]
            R, tg = gt[i]
            t = (np.asarray(tg, np.float32) - off_m).astype(np.float32)
            eng.integrate_at(d, R, t, c)
            s.upload(d, c)
            s.set_pose(R, t)
            s.integrate()
        xg, rg, n = s.point_cloud()
        assert n == len(xg) > 1000
        cap = 1 << 22
        xo, ro = np.zeros((cap, 3), np.float32), np.zeros((cap, 4), np.float32)
        tp = eng.tsdf
        rng = np.ascontiguousarray(cfg.res[:], np.int32)
        zero = np.zeros(3, np.int32)
        voff = np.ascontiguousarray(eng.shift_state(), np.int32)
        import ctypes as C
        no = O.oracle().orc_fetch_points(O.p(eng.volume()), O.p(eng.color_volume()), C.byref(tp), O.p(rng), O.p(zero),
                                         O.p(voff), O.p(xo), O.p(ro), cap)
        assert no == n
        assert np.array_equal(_point_set(xg, rg), _point_set(xo[:no], ro[:no]))
        if vs:
            assert np.any(voff != 0)
        s.close()
