"""GPU parity against the oracle at the sizes of the measured workloads, and of the parts whose
results depend only on given poses, so that every comparison runs unconditionally.

- Voxel hash at given poses: allocation, visible list, voxels, raycast maps (vertex, normal,
  colour, expected range) and the block mesh, bit for bit, after every frame; once with a
  small table whose excess chains are long, once at 640x480 with 2^20 buckets and a 2^19-block
  pool (the serving configuration's table sizes).
- The half-sdf pool of the served streams at given poses: the table bit for bit, voxels and
  raycast maps within tolerance of the oracle's int16 pool.
- Dense 256^3 over 3 m (truncation 46.875 mm, ICP 10/5/4): per-frame pose within 1e-4 rad and
  0.1 mm of the oracle over 32 tracked frames.
- Dense 512^3 over 4 m at given poses: the int16 volume and the raycast maps bit for bit.
- The integration gate (NuiKinfuTrackingEngine.cpp:114-127 with rodrigues2,
  NuiMatrixUtilities.cpp:7-52) at its default threshold 0.15: the same frames integrate.
- Pool exhaustion: a frame that finds the block pool empty reports NUI_ERR_HASH_FULL and
  leaves exactly the oracle's table.
"""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import cfg_for, cfg_hash, frames, relative_gt, rot_angle, same_bits

pytestmark = pytest.mark.gpu


def _oracle_voxels(oh):
    sdf, w, rgb = oh.voxels()
    vox = np.zeros(sdf.size, O.REF_VOXEL)
    vox["sdf"], vox["w"], vox["rgb"] = sdf, w, rgb
    return vox.view(np.uint8)


def _pass_depth(raw, cfg):
    W, H = cfg.width, cfg.height
    d = np.zeros(W * H, np.float32)
    O.oracle().orc_pass_filter(O.p(raw.reshape(-1)), W * H, cfg.depth_min, cfg.depth_max, O.p(d))
    return d


def _hash_given_poses(gpu_ctx, cfg, seq, mesh_at, color):
    """Runs `seq` at its true poses through a GPU hash session (step-wise C ABI) and the
    oracle's hash scene, comparing everything after every frame."""
    W, H = cfg.width, cfg.height
    s = L.Session(gpu_ctx, cfg)
    oh = O.OracleHash(cfg.hash_buckets, cfg.hash_excess, cfg.hash_pool_blocks, voxel=cfg.voxel_size,
                      mu=cfg.trunc_scale, max_w=cfg.hash_max_weight)
    cam = O.OrcCam.make(W, H, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.depth_min, cfg.depth_max)
    meshed = 0
    try:
        for k, ((raw, bgra, _, _), (R, t)) in enumerate(zip(seq, relative_gt(seq))):
            bgra = np.ascontiguousarray(bgra) if color else None
            x = O.make_xform(R, t)
            d = _pass_depth(raw, cfg)
            oh.allocate(d, cam, x)
            oh.integrate(d, bgra.reshape(-1) if color else None, cam, x)
            vm, nm, cm, rg = oh.raycast(cam, x, color=color)
            s.upload(raw, bgra)
            s.set_pose(R, t)
            s.integrate()
            s.raycast()
            assert np.array_equal(s.hash_download(21), oh.visible()), k
            assert np.array_equal(s.hash_download(20), oh.entries().view(np.uint8)), k
            assert np.array_equal(s.hash_download(22), _oracle_voxels(oh)), k
            _, lb, le, failed = s.hash_stats()
            assert [lb, le] == list(oh.counters()[:2]) and failed == 0, k
            assert same_bits(s.hash_download(23).reshape(-1), rg), k
            assert same_bits(s.download(3)[..., :3].reshape(-1), vm), k
            assert same_bits(s.download(4)[..., :3].reshape(-1), nm), k
            if color:
                assert np.array_equal(s.download(8).reshape(-1), cm), k
            assert np.mean(~np.isnan(vm)) > 0.3, k  # the maps are not trivially empty
            if k in mesh_at:
                cap = 6_000_000
                pg, cg, ng = s.mesh(cap)
                po, co, no = oh.mesh(cap)
                assert ng == no > 0, k
                assert same_bits(pg, po) and same_bits(cg, co), k
                meshed += 1
        assert meshed == len(mesh_at)
    finally:
        s.close()


def test_hash_given_poses_raycast_and_mesh_bit_exact(gpu_ctx):
    """320x240 with a 2^16-bucket table (many excess chains), colour on, a turning camera."""
    cfg = cfg_hash(color=True)
    seq = frames(5, W=320, H=240, seed=5, kind=L.SYNTH_ROOM, deg=3.0, color=True)
    _hash_given_poses(gpu_ctx, cfg, seq, mesh_at=(2, 4), color=True)


def test_hash_serving_table_sizes_bit_exact(gpu_ctx):
    """640x480 with 2^20 buckets and a 2^19-block pool (hash index masking, excess
    allocation and pool-pointer ranks at the served table sizes)."""
    cfg = cfg_hash(W=640, H=480, buckets=1 << 20, excess=1 << 17, pool=1 << 19, fmt=L.TSDF_I16)
    seq = frames(3, W=640, H=480, seed=9, kind=L.SYNTH_ROOM, deg=3.0, color=False)
    _hash_given_poses(gpu_ctx, cfg, seq, mesh_at=(2,), color=False)


def test_hash_half_format_given_poses_within_tolerance(gpu_ctx):
    """The half-sdf pool of the serving mix (tolerance-mode voxel update) at given poses
    against the oracle's int16 pool: the same table (entries and visible list) bit for bit,
    and over the voxels either side has updated, sdf within 1e-3 truncation units at the
    0.999 quantile (the half quantum is at most 4.9e-4 there), weights equal on all but 1e-3
    of them and colours within one level on all but 1e-3.  The raycast of the half pool
    against the oracle's: hit masks agree on all but 1 % of the pixels, and where both hit
    the surface points agree within 0.5 mm at the 0.99 quantile."""
    cfg = cfg_hash(fmt=L.TSDF_F16_U8, color=True)
    seq = frames(5, W=320, H=240, seed=5, kind=L.SYNTH_ROOM, deg=3.0, color=True)
    W, H = cfg.width, cfg.height
    s = L.Session(gpu_ctx, cfg)
    oh = O.OracleHash(cfg.hash_buckets, cfg.hash_excess, cfg.hash_pool_blocks, voxel=cfg.voxel_size,
                      mu=cfg.trunc_scale, max_w=cfg.hash_max_weight)
    cam = O.OrcCam.make(W, H, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.depth_min, cfg.depth_max)
    try:
        for k, ((raw, bgra, _, _), (R, t)) in enumerate(zip(seq, relative_gt(seq))):
            bgra = np.ascontiguousarray(bgra)
            x = O.make_xform(R, t)
            d = _pass_depth(raw, cfg)
            oh.allocate(d, cam, x)
            oh.integrate(d, bgra.reshape(-1), cam, x)
            vm, _, _, _ = oh.raycast(cam, x, color=True)
            s.upload(raw, bgra)
            s.set_pose(R, t)
            s.integrate()
            s.raycast()
            assert np.array_equal(s.hash_download(21), oh.visible()), k
            assert np.array_equal(s.hash_download(20), oh.entries().view(np.uint8)), k
            g = s.hash_download(22).view(O.REF_VOXEL)
            o = _oracle_voxels(oh).view(O.REF_VOXEL)
            upd = (g["w"] > 0) | (o["w"] > 0)
            assert upd.sum() > 10000, k
            dsdf = np.abs(g["sdf"][upd].astype(np.int64) - o["sdf"][upd]) / 32767.0
            assert np.quantile(dsdf, 0.999) <= 1e-3, (k, float(np.quantile(dsdf, 0.999)))
            assert np.mean(g["w"][upd] != o["w"][upd]) <= 1e-3, k
            dc = np.abs(g["rgb"][upd].astype(np.int64) - o["rgb"][upd]).max(axis=1)
            assert np.mean(dc > 1) <= 1e-3, k
            gv = s.download(3)[..., :3].reshape(-1, 3).astype(np.float64)
            ov = vm.reshape(-1, 3).astype(np.float64)
            hg, ho = ~np.isnan(gv[:, 0]), ~np.isnan(ov[:, 0])
            assert ho.mean() > 0.3, k
            assert np.mean(hg != ho) <= 0.01, (k, float(np.mean(hg != ho)))
            both = hg & ho
            dist = np.linalg.norm(gv[both] - ov[both], axis=1)
            assert np.quantile(dist, 0.99) <= 5e-4, (k, float(np.quantile(dist, 0.99)), float(dist.max()))
    finally:
        s.close()


def test_dense_256_config_poses_over_32_frames(gpu_ctx):
    """256^3 over 3 m, truncation 46.875 mm, ICP 10/5/4, 640x480 with sensor noise."""
    cfg = cfg_for(res=(256, 256, 256), dim=3.0, trunc=0.046875, iters=(10, 5, 4))
    seq = frames(32, W=640, H=480, seed=17)
    s = L.Session(gpu_ctx, cfg)
    eng = O.Engine(cfg)
    worst = (0.0, 0.0)
    try:
        for i, (d, _, _, _) in enumerate(seq):
            ok, pose = s.process(d)
            assert ok and eng.frame(d), i
            Ro, to = eng.pose()
            da, dt = rot_angle(pose[:9].reshape(3, 3), Ro), float(np.max(np.abs(pose[9:] - to)))
            worst = (max(worst[0], da), max(worst[1], dt))
            assert da < 1e-4 and dt < 1e-4, (i, da, dt)
    finally:
        s.close()
    assert worst[0] < 1e-4 and worst[1] < 1e-4


def test_dense_512_given_poses_bit_exact(gpu_ctx):
    """512^3 over 4 m: the int16 volume and the raycast maps after every frame."""
    cfg = cfg_for(res=(512, 512, 512), dim=4.0, trunc=0.03125)
    seq = frames(3, W=640, H=480, seed=21, extent=4.0)
    s = L.Session(gpu_ctx, cfg)
    eng = O.Engine(cfg)
    try:
        for k, ((d, _, _, _), (R, t)) in enumerate(zip(seq, relative_gt(seq))):
            eng.integrate_at(d, R, t)
            s.upload(d)
            s.set_pose(R, t)
            s.integrate()
            s.raycast()
            assert s.touched() == eng.touched() > 0, k
            assert np.array_equal(s.volume_ref_layout(), eng.volume()), k
            vg = s.download(3)[..., :3]
            assert same_bits(vg, eng.refmap(0)), k
            assert same_bits(s.download(4)[..., :3], eng.refmap(1)), k
            assert np.mean(~np.isnan(vg[..., 2])) > 0.3, k
    finally:
        s.close()


def test_integration_gate_at_default_threshold(gpu_ctx):
    """With the reference's default threshold (0.15) only frames whose motion since the last
    integration reaches (|rodrigues2(R^-1 R_last)| + |t - t_last|) / 2 >= 0.15 integrate; the
    GPU integrates exactly the frames the oracle does, and tracks within the tolerances."""
    cfg = cfg_for(res=(128, 128, 128), integ_thr=0.15)
    seq = frames(14, W=640, H=480, seed=3, deg=3.0)
    s = L.Session(gpu_ctx, cfg)
    eng = O.Engine(cfg)
    decisions = []
    try:
        for i, (d, _, _, _) in enumerate(seq):
            ok, pose = s.process(d)
            assert ok and eng.frame(d), i
            Ro, to = eng.pose()
            assert rot_angle(pose[:9].reshape(3, 3), Ro) < 1e-4 and np.max(np.abs(pose[9:] - to)) < 1e-4, i
            g, o = s.touched(), eng.touched()
            assert (g > 0) == (o > 0), (i, g, o)
            if o > 0:  # poses agree to 1e-4, so the updated voxel sets nearly coincide
                assert abs(g - o) <= 1e-3 * o, (i, g, o)
            decisions.append(o > 0)
    finally:
        s.close()
    # frame 0 always integrates; the gate both skipped and passed later frames
    assert decisions[0] and any(decisions[1:]) and not all(decisions[1:]), decisions


def test_hash_pool_exhaustion_reports_hash_full(gpu_ctx):
    """A 96-block pool cannot hold a 320x240 frame's blocks: the frame reports
    NUI_ERR_HASH_FULL (the reference drops the blocks silently), the table equals the
    oracle's (the first 96 requests in entry order got blocks), and the whole frame path
    returns the same status."""
    cfg = cfg_hash(pool=96)
    seq = frames(1, W=320, H=240, seed=5, kind=L.SYNTH_ROOM, deg=0.0)
    raw = seq[0][0]
    W, H = cfg.width, cfg.height
    s = L.Session(gpu_ctx, cfg)
    oh = O.OracleHash(cfg.hash_buckets, cfg.hash_excess, cfg.hash_pool_blocks, voxel=cfg.voxel_size,
                      mu=cfg.trunc_scale, max_w=cfg.hash_max_weight)
    cam = O.OrcCam.make(W, H, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.depth_min, cfg.depth_max)
    R, t = np.eye(3, dtype=np.float32), np.zeros(3, np.float32)
    x = O.make_xform(R, t)
    d = _pass_depth(raw, cfg)
    oh.allocate(d, cam, x)
    oh.integrate(d, None, cam, x)
    try:
        s.upload(raw)
        s.set_pose(R, t)
        with pytest.raises(L.NuiError) as e:
            s.integrate()
        assert e.value.status == L.NUI_ERR_HASH_FULL
        _, lb, le, failed = s.hash_stats()
        ob, oe, of = oh.counters()
        assert failed == of > 0 and lb == ob < 0 and le == oe
        assert np.array_equal(s.hash_download(20), oh.entries().view(np.uint8))
        assert np.array_equal(s.hash_download(22), _oracle_voxels(oh))
    finally:
        s.close()
    s2 = L.Session(gpu_ctx, cfg)
    try:
        with pytest.raises(L.NuiError) as e:
            s2.process(raw)
        assert e.value.status == L.NUI_ERR_HASH_FULL
        st, _ = gpu_ctx.batch_tick([s2], [raw])
        assert st[0] == L.NUI_ERR_HASH_FULL
    finally:
        s2.close()
