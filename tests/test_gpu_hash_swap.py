"""GPU parity of the voxel hash's global cache (hash swapping, NuiKinfuOpenCLHashGlobalCache)
against the oracle, itself pinned to the reference's swapping kernels.  At given poses a
camera turns away from a room and back: blocks leave the view, are merged, swapped out to
the host store (cleared, their pool blocks freed), come back, are re-allocated and merged
with their stored copies.  After every frame: the same hash entries, visible list, voxels,
swap states and free-list counters, and the same stored blocks."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import cfg_hash

pytestmark = pytest.mark.gpu


def _oracle_voxels(oh):
    sdf, w, rgb = oh.voxels()
    vox = np.zeros(sdf.size, O.REF_VOXEL)
    vox["sdf"], vox["w"], vox["rgb"] = sdf, w, rgb
    return vox.view(np.uint8)


def test_global_cache_at_given_poses_bit_exact(gpu_ctx):
    W, H = 160, 120
    cfg = cfg_hash(W=W, H=H, voxel=0.02, mu=0.08, color=True)
    cfg.hash_swapping = 1
    cfg.hash_store_blocks = 1 << 14
    s = L.Session(gpu_ctx, cfg)
    oh = O.OracleHash(cfg.hash_buckets, cfg.hash_excess, cfg.hash_pool_blocks, voxel=cfg.voxel_size,
                      mu=cfg.trunc_scale, max_w=cfg.hash_max_weight, swapping=True)
    f = cfg.fx
    cam = O.OrcCam.make(W, H, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.depth_min, cfg.depth_max)
    sc = L.SynthScene(L.SYNTH_ROOM, seed=5)
    path = [0, 20, 40, 60, 40, 20, 0]
    back = 0
    for k, i in enumerate(path):
        R, t = sc.pose(i, radius=1.5, deg_per_frame=2.0)
        raw, bgra = sc.render(R, t, W, H, fx=f, fy=f, cx=cfg.cx, cy=cfg.cy, frame=k, color=True)
        bgra = np.ascontiguousarray(bgra)
        d = np.zeros(W * H, np.float32)
        O.oracle().orc_pass_filter(O.p(raw.reshape(-1)), W * H, cfg.depth_min, cfg.depth_max, O.p(d))
        x = O.make_xform(R, t)
        oh.allocate(d, cam, x)
        oh.integrate(d, bgra.reshape(-1), cam, x)
        oh.swap()
        s.upload(raw, bgra)
        s.set_pose(R, t)
        s.integrate()
        assert np.array_equal(s.hash_download(21), oh.visible()), k
        assert np.array_equal(s.hash_download(20), oh.entries().view(np.uint8)), k
        assert np.array_equal(s.hash_download(22), _oracle_voxels(oh)), k
        st = s.hash_download(24)
        assert np.array_equal(st, oh.swap_states()), k
        _, lb, le, failed = s.hash_stats()
        assert [lb, le] == list(oh.counters()[:2]) and failed == 0, k
        ids = oh.stored_ids()
        sin, sout, used, refused = s.hash_swap_stats()
        assert used == ids.size and refused == 0, k
        for e in ids:
            g = s.hash_stored(e)
            o = oh.stored(e)
            assert g is not None, (k, e)
            assert np.array_equal(g[0], o[0]) and np.array_equal(g[1], o[1]), (k, e)
            assert np.array_equal(g[2][:, :3], o[2]), (k, e)
        back += int(np.sum((st == 2) & np.isin(np.arange(st.size), ids)))
    assert ids.size > 100 and back > 0
    s.close()


def test_swapping_session_tracks_and_snapshots(gpu_ctx):
    """Through the batched tick: a swapping hash session tracks like the oracle engine with
    the global cache on, and a restored snapshot continues identically."""
    from _util import frames, rot_angle
    seq = frames(6, W=320, H=240, seed=3)
    cfg = cfg_hash()
    cfg.hash_swapping = 1
    cfg.hash_store_blocks = 1 << 15
    s = L.Session(gpu_ctx, cfg)
    eng = O.Engine(cfg)
    for i, (d, _, _, _) in enumerate(seq[:4]):
        ok, pose = s.process(d)
        assert ok and eng.frame(d), i
        Ro, to = eng.pose()
        assert rot_angle(pose[:9].reshape(3, 3), Ro) < 1e-4 and np.max(np.abs(pose[9:] - to)) < 1e-4, i
    snap = s.snapshot()
    a = [s.process(d)[1] for d, _, _, _ in seq[4:]]
    r = L.Session(gpu_ctx, cfg)
    r.restore(snap)
    b = [r.process(d)[1] for d, _, _, _ in seq[4:]]
    for p1, p2 in zip(a, b):
        assert np.array_equal(p1, p2)
    s.close()
    r.close()
