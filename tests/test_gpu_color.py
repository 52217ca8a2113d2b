"""GPU parity of colour tracking (A8): the depth ICP joined by the photometric term of
the colour tracker, against the oracle (itself pinned to the reference's colour kernels).

Bit-exact: the colour gradients of the current frame and the model colours kept for the
next frame.  Tolerance: per-frame pose within 1e-4 rad and 0.1 mm (the normal equations
are summed in another order).  A photometric weight of 0 tracks exactly like depth-only
ICP, and the compact FP16 TSDF tracks like FP32 (ATE within 1 mm)."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import cfg_for, cfg_hash, frames, rot_angle

pytestmark = pytest.mark.gpu


def _ccfg(res=(128, 128, 128), W=640, H=480, fmt=L.TSDF_I16, w=0.1):
    cfg = cfg_for(W=W, H=H, res=res, fmt=fmt, color=True)
    cfg.photometric_weight = w
    return cfg


@pytest.fixture(scope="module")
def tex():
    return frames(6, W=640, H=480, seed=3, color=True)


def test_gradients_and_model_colours_bit_exact(gpu_ctx):
    seq = frames(2, W=320, H=240, seed=7, color=True)
    s = L.Session(gpu_ctx, _ccfg(res=(96, 96, 96), W=320, H=240))
    for d, c, _, _ in seq:
        ok, _ = s.process(d, np.ascontiguousarray(c))
        assert ok
    c1 = np.ascontiguousarray(seq[1][1])
    gx = np.zeros_like(c1)
    gy = np.zeros_like(c1)
    O.oracle().orc_color_gradient(O.p(c1), 320, 240, O.p(gx), O.p(gy))
    assert np.array_equal(s.download(11, 0), gx)
    assert np.array_equal(s.download(12, 0), gy)
    assert np.array_equal(s.download(10, 0), c1)


def test_color_tracking_sequence_against_oracle(gpu_ctx, tex):
    cfg = _ccfg()
    s = L.Session(gpu_ctx, cfg)
    eng = O.Engine(cfg)
    for i, (d, c, R_gt, t_gt) in enumerate(tex):
        c = np.ascontiguousarray(c)
        ok, pose = s.process(d, c)
        assert ok and eng.frame(d, c), i
        Rg, tg = pose[:9].reshape(3, 3), pose[9:]
        Ro, to = eng.pose()
        assert rot_angle(Rg, Ro) < 1e-4, i
        assert np.max(np.abs(tg - to)) < 1e-4, i
        assert rot_angle(Rg, R_gt) < 0.03 and np.max(np.abs(tg - t_gt)) < 0.03, i


def test_zero_photometric_weight_is_depth_only(gpu_ctx, tex):
    a = L.Session(gpu_ctx, _ccfg(w=0.0))
    b = L.Session(gpu_ctx, cfg_for(res=(128, 128, 128)))
    for d, c, _, _ in tex:
        ok1, p1 = a.process(d, np.ascontiguousarray(c))
        ok2, p2 = b.process(d)
        assert ok1 and ok2 and np.array_equal(p1, p2)


def test_hash_color_tracking_against_oracle(gpu_ctx):
    seq = frames(5, W=320, H=240, seed=3, color=True)
    cfg = cfg_hash(color=True)
    cfg.photometric_weight = 0.1
    s = L.Session(gpu_ctx, cfg)
    eng = O.Engine(cfg)
    for i, (d, c, _, _) in enumerate(seq):
        c = np.ascontiguousarray(c)
        ok, pose = s.process(d, c)
        assert ok and eng.frame(d, c), i
        Ro, to = eng.pose()
        assert rot_angle(pose[:9].reshape(3, 3), Ro) < 1e-4 and np.max(np.abs(pose[9:] - to)) < 1e-4, i


def test_hash_half_color_tracking_close_to_oracle(gpu_ctx):
    """The served voxel-hash streams' configuration -- half-sdf pool, colour ICP in
    tolerance mode (one reciprocal of the depth per photometric row) -- stays frame by frame
    within 4 mrad / 4 mm of the oracle tracking the reference's int16 pool."""
    seq = frames(6, W=320, H=240, seed=3, color=True)
    cfg = cfg_hash(color=True, fmt=L.TSDF_F16_U8)
    cfg.photometric_weight = 0.1
    ocfg = cfg_hash(color=True)
    ocfg.photometric_weight = 0.1
    s = L.Session(gpu_ctx, cfg)
    eng = O.Engine(ocfg)
    for i, (d, c, _, _) in enumerate(seq):
        c = np.ascontiguousarray(c)
        ok, pose = s.process(d, c)
        assert ok and eng.frame(d, c), i
        Ro, to = eng.pose()
        assert rot_angle(pose[:9].reshape(3, 3), Ro) < 4e-3 and np.max(np.abs(pose[9:] - to)) < 4e-3, i
    s.close()


def test_color_tracking_fp16_ate_within_1mm_of_fp32(gpu_ctx):
    seq = frames(16, W=640, H=480, seed=4, color=True)
    ate = {}
    for fmt in (L.TSDF_F32, L.TSDF_F16_U8):
        s = L.Session(gpu_ctx, _ccfg(res=(256, 256, 256), fmt=fmt))
        err = []
        for d, c, _, t in seq:
            ok, p = s.process(d, np.ascontiguousarray(c))
            assert ok
            err.append(np.sum((p[9:] - t) ** 2))
        ate[fmt] = float(np.sqrt(np.mean(err)))
        s.close()
    assert abs(ate[L.TSDF_F16_U8] - ate[L.TSDF_F32]) <= 1e-3, ate


def test_kernel_level_color_pyramid_bit_exact(gpu_ctx):
    torch = pytest.importorskip("torch")
    import ctypes as C
    bgra = np.ascontiguousarray(frames(1, W=640, H=480, seed=9, color=True)[0][1])
    H, W, levels = 480, 640, 3
    d_in = torch.from_numpy(bgra).cuda()
    lv = [None] + [torch.zeros((H >> l, W >> l, 4), dtype=torch.uint8, device="cuda") for l in range(1, levels)]
    gx = [torch.zeros((H >> l, W >> l, 4), dtype=torch.uint8, device="cuda") for l in range(levels)]
    gy = [torch.zeros((H >> l, W >> l, 4), dtype=torch.uint8, device="cuda") for l in range(levels)]
    arr = C.c_void_p * levels
    pl = arr(*[None] + [t.data_ptr() for t in lv[1:]])
    pgx = arr(*[t.data_ptr() for t in gx])
    pgy = arr(*[t.data_ptr() for t in gy])
    L.check(L.lib().nui_k_color_pyramid(gpu_ctx.h, C.c_void_p(d_in.data_ptr()), W, H, levels, pl, pgx, pgy))
    src = bgra
    for l in range(levels):
        if l > 0:
            want = np.zeros((H >> l, W >> l, 4), np.uint8)
            O.oracle().orc_color_half_sample(O.p(src), W >> l, H >> l, 1, O.p(want))
            assert np.array_equal(lv[l].cpu().numpy(), want), l
            src = want
        ox = np.zeros_like(src)
        oy = np.zeros_like(src)
        O.oracle().orc_color_gradient(O.p(src), W >> l, H >> l, O.p(ox), O.p(oy))
        assert np.array_equal(gx[l].cpu().numpy(), ox), l
        assert np.array_equal(gy[l].cpu().numpy(), oy), l
