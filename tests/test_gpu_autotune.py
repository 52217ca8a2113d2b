"""Launch shapes and the autotuner that picks them.  No launch shape changes a result bit
except the ICP pixels per thread, which regroups the float partial sums of the normal
equations (poses then agree within 1e-5 rad and 1e-5 m); the autotuner keeps a valid
choice in the context and frees its scratch sessions.  Runs through batch ticks, so the
captured tick graphs (keyed by the launch shape) are exercised too."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L

from _util import cfg_for, cfg_hash, frames, rot_angle, same_bits

pytestmark = pytest.mark.gpu

DEFAULT = (18, 4, 8, 8, 12)


@pytest.fixture(scope="module")
def mix():
    big = frames(5, W=640, H=480, seed=3)
    small = frames(5, W=320, H=240, seed=5)
    cfgs = [cfg_for(res=(128, 128, 128)), cfg_for(W=320, H=240, res=(96, 96, 160), fmt=L.TSDF_F16_U8),
            cfg_hash()]
    return cfgs, [big, small, small]


def _run(ctx, mix):
    cfgs, seqs = mix
    ss = [L.Session(ctx, c) for c in cfgs]
    poses = []
    for f in range(len(seqs[0])):
        st, p = ctx.batch_tick(ss, [q[f][0] for q in seqs])
        assert np.all(st == L.NUI_OK), f
        poses.append(p.copy())
    maps = [s.download(3) for s in ss]
    for s in ss:
        s.close()
    return np.array(poses), maps


def test_shapes_change_no_result_bit(gpu_ctx, mix):
    gpu_ctx.set_tuning(L.Tuning(*DEFAULT))
    base_p, base_m = _run(gpu_ctx, mix)
    for t in [L.Tuning(14, 4, 4, 32), L.Tuning(22, 4, 32, 4), L.Tuning(16, 4, 16, 16)]:
        gpu_ctx.set_tuning(t)
        p, m = _run(gpu_ctx, mix)
        assert np.array_equal(p, base_p), t.as_dict()
        for a, b in zip(m, base_m):
            assert same_bits(a, b), t.as_dict()
    gpu_ctx.set_tuning(L.Tuning(*DEFAULT))


def test_icp_shapes_regroup_sums_only(gpu_ctx, mix):
    """Pixels per thread and blocks per session (cluster sizes 2 .. 16, 16 being the
    non-portable size) change only the grouping of the FP64 partial sums."""
    gpu_ctx.set_tuning(L.Tuning(*DEFAULT))
    base, _ = _run(gpu_ctx, mix)
    for ppt, cl in ((2, 16), (8, 16), (16, 16), (4, 2), (4, 4), (8, 8), (4, 10), (4, 16)):
        gpu_ctx.set_tuning(L.Tuning(18, ppt, 8, 8, cl))
        p, _ = _run(gpu_ctx, mix)
        for f in range(p.shape[0]):
            for i in range(p.shape[1]):
                a, b = p[f, i], base[f, i]
                assert rot_angle(a[:9].reshape(3, 3), b[:9].reshape(3, 3)) < 1e-5, (ppt, cl, f, i)
                assert np.max(np.abs(a[9:] - b[9:])) < 1e-5, (ppt, cl, f, i)
    gpu_ctx.set_tuning(L.Tuning(*DEFAULT))


def test_out_of_range_tuning_is_rejected(gpu_ctx):
    before = gpu_ctx.tuning().as_dict()
    for bad in [L.Tuning(13, 4, 8, 8), L.Tuning(18, 3, 8, 8), L.Tuning(18, 4, 12, 8), L.Tuning(18, 4, 8, 64),
                L.Tuning(18, 4, 8, 8, 1), L.Tuning(18, 4, 8, 8, 17), L.Tuning(18, 4, 8, 8, 32)]:
        with pytest.raises(L.NuiError):
            gpu_ctx.set_tuning(bad)
    assert gpu_ctx.tuning().as_dict() == before


def test_autotune_keeps_a_valid_choice_and_frees_its_sessions(gpu_ctx, mix):
    torch = pytest.importorskip("torch")
    cfgs, seqs = mix
    free0 = torch.cuda.mem_get_info()[0]
    t, ms = gpu_ctx.autotune(cfgs, [[x[0] for x in q[:3]] for q in seqs], repeats=3)
    d = t.as_dict()
    assert d == gpu_ctx.tuning().as_dict()
    assert 16 <= d["integrate_threads_log2"] <= 20
    assert d["icp_pixels_per_thread"] in (2, 4, 8, 16) and d["icp_cluster_blocks"] in (8, 12, 16)
    assert d["raycast_tile_width"] in (4, 8, 16, 32) and d["hash_raycast_tile_width"] in (4, 8, 16, 32)
    assert ms > 0
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)
    # the tuned context still tracks like the default one
    p, _ = _run(gpu_ctx, mix)
    gpu_ctx.set_tuning(L.Tuning(*DEFAULT))
    base, _ = _run(gpu_ctx, mix)
    assert np.max(np.abs(p[..., 9:] - base[..., 9:])) < 1e-5
