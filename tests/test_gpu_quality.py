"""Accuracy against the analytic truth of the synthetic scenes, for the plain FP32 volume
and the compact formats, on the colour-tracking configuration (512^3 over 4 m, RGB texture,
photometric weight 0.1): trajectory error (ATE) against the true poses, TSDF error against
the true signed distance at weighted voxels of the truncation band, and the distance of
the marching-cubes vertices to the true surface.  The compact formats must stay within
1 mm of FP32 on each.  Run with -s to see the figures."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L

from _util import cfg_for, frames

pytestmark = pytest.mark.gpu


def _quality(gpu_ctx, fmt, seq, scene):
    cfg = cfg_for(res=(512, 512, 512), dim=4.0, fmt=fmt, color=True, trunc=0.03)
    cfg.photometric_weight = 0.1
    s = L.Session(gpu_ctx, cfg)
    err = []
    for d, c, _, t in seq:
        ok, p = s.process(d, np.ascontiguousarray(c))
        assert ok
        err.append(np.sum((p[9:] - t) ** 2))
    ate = float(np.sqrt(np.mean(err)))
    # TSDF against the true distance at weighted voxels of the band
    vol = s.volume_ref_layout()
    rx, ry, rz = cfg.res
    c = np.float32(4.0) / np.float32(512)
    trunc = max(0.03, 2.1 * float(c))
    w = vol[:, 1] > 0
    f = vol[:, 0].astype(np.float32) / 32766.0
    band = np.flatnonzero(w & (np.abs(f) < 0.999))
    z = band % rz
    xy = band // rz
    x, y = xy % rx, xy // rx
    pts = np.stack([(x - rx // 2 + 0.5) * c, (y - ry // 2 + 0.5) * c, (z + 0.5) * c], 1).astype(np.float32)
    true = np.clip(scene.sdf_many(pts), -trunc, trunc)
    tsdf_rms = float(np.sqrt(np.mean((f[band] * trunc - true) ** 2)))
    # mesh vertices against the true surface (positions flip y: marchingCube.cl:81-84)
    pos, _, n = s.mesh(6_000_000)
    world = np.stack([pos[:, 0], -pos[:, 1], pos[:, 2]], 1)
    dist = np.abs(scene.sdf_many(world))
    s.close()
    return {"ate_mm": ate * 1e3, "tsdf_rms_mm": tsdf_rms * 1e3, "mesh_mean_mm": float(dist.mean()) * 1e3,
            "mesh_p99_mm": float(np.percentile(dist, 99)) * 1e3, "vertices": int(n)}


def test_compact_formats_within_1mm_of_fp32_against_truth(gpu_ctx):
    seq = frames(16, W=640, H=480, seed=3, color=True)
    scene = L.SynthScene(L.SYNTH_TABLETOP, seed=3, extent=3.0)
    q = {f: _quality(gpu_ctx, f, seq, scene) for f in (L.TSDF_F32, L.TSDF_F16_U8, L.TSDF_F16_F16)}
    for f, v in q.items():
        print("format", f, {k: round(x, 3) for k, x in v.items()})
    ref = q[L.TSDF_F32]
    assert ref["ate_mm"] < 30 and ref["mesh_mean_mm"] < 10
    for f in (L.TSDF_F16_U8, L.TSDF_F16_F16):
        for k in ("ate_mm", "tsdf_rms_mm", "mesh_mean_mm"):
            assert abs(q[f][k] - ref[k]) <= 1.0, (f, k, q[f][k], ref[k])
