"""Errors of the GPU volumes against an FP64 integration of the same frames at the same poses.

The FP64 oracle here is the reference's integration (integrateTsdfVolumeKernel,
tsdfVolume.cl:31-190: voxel centre, projection with round-half-away, ray-length depth of the
pass-filtered frame, sdf >= -trunc, running average capped at weight 128) evaluated in double
precision with numpy.  Reported (run with -s): per format the TSDF RMS and 0.999 quantile
against it in truncation units over the voxels weighted in both, the share of voxels whose
weights differ, and the symmetric Hausdorff distance between the format's marching-cubes mesh
and the mesh of the FP64 volume (meshed by the oracle from its int16 quantisation, 3e-5
truncation units, far below the distances measured).  Bounds: the north-star TSDF tolerance
(1e-3 truncation units at the 0.999 quantile) for every format, and a Hausdorff distance
below one voxel.
"""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import cfg_for, frames, relative_gt

pytestmark = pytest.mark.gpu

RES, DIM, TRUNC = (128, 128, 128), 3.0, 0.046875


def _fp64_integrate(F, Wt, raw, R, t, cfg, cell, trunc):
    """One frame into the float64 volume (F, Wt shaped (rz, ry, rx))."""
    W, H = cfg.width, cfg.height
    d = raw.astype(np.float64) * 0.001
    d[(d <= cfg.depth_min) | (d >= cfg.depth_max)] = np.nan
    u, v = np.meshgrid(np.arange(W), np.arange(H))
    d = d * np.sqrt(((u - cfg.cx) / cfg.fx) ** 2 + ((v - cfg.cy) / cfg.fy) ** 2 + 1.0)
    rx, ry, rz = RES
    x = (np.arange(rx) - rx // 2 + 0.5) * cell - t[0]
    y = (np.arange(ry) - ry // 2 + 0.5) * cell - t[1]
    z = (np.arange(rz) + 0.5) * cell - t[2]
    gz, gy, gx = np.meshgrid(z, y, x, indexing="ij")
    Ri = np.asarray(R, np.float64).T
    vx = Ri[0, 0] * gx + Ri[0, 1] * gy + Ri[0, 2] * gz
    vy = Ri[1, 0] * gx + Ri[1, 1] * gy + Ri[1, 2] * gz
    vz = Ri[2, 0] * gx + Ri[2, 1] * gy + Ri[2, 2] * gz
    with np.errstate(divide="ignore", invalid="ignore"):
        qx, qy = vx * cfg.fx / vz + cfg.cx, vy * cfg.fy / vz + cfg.cy
    px = np.trunc(qx + np.copysign(0.5, qx))
    py = np.trunc(qy + np.copysign(0.5, qy))
    ok = (vz > 0) & (px >= 0) & (py >= 0) & (px < W) & (py < H)
    pxi, pyi = np.where(ok, px, 0).astype(np.int64), np.where(ok, py, 0).astype(np.int64)
    D = np.where(ok, d[pyi, pxi], np.nan)
    sdf = D - np.sqrt(gx * gx + gy * gy + gz * gz)
    upd = ok & ~np.isnan(D) & (sdf >= -trunc)
    tsdf = np.minimum(1.0, sdf / trunc)
    F[upd] = (F[upd] * Wt[upd] + tsdf[upd]) / (Wt[upd] + 1)
    Wt[upd] = np.minimum(Wt[upd] + 1, 128)


def _gpu_volume(s, fmt):
    rx, ry, rz = RES
    raw = s.download(6)
    if fmt == L.TSDF_F16_U8:
        F, Wt = raw.astype(np.float64), s.download(14).astype(np.float64)
    else:
        F, Wt = raw[:, 0].astype(np.float64), raw[:, 1].astype(np.float64)
    return F.reshape(rz, ry, rx), Wt.reshape(rz, ry, rx)


def _hausdorff(a, b):
    from scipy.spatial import cKDTree
    da, _ = cKDTree(b).query(a)
    db, _ = cKDTree(a).query(b)
    return float(max(da.max(), db.max())), float(np.percentile(np.concatenate([da, db]), 99))


def test_volumes_against_fp64_integration(gpu_ctx):
    seq = frames(8, W=640, H=480, seed=3)
    gt = relative_gt(seq)
    cfg0 = cfg_for(res=RES, dim=DIM, trunc=TRUNC)
    cell = float(np.float32(DIM) / np.float32(RES[0]))
    trunc = max(TRUNC, 2.1 * cell)
    rx, ry, rz = RES
    F64, W64 = np.ones((rz, ry, rx)), np.zeros((rz, ry, rx))
    for (raw, _, _, _), (R, t) in zip(seq, gt):
        _fp64_integrate(F64, W64, raw, R, t, cfg0, cell, trunc)
    # the FP64 volume's mesh, through the oracle's marching cubes on its int16 quantisation
    vol16 = np.zeros((ry, rx, rz, 2), np.int16)  # reference layout: (x + y rx) rz + z
    vol16[..., 0] = np.trunc(F64.transpose(1, 2, 0) * 32766.0).astype(np.int16)
    vol16[..., 1] = W64.transpose(1, 2, 0).astype(np.int16)
    tp = O.OrcTsdf.make(RES, (DIM, DIM, DIM), TRUNC)
    cap = 4_000_000
    pos64 = np.zeros((cap, 3), np.float32)
    import ctypes as C
    n64 = O.oracle().orc_marching_cubes(O.p(vol16.reshape(-1)), None, C.byref(tp), None, O.p(pos64), None, cap)
    pos64 = pos64[:min(n64, cap)]
    assert n64 > 1000
    report = {}
    for fmt in (L.TSDF_F32, L.TSDF_F16_U8, L.TSDF_F16_F16):
        s = L.Session(gpu_ctx, cfg_for(res=RES, dim=DIM, trunc=TRUNC, fmt=fmt))
        for (raw, _, _, _), (R, t) in zip(seq, gt):
            s.upload(raw)
            s.set_pose(R, t)
            s.integrate()
        F, Wt = _gpu_volume(s, fmt)
        both = (Wt > 0) & (W64 > 0)
        diff = np.abs(F[both] - F64[both])
        pos, _, n = s.mesh(cap)
        hd, hd99 = _hausdorff(pos.astype(np.float64), pos64.astype(np.float64))
        report[fmt] = {"tsdf_rms": float(np.sqrt(np.mean(diff ** 2))), "tsdf_q999": float(np.quantile(diff, 0.999)),
                       "weights_differ": float(np.mean(Wt != W64)), "hausdorff_mm": hd * 1e3,
                       "hausdorff_p99_mm": hd99 * 1e3, "vertices": int(n)}
        s.close()
    for fmt, r in report.items():
        print("format", fmt, {k: round(v, 6) for k, v in r.items()})
    for fmt, r in report.items():
        assert r["tsdf_q999"] <= 1e-3, (fmt, r)
        assert r["weights_differ"] <= 1e-4, (fmt, r)
        assert r["hausdorff_mm"] < cell * 1e3, (fmt, r)
