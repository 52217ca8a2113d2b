"""Shared helpers of the tests: synthetic frames and the oracle pipeline pieces."""
import ctypes as C

import numpy as np

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32 if a.dtype == np.float32 else np.uint16)


def same_bits(a, b):
    """Bit-exact float comparison (NaN == NaN when the bit patterns agree)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    if not np.array_equal(na, nb):
        return False
    return np.array_equal(a[~na].view(np.uint32), b[~nb].view(np.uint32))


def frames(n, W=640, H=480, seed=3, noise=True, color=False, deg=2.0, kind=L.SYNTH_TABLETOP, extent=3.0):
    sc = L.SynthScene(kind, seed=seed, extent=extent)
    out = []
    f = 525.0 * W / 640.0
    cx, cy = (W - 1) / 2.0, (H - 1) / 2.0
    for i in range(n):
        R, t = sc.pose(i, radius=extent / 2, deg_per_frame=deg)
        d, c = sc.render(R, t, W, H, fx=f, fy=f, cx=cx, cy=cy, frame=i, noise=noise, color=color)
        out.append((d, c, R, t))
    return out


def cfg_for(W=640, H=480, res=(256, 256, 256), dim=3.0, fmt=L.TSDF_I16, color=False, iters=(10, 5, 4),
            trunc=0.046875, integ_thr=0.0):
    f = 525.0 * W / 640.0
    return L.default_cfg(width=W, height=H, fx=f, fy=f, cx=(W - 1) / 2.0, cy=(H - 1) / 2.0, res=res,
                         dim=(dim, dim, dim), tsdf_format=fmt, color_volume=1 if color else 0,
                         iterations=list(iters) + [0] * (4 - len(iters)), levels=len(iters), trunc_dist=trunc,
                         integration_threshold=integ_thr)


def oracle_preprocess(raw, cfg):
    """Oracle pass filter + bilateral + vertex + pyramid + scaled depth of one frame."""
    orc = O.oracle()
    W, H = cfg.width, cfg.height
    N = W * H
    cam = O.OrcCam.make(W, H, cfg.fx, cfg.fy, cfg.cx, cfg.cy, cfg.depth_min, cfg.depth_max)
    a = np.zeros(N, np.float32)
    orc.orc_pass_filter(O.p(raw.reshape(-1)), N, cfg.depth_min, cfg.depth_max, O.p(a))
    g = np.zeros(2 * cfg.filter_radius + 1, np.float32)
    orc.orc_gaussian_table(cfg.filter_radius, cfg.sigma_space2_inv_half, O.p(g))
    f = np.zeros(N, np.float32)
    orc.orc_bilateral(O.p(a), W, H, O.p(g), cfg.filter_radius, cfg.sigma_depth2_inv_half, cfg.depth_threshold,
                      O.p(f))
    v = np.zeros(N * 3, np.float32)
    orc.orc_depth2vertex(O.p(f), W, H, C.byref(cam), 1, O.p(v))
    s = a.copy()
    orc.orc_scale_depths(O.p(s), W, H, C.byref(cam))
    levels = [(f.reshape(H, W), v.reshape(H, W, 3))]
    src = f
    for l in range(1, cfg.levels):
        h = np.zeros((W >> l) * (H >> l), np.float32)
        orc.orc_half_sample(O.p(src), W >> l, H >> l, 1, cfg.depth_threshold, O.p(h))
        vv = np.zeros(h.size * 3, np.float32)
        orc.orc_depth2vertex(O.p(h), W >> l, H >> l, C.byref(cam), 1 << l, O.p(vv))
        levels.append((h.reshape(H >> l, W >> l), vv.reshape(H >> l, W >> l, 3)))
        src = h
    return dict(passd=a.reshape(H, W), scaled=s.reshape(H, W), levels=levels, cam=cam)


def rot_angle(Ra, Rb):
    """Angle of Ra^T Rb, robust near zero (atan2 of the skew and symmetric parts)."""
    M = np.asarray(Ra, np.float64).T @ np.asarray(Rb, np.float64)
    s = 0.5 * np.linalg.norm([M[2, 1] - M[1, 2], M[0, 2] - M[2, 0], M[1, 0] - M[0, 1]])
    c = (np.trace(M) - 1) / 2
    return float(np.arctan2(s, c))


def cfg_hash(W=320, H=240, buckets=1 << 16, excess=1 << 14, pool=1 << 16, voxel=0.005, mu=0.02, fmt=L.TSDF_I16,
             color=False, iters=(10, 5, 4), integ_thr=0.0):
    f = 525.0 * W / 640.0
    return L.default_cfg(width=W, height=H, fx=f, fy=f, cx=(W - 1) / 2.0, cy=(H - 1) / 2.0, volume_kind=L.VOLUME_HASH,
                         tsdf_format=fmt, color_volume=1 if color else 0, hash_buckets=buckets, hash_excess=excess,
                         hash_pool_blocks=pool, voxel_size=voxel, trunc_scale=mu,
                         iterations=list(iters) + [0] * (4 - len(iters)), levels=len(iters),
                         integration_threshold=integ_thr, depth_min=0.4)


def relative_gt(seq):
    """Ground-truth poses expressed in the first camera's frame (the tracker starts at I)."""
    R0, t0 = np.asarray(seq[0][2], np.float64), np.asarray(seq[0][3], np.float64)
    out = []
    for _, _, R, t in seq:
        out.append((R0.T @ np.asarray(R, np.float64), R0.T @ (np.asarray(t, np.float64) - t0)))
    return out


def integration_near_ties(cfg, tp, R, t, scaled, eps_px=1e-4, eps_m=1e-5):
    """Voxels (reference layout, flattened) whose integration decision is a near tie at pose
    (R, t): the exact (FP64) projection lies within eps_px of a rounding boundary (a half
    pixel) in u or v, or the signed distance within eps_m of -trunc.  There any float
    evaluation -- the reference's running sums or a direct one -- may take the other side,
    i.e. the neighbouring pixel's depth or the other update decision.  scaled: the
    frame's ray-length depth (oracle_preprocess(...)["scaled"])."""
    rx, ry, rz = (int(v) for v in tp.res)
    cell = [float(np.float32(c)) for c in tp.cell[:3]]
    Ri = np.asarray(R, np.float64).T
    t = np.asarray(t, np.float64)
    x = (np.arange(rx) - rx // 2 + 0.5) * cell[0] - t[0]
    y = (np.arange(ry) - ry // 2 + 0.5) * cell[1] - t[1]
    z = (np.arange(rz) + 0.5) * cell[2] - t[2]
    gy, gx, gz = np.meshgrid(y, x, z, indexing="ij")  # reference layout: (x + y rx) rz + z
    vx = Ri[0, 0] * gx + Ri[0, 1] * gy + Ri[0, 2] * gz
    vy = Ri[1, 0] * gx + Ri[1, 1] * gy + Ri[1, 2] * gz
    vz = Ri[2, 0] * gx + Ri[2, 1] * gy + Ri[2, 2] * gz
    with np.errstate(divide="ignore", invalid="ignore"):
        qx, qy = vx * cfg.fx / vz + cfg.cx, vy * cfg.fy / vz + cfg.cy
        tie = (np.abs(qx - np.floor(qx) - 0.5) < eps_px) | (np.abs(qy - np.floor(qy) - 0.5) < eps_px)
        px, py = np.trunc(qx + np.copysign(0.5, qx)), np.trunc(qy + np.copysign(0.5, qy))
        W, H = cfg.width, cfg.height
        ok = (vz > 0) & (px >= 0) & (py >= 0) & (px < W) & (py < H)
        D = np.where(ok, scaled[np.where(ok, py, 0).astype(np.int64), np.where(ok, px, 0).astype(np.int64)], np.nan)
        sd = D - np.sqrt(gx * gx + gy * gy + gz * gz)
        tie |= np.abs(sd + float(tp.trunc)) < eps_m
    return (tie & (vz > 0)).reshape(-1)
