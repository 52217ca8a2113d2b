"""Pins the colour-tracking oracle (A8) against the reference's own kernels.

The reference's colour kernels (transformMaps.cl half_sample_bgra_kernel and
bgra_gradient_kernel, colorIcp.cl color_icp_block_kernel), compiled for the host by
oracle/build_ref.py, run on the same seeded textured frames as the oracle:

* the colour pyramid agrees byte for byte;
* the gradients agree byte for byte where the reference's index walk is a Sobel at all:
  on a square image, whose result the reference stores one row and one pixel past the
  centre (the oracle stores it at the centre);
* the photometric rows, evaluated in the kernel's own convention (ref_mode = 1), agree
  per work-group of 128 model points with the kernel's float tree reduction.

The tracker's own convention (ref_mode = 0: camera-to-world pose, the depth ICP's
parameters, signed gradients) is checked against its derivation: the camera-point
derivatives by central differences of the pose update, and each row against an
independent numpy evaluation.
"""
import ctypes as C

import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import frames

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels not built (no reference tree)")


@pytest.fixture(scope="module")
def textured():
    return frames(2, W=320, H=240, seed=7, color=True)


def _pyramid(bgra, levels=3):
    orc = O.oracle()
    H, W = bgra.shape[:2]
    pyr = [np.ascontiguousarray(bgra)]
    for l in range(1, levels):
        d = np.zeros((H >> l, W >> l, 4), np.uint8)
        orc.orc_color_half_sample(O.p(pyr[-1]), W >> l, H >> l, 1, O.p(d))
        pyr.append(d)
    return pyr


def _gradients(img):
    H, W = img.shape[:2]
    gx = np.zeros_like(img)
    gy = np.zeros_like(img)
    O.oracle().orc_color_gradient(O.p(img), W, H, O.p(gx), O.p(gy))
    return gx, gy


@needs_ref
def test_color_pyramid_matches_reference(textured):
    bgra = textured[1][1]
    H, W = bgra.shape[:2]
    src = np.ascontiguousarray(bgra)
    for l in (1, 2):
        w, h = W >> l, H >> l
        mine = np.zeros((h, w, 4), np.uint8)
        ref = np.zeros((h, w, 4), np.uint8)
        O.oracle().orc_color_half_sample(O.p(src), w, h, 1, O.p(mine))
        O.ref().ref_half_sample_bgra(O.p(src.copy()), O.p(ref), w, h, 1)
        assert np.array_equal(mine, ref), l
        src = mine


@needs_ref
def test_color_gradient_matches_reference_on_square_image(textured):
    img = np.ascontiguousarray(textured[0][1][:128, 40:168])  # 128 x 128
    n = img.shape[0]
    gx, gy = _gradients(img)
    rx = np.zeros_like(img)
    ry = np.zeros_like(img)
    O.ref().ref_bgra_gradient(O.p(img.copy()), O.p(rx), O.p(ry), n, n)
    # reference pixel (x + 1, y + 1) holds the Sobel of (x, y); compare where only one
    # work-item writes it
    assert np.array_equal(rx[2:n - 1, 2:n - 1], gx[1:n - 2, 1:n - 2])
    assert np.array_equal(ry[2:n - 1, 2:n - 1], gy[1:n - 2, 1:n - 2])
    assert np.any(gx[1:-1, 1:-1, :3].view(np.int8) < 0)  # negative gradients wrap


def test_color_gradient_is_sobel_over_eight(textured):
    img = textured[1][1]
    gx, gy = _gradients(img)
    f = img[..., :3].astype(np.float32)
    sx = ((f[:-2, 2:] - f[:-2, :-2]) + 2 * (f[1:-1, 2:] - f[1:-1, :-2]) + (f[2:, 2:] - f[2:, :-2])) / np.float32(8)
    sy = ((f[2:, :-2] - f[:-2, :-2]) + 2 * (f[2:, 1:-1] - f[:-2, 1:-1]) + (f[2:, 2:] - f[:-2, 2:])) / np.float32(8)
    assert np.array_equal(gx[1:-1, 1:-1, :3].view(np.int8), np.trunc(sx).astype(np.int8))
    assert np.array_equal(gy[1:-1, 1:-1, :3].view(np.int8), np.trunc(sy).astype(np.int8))
    assert np.all(gx[1:-1, 1:-1, 3] == 255) and np.all(gx[0] == 0) and np.all(gy[:, -1] == 0)


def _model(fr, W, H):
    """World vertex map and colours of frame 0 at its ground-truth pose."""
    orc = O.oracle()
    d, bgra, R0, t0 = fr
    cam = O.OrcCam.make(W, H, 525.0 * W / 640, 525.0 * W / 640, (W - 1) / 2, (H - 1) / 2)
    a = np.zeros(W * H, np.float32)
    orc.orc_pass_filter(O.p(d.reshape(-1)), W * H, 0.5, 4.5, O.p(a))
    v = np.zeros(W * H * 3, np.float32)
    orc.orc_depth2vertex(O.p(a), W, H, C.byref(cam), 1, O.p(v))
    n = np.zeros_like(v)
    orc.orc_normals(O.p(v), W, H, 0.3, O.p(n))
    x0 = O.make_xform(R0, t0)
    vw, nw = np.zeros_like(v), np.zeros_like(v)
    orc.orc_transform_maps(O.p(v), O.p(n), W, H, C.byref(x0), O.p(vw), O.p(nw))
    mc = np.ascontiguousarray(bgra).copy()
    mc[..., 3] = 255
    return cam, vw, mc


@needs_ref
@pytest.mark.parametrize("level", [0, 1, 2])
def test_color_rows_match_reference_kernel(textured, level):
    H, W = textured[0][0].shape
    cam, mv, mc = _model(textured[0], W, H)
    _, bgra1, R1, t1 = textured[1]
    pyr = _pyramid(bgra1)
    gx, gy = _gradients(pyr[level])
    # the kernel moves the model by (R, t) as given: pass world -> camera of frame 1
    Rw = np.ascontiguousarray(np.asarray(R1, np.float32).T).reshape(9)
    tw = np.ascontiguousarray(-(np.asarray(R1, np.float32).T @ np.asarray(t1, np.float32)), np.float32)
    n = W * H
    rows = np.zeros((n, 29), np.float32)
    sums = np.zeros(29)
    O.oracle().orc_color_rows(O.p(mv), O.p(mc), C.byref(cam), level, O.p(pyr[level]), O.p(gx), O.p(gy), O.p(Rw),
                              O.p(tw), 1, O.p(rows), O.p(sums))
    out = np.zeros((n // 128, 29), np.float32)
    O.ref().ref_color_icp_blocks(O.p(cam.flat()), O.p(mv.copy()), O.p(mc.copy()), O.p(pyr[level].copy()),
                                 O.p(gx.copy()), O.p(gy.copy()), O.p(Rw), O.p(tw), level, O.p(out))
    blk = rows.reshape(n // 128, 128, 29).astype(np.float64)
    mine = blk.sum(axis=1)
    scale = np.abs(blk).sum(axis=1)
    assert sums[28] > 1000
    assert np.array_equal(mine[:, 28], out[:, 28])
    assert np.all(np.abs(mine - out) <= 2e-6 * scale + 1e-30)


def _rinc(a, b, g):
    ca, sa, cb, sb, cg, sg = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(g), np.sin(g)
    Rz = np.array([[cg, -sg, 0], [sg, cg, 0], [0, 0, 1]])
    Ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    Rx = np.array([[1, 0, 0], [0, ca, -sa], [0, sa, ca]])
    return Rz @ Ry @ Rx


def _cam_point(R, t, m, x):
    """Camera coordinates of world point m after the depth ICP's update with increment x."""
    Ri = _rinc(*x[:3])
    Rn = Ri.T @ R
    tn = Ri.T @ t + x[3:]
    return Rn.T @ (m - tn)


def test_camera_point_derivatives_by_central_differences():
    rng = np.random.default_rng(3)
    R = _rinc(*rng.uniform(-0.5, 0.5, 3))
    t = rng.uniform(-1, 1, 3)
    m = rng.uniform(-2, 2, 3)
    E = np.eye(3)
    analytic = [R.T @ np.cross(E[k], m) for k in range(3)] + [-R.T @ E[k] for k in range(3)]
    for k in range(6):
        h = np.zeros(6)
        h[k] = 1e-6
        fd = (_cam_point(R, t, m, h) - _cam_point(R, t, m, -h)) / 2e-6
        assert np.allclose(fd, analytic[k], atol=1e-6), k


def test_color_rows_tracker_convention_against_numpy(textured):
    H, W = textured[0][0].shape
    cam, mv, mc = _model(textured[0], W, H)
    _, bgra1, R1, t1 = textured[1]
    pyr = _pyramid(bgra1)
    level = 1
    gx, gy = _gradients(pyr[level])
    R = np.ascontiguousarray(R1, np.float32).reshape(9)
    t = np.ascontiguousarray(t1, np.float32)
    n = W * H
    rows = np.zeros((n, 29), np.float32)
    sums = np.zeros(29)
    O.oracle().orc_color_rows(O.p(mv), O.p(mc), C.byref(cam), level, O.p(pyr[level]), O.p(gx), O.p(gy), O.p(R),
                              O.p(t), 0, O.p(rows), O.p(sums))
    assert sums[28] > 1000
    Rd, td = R.reshape(3, 3).astype(np.float64), t.astype(np.float64)
    fx, fy, cx, cy = cam.fx / 2, cam.fy / 2, cam.cx / 2, cam.cy / 2
    E = np.eye(3)
    idx = np.flatnonzero(rows[:, 28] == 1)
    for i in idx[:: max(1, len(idx) // 300)]:
        m = mv.reshape(-1, 3)[i].astype(np.float64)
        p = Rd.T @ (m - td)
        u, v = int(np.round(p[0] * fx / p[2] + cx)), int(np.round(p[1] * fy / p[2] + cy))
        obs = pyr[level][v, u, :3].astype(np.float64)
        g1 = gx[v, u, :3].view(np.int8).astype(np.float64) / 255
        g2 = gy[v, u, :3].view(np.int8).astype(np.float64) / 255
        diff = (obs - mc.reshape(-1, 4)[i, :3]) / 255
        dps = [Rd.T @ np.cross(E[k], m) for k in range(3)] + [-Rd.T @ E[k] for k in range(3)]
        D = []
        for dp in dps:
            jx = fx * (p[2] * dp[0] - dp[2] * p[0]) / p[2] ** 2
            jy = fy * (p[2] * dp[1] - dp[2] * p[1]) / p[2] ** 2
            D.append(jx * g1 + jy * g2)
        want = []
        for a in range(6):
            for b in range(a, 6):
                want.append(D[a] @ D[b])
            want.append(-(D[a] @ diff))
        want += [diff @ diff, 1.0]
        want = np.array(want)
        assert np.allclose(rows[i], want, rtol=2e-4, atol=2e-4 * np.abs(want).max() + 1e-9), i
