"""Pins the oracle's shifting dense volume -- the reference's eScene_ShiftingVolume
(NuiKinfuOpenCLShiftScene) -- against the reference's own kernels compiled for the host:
integration and raycast through a voxel wrap, slab clearing (initializeVolume with an
offset) and the point fetches of extract.cl.  The scene's host logic (shiftVolume and
fetchAndClearX/Y/Z, NuiKinfuOpenCLShiftScene.cpp:235-351) is plain C++ that cannot be
built here; the engine that restates it is checked through the invariants it must keep.

One difference is deliberate.  The reference's trilinear read (interpolateTrilineary,
raycast.cl:36-120) wraps only its first voxel and reaches the other seven by adding
buffer strides, so a read that straddles the wrap seam takes voxels of the neighbouring
buffer row (or, on the last row, past the buffer's end).  The oracle -- and the CUDA path,
which keeps the volume unwrapped -- read the voxel's true neighbours.  The raycast pin runs
the oracle once with the reference's strides (bit-exact against the reference; y wrap 0, so
that the reference build never reads past its buffer) and once as the product does, which
must equal the raycast of the unwrapped volume bit for bit."""
import ctypes as C

import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import cfg_for, frames, relative_gt, same_bits

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels not built (no reference tree)")

RES = (64, 48, 40)
WRAPS = [(17, 5, 39), (0, 47, 1), (63, 0, 0)]


def _pre(raw, W, H):
    a = np.zeros(W * H, np.float32)
    O.oracle().orc_pass_filter(O.p(raw.reshape(-1)), W * H, 0.5, 4.5, O.p(a))
    return a


def _ivec(v):
    return np.ascontiguousarray(v, np.int32)


@pytest.fixture(scope="module")
def seq():
    return frames(2, W=160, H=120, seed=5)


def _integrate(seq, wrap, ref):
    """Two frames into a RES volume at voxel wrap `wrap`, by the oracle or the reference."""
    orc = O.oracle()
    W, H = 160, 120
    cam = O.OrcCam.make(W, H, 525.0 * W / 640, 525.0 * W / 640, (W - 1) / 2, (H - 1) / 2)
    tp = O.OrcTsdf.make(RES, (3.0, 3.0, 3.0), 0.03)
    nv = int(np.prod(RES))
    vol = np.zeros(nv * 2, np.int16)
    col = np.zeros(nv * 4, np.uint8)
    orc.orc_tsdf_init(O.p(vol), O.p(col), nv)
    w = _ivec(wrap)
    for raw, c, R, t in seq:
        x = O.make_xform(R, t)
        d = _pre(raw, W, H)
        orc.orc_scale_depths(O.p(d), W, H, C.byref(cam))
        bgra = np.ascontiguousarray(frames(1, W=W, H=H, seed=9, color=True)[0][1].reshape(-1))
        if ref:
            O.ref().ref_integrate_wrap(O.p(d), O.p(bgra), O.p(cam.flat()), O.p(x.flat()), O.p(vol), O.p(tp.flat()),
                                       O.p(col), 128, O.p(w))
        else:
            orc.orc_tsdf_integrate_wrap(O.p(d), O.p(bgra), C.byref(cam), C.byref(x), C.byref(tp), O.p(vol), O.p(col),
                                        128, None, O.p(w))
    return vol, col, tp, cam, x


@needs_ref
@pytest.mark.parametrize("wrap", WRAPS)
def test_integrate_through_a_wrap_matches_reference(seq, wrap):
    va, ca, _, _, _ = _integrate(seq, wrap, ref=False)
    vb, cb, _, _, _ = _integrate(seq, wrap, ref=True)
    assert np.array_equal(va, vb) and np.array_equal(ca, cb)
    assert (va[1::2] > 0).sum() > 1000
    # the wrapped volume is the unwrapped one rolled by the wrap (reference layout: index
    # (y * rx + x) * rz + z)
    v0, _, _, _, _ = _integrate(seq, (0, 0, 0), ref=False)
    rx, ry, rz = RES
    rolled = np.roll(v0.reshape(ry, rx, rz, 2), (wrap[1], wrap[0], wrap[2]), axis=(0, 1, 2))
    assert np.array_equal(rolled.reshape(-1), va)


@needs_ref
@pytest.mark.parametrize("wrap", [(17, 0, 39), (0, 0, 1), (63, 0, 0), (5, 0, 20)])
def test_raycast_through_a_wrap_matches_reference(seq, wrap):
    va, ca, tp, cam, x = _integrate(seq, wrap, ref=False)
    vb, cb, _, _, _ = _integrate(seq, wrap, ref=True)
    assert np.array_equal(va, vb)
    W, H = 160, 120
    m = [np.zeros(W * H * 3, np.float32) for _ in range(6)]
    w = _ivec(wrap)
    O.oracle().orc_raycast_wrap_mode(O.p(va), O.p(ca), C.byref(tp), C.byref(cam), C.byref(x), W, H, O.p(m[0]),
                                     O.p(m[1]), None, None, O.p(w), 1)
    O.ref().ref_raycast_wrap(O.p(vb), O.p(cb), O.p(tp.flat()), O.p(cam.flat()), O.p(x.flat()), O.p(m[2]),
                             O.p(m[3]), None, W, H, O.p(w))
    assert same_bits(m[0], m[2]) and same_bits(m[1], m[3])
    assert (~np.isnan(m[0])).mean() > 0.1
    # the product's reading: the wrapped volume raycasts exactly like the unwrapped one
    v0, c0, _, _, _ = _integrate(seq, (0, 0, 0), ref=False)
    O.oracle().orc_raycast_wrap(O.p(va), O.p(ca), C.byref(tp), C.byref(cam), C.byref(x), W, H, O.p(m[4]),
                                O.p(m[5]), None, None, O.p(w))
    O.oracle().orc_raycast(O.p(v0), O.p(c0), C.byref(tp), C.byref(cam), C.byref(x), W, H, O.p(m[0]), O.p(m[1]),
                           None, None)
    assert same_bits(m[4], m[0]) and same_bits(m[5], m[1])


@needs_ref
def test_clear_slice_matches_reference():
    rng = np.random.default_rng(4)
    nv = int(np.prod(RES))
    tp = O.OrcTsdf.make(RES, (3.0, 3.0, 3.0), 0.03)
    va = rng.integers(-30000, 30000, nv * 2).astype(np.int16)
    ca = rng.integers(0, 255, nv * 4).astype(np.uint8)
    vb, cb = va.copy(), ca.copy()
    for off, rng_ in [((60, 0, 0), (7, 48, 40)), ((0, 45, 0), (64, 5, 40)), ((0, 0, 38), (64, 48, 4))]:
        O.oracle().orc_tsdf_clear_slice(O.p(va), O.p(ca), C.byref(tp), O.p(_ivec(off)), O.p(_ivec(rng_)))
        O.ref().ref_clear_slice(O.p(vb), O.p(cb), O.p(tp.flat()), O.p(_ivec(off)), O.p(_ivec(rng_)))
        assert np.array_equal(va, vb) and np.array_equal(ca, cb)
    assert (va[1::2] == 0).sum() > 0.2 * nv


def _point_set(xyz, rgba, n):
    return np.unique(np.concatenate([xyz[:n], rgba[:n]], axis=1), axis=0)


@needs_ref
@pytest.mark.parametrize("rng_,wrap,voff", [
    ((64, 48, 40), (0, 0, 0), (0, 0, 0)),        # Volume2CLVertices of the static scene
    ((64, 48, 40), (0, 0, 0), (-81, 30, 140)),   # the shifting scene's Volume2CLVertices
    ((6, 48, 40), (29, 0, 0), (-35, 0, 0)),      # fetchAndClearX of a negative shift
    ((64, 6, 40), (0, 20, 0), (0, 20, 2)),       # fetchAndClearY
    ((64, 48, 6), (0, 0, 6), (3, -50, 6)),       # fetchAndClearZ (its z loop adds the wrap twice)
])
def test_point_fetch_matches_reference(seq, rng_, wrap, voff):
    vol, col, tp, _, _ = _integrate(seq, (0, 0, 0), ref=False)
    cap = 1 << 20
    xa, ra = np.zeros((cap, 3), np.float32), np.zeros((cap, 4), np.float32)
    xb, rb = np.zeros((cap, 3), np.float32), np.zeros((cap, 4), np.float32)
    n_a = O.oracle().orc_fetch_points(O.p(vol), O.p(col), C.byref(tp), O.p(_ivec(rng_)), O.p(_ivec(wrap)),
                                      O.p(_ivec(voff)), O.p(xa), O.p(ra), cap)
    cnt = np.zeros(1, np.int32)
    if wrap == (0, 0, 0) and voff == (0, 0, 0):
        O.ref().ref_fetch_volume(O.p(vol), O.p(col), O.p(tp.flat()), O.p(_ivec(rng_)), O.p(xb), O.p(rb), O.p(cnt))
    else:
        O.ref().ref_fetch_shift_volume(O.p(vol), O.p(col), O.p(tp.flat()), O.p(_ivec(rng_)), O.p(_ivec(wrap)),
                                       O.p(_ivec(voff)), O.p(xb), O.p(rb), O.p(cnt))
    assert n_a == int(cnt[0]) > 0
    assert np.array_equal(_point_set(xa, ra, n_a), _point_set(xb, rb, n_a))


def test_shifting_engine_keeps_the_camera_inside_and_tracks():
    """An orbiting camera (1.5 m radius, 0.5 degrees per frame) moves the 128^3 volume of
    3 m (2.3 cm voxels) with a shift of 2 voxels several times.  After every frame the local
    translation stays within the shift distance of the basis; the global translation
    (local + offset) follows the truth like a fixed volume's does; the slabs that left the
    volume gave points."""
    seq = frames(12, W=160, H=120, seed=5, deg=0.5)
    gt = relative_gt(seq)
    cell = np.float32(3.0) / np.float32(128)
    err = {}
    for vs in (0, 2):
        cfg = cfg_for(W=160, H=120, res=(128, 128, 128), dim=3.0)
        cfg.voxel_shift = vs
        cfg.shift_point_cap = 1 << 20
        eng = O.Engine(cfg)
        err[vs] = []
        for i, (d, _, _, _) in enumerate(seq):
            assert eng.frame(d), (vs, i)
            _, t = eng.pose()
            if vs:
                assert np.all(np.abs(t) < vs * cell), (i, t)
            g = t + eng.shift_state().astype(np.float32) * cell
            err[vs].append(float(np.linalg.norm(g - gt[i][1])))
        if vs:
            assert np.any(eng.shift_state() != 0)
            xyz, rgba, n = eng.points()
            assert n > 0 and len(xyz) == n and np.all(rgba[:, 3] == 1.0)
    assert max(err[2]) < max(err[0]) + 0.03, err


def test_engine_without_shift_distance_is_the_fixed_volume():
    """A shift distance larger than the motion never shifts: the shifting engine then gives
    the fixed volume's tracking outcomes, poses and volume bit for bit (this coarse
    configuration -- 4.7 cm voxels, 160 x 120 -- may lose track; both must lose it alike)."""
    seq = frames(4, W=160, H=120, seed=5)
    cfg = cfg_for(W=160, H=120, res=(64, 64, 64), dim=3.0)
    a = O.Engine(cfg)
    cfg.voxel_shift = 60
    b = O.Engine(cfg)
    tracked = 0
    for d, _, _, _ in seq:
        ra, rb = a.frame(d), b.frame(d)
        assert ra == rb
        tracked += ra
        assert np.array_equal(a.pose()[1], b.pose()[1])
    assert tracked >= 3
    assert np.array_equal(a.volume(), b.volume())
    assert np.all(b.shift_state() == 0)
