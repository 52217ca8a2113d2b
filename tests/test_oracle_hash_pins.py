"""Pins the voxel-hash oracle against the reference's own hash kernels (KinfuHashScene.cl,
KinfuHashRaycast.cl, KinfuHashVisualization.cl compiled for the host with test-sized tables
and run one work-item at a time, which resolves the kernels' races in raster order)."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import same_bits

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels not built (no reference tree)")


def _run(kind, W, H, frames, mesh):
    f = 525.0 * W / 640
    cx, cy = (W - 1) / 2.0, (H - 1) / 2.0
    sc = L.SynthScene(kind, seed=5)
    cam = O.OrcCam.make(W, H, f, f, cx, cy, 0.4, 4.5)
    rh = O.RefHash()
    oh = O.OracleHash(rh.buckets, rh.excess, rh.pool)
    for fr in range(frames):
        R, t = sc.pose(fr * 5)
        raw, bgra = sc.render(R, t, W, H, fx=f, fy=f, cx=cx, cy=cy, frame=fr, color=True)
        d = np.zeros(W * H, np.float32)
        O.oracle().orc_pass_filter(O.p(raw.reshape(-1)), W * H, 0.4, 4.5, O.p(d))
        x = O.make_xform(R, t)
        b = np.ascontiguousarray(bgra.reshape(-1))
        nr = rh.frame(d, b, cam, x)
        no = oh.allocate(d, cam, x)
        oh.integrate(d, b, cam, x)
        assert nr == no > 0
        assert np.array_equal(rh.visible(), oh.visible())
        assert np.array_equal(rh.entries.view(np.uint8), oh.entries().view(np.uint8))
        sdf, w, rgb = oh.voxels()
        assert np.array_equal(rh.voxels["sdf"], sdf)
        assert np.array_equal(rh.voxels["w"], w)
        assert np.array_equal(rh.voxels["rgb"], rgb)
        lb, le, _ = oh.counters()
        assert [lb, le] == list(rh.last)
        vr, nr_, cr, rgr = rh.raycast(cam, x, color=True)
        vo, no_, co, rgo = oh.raycast(cam, x, color=True)
        assert same_bits(rgr, rgo) and same_bits(vr, vo) and same_bits(nr_, no_) and np.array_equal(cr, co)
        assert (~np.isnan(vo)).mean() > 0.5
        xr, cr_, n_r = rh.fetch()  # fetchHashScene_kernel, in the sequential order
        xo, co_, n_o = oh.fetch()
        assert n_r == n_o > 0 and same_bits(xr, xo) and same_bits(cr_, co_)
        if mesh:
            pr, colr, n_r = rh.mesh()
            po, colo, n_o = oh.mesh(5_000_000)
            assert n_r == n_o > 0
            assert same_bits(pr, po) and same_bits(colr, colo)


@needs_ref
def test_hash_alloc_integrate_raycast_room_matches_reference():
    _run(L.SYNTH_ROOM, 160, 120, 2, mesh=False)


@needs_ref
def test_hash_pipeline_with_mesh_matches_reference():
    _run(L.SYNTH_TABLETOP, 64, 48, 2, mesh=True)


@needs_ref
def test_hash_forward_render_matches_reference():
    """The forward-render path of the hash scene (ForwardRender: forwardProject_kernel,
    findMissingPoints_kernel, genericRaycastMissingPoints_kernel, then the simple normals)
    from the previous frame's maps: landed vertices, missing flags, cast vertices and the
    normals bit for bit; colours where a vertex exists (the reference copies colours within
    one buffer while it reads it, so the input colours are uniform here)."""
    W, H = 160, 120
    f = 525.0 * W / 640
    cx, cy = (W - 1) / 2.0, (H - 1) / 2.0
    sc = L.SynthScene(L.SYNTH_ROOM, seed=5)
    cam = O.OrcCam.make(W, H, f, f, cx, cy, 0.4, 4.5)
    rh = O.RefHash()
    oh = O.OracleHash(rh.buckets, rh.excess, rh.pool)
    vprev = None
    landed_total = 0
    for fr in range(3):
        R, t = sc.pose(fr * 3)
        raw, bgra = sc.render(R, t, W, H, fx=f, fy=f, cx=cx, cy=cy, frame=fr, color=True)
        d = np.zeros(W * H, np.float32)
        O.oracle().orc_pass_filter(O.p(raw.reshape(-1)), W * H, 0.4, 4.5, O.p(d))
        x = O.make_xform(R, t)
        b = np.ascontiguousarray(bgra.reshape(-1))
        rh.frame(d, b, cam, x)
        oh.allocate(d, cam, x)
        oh.integrate(d, b, cam, x)
        if vprev is None:
            vprev = oh.raycast(cam, x, color=True)[0]
            continue
        cprev = np.tile(np.array([10, 20, 30, 255], np.uint8), W * H)
        vr, cr, rgr, flr, nr = rh.forward_render(cam, x, vprev, cprev)
        vo, no, co, rgo, flo, n_o = oh.forward_render(cam, x, vprev, cprev, color=True)
        assert nr == n_o > 0 and np.array_equal(flr, flo)
        assert same_bits(rgr, rgo) and same_bits(vr, vo)
        nref = np.zeros(W * H * 3, np.float32)
        O.ref().ref_normals_simple(O.p(vr), O.p(nref), W, H, 0.3)
        assert same_bits(nref, no)
        valid = ~np.isnan(vo.reshape(-1, 3)[:, 0])
        assert np.array_equal(cr.reshape(-1, 4)[valid], co.reshape(-1, 4)[valid])
        landed_total += int(np.sum(valid & (flo == 0)))
        vprev = vo
    assert landed_total > 1000  # vertices carried forward, not only cast
