"""Pins the oracle's global cache of the voxel hash -- NuiKinfuOpenCLHashGlobalCache, the
host-side store that blocks leaving the view swap out to and back in from
(KinfuHashSwapping.cl) -- against the reference's own kernels compiled for the host, run
one work-item at a time, with the host half of the cache restated in the launcher.

The camera turns away from the scene and back, so that blocks leave the view, are merged,
swapped out (cleared, their blocks returned to the free list), and later come back and are
merged with their stored copies.  After every frame: the same visible list, hash entries,
voxels, swap states, free-list counters and stored blocks."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference kernels not built (no reference tree)")


@needs_ref
def test_global_cache_matches_reference():
    W, H = 96, 72
    f = 525.0 * W / 640
    cx, cy = (W - 1) / 2.0, (H - 1) / 2.0
    sc = L.SynthScene(L.SYNTH_ROOM, seed=5)
    cam = O.OrcCam.make(W, H, f, f, cx, cy, 0.4, 4.5)
    rh = O.RefHash(voxel=0.02, mu=0.08, swapping=True)
    oh = O.OracleHash(rh.buckets, rh.excess, rh.pool, voxel=0.02, mu=0.08, swapping=True)
    # orbit frames: out and back (blocks leave the view and return)
    path = [0, 20, 40, 60, 40, 20, 0]
    swapped_out = stored_back = 0
    for k, i in enumerate(path):
        R, t = sc.pose(i, radius=1.5, deg_per_frame=2.0)
        raw, bgra = sc.render(R, t, W, H, fx=f, fy=f, cx=cx, cy=cy, frame=k, color=True)
        d = np.zeros(W * H, np.float32)
        O.oracle().orc_pass_filter(O.p(raw.reshape(-1)), W * H, 0.4, 4.5, O.p(d))
        x = O.make_xform(R, t)
        b = np.ascontiguousarray(bgra.reshape(-1))
        nr = rh.frame(d, b, cam, x)
        oh.allocate(d, cam, x)
        oh.integrate(d, b, cam, x)
        oh.swap()
        assert nr == oh.visible().size, k
        assert np.array_equal(rh.visible(), oh.visible()), k
        assert np.array_equal(rh.entries.view(np.uint8), oh.entries().view(np.uint8)), k
        sdf, w, rgb = oh.voxels()
        assert np.array_equal(rh.voxels["sdf"], sdf), k
        assert np.array_equal(rh.voxels["w"], w), k
        assert np.array_equal(rh.voxels["rgb"], rgb), k
        assert np.array_equal(rh.swap_states, oh.swap_states()), k
        lb, le, _ = oh.counters()
        assert [lb, le] == list(rh.last), k
        ids = np.nonzero(rh.has_stored)[0]
        assert ids.size == oh.stored_count(), k
        st = rh.store.reshape(-1, 512)
        for e in ids:
            o = oh.stored(e)
            assert o is not None
            assert np.array_equal(st[e]["sdf"], o[0]) and np.array_equal(st[e]["w"], o[1])
            assert np.array_equal(st[e]["rgb"], o[2])
        swapped_out = max(swapped_out, ids.size)
        stored_back += int(np.sum((oh.swap_states() == 2) & (rh.has_stored > 0)))
    assert swapped_out > 100  # blocks left the view and went to the host
    assert stored_back > 0    # and some came back and merged with their stored copies
