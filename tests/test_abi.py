"""The C-ABI library loads and exports every entry point its headers declare (no GPU
needed), and host-only entry points behave (config defaults, argument validation,
synthetic input generator)."""
import glob
import os
import re
import ctypes as C

import numpy as np

from natureuserinterfacestudio_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        for m in re.finditer(r"NUI_API\s+[^;{]*?\b(nui_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    names = declared_symbols()
    assert len(names) > 25
    lib = C.CDLL(L.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declarations():
    assert declared_symbols() <= set(L._SIGS)


def test_cfg_defaults_are_reference_defaults():
    c = L.default_cfg()
    assert (c.width, c.height, c.fx, c.cx) == (640, 480, 525.0, 319.5)
    assert list(c.res) == [256, 256, 256] and abs(c.dim[0] - 3.0) < 1e-6
    assert c.levels == 3 and list(c.iterations)[:3] == [10, 10, 10]
    assert c.filter_radius == 3 and abs(c.sigma_depth2_inv_half - 50.0) < 1e-6
    assert abs(c.depth_threshold - 0.3) < 1e-6 and abs(c.dist_threshold - 0.1) < 1e-6
    assert abs(c.integration_threshold - 0.15) < 1e-6 and c.max_color_weight == 128


def test_device_bytes_and_validation():
    c = L.default_cfg()
    b = L.lib().nui_session_device_bytes(C.byref(c))
    assert b >= 256 ** 3 * 4
    bad = L.default_cfg(levels=7)
    assert L.lib().nui_session_device_bytes(C.byref(bad)) == 0
    assert L.lib().nui_ctx_create(0, None) == L.NUI_ERR_INVALID_ARG


def test_synthetic_frames_are_deterministic_and_plausible():
    sc = L.SynthScene(L.SYNTH_TABLETOP, seed=2)
    R, t = sc.pose(0)
    assert np.allclose(R, np.eye(3)) and np.allclose(t, 0)
    d1, c1 = sc.render(R, t, 160, 120, fx=131.25, fy=131.25, cx=79.5, cy=59.5, frame=0, color=True)
    d2, c2 = sc.render(R, t, 160, 120, fx=131.25, fy=131.25, cx=79.5, cy=59.5, frame=0, color=True)
    assert np.array_equal(d1, d2) and np.array_equal(c1, c2)
    valid = d1[d1 > 0]
    assert 0.3 < valid.size / d1.size < 0.99
    assert valid.min() >= 400 and valid.max() <= 4500
    d3, _ = sc.render(R, t, 160, 120, fx=131.25, fy=131.25, cx=79.5, cy=59.5, frame=1)
    assert not np.array_equal(d1, d3)  # fresh noise per frame
    R5, t5 = sc.pose(45, deg_per_frame=2.0)
    # orbit: 90 degrees later the camera sits at (-r, 0, r) looking along +x
    assert np.allclose(t5, [-1.5, 0, 1.5], atol=0.01)
    room = L.SynthScene(L.SYNTH_ROOM, seed=2)
    Rr, tr = room.pose(0)
    dr, _ = room.render(Rr, tr, 160, 120, fx=131.25, fy=131.25, cx=79.5, cy=59.5)
    assert (dr > 0).mean() > 0.5
