"""Seeded synthetic RGB-D input (libnui_synth.so): analytic scenes, camera trajectories and
a Kinect-like renderer with the noise model sigma(z) = 0.0012 + 0.0019 (z - 0.4)^2 m, 1 mm
quantisation and 2 % dropouts.  Input generation for the tests and the benchmark; it never
loads the product library."""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SYNTH_PATH = os.path.join(_HERE, "libnui_synth.so")

SYNTH_TABLETOP, SYNTH_ROOM = 0, 1

_P = C.c_void_p
_SIGS = {
    "nui_synth_scene_create": (_P, [C.c_int, C.c_uint64, C.c_float]),
    "nui_synth_scene_destroy": (None, [_P]),
    "nui_synth_scene_sdf": (C.c_float, [_P, C.c_float, C.c_float, C.c_float]),
    "nui_synth_scene_sdf_many": (None, [_P, _P, C.c_long, _P]),
    "nui_synth_trajectory": (None, [C.c_int, C.c_uint64, C.c_int, C.c_float, C.c_float, _P, _P]),
    "nui_synth_render": (None, [_P, _P, _P, C.c_int, C.c_int] + [C.c_float] * 4 + [C.c_uint64, C.c_int, C.c_int, _P, _P]),
}
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SYNTH_PATH):
            from .. import build as B
            B.build_synth()
        L = C.CDLL(SYNTH_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


class SynthScene:
    def __init__(self, kind=SYNTH_TABLETOP, seed=1, extent=3.0):
        self.h = lib().nui_synth_scene_create(kind, seed, extent)
        self.kind = kind
        self.seed = seed

    def __del__(self):
        try:
            if self.h:
                lib().nui_synth_scene_destroy(self.h)
        except Exception:
            pass

    def sdf(self, x, y, z):
        return lib().nui_synth_scene_sdf(self.h, x, y, z)

    def sdf_many(self, xyz):
        p = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        out = np.zeros(len(p), np.float32)
        lib().nui_synth_scene_sdf_many(self.h, _ptr(p), len(p), _ptr(out))
        return out

    def pose(self, frame, radius=1.5, deg_per_frame=2.0, traj_seed=None):
        R = np.zeros(9, np.float32)
        t = np.zeros(3, np.float32)
        lib().nui_synth_trajectory(self.kind, self.seed if traj_seed is None else traj_seed, frame, radius,
                                   deg_per_frame, _ptr(R), _ptr(t))
        return R.reshape(3, 3), t

    def render(self, R, t, W=640, H=480, fx=525.0, fy=525.0, cx=319.5, cy=239.5, noise_seed=7, frame=0,
               noise=True, color=False):
        d = np.zeros((H, W), np.uint16)
        c = np.zeros((H, W, 4), np.uint8) if color else None
        Rf = np.ascontiguousarray(R, np.float32).reshape(9)
        tf = np.ascontiguousarray(t, np.float32).reshape(3)
        lib().nui_synth_render(self.h, _ptr(Rf), _ptr(tf), W, H, fx, fy, cx, cy, noise_seed, frame,
                               1 if noise else 0, _ptr(d), _ptr(c))
        return d, c
