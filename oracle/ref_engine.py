"""The reference's dense KinectFusion frame (NuiKinfuTrackingEngine::RunTracking over
NuiKinfuOpenCLScene, NuiKinfuTrackingEngine.cpp:68-142) run on the host cores with the
reference's own OpenCL kernels compiled for the host (oracle/_ref/libnui_ref.so): pass
filter, bilateral filter, vertex and half-sample pyramid, icp_block_kernel + compute_sums
per ICP iteration, scaleDepthsKernel + integrateTsdfVolumeKernel, raycastKernel, and the
frame-0 normals and world maps.  The host steps the reference writes in C++ with Eigen
(the Gaussian table, the Levenberg-Marquardt / Cholesky step of
NuiKinfuOpenCLDepthTracker::IterativeClosestPoint) come from the oracle's restatement.

Test and benchmark infrastructure: the CPU reference arm of bench.py times it.
"""
import ctypes as C

import numpy as np

from . import oracle as O

_ROWS_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                       C.POINTER(C.c_double))


class RefEngine:
    def __init__(self, session_cfg):
        c = session_cfg
        self.c = c
        self.W, self.H = c.width, c.height
        self.N = self.W * self.H
        self.cam = O.OrcCam.make(self.W, self.H, c.fx, c.fy, c.cx, c.cy, c.depth_min, c.depth_max)
        self.camf = self.cam.flat()
        self.tp = O.OrcTsdf.make(list(c.res), list(c.dim), c.trunc_dist)
        self.tpf = self.tp.flat()
        nvox = c.res[0] * c.res[1] * c.res[2]
        self.vol = np.zeros(2 * nvox, np.int16)
        O.ref().ref_init_volume(O.p(self.vol), None, O.p(self.tpf))
        self.gauss = np.zeros(2 * c.filter_radius + 1, np.float32)
        O.oracle().orc_gaussian_table(c.filter_radius, c.sigma_space2_inv_half, O.p(self.gauss))
        self.levels = c.levels
        self.iters = (C.c_int * 4)(*list(c.iterations))
        # reference maps, padded with NaN past the image (the ICP kernel's bilinear taps read
        # one row beyond it at the bottom edge)
        self.vref = np.full((self.N + self.W) * 3, np.nan, np.float32)
        self.nref = np.full((self.N + self.W) * 3, np.nan, np.float32)
        self.R = np.eye(3, dtype=np.float32)
        self.t = np.zeros(3, np.float32)
        self.frames = 0
        step = np.float32(c.dist_threshold) / np.float32(c.levels)
        self.dist_thr = float(np.float32(c.dist_threshold) + step)
        O.oracle().orc_icp_with_rows.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, _ROWS_FN, C.c_void_p]
        O.oracle().orc_icp_with_rows.restype = C.c_int

    def _preprocess(self, raw):
        W, H, c = self.W, self.H, self.c
        ref = O.ref()
        d = np.zeros(self.N, np.float32)
        ref.ref_pass_filter(O.p(np.ascontiguousarray(raw).reshape(-1)), O.p(d), self.N, c.depth_min, c.depth_max)
        f = np.zeros(self.N, np.float32)
        ref.ref_bilateral(O.p(d), O.p(f), O.p(self.gauss), W, H, c.filter_radius, c.sigma_depth2_inv_half,
                          c.depth_threshold)
        levels = []
        src = f
        for l in range(self.levels):
            w, h = W >> l, H >> l
            if l > 0:
                dst = np.zeros(w * h, np.float32)
                ref.ref_half_sample(O.p(src), O.p(dst), w, h, 1, c.depth_threshold)
                src = dst
            v = np.zeros(w * h * 3, np.float32)
            ref.ref_depth2vertex(O.p(src), O.p(v), O.p(self.camf), w, h, 1 << l)
            levels.append(v)
        return d, levels

    def _integrate(self, d):
        s = d.copy()
        O.ref().ref_scale_depths(O.p(s), O.p(self.camf), self.W, self.H)
        xf = O.make_xform(self.R, self.t).flat()
        O.ref().ref_integrate(O.p(s), None, O.p(self.camf), O.p(xf), O.p(self.vol), O.p(self.tpf), None, 0)

    def _raycast(self):
        xf = O.make_xform(self.R, self.t).flat()
        O.ref().ref_raycast(O.p(self.vol), None, O.p(self.tpf), O.p(self.camf), O.p(xf), O.p(self.vref),
                            O.p(self.nref), None, self.W, self.H)

    def frame(self, raw):
        """One frame; False when tracking is lost (the frame then changes nothing)."""
        d, levels = self._preprocess(raw)
        W, H = self.W, self.H
        if self.frames == 0:
            n0 = np.zeros(self.N * 3, np.float32)
            O.ref().ref_normals_simple(O.p(levels[0]), O.p(n0), W, H, self.c.depth_threshold)
            xf = O.make_xform(self.R, self.t).flat()
            O.ref().ref_transform_maps(O.p(levels[0]), O.p(n0), O.p(self.vref), O.p(self.nref), O.p(xf), W, H)
            self._integrate(d)
            self.frames += 1
            return True
        prev = O.make_xform(self.R, self.t).flat()
        out29 = np.zeros(29, np.float32)

        def rows(user, lv, Rp, tp, sums):
            Rm = np.ctypeslib.as_array(Rp, shape=(9,)).copy()
            tv = np.ctypeslib.as_array(tp, shape=(3,)).copy()
            O.ref().ref_icp_iteration(O.p(self.camf), O.p(levels[lv]), W >> lv, H >> lv, O.p(Rm), O.p(tv),
                                      O.p(self.vref), O.p(self.nref), O.p(prev), self.dist_thr, O.p(out29))
            for k in range(29):
                sums[k] = float(out29[k])

        R = np.ascontiguousarray(self.R, np.float32).reshape(-1).copy()
        t = np.ascontiguousarray(self.t, np.float32).copy()
        st = O.OrcIcpStats()
        r = O.oracle().orc_icp_with_rows(self.iters, self.levels, C.byref(self.cam), O.p(R), O.p(t), C.byref(st),
                                         _ROWS_FN(rows), None)
        if r != 0:
            return False
        self.R, self.t = R.reshape(3, 3), t
        self._integrate(d)  # integration gate 0: every tracked frame integrates
        self._raycast()
        self.frames += 1
        return True

    def pose(self):
        return self.R.copy(), self.t.copy()
