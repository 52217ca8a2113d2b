"""ctypes access to the CPU oracle (libnui_oracle.so) and to the reference's own kernels
compiled for the host (oracle/_ref/libnui_ref.so).  Test infrastructure: imported only by
tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libnui_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libnui_ref.so")
# where the reference source tree is read from when oracle/_ref is built (NUI_REFERENCE_TREE)
REFERENCE_TREE = os.environ.get("NUI_REFERENCE_TREE", "/root/reference")

_P = C.c_void_p


def build(reference=True):
    """Compile the oracle (always) and, when the reference tree is present, oracle/_ref."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if reference and os.path.isdir(os.path.join(REFERENCE_TREE, "src", "Kernels")):
        subprocess.run(["python", os.path.join(HERE, "build_ref.py"), "--reference", REFERENCE_TREE], check=True,
                       stdout=subprocess.DEVNULL)


def p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(_P)


class OrcCam(C.Structure):
    _fields_ = [("fx", C.c_float), ("fy", C.c_float), ("fx_inv", C.c_float), ("fy_inv", C.c_float),
                ("cx", C.c_float), ("cy", C.c_float), ("W", C.c_uint32), ("H", C.c_uint32),
                ("dmin", C.c_float), ("dmax", C.c_float)]

    @staticmethod
    def make(W, H, fx=525.0, fy=525.0, cx=319.5, cy=239.5, dmin=0.5, dmax=4.5):
        f32 = np.float32
        return OrcCam(f32(fx), f32(fy), f32(1) / f32(fx), f32(1) / f32(fy), f32(cx), f32(cy), W, H, f32(dmin), f32(dmax))

    def flat(self):
        return np.array([self.fx, self.fy, self.fx_inv, self.fy_inv, self.cx, self.cy, self.W, self.H, self.dmin,
                         self.dmax], np.float32)


class OrcXform(C.Structure):
    _fields_ = [("R", C.c_float * 9), ("R_inv", C.c_float * 9), ("t", C.c_float * 3)]

    def flat(self):
        return np.array(list(self.R) + list(self.R_inv) + list(self.t), np.float32)


class OrcTsdf(C.Structure):
    _fields_ = [("res", C.c_float * 3), ("dim", C.c_float * 3), ("cell", C.c_float * 3), ("trunc", C.c_float)]

    @staticmethod
    def make(res, dim, trunc_cfg):
        t = OrcTsdf()
        cells = []
        for i in range(3):
            t.res[i] = float(res[i])
            t.dim[i] = float(dim[i])
            c = np.float32(dim[i]) / np.float32(res[i])
            t.cell[i] = float(c)
            cells.append(c)
        t.trunc = float(max(np.float32(trunc_cfg), np.float32(2.1) * max(cells)))
        return t

    def flat(self):
        return np.array(list(self.res) + list(self.dim) + list(self.cell) + [self.trunc], np.float32)


class OrcIcpStats(C.Structure):
    _fields_ = [("error", C.c_float), ("count", C.c_float), ("iterations", C.c_int), ("status", C.c_int)]


class OrcEngineCfg(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float),
                ("cy", C.c_float), ("dmin", C.c_float), ("dmax", C.c_float), ("res", C.c_int * 3),
                ("dim", C.c_float * 3), ("trunc_cfg", C.c_float), ("color", C.c_int), ("max_color_weight", C.c_int),
                ("levels", C.c_int), ("iters", C.c_int * 4), ("filter_radius", C.c_int),
                ("sigma_space2_inv_half", C.c_float), ("sigma_depth2_inv_half", C.c_float),
                ("depth_threshold", C.c_float), ("dist_threshold", C.c_float), ("integration_threshold", C.c_float),
                ("hash", C.c_int), ("voxel", C.c_float), ("mu", C.c_float), ("buckets", C.c_int), ("excess", C.c_int),
                ("pool", C.c_int), ("max_w", C.c_int), ("photometric_weight", C.c_float),
                ("voxel_shift", C.c_int), ("shift_basis", C.c_float * 3), ("point_cap", C.c_long),
                ("swapping", C.c_int), ("forward_render", C.c_int)]

    @staticmethod
    def from_session_cfg(c):
        e = OrcEngineCfg()
        e.W, e.H = c.width, c.height
        e.fx, e.fy, e.cx, e.cy = c.fx, c.fy, c.cx, c.cy
        e.dmin, e.dmax = c.depth_min, c.depth_max
        for i in range(3):
            e.res[i] = c.res[i]
            e.dim[i] = c.dim[i]
        e.trunc_cfg = c.trunc_dist
        e.color = c.color_volume
        e.max_color_weight = c.max_color_weight
        e.levels = c.levels
        for i in range(4):
            e.iters[i] = c.iterations[i]
        e.filter_radius = c.filter_radius
        e.sigma_space2_inv_half = c.sigma_space2_inv_half
        e.sigma_depth2_inv_half = c.sigma_depth2_inv_half
        e.depth_threshold = c.depth_threshold
        e.dist_threshold = c.dist_threshold
        e.integration_threshold = c.integration_threshold
        e.hash = 1 if c.volume_kind == 1 else 0
        e.voxel, e.mu = c.voxel_size, c.trunc_scale
        e.buckets, e.excess, e.pool, e.max_w = c.hash_buckets, c.hash_excess, c.hash_pool_blocks, c.hash_max_weight
        e.photometric_weight = getattr(c, "photometric_weight", 0.0)
        e.voxel_shift = getattr(c, "voxel_shift", 0)
        for i in range(3):
            e.shift_basis[i] = c.shift_basis[i] if hasattr(c, "shift_basis") else 0.0
        e.point_cap = getattr(c, "shift_point_cap", 0)
        e.forward_render = getattr(c, "hash_forward_render", 0)
        e.swapping = getattr(c, "hash_swapping", 0)
        return e


_orc = None
_ref = None


def oracle():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            build(reference=False)
        L = C.CDLL(ORACLE_SO)
        sig = {
            "oracle_expf": (C.c_float, [C.c_float]),
            "orc_pass_filter": (None, [_P, C.c_long, C.c_float, C.c_float, _P]),
            "orc_gaussian_table": (None, [C.c_int, C.c_float, _P]),
            "orc_bilateral": (None, [_P, C.c_int, C.c_int, _P, C.c_int, C.c_float, C.c_float, _P]),
            "orc_half_sample": (None, [_P, C.c_int, C.c_int, C.c_int, C.c_float, _P]),
            "orc_depth2vertex": (None, [_P, C.c_int, C.c_int, _P, C.c_int, _P]),
            "orc_normals": (None, [_P, C.c_int, C.c_int, C.c_float, _P]),
            "orc_transform_maps": (None, [_P, _P, C.c_int, C.c_int, _P, _P, _P]),
            "orc_scale_depths": (None, [_P, C.c_int, C.c_int, _P]),
            "orc_tsdf_init": (None, [_P, _P, C.c_long]),
            "orc_tsdf_integrate": (None, [_P, _P, _P, _P, _P, _P, _P, C.c_int, _P]),
            "orc_raycast": (None, [_P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P, _P]),
            "orc_tsdf_integrate_wrap": (None, [_P, _P, _P, _P, _P, _P, _P, C.c_int, _P, _P]),
            "orc_raycast_wrap": (None, [_P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P, _P, _P]),
            "orc_raycast_wrap_mode": (None, [_P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P, _P, _P, _P, C.c_int]),
            "orc_raycast_values": (None, [_P, _P, _P, _P, _P, C.c_int, C.c_int, _P, _P]),
            "orc_tsdf_clear_slice": (None, [_P, _P, _P, _P, _P]),
            "orc_fetch_points": (C.c_long, [_P, _P, _P, _P, _P, _P, _P, _P, C.c_long]),
            "orc_engine_shift_state": (None, [_P, _P]),
            "orc_engine_points": (C.c_long, [_P, _P, _P, C.c_long]),
            "orc_engine_integrate_at": (None, [_P, _P, _P, _P, _P]),
            "orc_icp_rows": (None, [_P, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P, C.c_float, _P, _P]),
            "orc_inverse3": (None, [_P, _P]),
            "orc_make_xform": (None, [_P, _P, _P]),
            "orc_icp": (C.c_int, [_P, _P, C.c_int, _P, _P, _P, _P, C.c_float, _P, _P, _P, _P]),
            "orc_color_half_sample": (None, [_P, C.c_int, C.c_int, C.c_int, _P]),
            "orc_color_gradient": (None, [_P, C.c_int, C.c_int, _P, _P]),
            "orc_color_rows": (None, [_P, _P, _P, C.c_int, _P, _P, _P, _P, _P, C.c_int, _P, _P]),
            "orc_marching_cubes": (C.c_long, [_P, _P, _P, _P, _P, _P, C.c_long]),
            "orc_scan_compact": (C.c_long, [_P, C.c_long, _P, _P]),
            "orc_engine_create": (_P, [_P]),
            "orc_engine_destroy": (None, [_P]),
            "orc_engine_frame": (C.c_int, [_P, _P, _P]),
            "orc_engine_pose": (None, [_P, _P, _P]),
            "orc_engine_volume": (_P, [_P]),
            "orc_engine_color_volume": (_P, [_P]),
            "orc_engine_refmap": (_P, [_P, C.c_int]),
            "orc_engine_tsdf_params": (None, [_P, _P]),
            "orc_engine_icp_stats": (None, [_P, _P]),
            "orc_engine_touched": (C.c_long, [_P]),
            "orc_engine_hash": (_P, [_P]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _orc = L
    return _orc


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError("oracle/_ref/libnui_ref.so is not built (needs the reference tree)")
        L = C.CDLL(REF_SO)
        sig = {
            "ref_pass_filter": (None, [_P, _P, C.c_long, C.c_float, C.c_float]),
            "ref_bilateral": (None, [_P, _P, _P, C.c_int, C.c_int, C.c_uint, C.c_float, C.c_float]),
            "ref_depth2vertex": (None, [_P, _P, _P, C.c_int, C.c_int, C.c_int]),
            "ref_half_sample": (None, [_P, _P, C.c_int, C.c_int, C.c_uint, C.c_float]),
            "ref_transform_maps": (None, [_P, _P, _P, _P, _P, C.c_int, C.c_int]),
            "ref_normals_simple": (None, [_P, _P, C.c_int, C.c_int, C.c_float]),
            "ref_scale_depths": (None, [_P, _P, C.c_int, C.c_int]),
            "ref_integrate": (None, [_P, _P, _P, _P, _P, _P, _P, C.c_uint8]),
            "ref_init_volume": (None, [_P, _P, _P]),
            "ref_raycast": (None, [_P, _P, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int]),
            "ref_integrate_wrap": (None, [_P, _P, _P, _P, _P, _P, _P, C.c_uint8, _P]),
            "ref_raycast_wrap": (None, [_P, _P, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int, _P]),
            "ref_clear_slice": (None, [_P, _P, _P, _P, _P]),
            "ref_fetch_volume": (None, [_P, _P, _P, _P, _P, _P, _P]),
            "ref_fetch_shift_volume": (None, [_P, _P, _P, _P, _P, _P, _P, _P, _P]),
            "ref_marching_cubes": (C.c_int, [_P, _P, _P, _P, _P]),
            "ref_icp_iteration": (None, [_P, _P, C.c_int, C.c_int, _P, _P, _P, _P, _P, C.c_float, _P]),
            "ref_half_sample_bgra": (None, [_P, _P, C.c_int, C.c_int, C.c_uint]),
            "ref_bgra_gradient": (None, [_P, _P, _P, C.c_int, C.c_int]),
            "ref_color_icp_blocks": (None, [_P, _P, _P, _P, _P, _P, _P, _P, C.c_int, _P]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _ref = L
    return _ref


def make_xform(R, t):
    x = OrcXform()
    Rf = np.ascontiguousarray(R, np.float32).reshape(9)
    tf = np.ascontiguousarray(t, np.float32).reshape(3)
    oracle().orc_make_xform(p(Rf), p(tf), C.byref(x))
    return x


class Engine:
    """The oracle's frame driver (RunTracking over the dense scene)."""

    def __init__(self, session_cfg):
        self.cfg = OrcEngineCfg.from_session_cfg(session_cfg)
        self.h = oracle().orc_engine_create(C.byref(self.cfg))
        t = OrcTsdf()
        oracle().orc_engine_tsdf_params(self.h, C.byref(t))
        self.tsdf = t
        self.nvox = session_cfg.res[0] * session_cfg.res[1] * session_cfg.res[2]
        self.W, self.H = session_cfg.width, session_cfg.height

    def __del__(self):
        try:
            oracle().orc_engine_destroy(self.h)
        except Exception:
            pass

    def frame(self, depth, bgra=None):
        return oracle().orc_engine_frame(self.h, p(depth), p(bgra)) == 0

    def pose(self):
        R = np.zeros(9, np.float32)
        t = np.zeros(3, np.float32)
        oracle().orc_engine_pose(self.h, p(R), p(t))
        return R.reshape(3, 3), t

    def volume(self):
        ptr_ = oracle().orc_engine_volume(self.h)
        return np.ctypeslib.as_array(C.cast(ptr_, C.POINTER(C.c_int16)), shape=(self.nvox, 2)).copy()

    def integrate_at(self, depth, R, t, bgra=None):
        """A frame at the given pose without tracking: integrate (shifting first) and raycast."""
        Rf = np.ascontiguousarray(R, np.float32).reshape(9)
        tf = np.ascontiguousarray(t, np.float32).reshape(3)
        oracle().orc_engine_integrate_at(self.h, p(depth), p(bgra), p(Rf), p(tf))

    def color_volume(self):
        ptr_ = oracle().orc_engine_color_volume(self.h)
        if not ptr_:
            return None
        return np.ctypeslib.as_array(C.cast(ptr_, C.POINTER(C.c_uint8)), shape=(self.nvox, 4)).copy()

    def shift_state(self):
        """The shifting volume's voxel offset (m_voxel_offset)."""
        v = np.zeros(3, np.int32)
        oracle().orc_engine_shift_state(self.h, p(v))
        return v

    def points(self, cap=1 << 22):
        """(xyz[n, 3], rgba[n, 4], found) of the slabs that left the shifting volume."""
        xyz = np.zeros((cap, 3), np.float32)
        rgba = np.zeros((cap, 4), np.float32)
        n = oracle().orc_engine_points(self.h, p(xyz), p(rgba), cap)
        k = min(n, cap, int(self.cfg.point_cap))
        return xyz[:k].copy(), rgba[:k].copy(), n

    def refmap(self, which):
        ptr_ = oracle().orc_engine_refmap(self.h, which)
        return np.ctypeslib.as_array(C.cast(ptr_, C.POINTER(C.c_float)), shape=(self.H, self.W, 3)).copy()

    def icp_stats(self):
        s = OrcIcpStats()
        oracle().orc_engine_icp_stats(self.h, C.byref(s))
        return s

    def touched(self):
        return oracle().orc_engine_touched(self.h)

    def hash_scene(self):
        """The engine's OracleHash view (hash sessions only)."""
        h = OracleHash.__new__(OracleHash)
        _bind(oracle(), _hash_sigs)
        c = self.cfg
        h.cfg = OrcHashCfg(c.buckets, c.excess, c.pool, c.buckets - 1, c.voxel, c.mu, c.max_w, c.swapping)
        h.h = oracle().orc_engine_hash(self.h)
        h.n_entries = c.buckets + c.excess
        h._borrowed = True
        return h


# ------------------------------------------------------------------ voxel-block hashing
class OrcHashCfg(C.Structure):
    _fields_ = [("buckets", C.c_int), ("excess", C.c_int), ("pool", C.c_int), ("mask", C.c_uint32),
                ("voxel", C.c_float), ("mu", C.c_float), ("max_w", C.c_int), ("swapping", C.c_int)]


HASH_ENTRY = np.dtype([("pos", np.int16, 3), ("pad", np.int16), ("ptr", np.int32), ("offset", np.uint32)])
REF_VOXEL = np.dtype([("sdf", np.int16), ("rgb", np.uint8, 3), ("w", np.uint8)])

_hash_sigs = {
    "orc_hash_create": (_P, [_P]),
    "orc_hash_destroy": (None, [_P]),
    "orc_hash_reset": (None, [_P]),
    "orc_hash_allocate": (C.c_long, [_P, _P, _P, _P]),
    "orc_hash_integrate": (None, [_P, _P, _P, _P, _P, _P]),
    "orc_hash_raycast": (None, [_P, _P, _P, _P, _P, _P, _P]),
    "orc_hash_forward_render": (C.c_long, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.c_int]),
    "orc_hash_mesh": (C.c_long, [_P, _P, _P, C.c_long]),
    "orc_hash_fetch_points": (C.c_long, [_P, _P, _P, C.c_long]),
    "orc_hash_visible": (C.c_long, [_P, _P, C.c_long]),
    "orc_hash_entries": (_P, [_P]),
    "orc_hash_sdf": (_P, [_P]),
    "orc_hash_weight": (_P, [_P]),
    "orc_hash_rgb": (_P, [_P]),
    "orc_hash_counters": (None, [_P, _P, _P, _P]),
    "orc_hash_swap": (None, [_P]),
    "orc_hash_swap_states": (_P, [_P]),
    "orc_hash_stored": (C.c_int, [_P, C.c_int, _P, _P, _P]),
    "orc_hash_stored_count": (C.c_long, [_P]),
    "orc_hash_stored_ids": (C.c_long, [_P, _P, C.c_long]),
}
_ref_hash_sigs = {
    "ref_hash_sizes": (None, [_P, _P, _P]),
    "ref_hash_reset": (None, [_P, _P, _P, _P, _P, _P]),
    "ref_hash_frame": (None, [_P] * 15 + [C.c_float, C.c_float, C.c_int, C.c_int]),
    "ref_hash_raycast": (None, [_P, _P, _P, C.c_int, _P, _P, C.c_float, C.c_float, _P, _P, _P, _P]),
    "ref_hash_forward_render": (C.c_int, [_P, _P, _P, C.c_int, _P, _P, C.c_float, C.c_float, _P, _P, _P, _P, _P]),
    "ref_hash_mesh": (C.c_int, [_P, _P, _P, C.c_int, C.c_float, _P, _P]),
    "ref_hash_fetch": (C.c_int, [_P, _P, _P, C.c_int, C.c_float, C.c_float, _P, _P]),
    "ref_hash_alloc_swap": (None, [_P] * 13 + [C.c_float, C.c_float, _P]),
    "ref_hash_integrate_visible": (None, [_P, _P, _P, C.c_int, _P, _P, _P, _P, C.c_float, C.c_float, C.c_int]),
    "ref_hash_realloc": (None, [_P, _P, _P, _P]),
    "ref_hash_global_cache": (None, [_P, _P, _P, _P, _P, _P, C.c_int, _P, _P]),
}


def _bind(L, sigs):
    for k, (r, a) in sigs.items():
        f = getattr(L, k)
        f.restype = r
        f.argtypes = a


class OracleHash:
    """The oracle's voxel-block hash scene."""

    def __init__(self, buckets, excess, pool, voxel=0.005, mu=0.02, max_w=255, mask=None, swapping=False):
        L = oracle()
        _bind(L, _hash_sigs)
        self.cfg = OrcHashCfg(buckets, excess, pool, (buckets - 1) if mask is None else mask, voxel, mu, max_w,
                              1 if swapping else 0)
        self.h = L.orc_hash_create(C.byref(self.cfg))
        self.n_entries = buckets + excess

    def __del__(self):
        try:
            if not getattr(self, "_borrowed", False):
                oracle().orc_hash_destroy(self.h)
        except Exception:
            pass

    def allocate(self, depth, cam, xform):
        return oracle().orc_hash_allocate(self.h, p(depth), C.byref(cam), C.byref(xform))

    def integrate(self, depth, bgra, cam, xform):
        t = C.c_long()
        oracle().orc_hash_integrate(self.h, p(depth), p(bgra), C.byref(cam), C.byref(xform), C.byref(t))
        return t.value

    def raycast(self, cam, xform, color=False):
        N = cam.W * cam.H
        vm = np.zeros(N * 3, np.float32)
        nm = np.zeros(N * 3, np.float32)
        cm = np.zeros(N * 4, np.uint8) if color else None
        rg = np.zeros(N * 2, np.float32)
        oracle().orc_hash_raycast(self.h, C.byref(cam), C.byref(xform), p(vm), p(nm), p(cm), p(rg))
        return vm, nm, cm, rg

    def forward_render(self, cam, xform, vprev, cprev=None, color=False, mode=1):
        """ForwardRender of the hash scene from the previous world vertex map (N x 3 floats) and
        colours (N x 4 bytes): (vmap, nmap, cmap, range, missing flags, missing count)."""
        N = cam.W * cam.H
        vm = np.zeros(N * 3, np.float32)
        nm = np.zeros(N * 3, np.float32)
        cm = np.zeros(N * 4, np.uint8) if color else None
        rg = np.zeros(N * 2, np.float32)
        miss = np.zeros(N, np.uint8)
        vp = np.ascontiguousarray(vprev, np.float32).reshape(-1)
        cp = None if cprev is None else np.ascontiguousarray(cprev, np.uint8).reshape(-1)
        n = oracle().orc_hash_forward_render(self.h, C.byref(cam), C.byref(xform), p(vp), p(cp), p(vm), p(nm), p(cm),
                                             p(rg), p(miss), mode)
        return vm, nm, cm, rg, miss, n

    def mesh(self, cap):
        pos = np.zeros((cap, 3), np.float32)
        col = np.zeros((cap, 4), np.float32)
        n = oracle().orc_hash_mesh(self.h, p(pos), p(col), cap)
        return pos[:min(n, cap)], col[:min(n, cap)], n

    def fetch(self, cap=1 << 22):
        """fetchHashScene_kernel's points: (xyz[n, 3], rgba[n, 4], found)."""
        xyz = np.zeros((cap, 3), np.float32)
        rgba = np.zeros((cap, 4), np.float32)
        n = oracle().orc_hash_fetch_points(self.h, p(xyz), p(rgba), cap)
        return xyz[:min(n, cap)], rgba[:min(n, cap)], n

    def visible(self):
        ids = np.zeros(self.n_entries, np.int32)
        n = oracle().orc_hash_visible(self.h, p(ids), ids.size)
        return ids[:n].copy()

    def entries(self):
        ptr_ = oracle().orc_hash_entries(self.h)
        raw = np.ctypeslib.as_array(C.cast(ptr_, C.POINTER(C.c_uint8)), shape=(self.n_entries * 16,))
        return raw.copy().view(HASH_ENTRY)

    def voxels(self):
        n = self.cfg.pool * 512
        L = oracle()
        sdf = np.ctypeslib.as_array(C.cast(L.orc_hash_sdf(self.h), C.POINTER(C.c_int16)), shape=(n,)).copy()
        w = np.ctypeslib.as_array(C.cast(L.orc_hash_weight(self.h), C.POINTER(C.c_uint8)), shape=(n,)).copy()
        rgb = np.ctypeslib.as_array(C.cast(L.orc_hash_rgb(self.h), C.POINTER(C.c_uint8)), shape=(n, 3)).copy()
        return sdf, w, rgb

    def swap(self):
        """The global cache's swap-in merge and swap-out, after an integration."""
        oracle().orc_hash_swap(self.h)

    def swap_states(self):
        ptr_ = oracle().orc_hash_swap_states(self.h)
        return np.ctypeslib.as_array(C.cast(ptr_, C.POINTER(C.c_uint8)), shape=(self.n_entries,)).copy()

    def stored(self, entry):
        """(sdf int16[512], w uint8[512], rgb uint8[512, 3]) kept on the host for entry, or None."""
        sdf = np.zeros(512, np.int16)
        w = np.zeros(512, np.uint8)
        rgb = np.zeros((512, 3), np.uint8)
        if not oracle().orc_hash_stored(self.h, int(entry), p(sdf), p(w), p(rgb)):
            return None
        return sdf, w, rgb

    def stored_count(self):
        return oracle().orc_hash_stored_count(self.h)

    def stored_ids(self):
        ids = np.zeros(self.n_entries, np.int32)
        n = oracle().orc_hash_stored_ids(self.h, p(ids), ids.size)
        return ids[:n].copy()

    def counters(self):
        a, b, c = C.c_int(), C.c_int(), C.c_long()
        oracle().orc_hash_counters(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value


class RefHash:
    """The reference's own hash kernels (host build, test table sizes), run sequentially."""

    def __init__(self, voxel=0.005, mu=0.02, max_w=255, swapping=False):
        L = ref()
        _bind(L, _ref_hash_sigs)
        b, e, pl = C.c_int(), C.c_int(), C.c_int()
        L.ref_hash_sizes(C.byref(b), C.byref(e), C.byref(pl))
        self.buckets, self.excess, self.pool = b.value, e.value, pl.value
        ne = self.buckets + self.excess
        self.entries = np.zeros(ne, HASH_ENTRY)
        self.voxels = np.zeros(self.pool * 512, REF_VOXEL)
        self.alloc_list = np.zeros(self.pool, np.int32)
        self.excess_list = np.zeros(self.excess, np.int32)
        self.last = np.zeros(2, np.int32)
        self.alloc_type = np.zeros(ne, np.uint8)
        self.vis_type = np.zeros(ne, np.uint8)
        self.coords = np.zeros(ne * 4, np.int16)
        self.vis_ids = np.zeros(ne, np.int32)
        self.nvis = C.c_int(0)
        self.voxel, self.mu, self.max_w = voxel, mu, max_w
        self.swapping = swapping
        if swapping:  # NuiKinfuOpenCLHashGlobalCache: swap states and the host store
            self.swap_states = np.zeros(ne, np.uint8)
            self.store = np.zeros(ne * 512, REF_VOXEL)
            self.has_stored = np.zeros(ne, np.uint8)
        last_b, last_e = C.c_int(), C.c_int()
        L.ref_hash_reset(p(self.entries), p(self.voxels), p(self.alloc_list), p(self.excess_list), C.byref(last_b),
                         C.byref(last_e))
        self.last[:] = [last_b.value, last_e.value]

    def frame(self, depth, bgra, cam, xform, integrate=True):
        lb = self.last[0:1]
        le = self.last[1:2]
        if self.swapping:  # NuiKinfuOpenCLHashScene::integrateVolume with the global cache
            L = ref()
            L.ref_hash_alloc_swap(p(self.entries), p(self.alloc_list), p(self.excess_list), p(lb), p(le),
                                  p(self.alloc_type), p(self.vis_type), p(self.coords), p(self.vis_ids),
                                  C.byref(self.nvis), p(depth), p(cam.flat()), p(xform.flat()), self.voxel, self.mu,
                                  p(self.swap_states))
            L.ref_hash_realloc(p(self.entries), p(self.vis_type), p(self.alloc_list), p(lb))
            L.ref_hash_integrate_visible(p(self.entries), p(self.voxels), p(self.vis_ids), self.nvis.value, p(depth),
                                         p(bgra), p(cam.flat()), p(xform.flat()), self.voxel, self.mu, self.max_w)
            L.ref_hash_global_cache(p(self.entries), p(self.voxels), p(self.vis_type), p(self.swap_states),
                                    p(self.alloc_list), p(lb), self.max_w, p(self.store), p(self.has_stored))
            return self.nvis.value
        ref().ref_hash_frame(p(self.entries), p(self.voxels), p(self.alloc_list), p(self.excess_list), p(lb), p(le),
                             p(self.alloc_type), p(self.vis_type), p(self.coords), p(self.vis_ids),
                             C.byref(self.nvis), p(depth), p(bgra), p(cam.flat()), p(xform.flat()), self.voxel,
                             self.mu, self.max_w, 1 if integrate else 0)
        return self.nvis.value

    def visible(self):
        return self.vis_ids[:self.nvis.value].copy()

    def raycast(self, cam, xform, color=False):
        N = cam.W * cam.H
        vm = np.zeros(N * 3, np.float32)
        nm = np.zeros(N * 3, np.float32)
        cm = np.zeros(N * 4, np.uint8) if color else None
        rg = np.zeros(N * 2, np.float32)
        ref().ref_hash_raycast(p(self.entries), p(self.voxels), p(self.vis_ids), self.nvis.value, p(cam.flat()),
                               p(xform.flat()), self.voxel, self.mu, p(rg), p(vm), p(nm), p(cm))
        return vm, nm, cm, rg

    def forward_render(self, cam, xform, vprev, cprev):
        """The reference's ForwardRender kernels up to the normals (see the launcher):
        (vmap, cmap, range, flags, count); vprev / cprev are copied, not modified."""
        N = cam.W * cam.H
        vm = np.ascontiguousarray(vprev, np.float32).reshape(-1).copy()
        nm = np.zeros(N * 3, np.float32)
        cm = np.ascontiguousarray(cprev, np.uint8).reshape(-1).copy()
        rg = np.zeros(N * 2, np.float32)
        fl = np.zeros(N, np.uint8)
        n = ref().ref_hash_forward_render(p(self.entries), p(self.voxels), p(self.vis_ids), self.nvis.value,
                                          p(cam.flat()), p(xform.flat()), self.voxel, self.mu, p(rg), p(vm), p(nm),
                                          p(cm), p(fl))
        return vm, cm, rg, fl, n

    def fetch(self):
        cap = 5_000_000  # MAX_OUTPUT_VERTEX_SIZE
        xyz = np.zeros((cap, 3), np.float32)
        rgba = np.zeros((cap, 4), np.float32)
        n = ref().ref_hash_fetch(p(self.entries), p(self.voxels), p(self.vis_ids), self.nvis.value, self.voxel,
                                 self.mu, p(xyz), p(rgba))
        return xyz[:n], rgba[:n], n

    def mesh(self):
        cap = 5_000_000 + 3  # the kernel stops at MAX_OUTPUT_VERTEX_SIZE (+2, its `>` check)
        pos = np.zeros((cap, 3), np.float32)
        col = np.zeros((cap, 4), np.float32)
        n = ref().ref_hash_mesh(p(self.entries), p(self.voxels), p(self.vis_ids), self.nvis.value, self.voxel, p(pos),
                                p(col))
        return pos[:n], col[:n], n
