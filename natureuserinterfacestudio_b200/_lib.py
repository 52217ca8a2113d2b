"""ctypes binding of libnui_b200.so (the C ABI declared in include/nui_b200.h).

The library is the only implementation: if it is missing or cannot be loaded, every call
raises -- there is no CPU fallback.
"""
import ctypes as C
import os
import weakref

import numpy as np

# test and benchmark input (its own library, libnui_synth.so); re-exported for the callers
from .synth import SYNTH_ROOM, SYNTH_TABLETOP, SynthScene  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnui_b200.so")

NUI_OK = 0
NUI_ERR_INVALID_ARG = 1
NUI_ERR_OOM = 2
NUI_ERR_TRACKING_LOST = 3
NUI_ERR_HASH_FULL = 4
NUI_ERR_MESH_OVERFLOW = 5
NUI_ERR_TIMEOUT = 6
NUI_ERR_DEVICE = 7
NUI_ERR_UNSUPPORTED = 8

TSDF_I16, TSDF_F32, TSDF_F16_U8, TSDF_F16_F16 = 0, 1, 2, 3
VOLUME_DENSE, VOLUME_HASH = 0, 1


class SessionCfg(C.Structure):
    _fields_ = [
        ("width", C.c_int), ("height", C.c_int),
        ("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
        ("depth_min", C.c_float), ("depth_max", C.c_float),
        ("volume_kind", C.c_int), ("tsdf_format", C.c_int),
        ("res", C.c_int * 3), ("dim", C.c_float * 3), ("trunc_dist", C.c_float),
        ("color_volume", C.c_int), ("max_color_weight", C.c_int),
        ("levels", C.c_int), ("iterations", C.c_int * 4), ("filter_radius", C.c_int),
        ("sigma_space2_inv_half", C.c_float), ("sigma_depth2_inv_half", C.c_float),
        ("depth_threshold", C.c_float), ("dist_threshold", C.c_float),
        ("integration_threshold", C.c_float),
        ("voxel_size", C.c_float), ("trunc_scale", C.c_float), ("hash_buckets", C.c_int),
        ("hash_excess", C.c_int), ("hash_pool_blocks", C.c_int), ("hash_max_weight", C.c_int),
        ("photometric_weight", C.c_float),
        ("voxel_shift", C.c_int), ("shift_basis", C.c_float * 3), ("shift_point_cap", C.c_int),
        ("hash_swapping", C.c_int), ("hash_store_blocks", C.c_int), ("hash_forward_render", C.c_int),
    ]


class Tuning(C.Structure):
    """Launch shapes of a context's tick (nui_tuning)."""
    _fields_ = [
        ("integrate_threads_log2", C.c_int), ("icp_pixels_per_thread", C.c_int),
        ("raycast_tile_width", C.c_int), ("hash_raycast_tile_width", C.c_int), ("icp_cluster_blocks", C.c_int),
    ]

    def __init__(self, *args, **kw):
        # the ICP cluster size defaults to the library's default when left out
        super().__init__(*args, **kw)
        if len(args) < 5 and "icp_cluster_blocks" not in kw:
            self.icp_cluster_blocks = 12

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class NuiError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("nui status %d: %s" % (status, msg))
        self.status = status


_lib = None

_P = C.c_void_p
_SIGS = {
    "nui_session_cfg_default": (None, [_P]),
    "nui_last_error_string": (C.c_char_p, []),
    "nui_ctx_create": (C.c_int, [C.c_int, _P]),
    "nui_ctx_destroy": (C.c_int, [_P]),
    "nui_ctx_set_stream": (C.c_int, [_P, _P]),
    "nui_ctx_synchronize": (C.c_int, [_P]),
    "nui_ctx_trim": (C.c_int, [_P]),
    "nui_session_device_bytes": (C.c_size_t, [_P]),
    "nui_session_create": (C.c_int, [_P, _P, _P]),
    "nui_session_destroy": (C.c_int, [_P]),
    "nui_reset": (C.c_int, [_P]),
    "nui_process_frame": (C.c_int, [_P, _P, _P, _P]),
    "nui_process_frame_device": (C.c_int, [_P, _P, _P, _P]),
    "nui_frame_upload": (C.c_int, [_P, _P, _P]),
    "nui_feedback_update": (C.c_int, [_P]),
    "nui_track": (C.c_int, [_P, _P, _P]),
    "nui_integrate": (C.c_int, [_P]),
    "nui_raycast": (C.c_int, [_P]),
    "nui_set_pose": (C.c_int, [_P, _P]),
    "nui_get_pose": (C.c_int, [_P, _P]),
    "nui_mesh": (C.c_int, [_P, _P, _P, C.c_uint64, _P]),
    "nui_mesh_cases": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "nui_mesh_device_noalloc": (C.c_int, [_P, _P, _P, C.c_uint64, _P]),
    "nui_debug_allocation_count": (C.c_int, [_P]),
    "nui_k_color_pyramid": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_int, _P, _P, _P]),
    "nui_server_create": (C.c_int, [_P, C.c_size_t, C.c_int, _P]),
    "nui_server_destroy": (C.c_int, [_P]),
    "nui_server_clock": (C.c_double, [_P]),
    "nui_server_admit": (C.c_int, [_P, _P, _P]),
    "nui_server_release": (C.c_int, [_P, C.c_int]),
    "nui_server_reserve": (C.c_int, [_P, _P, C.c_int]),
    "nui_server_submit": (C.c_int, [_P, C.c_int, _P, _P, C.c_uint64, C.c_double]),
    "nui_server_step": (C.c_int, [_P, _P]),
    "nui_server_drain": (C.c_int, [_P]),
    "nui_server_poll": (C.c_int, [_P, _P, C.c_int, _P]),
    "nui_server_stats": (C.c_int, [_P, _P, _P, _P]),
    "nui_server_session": (_P, [_P, C.c_int]),
    "nui_debug_download": (C.c_int, [_P, C.c_int, C.c_int, _P, C.c_size_t]),
    "nui_debug_upload_volume": (C.c_int, [_P, _P]),
    "nui_hash_stats": (C.c_int, [_P, _P, _P, _P, _P]),
    "nui_batch_tick": (C.c_int, [_P, _P, C.c_int, _P, _P, _P, _P]),
    "nui_batch_tick_device": (C.c_int, [_P, _P, C.c_int, _P, _P, _P, _P]),
    "nui_ctx_enable_timing": (C.c_int, [_P, C.c_int]),
    "nui_ctx_stage_ms": (C.c_int, [_P, C.c_int, _P]),
    "nui_ctx_last_tick_kernels": (C.c_int, [_P, _P]),
    "nui_ctx_get_tuning": (C.c_int, [_P, _P]),
    "nui_shift_state": (C.c_int, [_P, _P, _P, _P]),
    "nui_hash_swap_stats": (C.c_int, [_P, _P, _P, _P, _P]),
    "nui_hash_stored_block": (C.c_int, [_P, C.c_int, _P, _P, _P, _P]),
    "nui_session_snapshot_bytes": (C.c_size_t, [_P]),
    "nui_session_snapshot": (C.c_int, [_P, _P, C.c_size_t]),
    "nui_session_restore": (C.c_int, [_P, _P, C.c_size_t]),
    "nui_shift_points": (C.c_int, [_P, _P, _P, C.c_uint64, _P]),
    "nui_shift_points_clear": (C.c_int, [_P]),
    "nui_point_cloud_device": (C.c_int, [_P, _P, _P, C.c_uint64, _P]),
    "nui_ctx_set_tuning": (C.c_int, [_P, _P]),
    "nui_ctx_autotune": (C.c_int, [_P, _P, C.c_int, _P, _P, C.c_int, C.c_int, _P, _P]),
    "nui_session_touched_voxels": (C.c_int, [_P, _P]),
    "nui_session_work_counters": (C.c_int, [_P, _P]),
    "nui_k_preprocess": (C.c_int, [_P, _P, C.c_int, C.c_int] + [C.c_float] * 6 + [C.c_int] + [C.c_float] * 3 + [_P, _P, _P]),
    "nui_k_pyramid_level": (C.c_int, [_P, _P, C.c_int, C.c_int] + [C.c_float] * 4 + [C.c_int, C.c_float, _P, _P]),
    "nui_k_feedback_maps": (C.c_int, [_P, _P, C.c_int, C.c_int, C.c_float, _P, _P, _P]),
    "nui_frame_file_write": (C.c_int, [C.c_char_p, C.c_int, C.c_int64, C.c_uint32, C.c_uint32, _P, C.c_uint32]),
    "nui_frame_file_header": (C.c_int, [C.c_char_p, _P, _P, _P]),
    "nui_frame_file_read": (C.c_int, [C.c_char_p, _P, C.c_uint32]),
    "nui_camera_file_write": (C.c_int, [C.c_char_p, _P]),
    "nui_camera_file_read": (C.c_int, [C.c_char_p, _P]),
    "nui_recording_frame": (C.c_int, [C.c_char_p, C.c_int, _P, _P, _P, _P, C.c_uint32, C.c_uint32]),
}


def lib():
    """Load libnui_b200.so (raises if it is absent: the CUDA library is the only path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libnui_b200.so not built: run `python -m natureuserinterfacestudio_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != NUI_OK:
        raise NuiError(status, lib().nui_last_error_string().decode())
    return status


def ptr(a):
    """Host pointer of a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def default_cfg(**kw):
    c = SessionCfg()
    lib().nui_session_cfg_default(C.byref(c))
    for k, v in kw.items():
        if k in ("res", "dim", "iterations"):
            arr = getattr(c, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(c, k, v)
    return c


class Context:
    def __init__(self, device=0):
        h = C.c_void_p()
        check(lib().nui_ctx_create(device, C.byref(h)))
        self.h = h
        self._sessions = weakref.WeakSet()

    def trim(self):
        """Returns the context's unused session memory to the device."""
        check(lib().nui_ctx_trim(self.h))

    def close(self):
        """Destroys the context; sessions still open on it are closed first (a session
        must never outlive its context)."""
        if self.h:
            for s in list(self._sessions):
                s.close()
            lib().nui_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        check(lib().nui_ctx_set_stream(self.h, C.c_void_p(stream_handle) if stream_handle else None))

    def sync(self):
        check(lib().nui_ctx_synchronize(self.h))

    def enable_timing(self, on=True):
        check(lib().nui_ctx_enable_timing(self.h, 1 if on else 0))

    def last_tick_kernels(self):
        v = C.c_int()
        check(lib().nui_ctx_last_tick_kernels(self.h, C.byref(v)))
        return v.value

    def stage_ms(self, stage):
        v = C.c_float()
        check(lib().nui_ctx_stage_ms(self.h, stage, C.byref(v)))
        return v.value

    def tuning(self):
        t = Tuning()
        check(lib().nui_ctx_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, t=None, **kw):
        """Sets the launch shapes: a Tuning, or fields by keyword over the current ones."""
        t = t or self.tuning()
        for k, v in kw.items():
            setattr(t, k, v)
        check(lib().nui_ctx_set_tuning(self.h, C.byref(t)))

    def autotune(self, cfgs, seqs, bgras=None, repeats=5):
        """Times the launch-shape candidates on scratch sessions of cfgs fed seqs[i] (a
        list of >= 2 uint16 depth frames per session, bgras likewise or None) and keeps
        the fastest in the context.  Returns (Tuning, whole-tick median ms)."""
        n, frames = len(cfgs), len(seqs[0])
        assert all(len(q) == frames for q in seqs)
        cf = (SessionCfg * n)(*cfgs)
        keep = [np.ascontiguousarray(x) for q in seqs for x in q]
        d = (C.c_void_p * (n * frames))(*[x.ctypes.data for x in keep])
        b = None
        if bgras is not None:  # None entries: sessions without colour frames
            keepc = [None if x is None else np.ascontiguousarray(x) for q in bgras for x in q]
            keep += [x for x in keepc if x is not None]
            b = (C.c_void_p * (n * frames))(*[None if x is None else x.ctypes.data for x in keepc])
        t, ms = Tuning(), C.c_float()
        check(lib().nui_ctx_autotune(self.h, cf, n, d, b, frames, repeats, C.byref(t), C.byref(ms)))
        return t, ms.value

    def batch_tick(self, sessions, depths, bgras=None, device=False):
        """One frame for every session.  depths: list of uint16 arrays (host) or device
        pointers (ints) when device=True.  Returns (statuses, poses[n,12])."""
        n = len(sessions)
        arr = (C.c_void_p * n)(*[s.h.value for s in sessions])
        if device:
            d = (C.c_void_p * n)(*depths)
            b = (C.c_void_p * n)(*(bgras or [None] * n))
        else:
            d = (C.c_void_p * n)(*[x.ctypes.data for x in depths])
            b = (C.c_void_p * n)(*[(x.ctypes.data if x is not None else None) for x in (bgras or [None] * n)])
        st = np.zeros(n, np.int32)
        poses = np.zeros((n, 12), np.float32)
        fn = lib().nui_batch_tick_device if device else lib().nui_batch_tick
        r = fn(self.h, arr, n, d, b, ptr(st), ptr(poses))
        if r not in (NUI_OK, NUI_ERR_TRACKING_LOST, NUI_ERR_HASH_FULL):
            check(r)
        return st, poses


class Session:
    def __init__(self, ctx, cfg):
        h = C.c_void_p()
        check(lib().nui_session_create(ctx.h, C.byref(cfg), C.byref(h)))
        self.h = h
        self.ctx = ctx
        ctx._sessions.add(self)
        self.cfg = cfg
        self.W, self.H = cfg.width, cfg.height
        self.res = tuple(cfg.res)

    def close(self):
        if self.h and self.ctx.h:
            lib().nui_session_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def process(self, depth, bgra=None):
        pose = np.zeros(12, np.float32)
        r = lib().nui_process_frame(self.h, ptr(depth), ptr(bgra), ptr(pose))
        if r == NUI_ERR_TRACKING_LOST:
            return False, pose
        check(r)
        return True, pose

    def process_device(self, depth_ptr, bgra_ptr=None):
        pose = np.zeros(12, np.float32)
        r = lib().nui_process_frame_device(self.h, C.c_void_p(depth_ptr), C.c_void_p(bgra_ptr) if bgra_ptr else None,
                                           ptr(pose))
        if r == NUI_ERR_TRACKING_LOST:
            return False, pose
        check(r)
        return True, pose

    def reset(self):
        check(lib().nui_reset(self.h))

    def upload(self, depth, bgra=None):
        check(lib().nui_frame_upload(self.h, ptr(depth), ptr(bgra)))

    def feedback_update(self):
        check(lib().nui_feedback_update(self.h))

    def track(self):
        err = C.c_float()
        cnt = C.c_int()
        r = lib().nui_track(self.h, C.byref(err), C.byref(cnt))
        if r == NUI_ERR_TRACKING_LOST:
            return False, err.value, cnt.value
        check(r)
        return True, err.value, cnt.value

    def integrate(self):
        check(lib().nui_integrate(self.h))

    def raycast(self):
        check(lib().nui_raycast(self.h))

    def set_pose(self, R, t):
        p = np.concatenate([np.asarray(R, np.float32).reshape(9), np.asarray(t, np.float32).reshape(3)])
        check(lib().nui_set_pose(self.h, ptr(p)))

    def get_pose(self):
        p = np.zeros(12, np.float32)
        check(lib().nui_get_pose(self.h, ptr(p)))
        return p[:9].reshape(3, 3), p[9:]

    def touched(self):
        v = C.c_uint64()
        check(lib().nui_session_touched_voxels(self.h, C.byref(v)))
        return v.value

    def snapshot(self):
        """The session's state as bytes (numpy uint8) for restore() into a session of the
        same configuration."""
        n = lib().nui_session_snapshot_bytes(self.h)
        buf = np.zeros(n, np.uint8)
        check(lib().nui_session_snapshot(self.h, ptr(buf), n))
        return buf

    def restore(self, snap):
        snap = np.ascontiguousarray(snap, np.uint8)
        check(lib().nui_session_restore(self.h, ptr(snap), snap.size))

    def hash_swap_stats(self):
        """(swapped in, swapped out by the last frame, store blocks used, refused swap-outs)."""
        v = [C.c_int() for _ in range(4)]
        check(lib().nui_hash_swap_stats(self.h, *[C.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def hash_stored(self, entry):
        """(sdf[512] raw int16 bits, weight[512], rgb[512, 4]) stored for a hash entry, or None."""
        sdf = np.zeros(512, np.int16)
        w = np.zeros(512, np.uint8)
        rgb = np.zeros((512, 4), np.uint8)
        f = C.c_int()
        check(lib().nui_hash_stored_block(self.h, int(entry), ptr(sdf), ptr(w), ptr(rgb), C.byref(f)))
        return (sdf, w, rgb) if f.value else None

    def shift_state(self):
        """(voxel offset int32[3], offset in metres float32[3], points found) of a shifting
        volume; the camera's global translation is its pose's plus the offset."""
        vo = np.zeros(3, np.int32)
        om = np.zeros(3, np.float32)
        n = C.c_uint64()
        check(lib().nui_shift_state(self.h, ptr(vo), ptr(om), C.byref(n)))
        return vo, om, n.value

    def shift_points(self, cap=None):
        """(xyz[n, 3], rgba[n, 4]) of the point cache of the slabs that left the volume."""
        n = C.c_uint64()
        check(lib().nui_shift_points(self.h, None, None, 0, C.byref(n)))
        k = n.value if cap is None else min(cap, n.value)
        xyz = np.zeros((k, 3), np.float32)
        rgba = np.zeros((k, 4), np.float32)
        if k:
            check(lib().nui_shift_points(self.h, ptr(xyz), ptr(rgba), k, C.byref(n)))
        return xyz, rgba

    def clear_shift_points(self):
        check(lib().nui_shift_points_clear(self.h))

    def point_cloud(self, cap=1 << 22):
        """Point cloud of the scene (fetchVolumeKernel / fetchShiftVolumeKernel for dense volumes,
        fetchHashScene_kernel for the voxel hash): (xyz[n, 3], rgba[n, 4], found)."""
        import torch
        xyz = torch.empty((cap, 3), dtype=torch.float32, device="cuda")
        rgba = torch.empty((cap, 4), dtype=torch.float32, device="cuda")
        n = C.c_uint64()
        check(lib().nui_point_cloud_device(self.h, C.c_void_p(xyz.data_ptr()), C.c_void_p(rgba.data_ptr()), cap,
                                           C.byref(n)))
        k = min(n.value, cap)
        return xyz[:k].cpu().numpy(), rgba[:k].cpu().numpy(), n.value

    def download(self, what, level=0):
        W, H = self.W >> level, self.H >> level
        nv = self.res[0] * self.res[1] * self.res[2]
        shapes = {0: ((H, W), np.float32), 1: ((H, W), np.float32), 2: ((H, W, 4), np.float32),
                  3: ((self.H, self.W, 4), np.float32), 4: ((self.H, self.W, 4), np.float32),
                  5: ((nv, 2), np.int16), 7: ((H, W), np.float32), 8: ((self.H, self.W, 4), np.uint8),
                  9: ((nv, 4), np.uint8), 10: ((self.H, self.W, 4), np.uint8), 11: ((H, W, 4), np.uint8),
                  12: ((H, W, 4), np.uint8),
                  13: ((((self.res[0] + 7) // 8) * ((self.res[1] + 7) // 8) * ((self.res[2] + 7) // 8),), np.uint8),
                  14: ((nv,), np.uint8)}
        fmt = self.cfg.tsdf_format
        shapes[6] = {TSDF_I16: ((nv, 2), np.int16), TSDF_F32: ((nv, 2), np.float32),
                     TSDF_F16_U8: ((nv,), np.float16), TSDF_F16_F16: ((nv, 2), np.float16)}[fmt]
        shape, dt = shapes[what]
        out = np.zeros(shape, dt)
        check(lib().nui_debug_download(self.h, what, level, ptr(out), out.nbytes))
        return out

    def hash_stats(self):
        v, b, e, f = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib().nui_hash_stats(self.h, C.byref(v), C.byref(b), C.byref(e), C.byref(f)))
        return v.value, b.value, e.value, f.value

    def hash_download(self, what):
        """20 entries, 21 visible list, 22 voxels (reference layout), 23 range image, 24 swap
        states (global cache)."""
        c = self.cfg
        ne = c.hash_buckets + c.hash_excess
        if what == 24:
            out = np.zeros(ne, np.uint8)
        elif what == 20:
            out = np.zeros(ne * 16, np.uint8)
        elif what == 21:
            out = np.zeros(self.hash_stats()[0], np.int32)
        elif what == 22:
            out = np.zeros(c.hash_pool_blocks * 512 * 6, np.uint8)
        else:
            out = np.zeros(self.W * self.H * 2, np.float32)
        if out.size:
            check(lib().nui_debug_download(self.h, what, 0, ptr(out), out.nbytes))
        return out

    def work_counters(self):
        """Work of the last frame: updated voxels, re-classified bricks, raycast voxel reads,
        samples visited, refined crossings, ICP iterations per level (4), integration tiles run."""
        out = np.zeros(10, np.uint64)
        check(lib().nui_session_work_counters(self.h, ptr(out)))
        return {"touched": int(out[0]), "bricks": int(out[1]), "ray_reads": int(out[2]),
                "ray_samples": int(out[3]), "ray_hits": int(out[4]), "icp_iters": [int(x) for x in out[5:9]],
                "tiles": int(out[9])}

    def volume_ref_layout(self):
        """Volume as the reference stores it: short2 at ((x + y*rx)*rz + z)."""
        return self.download(5)

    def upload_volume(self, ref_short2):
        a = np.ascontiguousarray(ref_short2, np.int16)
        check(lib().nui_debug_upload_volume(self.h, ptr(a)))

    def mesh(self, cap):
        pos = np.zeros((cap, 3), np.float32)
        col = np.zeros((cap, 4), np.float32)
        n = C.c_uint64()
        r = lib().nui_mesh(self.h, ptr(pos), ptr(col), cap, C.byref(n))
        if r not in (NUI_OK, NUI_ERR_MESH_OVERFLOW):
            check(r)
        k = min(n.value, cap)
        return pos[:k], col[:k], n.value

    def mesh_into(self, pos):
        """Marching cubes into a caller's (cap, 3) float32 array (no colours); the vertex count
        (more than cap: the mesh was cut)."""
        n = C.c_uint64()
        r = lib().nui_mesh(self.h, ptr(pos), None, pos.shape[0], C.byref(n))
        if r not in (NUI_OK, NUI_ERR_MESH_OVERFLOW):
            check(r)
        return n.value

    def mesh_cases(self):
        rx, ry, rz = self.res
        out = np.zeros((ry - 1) * (rx - 1) * (rz - 1), np.uint8)
        n = C.c_uint64()
        check(lib().nui_mesh_cases(self.h, ptr(out), out.nbytes, C.byref(n)))
        return out, n.value


class ServerResult(C.Structure):
    _fields_ = [("slot", C.c_int), ("status", C.c_int), ("tag", C.c_uint64), ("t_submit", C.c_double),
                ("t_done", C.c_double), ("pose", C.c_float * 12)]


class Server:
    """Continuous batching of many streams on one context (nui_server_*).

    Frames passed to submit() must stay alive until their result is polled; pinned
    (page-locked) host arrays let the upload overlap the previous batch."""

    def __init__(self, ctx, hbm_budget_bytes, max_streams=64):
        h = C.c_void_p()
        check(lib().nui_server_create(ctx.h, int(hbm_budget_bytes), int(max_streams), C.byref(h)))
        self.h = h
        self.ctx = ctx
        self._keep = {}
        ctx._sessions.add(self)  # closed before its context

    def close(self):
        if self.h:
            lib().nui_server_destroy(self.h)
            self.h = None
            self._keep = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clock(self):
        return lib().nui_server_clock(self.h)

    def admit(self, cfg):
        """Slot of the new stream, or None when it does not fit (budget or slots)."""
        k = C.c_int()
        r = lib().nui_server_admit(self.h, C.byref(cfg), C.byref(k))
        if r == NUI_ERR_OOM:
            return None
        check(r)
        return k.value

    def reserve(self, cfg, count):
        """Idle sessions of cfg for later admissions (None when the budget is short)."""
        r = lib().nui_server_reserve(self.h, C.byref(cfg), int(count))
        if r == NUI_ERR_OOM:
            return None
        check(r)
        return count

    def release(self, slot):
        check(lib().nui_server_release(self.h, slot))
        self._keep = {k: v for k, v in self._keep.items() if k[0] != slot}

    def submit(self, slot, depth, bgra=None, tag=0, t_submit=-1.0):
        self._keep[(slot, tag)] = (depth, bgra)
        check(lib().nui_server_submit(self.h, slot, ptr(depth), ptr(bgra), int(tag), float(t_submit)))

    def step(self):
        n = C.c_int()
        check(lib().nui_server_step(self.h, C.byref(n)))
        return n.value

    def drain(self):
        check(lib().nui_server_drain(self.h))

    def poll(self, cap=1024):
        if getattr(self, "_pollbuf", None) is None or len(self._pollbuf) < cap:
            self._pollbuf = (ServerResult * cap)()
        out = self._pollbuf
        res = []
        while True:
            n = C.c_int()
            check(lib().nui_server_poll(self.h, out, cap, C.byref(n)))
            res += [ServerResult.from_buffer_copy(out[i]) for i in range(n.value)]
            if n.value < cap:
                break
        for r in res:
            self._keep.pop((r.slot, r.tag), None)
        return res

    def stats(self):
        used, ns, nq = C.c_size_t(), C.c_int(), C.c_int()
        check(lib().nui_server_stats(self.h, C.byref(used), C.byref(ns), C.byref(nq)))
        return used.value, ns.value, nq.value


# ---------------------------------------------------------------- recorded frames
def write_recording(directory, frames, intrinsics, compressed=True, t0=0, dt=33333):
    """Writes frames [(depth uint16 HxW, bgra uint8 HxWx4 or None), ...] as a recording:
    <n>.depth, <n>.color, <n>.camIntri (the reference's layout and file format)."""
    os.makedirs(directory, exist_ok=True)
    cam = np.asarray(intrinsics, np.float32)
    for n, (d, c) in enumerate(frames):
        base = os.path.join(directory, str(n)).encode()
        d = np.ascontiguousarray(d, np.uint16)
        H, W = d.shape
        check(lib().nui_frame_file_write(base + b".depth", int(compressed), t0 + n * dt, W, H, ptr(d), 2))
        if c is not None:
            c = np.ascontiguousarray(c, np.uint8)
            check(lib().nui_frame_file_write(base + b".color", int(compressed), t0 + n * dt, W, H, ptr(c), 4))
        check(lib().nui_camera_file_write(base + b".camIntri", ptr(cam)))


def read_recording(directory, width, height, color=True):
    """Frames of a recording: [(depth, bgra or None, intrinsics[4], timestamp), ...]."""
    out = []
    n = 0
    while True:
        d = np.zeros((height, width), np.uint16)
        c = np.zeros((height, width, 4), np.uint8) if color else None
        cam = np.zeros(4, np.float32)
        ts = C.c_int64()
        r = lib().nui_recording_frame(directory.encode(), n, ptr(d), ptr(c), ptr(cam), C.byref(ts), width, height)
        if r != NUI_OK:
            break
        has_c = color and os.path.exists(os.path.join(directory, "%d.color" % n))
        out.append((d, c if has_c else None, cam, ts.value))
        n += 1
    return out
