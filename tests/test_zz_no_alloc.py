"""Meshing without device allocation (nui_mesh_device_noalloc) against nui_mesh.

Collected last on purpose: it must hold both in a fresh process and after every other
test has run on the same device.  Each call is compared bit for bit with the allocating
entry point, over consecutive calls on volumes of different sizes, so a result that
depended on what an earlier call left in the shared scratch array would show.
"""
import ctypes as C

import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L
from oracle import oracle as O

from _util import cfg_for, frames, same_bits

pytestmark = pytest.mark.gpu


def _noalloc(s, cap, colours=True):
    torch = pytest.importorskip("torch")
    pos = torch.full((max(cap, 1), 3), float("nan"), dtype=torch.float32, device="cuda")
    col = torch.full((max(cap, 1), 4), float("nan"), dtype=torch.float32, device="cuda")
    n = C.c_uint64()
    torch.cuda.synchronize()  # the output buffers must be idle when the call is made
    before = _allocations()
    r = L.lib().nui_mesh_device_noalloc(s.h, C.c_void_p(pos.data_ptr()),
                                        C.c_void_p(col.data_ptr()) if colours else None, cap, C.byref(n))
    # the defining property: the call makes no device or pinned-host allocation of its own
    assert _allocations() == before
    k = min(n.value, cap)
    return r, n.value, pos[:k].cpu().numpy(), col[:k].cpu().numpy()


def _allocations():
    n = C.c_uint64()
    assert L.lib().nui_debug_allocation_count(C.byref(n)) == L.NUI_OK
    return n.value


@pytest.fixture(scope="module")
def sessions(gpu_ctx):
    seq = frames(3, W=640, H=480, seed=5)
    out = []
    for res, color in (((160, 144, 128), True), ((96, 80, 112), False)):
        cfg = cfg_for(res=res, color=color)
        eng = O.Engine(cfg)
        for d, _, _, _ in seq:
            assert eng.frame(d)
        s = L.Session(gpu_ctx, cfg)
        s.upload_volume(eng.volume())
        out.append(s)
    yield out
    for s in out:
        s.close()


def test_consecutive_calls_match_allocating_entry(sessions):
    cap = 2_000_000
    expect = [s.mesh(cap) for s in sessions]
    assert all(e[2] > 0 for e in expect)
    for s, (pos_e, col_e, n_e) in zip(sessions + sessions[:1], expect + expect[:1]):
        r, n, pos, col = _noalloc(s, cap)
        assert r == L.NUI_OK and n == n_e
        assert same_bits(pos, pos_e)
        assert same_bits(col, col_e)


def test_overflow_and_positions_only(sessions):
    s = sessions[0]
    pos_e, _, n_e = s.mesh(2_000_000)
    small = n_e // 3
    r, n, pos, _ = _noalloc(s, small, colours=False)
    assert r == L.NUI_ERR_MESH_OVERFLOW and n == n_e and len(pos) == small
    assert same_bits(pos, pos_e[:small])
    r, n, pos, _ = _noalloc(s, 2_000_000, colours=False)
    assert r == L.NUI_OK and same_bits(pos, pos_e)


def test_rejects_oversize_volume_and_host_buffers(gpu_ctx, sessions):
    big = L.Session(gpu_ctx, cfg_for(res=(600, 600, 8)))  # 599 * 599 columns > 262144
    try:
        r, n, _, _ = _noalloc(big, 16)
        assert r == L.NUI_ERR_INVALID_ARG
        assert "too large" in L.lib().nui_last_error_string().decode()
    finally:
        big.close()
    host = np.zeros((16, 3), np.float32)
    n = C.c_uint64()
    r = L.lib().nui_mesh_device_noalloc(sessions[1].h, L.ptr(host), None, 16, C.byref(n))
    assert r == L.NUI_ERR_INVALID_ARG


def test_rejects_buffers_of_another_device(sessions):
    """A buffer on another GPU is refused before any launch (the kernels would otherwise
    write another device's memory from this one)."""
    torch = pytest.importorskip("torch")
    if torch.cuda.device_count() < 2:
        pytest.skip("needs a second CUDA device")
    other = torch.zeros((16, 3), dtype=torch.float32, device="cuda:1")
    torch.cuda.synchronize(1)
    n = C.c_uint64(12345)
    r = L.lib().nui_mesh_device_noalloc(sessions[1].h, C.c_void_p(other.data_ptr()), None, 16, C.byref(n))
    assert r == L.NUI_ERR_INVALID_ARG and n.value == 12345
    assert torch.count_nonzero(other).item() == 0
