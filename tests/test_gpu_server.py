"""The serving loop (continuous batching): each stream's results are the same alone and in
a mix whose members join and leave between steps, admission follows the HBM budget, and
the reported times are ordered.  Streams differ in image size, volume kind, format and
colour."""
import ctypes as C

import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L

from _util import cfg_for, cfg_hash, frames

pytestmark = pytest.mark.gpu


def _streams():
    c_col = cfg_for(res=(128, 128, 128), color=True)
    c_col.photometric_weight = 0.1
    return [
        (cfg_for(res=(128, 128, 128)), frames(6, W=640, H=480, seed=3), False),
        (cfg_for(W=320, H=240, res=(96, 96, 96), fmt=L.TSDF_F16_U8), frames(7, W=320, H=240, seed=8), False),
        (cfg_hash(), frames(5, W=320, H=240, seed=5), False),
        (c_col, frames(5, W=640, H=480, seed=12, color=True), True),
    ]


def test_results_same_alone_and_in_the_mix(gpu_ctx):
    streams = _streams()
    alone = []
    for cfg, seq, col in streams:
        s = L.Session(gpu_ctx, cfg)
        alone.append([s.process(d, np.ascontiguousarray(c) if col else None)[1] for d, c, _, _ in seq])
        s.close()
    srv = L.Server(gpu_ctx, 100 << 30, max_streams=8)
    # join schedule: stream k is admitted before step join[k]; every admitted stream
    # submits its frames two at a time, so queues build up and drain unevenly
    join = [0, 0, 2, 3]
    slot, nxt, got = {}, [0] * 4, {k: {} for k in range(4)}
    step = 0
    while any(len(got[k]) < len(streams[k][1]) for k in range(4)):
        for k in range(4):
            if k not in slot and step >= join[k]:
                slot[k] = srv.admit(streams[k][0])
                assert slot[k] is not None
            if k in slot and nxt[k] < len(streams[k][1]) and step % 2 == k % 2:
                for _ in range(2):
                    if nxt[k] < len(streams[k][1]):
                        d, c, _, _ = streams[k][1][nxt[k]]
                        srv.submit(slot[k], d, np.ascontiguousarray(c) if streams[k][2] else None, tag=nxt[k])
                        nxt[k] += 1
        srv.step()
        for r in srv.poll():
            k = [j for j in slot if slot[j] == r.slot][0]
            assert r.status == L.NUI_OK and r.t_done >= r.t_submit
            got[k][r.tag] = np.array(r.pose)
        # a stream that has all its results leaves at once
        for k in list(slot):
            if len(got[k]) == len(streams[k][1]) and slot[k] is not None:
                srv.release(slot[k])
                slot[k] = None
        step += 1
        assert step < 100
    for k in range(4):
        for i, p in enumerate(alone[k]):
            assert np.array_equal(got[k][i], p), (k, i)
    assert srv.stats()[1] == 0
    srv.close()


def test_admission_follows_the_budget(gpu_ctx):
    cfg = cfg_for(res=(128, 128, 128))
    need = L.lib().nui_session_device_bytes(C.byref(cfg))
    srv = L.Server(gpu_ctx, int(2.5 * need) + (8 << 20), max_streams=8)
    a, b = srv.admit(cfg), srv.admit(cfg)
    assert a is not None and b is not None
    assert srv.admit(cfg) is None  # over budget
    used, n, _ = srv.stats()
    assert n == 2 and used >= 2 * need
    srv.release(a)
    assert srv.admit(cfg) is not None
    srv.close()


def test_admission_that_evicts_a_pooled_session(gpu_ctx):
    """A released stream's session stays pooled; a stream of another configuration that
    needs its budget evicts it.  The eviction and the new session's allocation and reset are
    queued on the stream behind another stream's tick in flight (stream-ordered memory, no
    device synchronisation), and both live streams' results equal their runs alone."""
    c1 = cfg_for(res=(128, 128, 128))
    c2 = cfg_for(W=320, H=240, res=(96, 96, 160), fmt=L.TSDF_F16_U8)
    s1, s2 = frames(8, W=640, H=480, seed=3), frames(5, W=320, H=240, seed=8)
    expect = {}
    for key, cfg, seq in (("c", c1, s1), ("b", c2, s2)):
        alone = L.Session(gpu_ctx, cfg)
        expect[key] = [alone.process(d)[1] for d, _, _, _ in seq]
        alone.close()
    need = [L.lib().nui_session_device_bytes(C.byref(c)) + c.width * c.height * 12 for c in (c1, c2)]
    assert need[0] >= need[1] // 2
    srv = L.Server(gpu_ctx, 2 * need[0] + need[1] // 2, max_streams=4)
    a, c = srv.admit(c1), srv.admit(c1)
    assert a is not None and c is not None
    got = {"b": {}, "c": {}}
    slots = {c: "c"}

    def collect():
        for r in srv.poll():
            if r.slot in slots:
                assert r.status == L.NUI_OK
                got[slots[r.slot]][r.tag] = np.array(r.pose)
    for i in range(3):  # both streams run; a leaves, its session is pooled
        srv.submit(a, s1[i][0], tag=i)
        srv.submit(c, s1[i][0], tag=i)
        srv.step()
        collect()
    srv.release(a)
    collect()
    srv.submit(c, s1[3][0], tag=3)
    srv.step()  # c's tick is in flight
    b = srv.admit(c2)  # evicts a's pooled session
    assert b is not None
    slots[b] = "b"
    for i in range(5):
        srv.submit(b, s2[i][0], tag=i)
        if 4 + i < len(s1):
            srv.submit(c, s1[4 + i][0], tag=4 + i)
        srv.step()
        collect()
    srv.drain()
    collect()
    for key in ("b", "c"):
        for i, p in enumerate(expect[key]):
            assert np.array_equal(got[key][i], p), (key, i)
    srv.close()
