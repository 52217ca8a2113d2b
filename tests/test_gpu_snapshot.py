"""Session snapshot / restore: a session restored from a snapshot continues exactly as the
snapshotted one -- the same poses bit for bit, the same volume -- for a dense colour volume,
a voxel hash and a shifting volume; a snapshot does not load into another configuration."""
import numpy as np
import pytest

from natureuserinterfacestudio_b200 import _lib as L

from _util import cfg_for, cfg_hash, frames

pytestmark = pytest.mark.gpu


def _cases():
    shift = cfg_for(W=320, H=240, res=(96, 80, 112), dim=3.0, color=True)
    shift.voxel_shift = 3
    return [
        ("dense colour", cfg_for(W=320, H=240, res=(128, 128, 128), color=True), True),
        ("hash", cfg_hash(), False),
        ("shifting", shift, True),
    ]


@pytest.mark.parametrize("name,cfg,color", _cases(), ids=[c[0] for c in _cases()])
def test_restored_session_continues_identically(gpu_ctx, name, cfg, color):
    seq = frames(7, W=320, H=240, seed=5, deg=1.0, color=True, kind=L.SYNTH_ROOM)
    a = L.Session(gpu_ctx, cfg)
    for d, c, _, _ in seq[:4]:
        assert a.process(d, np.ascontiguousarray(c) if color else None)[0]
    snap = a.snapshot()
    first = [a.process(d, np.ascontiguousarray(c) if color else None)[1] for d, c, _, _ in seq[4:]]
    b = L.Session(gpu_ctx, cfg)
    b.restore(snap)
    second = [b.process(d, np.ascontiguousarray(c) if color else None)[1] for d, c, _, _ in seq[4:]]
    for p1, p2 in zip(first, second):
        assert np.array_equal(p1, p2), name
    if cfg.volume_kind == L.VOLUME_DENSE:
        assert np.array_equal(a.volume_ref_layout(), b.volume_ref_layout())
        assert np.array_equal(a.shift_state()[0], b.shift_state()[0])
    else:
        assert np.array_equal(a.hash_download(22), b.hash_download(22))
    other = L.Session(gpu_ctx, cfg_for(W=320, H=240, res=(64, 64, 64)))
    with pytest.raises(L.NuiError):
        other.restore(snap)
    for s in (a, b, other):
        s.close()
