"""Generates tests/golden/dense_small.npz from the reference's own kernels.

Runs the reference OpenCL kernels of the dense path (compiled for the host by
oracle/build_ref.py from the reference tree) on one seeded synthetic frame:
pass filter -> scaleDepths -> integrateTsdfVolume -> raycast -> marchingCube, and stores
their outputs.  The fixture lets the oracle be checked on machines without the reference
tree.  Run from the repository root:  python tests/golden/make_golden.py
"""
import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from natureuserinterfacestudio_b200 import _lib as L  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    W, H, f = 160, 120, 131.25
    res, dim, trunc_cfg = (40, 40, 40), (3.0, 3.0, 3.0), 0.0
    sc = L.SynthScene(L.SYNTH_TABLETOP, seed=11)
    R, t = sc.pose(3)
    raw, _ = sc.render(R, t, W, H, fx=f, fy=f, cx=(W - 1) / 2, cy=(H - 1) / 2, frame=3)
    ref = O.ref()
    N = W * H
    pas = np.zeros(N, np.float32)
    ref.ref_pass_filter(O.p(raw.reshape(-1)), O.p(pas), N, 0.5, 4.5)
    cam = O.OrcCam.make(W, H, f, f, (W - 1) / 2, (H - 1) / 2)
    tp = O.OrcTsdf.make(res, dim, trunc_cfg)
    nv = int(np.prod(res))
    vol = np.zeros(nv * 2, np.int16)
    ref.ref_init_volume(O.p(vol), None, O.p(tp.flat()))
    x = O.make_xform(R, t)
    s = pas.copy()
    ref.ref_scale_depths(O.p(s), O.p(cam.flat()), W, H)
    ref.ref_integrate(O.p(s), None, O.p(cam.flat()), O.p(x.flat()), O.p(vol), O.p(tp.flat()), None, 128)
    vm, nm = np.zeros(N * 3, np.float32), np.zeros(N * 3, np.float32)
    ref.ref_raycast(O.p(vol), None, O.p(tp.flat()), O.p(cam.flat()), O.p(x.flat()), O.p(vm), O.p(nm), None, W, H)
    cap = 500_000
    pos, col = np.zeros((cap, 3), np.float32), np.zeros((cap, 4), np.float32)
    n = ref.ref_marching_cubes(O.p(vol), None, O.p(tp.flat()), O.p(pos), O.p(col))
    tris = np.unique(pos[:n].reshape(-1, 9), axis=0)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dense_small.npz")
    np.savez_compressed(out, raw=raw, f=np.float32(f), res=np.array(res), dim=np.array(dim, np.float32),
                        trunc_cfg=np.float32(trunc_cfg), R=R, t=t, **{"pass": pas}, volume=vol, vmap=vm, nmap=nm,
                        mc_count=np.int64(n), mc_tris=tris)
    print(out, os.path.getsize(out), "bytes; mc vertices", n, "valid rays", int((~np.isnan(vm)).sum() // 3))


if __name__ == "__main__":
    main()
