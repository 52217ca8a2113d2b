"""Benchmark: aggregate frames/s and per-frame latency of many concurrent KinectFusion
sessions on one B200 (weak scaling: each GPU/rank serves its own sessions).

A step is one tick: every session advances one 640x480 frame (preprocess, 3-level ICP,
gated TSDF integration, raycast) in one batched launch sequence replayed from a CUDA graph.
value = sessions * steps / device time (frames already in HBM); e2e = the same through the
public C-ABI call with host (pinned) frames, host->device copies and the pose readback in
the timed region.  The in-GPU comparison is the plain FP32 path: one session per launch
sequence, FP32 TSDF, no graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W_IMG, H_IMG, FOCAL = 640, 480, 525.0
VOLUMES = (256, 384, 512)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def session_cfgs(L, n, fmt):
    cfgs = []
    for i in range(n):
        r = VOLUMES[i % len(VOLUMES)]
        dim = 3.0 if r == 256 else 4.0
        cfgs.append(L.default_cfg(res=(r, r, r), dim=(dim, dim, dim), tsdf_format=fmt, trunc_dist=0.03,
                                  iterations=[10, 5, 4, 0], integration_threshold=0.0))
    return cfgs


def render_sequences(L, nseq, nframes, seed0=100):
    seqs = []
    for k in range(nseq):
        sc = L.SynthScene(L.SYNTH_TABLETOP, seed=seed0 + k, extent=3.0)
        fr = []
        for i in range(nframes):
            R, t = sc.pose(i, radius=1.5, deg_per_frame=2.0)
            d, _ = sc.render(R, t, W_IMG, H_IMG, frame=i, noise_seed=seed0 * 7 + k)
            fr.append(d)
        seqs.append(fr)
    return seqs


def run_ours(args, rank, world):
    import torch
    from natureuserinterfacestudio_b200 import _lib as L

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    ctx = L.Context(dev)
    # a dedicated stream: graphs cannot be captured on the legacy default stream, and torch
    # events must be recorded on the stream the kernels run on
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    n = args.sessions
    nframes = args.warmup + args.steps + 1
    nseq = min(n, args.sequences)
    seqs = render_sequences(L, nseq, 2 * nframes + args.warmup + 1)
    # frames resident in HBM: one device tensor per (sequence, frame)
    dev_frames = [[torch.from_numpy(f.view(np.int16)).cuda() for f in s] for s in seqs]
    host_frames = [[torch.from_numpy(f.view(np.int16)).pin_memory() for f in s] for s in seqs]
    torch.cuda.synchronize()

    def make_sessions(fmt):
        return [L.Session(ctx, c) for c in session_cfgs(L, n, fmt)]

    sessions = make_sessions(L.TSDF_F16_U8)
    offs = [(i * 7) % 11 for i in range(n)]  # sessions sharing a sequence start at different frames

    def dframes(step):
        return [dev_frames[i % nseq][offs[i] + step].data_ptr() for i in range(n)]

    def hframes(step):
        return [host_frames[i % nseq][offs[i] + step].numpy() for i in range(n)]

    def tick_device(step):
        st, poses = ctx.batch_tick(sessions, dframes(step), device=True)
        return st

    # warm-up (also captures the graph)
    for w in range(args.warmup):
        tick_device(w)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    launches_per_tick = tick_launch_count(sessions)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tick_ms = []
    with ClockSampler(dev) as clk:
        e0.record(stream)
        for k in range(args.steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            st = tick_device(args.warmup + k)
            b.record(stream)
            tick_ms.append((a, b))
            lost = int(np.sum(st != 0))
        e1.record(stream)
        torch.cuda.synchronize()
    ms_total = e0.elapsed_time(e1)
    per_tick = [a.elapsed_time(b) for a, b in tick_ms]
    ms = max_over_ranks(ms_total, world)
    value = n * world * args.steps / (ms / 1e3)

    # e2e: same ticks through the public call with host frames (pinned), copies included
    base = args.warmup + args.steps
    for s in sessions:
        s.reset()
    for w in range(args.warmup):
        ctx.batch_tick(sessions, hframes(w))
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    e2e_tick = []
    t0.record(stream)
    for k in range(args.steps):
        a = time.perf_counter()
        ctx.batch_tick(sessions, hframes(args.warmup + k))
        e2e_tick.append((time.perf_counter() - a) * 1e3)
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(t0.elapsed_time(t1), world)
    e2e_value = n * world * args.steps / (e2e_ms / 1e3)

    # per-stage device times (un-graphed launches with stage events): roofline of the
    # integration kernel, the largest stage
    ctx.enable_timing(True)
    stage = np.zeros(6)
    reps = max(3, min(args.steps, 5))
    touched = 0
    for k in range(reps):
        ctx.batch_tick(sessions, dframes(base - reps + k), device=True)
        stage += np.array([ctx.stage_ms(i) for i in range(6)])
        touched += sum(s.touched() for s in sessions)
    ctx.enable_timing(False)
    stage /= reps
    touched /= reps
    bytes_per_voxel = 3  # FP16 tsdf + u8 weight
    # algorithmic bytes of one integration launch: every voxel's state read and written once
    # plus each session's depth image read once (N_vox * 2 * S + W * H * 4 per session)
    n_vox = sum(int(np.prod(c.res)) for c in session_cfgs(L, n, L.TSDF_F16_U8))
    integ_bytes = n_vox * 2 * bytes_per_voxel + n * W_IMG * H_IMG * 4
    touched_bytes = touched * 2 * bytes_per_voxel + n * W_IMG * H_IMG * 4
    integ_ms = stage[3]
    peak, peak_kind = peaks()
    achieved = integ_bytes / (integ_ms / 1e3) / 1e9

    plain = None
    if args.plain:
        for s in sessions:
            s.close()
        sessions = None
        torch.cuda.empty_cache()
        plain_sessions = make_sessions(L.TSDF_F32)
        for w in range(args.warmup):
            for i, s in enumerate(plain_sessions):
                s.process_device(dframes(w)[i])
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        psteps = max(2, args.steps // 2)
        for k in range(psteps):
            fr = dframes(args.warmup + k)
            for i, s in enumerate(plain_sessions):
                s.process_device(fr[i])
        p1.record(stream)
        torch.cuda.synchronize()
        pms = max_over_ranks(p0.elapsed_time(p1), world)
        plain = n * world * psteps / (pms / 1e3)
        for s in plain_sessions:
            s.close()

    if rank == 0:
        cpu = cpu_baseline(args) if world == 1 and not args.no_cpu else None
        lat = np.array(per_tick)
        line = {
            "metric": "aggregate frames/s + p99 frame latency @64 sessions, ATE<=1mm vs plain FP32",
            "value": round(value, 2), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f16",
            "data": "synthetic: seeded analytic tabletop scenes, Kinect noise model",
            "config": {"workload": "serving-dense-%dx640x480" % n, "sessions_per_gpu": n,
                       "volumes": "dense FP16 TSDF + u8 weight, %s^3 round-robin" % "/".join(map(str, VOLUMES)),
                       "icp_iterations": [10, 5, 4], "l2": "inputs larger than L2 (volumes ~13 GB per GPU)",
                       "graph": "one CUDA graph per tick"},
            "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 3),
                           "p99": round(float(np.percentile(lat, 99)), 3),
                           "e2e_p50": round(float(np.percentile(e2e_tick, 50)), 3),
                           "e2e_p99": round(float(np.percentile(e2e_tick, 99)), 3)},
            "plain_fp32_per_session_fps": round(plain, 2) if plain else None,
            "speedup_vs_plain_fp32": round(value / plain, 3) if plain else None,
            "stage_ms": {k: round(float(v), 4) for k, v in
                         zip(["preprocess", "pyramid+feedback", "icp", "integrate", "raycast", "tick"], stage)},
            "e2e": {"value": round(e2e_value, 2), "unit": "frames/s",
                    "h2d_bytes_per_step": n * W_IMG * H_IMG * 2, "d2h_bytes_per_step": n * (14 * 4 + 2 * 4)},
            "gpu_launches": launches_per_tick * args.steps,
            "roofline": {"kernel": "k_integrate<F16_U8>", "bound": "hbm", "achieved": round(achieved, 1),
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": profile_traffic("k_integrate"),
                         "algorithmic_bytes_per_launch": int(integ_bytes), "launch_ms": round(float(integ_ms), 4),
                         "touched_voxel_bytes_per_launch": int(touched_bytes),
                         "touched_voxel_gbs": round(touched_bytes / (integ_ms / 1e3) / 1e9, 1)},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "tracking_lost": lost,
        }
        print(json.dumps(line))
    return 0


def tick_launch_count(sessions):
    # tick_begin + preprocess + 2 pyramid + feedback + 19 icp + finalize + publish + integrate
    # + brick summary + raycast
    return 1 + 1 + 2 + 1 + 19 + 1 + 1 + 1 + 1 + 1


def profile_traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    try:
        for line in open(path):
            if line.startswith(kernel + " "):
                return float(line.split()[1])
    except Exception:
        pass
    return None


def max_over_ranks(ms, world):
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(args, seconds=10.0):
    """The oracle (CPU restatement of the reference path), one session at the bench's
    smallest volume, timed on the host cores for a bounded number of frames."""
    from natureuserinterfacestudio_b200 import _lib as L
    from oracle import oracle as O
    cfg = session_cfgs(L, 1, L.TSDF_I16)[0]
    eng = O.Engine(cfg)
    seq = render_sequences(L, 1, 40, seed0=900)[0]
    eng.frame(seq[0])
    t0 = time.perf_counter()
    k = 0
    while k < len(seq) - 1 and time.perf_counter() - t0 < seconds:
        eng.frame(seq[1 + k])
        k += 1
    dt = time.perf_counter() - t0
    cores = os.cpu_count()
    return {"value": round(k / dt, 3), "unit": "frames/s", "cores": cores, "kind": "port",
            "sample": "%d tracked frames of one 640x480 session, 256^3 int16 TSDF, %d OpenMP threads" % (k, cores)}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    cpu = cpu_baseline(args, seconds=max(5.0, min(60.0, 3.0 * args.steps)))
    line = {"impl": "reference", "metric": "aggregate frames/s + p99 frame latency @64 sessions, ATE<=1mm vs plain FP32",
            "value": cpu["value"], "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "serving-dense-%dx640x480" % args.sessions,
                                            "sample": "one session on the host cores"},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sessions", type=int, default=64)
    ap.add_argument("--sequences", type=int, default=8)
    ap.add_argument("--no-plain", dest="plain", action="store_false")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and args.impl == "ours":
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        if args.impl == "reference":
            return run_reference(args, rank, world)
        return run_ours(args, rank, world)
    finally:
        if world > 1 and args.impl == "ours":
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
