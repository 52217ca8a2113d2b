"""Benchmark: aggregate frames/s and per-frame latency of 64 concurrent KinectFusion streams
on one B200 (weak scaling: each GPU/rank serves its own streams).

Workload (the serving configuration): 64 streams of 640x480 depth, 60 % dense volumes
(FP16 TSDF + u8 weight, 256^3 over 3 m / 384^3 and 512^3 over 4 m, round robin) and 40 %
voxel-block hash scenes (5 mm voxels, 2^20 buckets, pools of 2^19 / 2^20 / 2^21 blocks,
half-precision sdf + u8 weight); 3-level point-to-plane ICP (10/5/4 iterations), every
frame integrated and raycast.  Inputs: seeded analytic tabletop scenes rendered with the
Kinect noise model, each stream on one of 8 orbit sequences (frames replayed forth and
back so that the motion stays continuous).

A step is one tick: every stream advances one frame, all streams in one batched launch
sequence replayed from a CUDA graph.
  value    streams * steps / device time, frames already resident in HBM;
  e2e      the same 64 streams through the serving loop (nui_server_*): frames from pinned
           host memory, uploads on a second stream overlapped with the previous tick,
           poses read back; wall-clock over the steps;
  serving  a real-time run of the serving loop: streams arrive as a Poisson process, send
           frames at 30 Hz +- 3 ms, live an exponential number of frames (mean 300) and are
           admitted under a 150 GB HBM budget; per-frame latency p50 / p99.
The in-GPU comparison is the plain FP32 path: one stream per launch sequence, FP32 dense
TSDF (int16 hash), no graph.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
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
HASH_POOLS = (1 << 19, 1 << 20, 1 << 21)
SEQ_FRAMES = 30
METRIC = "aggregate frames/s + p99 frame latency @64 sessions, ATE<=1mm vs plain FP32"


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
        self.active = False

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
            if len(parts) == 7 and self.active:
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


def stream_cfg(L, i, fmt_dense, fmt_hash):
    """Configuration of stream i: 3 of every 5 dense, 2 hash."""
    if i % 5 < 3:
        r = VOLUMES[(i // 5 * 3 + i % 5) % len(VOLUMES)]
        dim = 3.0 if r == 256 else 4.0
        return L.default_cfg(res=(r, r, r), dim=(dim, dim, dim), tsdf_format=fmt_dense, trunc_dist=0.03,
                             iterations=[10, 5, 4, 0], integration_threshold=0.0)
    # voxel-hash streams are RGB-D: colour volume and colour ICP (photometric weight 0.1)
    pool = HASH_POOLS[(i // 5 * 2 + i % 5 - 3) % len(HASH_POOLS)]
    return L.default_cfg(volume_kind=L.VOLUME_HASH, tsdf_format=fmt_hash, voxel_size=0.005, trunc_scale=0.02,
                         hash_buckets=1 << 20, hash_excess=1 << 16, hash_pool_blocks=pool,
                         iterations=[10, 5, 4, 0], integration_threshold=0.0, depth_min=0.4,
                         color_volume=1, photometric_weight=0.1)


def stream_cfgs(L, n, fmt_dense, fmt_hash):
    return [stream_cfg(L, i, fmt_dense, fmt_hash) for i in range(n)]


def is_hash(c):
    return c.volume_kind == 1


def render_sequences(L, nseq, nframes, seed0=100, poses=False, color=False):
    """nseq orbit sequences of nframes depth frames (with color=True, (depth, BGRA) pairs;
    with poses=True also their true camera poses (R, t) in the scene frame)."""
    seqs, gts = [], []
    for k in range(nseq):
        sc = L.SynthScene(L.SYNTH_TABLETOP, seed=seed0 + k, extent=3.0)
        fr, gt = [], []
        for i in range(nframes):
            R, t = sc.pose(i, radius=1.5, deg_per_frame=2.0)
            d, c = sc.render(R, t, W_IMG, H_IMG, frame=i, noise_seed=seed0 * 7 + k, color=color)
            fr.append((d, np.ascontiguousarray(c)) if color else d)
            gt.append((np.asarray(R, np.float64), np.asarray(t, np.float64)))
        seqs.append(fr)
        gts.append(gt)
    return (seqs, gts) if poses else seqs


def pingpong(k, n=SEQ_FRAMES):
    """Frame index of step k replaying a sequence forth and back."""
    p = 2 * n - 2
    k %= p
    return k if k < n else p - k


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
    nseq = min(n, args.sequences)
    seqs, gts = render_sequences(L, nseq, SEQ_FRAMES, poses=True, color=True)
    dev_frames = [[torch.from_numpy(d.view(np.int16)).cuda() for d, _ in s] for s in seqs]
    dev_colors = [[torch.from_numpy(c).cuda() for _, c in s] for s in seqs]
    host_frames = [[torch.from_numpy(d.view(np.int16)).pin_memory() for d, _ in s] for s in seqs]
    host_colors = [[torch.from_numpy(c).pin_memory() for _, c in s] for s in seqs]
    torch.cuda.synchronize()
    offs = [(i * 7) % 11 for i in range(n)]  # streams sharing a sequence start at different frames
    cfgs = stream_cfgs(L, n, L.TSDF_F16_U8, L.TSDF_F16_U8)
    n_hash = sum(is_hash(c) for c in cfgs)

    def dframes(step):
        return [dev_frames[i % nseq][pingpong(offs[i] + step)].data_ptr() for i in range(n)]

    def dcolors(step):  # BGRA for the RGB-D (voxel-hash) streams
        return [dev_colors[i % nseq][pingpong(offs[i] + step)].data_ptr() if is_hash(cfgs[i]) else None
                for i in range(n)]

    def hframe(i, step):
        return host_frames[i % nseq][pingpong(offs[i] + step)].numpy()

    def hcolor(i, step):
        return host_colors[i % nseq][pingpong(offs[i] + step)].numpy() if is_hash(cfgs[i]) else None

    # ---------------------------------------------------------------- launch shapes
    tuning, tune_s = None, 0.0
    if args.tuning:
        ctx.set_tuning(L.Tuning(*[int(x) for x in args.tuning.split(",")]))
        tuning = ctx.tuning().as_dict()
    elif not args.no_autotune:
        t0 = time.perf_counter()
        t, _ = ctx.autotune(cfgs, [[hframe(i, k) for k in range(8)] for i in range(n)], repeats=5,
                            bgras=[[hcolor(i, k) for k in range(8)] for i in range(n)])
        tune_s = time.perf_counter() - t0
        tuning = t.as_dict()
        torch.cuda.empty_cache()
    ctx.trim()

    # ---------------------------------------------------------------- value: device frames
    sessions = [L.Session(ctx, c) for c in cfgs]
    with ClockSampler(dev) as clk:
        for w in range(args.warmup):
            ctx.batch_tick(sessions, dframes(w), dcolors(w), device=True)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        clk.active = True
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tick_ev = []
        lost = 0
        e0.record(stream)
        for k in range(args.steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            st, _ = ctx.batch_tick(sessions, dframes(args.warmup + k), dcolors(args.warmup + k), device=True)
            b.record(stream)
            tick_ev.append((a, b))
            lost += int(np.sum(st != 0))
        e1.record(stream)
        torch.cuda.synchronize()
        clk.active = False
    kernels_per_tick = ctx.last_tick_kernels()
    ms_total = max_over_ranks(e0.elapsed_time(e1), world)
    per_tick = [a.elapsed_time(b) for a, b in tick_ev]
    value = n * world * args.steps / (ms_total / 1e3)

    # per-stage device times (un-graphed launches with stage events) and the work the
    # kernels counted in the same ticks
    ctx.enable_timing(True)
    stage = np.zeros(9)
    reps = 3
    work = {"touched": 0, "bricks": 0, "ray_reads": 0, "ray_samples": 0, "ray_hits": 0, "icp_px": 0, "icp_px_dense": 0,
            "tiles": 0}
    for k in range(reps):
        ctx.batch_tick(sessions, dframes(args.warmup + args.steps + k), dcolors(args.warmup + args.steps + k),
                       device=True)
        stage += np.array([ctx.stage_ms(i) for i in range(9)])
        for s, c in zip(sessions, cfgs):
            w = s.work_counters()
            if not is_hash(c):
                for key in ("touched", "bricks", "ray_reads", "ray_samples", "ray_hits", "tiles"):
                    work[key] += w[key]
            px = sum(it * (W_IMG >> l) * (H_IMG >> l) for l, it in enumerate(w["icp_iters"]))
            work["icp_px"] += px
            if not is_hash(c):
                work["icp_px_dense"] += px
    ctx.enable_timing(False)
    stage /= reps
    work = {k: v / reps for k, v in work.items()}
    hash_visible = [s.hash_stats()[0] for s, c in zip(sessions, cfgs) if is_hash(c)]
    for s in sessions:
        s.close()
    sessions = None
    torch.cuda.empty_cache()
    ctx.trim()

    # rooflines of the dominant kernels, from the work the kernels counted:
    #   integration (k_integrate_fast, stage 3): updated voxels read and written (3 B each
    #     way, FP16 + u8), the voxels of re-classified bricks read once, the depth image read;
    #   dense raycast (k_raycast_fast + k_raycast_finish_fast, stage 7): the voxels the march
    #     read, one brick-state byte per visited sample, 64 voxels per refined crossing, and
    #     the vertex / normal / colour maps written (12 + 12 + 4 B a pixel);
    #   ICP (k_icp_cluster over the dense sessions, stage 2 -- the hash sessions' tracking runs
    #     on the second stream): per pixel-iteration the depth (4 B) and one reference vertex
    #     and normal (16 + 16 B).
    dense = [c for c in cfgs if not is_hash(c)]
    npx = W_IMG * H_IMG
    peak, peak_kind = peaks()
    kernels = [
        ("k_integrate_fast<F16_U8>", stage[3],
         work["touched"] * 6 + work["bricks"] * 512 * 3 + len(dense) * npx * 4),
        ("k_raycast_fast<F16_U8>+k_raycast_finish_fast<F16_U8>", stage[7],
         work["ray_reads"] * 3 + work["ray_samples"] + work["ray_hits"] * 64 * 3 + len(dense) * npx * 28),
        ("k_icp_cluster", stage[2], work["icp_px_dense"] * 36),
    ]
    roof = []
    for name, ms, nbytes in kernels:
        ach = nbytes / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        roof.append({"kernel": name, "bound": "hbm", "achieved": round(ach, 1), "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": profile_traffic(name.split("<")[0]),
                     "algorithmic_bytes_per_launch": int(nbytes), "launch_ms": round(float(ms), 4)})
    top = max(roof, key=lambda r: r["launch_ms"])

    # ---------------------------------------------------------------- batched mixed sizes
    mixed = mixed_batch(L, ctx, torch, args.steps, args.warmup) if args.mixed else None
    torch.cuda.empty_cache()
    ctx.trim()
    if tuning is not None:  # the mixed batch autotuned the context for itself
        ctx.set_tuning(L.Tuning(**tuning))

    # ---------------------------------------------------------------- ATE vs plain FP32
    ate = ate_vs_plain(L, ctx, seqs, gts, args.ate_frames, args.ate_streams) if args.ate_frames > 0 else None
    torch.cuda.empty_cache()
    ctx.trim()

    # ---------------------------------------------------------------- e2e: serving loop
    srv = L.Server(ctx, 150 << 30, max_streams=max(64, n))
    slots = [srv.admit(c) for c in cfgs]
    assert all(s is not None for s in slots), "the 64 streams must fit the budget"
    for w in range(args.warmup):
        for i, sl in enumerate(slots):
            srv.submit(sl, hframe(i, w), hcolor(i, w), tag=w)
        srv.step()
    srv.drain()
    srv.poll()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lat = []
    for k in range(args.steps):
        for i, sl in enumerate(slots):
            srv.submit(sl, hframe(i, args.warmup + k), hcolor(i, args.warmup + k), tag=args.warmup + k)
        srv.step()
        lat += [r.t_done - r.t_submit for r in srv.poll()]
    srv.drain()
    lat += [r.t_done - r.t_submit for r in srv.poll()]
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s * 1e3, world) / 1e3
    e2e_value = n * world * args.steps / e2e_s
    e2e_lat = np.array(lat) * 1e3
    srv.close()
    torch.cuda.empty_cache()
    ctx.trim()

    # ---------------------------------------------------------------- serving simulation
    sim = serving_sim(L, ctx, host_frames, host_colors, args.serve_seconds, n) if args.serve_seconds > 0 else None
    torch.cuda.empty_cache()
    ctx.trim()

    # ---------------------------------------------------------------- plain FP32 path
    plain = None
    if args.plain:
        plain_sessions = [L.Session(ctx, c) for c in stream_cfgs(L, n, L.TSDF_F32, L.TSDF_I16)]
        for w in range(args.warmup):
            fr, co = dframes(w), dcolors(w)
            for i, s in enumerate(plain_sessions):
                s.process_device(fr[i], co[i])
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        psteps = max(2, min(args.steps, 10))
        p0.record(stream)
        for k in range(psteps):
            fr, co = dframes(args.warmup + k), dcolors(args.warmup + k)
            for i, s in enumerate(plain_sessions):
                s.process_device(fr[i], co[i])
        p1.record(stream)
        torch.cuda.synchronize()
        pms = max_over_ranks(p0.elapsed_time(p1), world)
        plain = n * world * psteps / (pms / 1e3)
        for s in plain_sessions:
            s.close()

    if rank == 0:
        cpu = cpu_baseline(args) if world == 1 and not args.no_cpu else None
        lat_t = np.array(per_tick)
        line = {
            "metric": METRIC,
            "value": round(value, 2), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_total / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f16",
            "data": "synthetic: seeded analytic tabletop scenes, Kinect noise model",
            "config": {"workload": "serving-%dx640x480-dense%d-hash%d" % (n, n - n_hash, n_hash),
                       "streams_per_gpu": n,
                       "dense": "FP16 TSDF + u8 weight, %s^3 round robin" % "/".join(map(str, VOLUMES)),
                       "hash": "RGB-D: 5 mm voxels, 2^20 buckets, pools 2^19/2^20/2^21 blocks, half sdf + u8 weight + "
                               "RGB, colour ICP (photometric weight 0.1)",
                       "icp_iterations": [10, 5, 4], "l2": "inputs larger than L2 (volumes ~60 GB per GPU)",
                       "graph": "one CUDA graph per tick",
                       "tuning": tuning, "autotune_s": round(tune_s, 2)},
            "latency_ms": {"tick_p50": round(float(np.percentile(lat_t, 50)), 3),
                           "tick_p99": round(float(np.percentile(lat_t, 99)), 3),
                           "e2e_p50": round(float(np.percentile(e2e_lat, 50)), 3),
                           "e2e_p99": round(float(np.percentile(e2e_lat, 99)), 3)},
            "serving": sim,
            "plain_fp32_per_session_fps": round(plain, 2) if plain else None,
            "speedup_vs_plain_fp32": round(value / plain, 3) if plain else None,
            "stage_ms": {k: round(float(v), 4) for k, v in zip(
                ["preprocess", "pyramid+feedback", "track", "integrate_dense_kernel", "summaries+hash_integrate",
                 "raycast", "tick", "raycast_dense_kernels", "hash_side_stream"], stage)},
            "work_per_tick": {k: int(v) for k, v in work.items()},
            "ate": ate,
            "batched_mixed": mixed,
            "hash_visible_blocks_mean": round(float(np.mean(hash_visible)), 1) if hash_visible else None,
            "e2e": {"value": round(e2e_value, 2), "unit": "frames/s",
                    "h2d_bytes_per_step": n * W_IMG * H_IMG * 2 + n_hash * W_IMG * H_IMG * 4,
                    "d2h_bytes_per_step": n * (14 * 4 + 2 * 4)},
            "gpu_launches": kernels_per_tick * args.steps,
            "roofline": top,
            "roofline_kernels": roof,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "tracking_lost": lost,
        }
        print(json.dumps(line))
    return 0


def serving_sim(L, ctx, host_frames, host_colors, seconds, n_target, warm=2.0, seed=11):
    """Real-time run of the serving loop.  Streams arrive as a Poisson process whose rate
    keeps n_target streams live at steady state (Little's law with a mean life of 300
    frames at 30 Hz), send frames every 1/30 s +- 3 ms, and are admitted under a 150 GB
    HBM budget (those that do not fit wait).  The run starts with n_target live streams."""
    rng = np.random.default_rng(seed)
    nseq = len(host_frames)
    life_mean = 300
    lam = n_target / (life_mean / 30.0)
    srv = L.Server(ctx, 150 << 30, max_streams=n_target + 32)
    live, waiting, lat, done_frames = {}, [], [], 0
    count = [0]

    def new_stream(now):
        i = count[0]
        count[0] += 1
        return {"id": i, "cfg": stream_cfg(L, i, L.TSDF_F16_U8, L.TSDF_F16_U8), "seq": i % nseq,
                "off": (i * 7) % 11, "life": max(1, int(rng.exponential(life_mean))), "sent": 0, "back": 0,
                "next": now + rng.uniform(0, 1 / 30.0), "arrived": now}

    waits = []

    admit_ms = []

    def try_admit(st, now):
        a0 = time.perf_counter()
        sl = srv.admit(st["cfg"])
        admit_ms.append((time.perf_counter() - a0) * 1e3)
        if sl is None:
            return False
        st["slot"] = sl
        st["next"] = max(st["next"], srv.clock())
        waits.append(srv.clock() - st["arrived"])
        live[sl] = st
        return True

    start = srv.clock()
    for _ in range(n_target):
        try_admit(new_stream(start), start)
    initial_admit_ms = list(admit_ms)
    admit_ms.clear()
    # warm pool: two idle sessions of every stream configuration for the arrivals to come
    # (about two seconds of arrivals of each kind)
    kinds = {}
    for i in range(15):
        c = stream_cfg(L, i, L.TSDF_F16_U8, L.TSDF_F16_U8)
        kinds[bytes(c)] = c
    for c in kinds.values():
        srv.reserve(c, 2)
    start = srv.clock()
    for st in live.values():
        st["next"] = start + rng.uniform(0, 1 / 30.0)
    t_end = start + warm + seconds
    next_arrival = start + rng.exponential(1 / lam)
    conc = []
    step_ms = []
    steps = 0
    while True:
        now = srv.clock()
        if now >= t_end:
            break
        while next_arrival <= now:
            waiting.append(new_stream(next_arrival))
            next_arrival += rng.exponential(1 / lam)
        while waiting and try_admit(waiting[0], now):
            waiting.pop(0)
        for st in live.values():
            while st["sent"] < st["life"] and st["next"] <= now:
                fi = pingpong(st["off"] + st["sent"])
                fr = host_frames[st["seq"]][fi].numpy()
                co = host_colors[st["seq"]][fi].numpy() if is_hash(st["cfg"]) else None
                srv.submit(st["slot"], fr, co, tag=st["sent"], t_submit=st["next"])
                st["sent"] += 1
                st["next"] += 1 / 30.0 + rng.uniform(-0.003, 0.003)
        s0 = time.perf_counter()
        launched = srv.step()
        step_ms.append((time.perf_counter() - s0) * 1e3)
        steps += 1
        for r in srv.poll():
            st = live[r.slot]
            st["back"] += 1
            if r.t_submit >= start + warm:
                lat.append(r.t_done - r.t_submit)
                done_frames += 1
        for sl in [s for s, st in live.items() if st["back"] >= st["life"]]:
            srv.release(sl)
            del live[sl]
        conc.append(len(live))
        if launched == 0:
            time.sleep(0.0005)
    srv.drain()
    srv.close()
    lat = np.array(lat) * 1e3
    return {"seconds": seconds, "arrivals_per_s": round(lam, 2), "mean_life_frames": life_mean, "frame_hz": 30,
            "hbm_budget_gb": 150, "mean_live_streams": round(float(np.mean(conc)), 1),
            "frames": int(done_frames), "fps": round(done_frames / seconds, 1),
            "latency_p50_ms": round(float(np.percentile(lat, 50)), 3) if lat.size else None,
            "latency_p99_ms": round(float(np.percentile(lat, 99)), 3) if lat.size else None,
            "admission_wait_p99_ms": round(float(np.percentile(np.array(waits) * 1e3, 99)), 1) if waits else None,
            "loop_steps": steps, "step_ms_p99": round(float(np.percentile(step_ms, 99)), 2),
            "step_ms_max": round(float(np.max(step_ms)), 2),
            "admit_ms_max": round(float(np.max(admit_ms)), 2) if admit_ms else None,
            "admit_ms_p99": round(float(np.percentile(admit_ms, 99)), 3) if admit_ms else None,
            "admissions": len(admit_ms), "admissions_over_5ms": int(sum(a > 5 for a in admit_ms)),
            "initial_admit_ms_max": round(float(np.max(initial_admit_ms)), 2) if initial_admit_ms else None}


def mixed_batch(L, ctx, torch, steps, warmup, seed=4):
    """The batched configuration: 32 independent sessions, one frame each per tick, all in
    one graphed tick; volumes drawn from {128^3, 256^3, 384^3, 512^3} as dense FP16 TSDF +
    u8 weight or voxel hash at 5-10 mm, images from {320x240, 640x480}, each session on its
    own seeded scene and orbit; launch shapes from the autotuner.  Reports frames/s and the
    tick's p50 / p99 (frames already on the device; inputs larger than L2)."""
    rng = np.random.default_rng(seed)
    nsess, nfr = 32, 12
    cfgs, frames_d = [], []
    for i in range(nsess):
        W, H = (320, 240) if rng.random() < 0.5 else (640, 480)
        f = 525.0 * W / 640.0
        common = dict(width=W, height=H, fx=f, fy=f, cx=(W - 1) / 2.0, cy=(H - 1) / 2.0, iterations=[10, 5, 4, 0],
                      integration_threshold=0.0)
        if rng.random() < 0.6:
            r = int(rng.choice([128, 256, 384, 512]))
            dim = 3.0 if r <= 256 else 4.0
            c = L.default_cfg(res=(r, r, r), dim=(dim, dim, dim), tsdf_format=L.TSDF_F16_U8, trunc_dist=0.03, **common)
        else:
            vox = float(rng.uniform(0.005, 0.010))
            c = L.default_cfg(volume_kind=L.VOLUME_HASH, tsdf_format=L.TSDF_F16_U8, voxel_size=vox,
                              trunc_scale=4 * vox, hash_buckets=1 << 20, hash_excess=1 << 16,
                              hash_pool_blocks=1 << 19, depth_min=0.4, **common)
        cfgs.append(c)
        sc = L.SynthScene(L.SYNTH_TABLETOP, seed=1000 + i, extent=3.0)
        fr = []
        for k in range(nfr):
            R, t = sc.pose(k, radius=1.5, deg_per_frame=2.0, traj_seed=2000 + i)
            d, _ = sc.render(R, t, W, H, fx=f, fy=f, cx=(W - 1) / 2.0, cy=(H - 1) / 2.0, frame=k, noise_seed=3000 + i)
            fr.append(d)
        frames_d.append(fr)
    dev = [[torch.from_numpy(d.view(np.int16)).cuda() for d in fr] for fr in frames_d]
    t0 = time.perf_counter()
    tune, _ = ctx.autotune(cfgs, [fr[:4] for fr in frames_d], repeats=3)
    tune_s = time.perf_counter() - t0
    sessions = [L.Session(ctx, c) for c in cfgs]
    stream = torch.cuda.current_stream()

    def fptr(k):
        return [dev[i][pingpong(k, nfr)].data_ptr() for i in range(nsess)]
    for k in range(warmup):
        ctx.batch_tick(sessions, fptr(k), device=True)
    torch.cuda.synchronize()
    ticks = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    lost = 0
    for k in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        st, _ = ctx.batch_tick(sessions, fptr(warmup + k), device=True)
        b.record(stream)
        ticks.append((a, b))
        lost += int(np.sum(st != 0))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    per = np.array([a.elapsed_time(b) for a, b in ticks])
    kinds = {"dense": sum(not is_hash(c) for c in cfgs), "hash": sum(is_hash(c) for c in cfgs),
             "640x480": sum(c.width == 640 for c in cfgs)}
    for s_ in sessions:
        s_.close()
    return {"workload": "batched-32-mixed", "sessions": nsess, "mix": kinds, "steps": steps,
            "frames_per_s": round(nsess * steps / (ms / 1e3), 1), "tick_ms_p50": round(float(np.percentile(per, 50)), 3),
            "tick_ms_p99": round(float(np.percentile(per, 99)), 3), "tracking_lost": lost,
            "kernels_per_tick": ctx.last_tick_kernels(), "tuning": tune.as_dict(), "autotune_s": round(tune_s, 2)}


def _rel(gt, i0, i):
    """Pose i of a sequence in the camera frame of pose i0 (trackers start at identity)."""
    R0, t0 = gt[i0]
    R, t = gt[i]
    return R0.T @ R, R0.T @ (t - t0)


def ate_vs_plain(L, ctx, seqs, gts, nframes, nstreams):
    """The metric's accuracy condition: the first nstreams streams of the mix run nframes
    frames (sequences replayed forth and back) in the served formats (FP16 TSDF + u8
    weight, half-precision hash, one batched tick per frame) and in the plain path (FP32
    dense TSDF / int16 hash, one stream at a time).  Reported per stream: the RMS distance
    between the two trajectories' camera positions, and each one's ATE against the true
    trajectory (RMS position error after both start at the first frame's pose).  The plain
    path also runs a second time with other ICP launch shapes (8-block clusters, 8 pixels a
    thread), which change nothing but the FP64 rounding of the ICP sums: the spread between
    the two plain runs is how far rounding alone moves a trajectory of that stream."""
    nseq = len(seqs)
    cfg16 = stream_cfgs(L, nstreams, L.TSDF_F16_U8, L.TSDF_F16_U8)
    cfg32 = stream_cfgs(L, nstreams, L.TSDF_F32, L.TSDF_I16)
    offs = [(i * 7) % 11 for i in range(nstreams)]
    idx = [[pingpong(offs[i] + k) for k in range(nframes)] for i in range(nstreams)]
    tune0 = ctx.tuning().as_dict()

    def frames(k):
        fr = [seqs[i % nseq][idx[i][k]][0] for i in range(nstreams)]
        co = [seqs[i % nseq][idx[i][k]][1] if is_hash(cfg16[i]) else None for i in range(nstreams)]
        return fr, co

    a = [L.Session(ctx, c) for c in cfg16]
    b = [L.Session(ctx, c) for c in cfg32]
    p16 = np.zeros((nstreams, nframes, 3))
    p32 = np.zeros((nstreams, nframes, 3))
    for k in range(nframes):
        fr, co = frames(k)
        _, poses = ctx.batch_tick(a, fr, co)
        p16[:, k] = poses[:, 9:]
        for i in range(nstreams):
            p32[i, k] = b[i].process(fr[i], co[i])[1][9:]
    for s in a + b:
        s.close()
    # the plain path again with other ICP launch shapes
    ctx.set_tuning(L.Tuning(**dict(tune0, icp_cluster_blocks=8, icp_pixels_per_thread=8)))
    b = [L.Session(ctx, c) for c in cfg32]
    p32b = np.zeros((nstreams, nframes, 3))
    for k in range(nframes):
        fr, co = frames(k)
        for i in range(nstreams):
            p32b[i, k] = b[i].process(fr[i], co[i])[1][9:]
    for s in b:
        s.close()
    ctx.set_tuning(L.Tuning(**tune0))

    def rms(x):
        return round(float(np.sqrt(np.mean(np.sum(x ** 2, 1)))) * 1e3, 3)

    out = []
    for i in range(nstreams):
        gt = np.array([_rel(gts[i % nseq], idx[i][0], idx[i][k])[1] for k in range(nframes)])
        out.append({"stream": i, "kind": "hash" if is_hash(cfg16[i]) else "dense %d^3" % cfg16[i].res[0],
                    "traj_rms_diff_mm": rms(p16[i] - p32[i]), "ate_fp16_mm": rms(p16[i] - gt),
                    "ate_plain_fp32_mm": rms(p32[i] - gt), "ate_plain_reshaped_mm": rms(p32b[i] - gt),
                    "plain_vs_reshaped_traj_rms_diff_mm": rms(p32[i] - p32b[i])})
    worst = max(abs(o["ate_fp16_mm"] - o["ate_plain_fp32_mm"]) for o in out)
    floor = max(abs(o["ate_plain_reshaped_mm"] - o["ate_plain_fp32_mm"]) for o in out)
    return {"frames": nframes, "streams": out, "max_abs_ate_diff_mm": round(worst, 3),
            "max_traj_rms_diff_mm": round(max(o["traj_rms_diff_mm"] for o in out), 3),
            "max_abs_ate_diff_plain_vs_reshaped_mm": round(floor, 3),
            "streams_within_1mm": int(sum(abs(o["ate_fp16_mm"] - o["ate_plain_fp32_mm"]) <= 1.0 for o in out)),
            "within_1mm": bool(worst <= 1.0)}


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
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_baseline(args, seconds=12.0):
    """The reference's own kernels (oracle/_ref: its OpenCL C compiled for the host, run on
    all host cores; the host-side ICP step from the oracle's restatement) on the dense part
    of the served mix: one stream each of 256^3 over 3 m, 384^3 and 512^3 over 4 m in the
    reference's int16 format, 640x480, ICP 10/5/4, every frame integrated and raycast, for
    a bounded number of frames each."""
    import types

    from natureuserinterfacestudio_b200 import synth  # input generation only: not the product library
    from oracle.ref_engine import RefEngine
    seq = render_sequences(synth, 1, 12, seed0=900)[0]
    frames, spent = 0, 0.0
    for r in VOLUMES:
        dim = 3.0 if r == 256 else 4.0
        # the stream's configuration; tracker values of NuiTrackerConfig (NuiTrackerConfig.cpp:5-24)
        cfg = types.SimpleNamespace(width=W_IMG, height=H_IMG, fx=FOCAL, fy=FOCAL, cx=(W_IMG - 1) / 2.0,
                                    cy=(H_IMG - 1) / 2.0, depth_min=0.5, depth_max=4.5, res=(r, r, r),
                                    dim=(dim, dim, dim), trunc_dist=0.03, filter_radius=3,
                                    sigma_space2_inv_half=0.08, sigma_depth2_inv_half=50.0, depth_threshold=0.3,
                                    dist_threshold=0.1, levels=3, iterations=[10, 5, 4, 0])
        eng = RefEngine(cfg)
        eng.frame(seq[0])  # the first frame only integrates
        t0 = time.perf_counter()
        k = 0
        while k < len(seq) - 1 and (k < 2 or time.perf_counter() - t0 < seconds / len(VOLUMES)):
            eng.frame(seq[1 + k])
            k += 1
        spent += time.perf_counter() - t0
        frames += k
    cores = os.cpu_count()
    return {"value": round(frames / spent, 3), "unit": "frames/s", "cores": cores, "kind": "reference",
            "sample": "%d tracked frames of 640x480 streams on 256^3 / 384^3 / 512^3 int16 volumes (the dense "
                      "part of the mix) through the reference's kernels compiled for the host, %d threads"
                      % (frames, cores)}


def _ate(poses, gt, idx0=0):
    """RMS position error (mm) of a trajectory against the true one, both from frame idx0."""
    err = [np.asarray(p, np.float64) - _rel(gt, idx0, k)[1] for k, p in enumerate(poses)]
    return round(float(np.sqrt(np.mean(np.sum(np.square(err), 1)))) * 1e3, 3)


STAGE_NAMES = ("preprocess", "pyramid+feedback", "track", "integrate", "summaries", "raycast", "tick")


def _run_stream(L, ctx, cfg, frames, colors, gt, mesh_every=0, mesh_cap=1 << 22, skip=3):
    """One stream frame by frame through the public per-frame call (host frames), with the
    per-stage device times of each frame; meshes every mesh_every frames.  Stage times and
    frames/s are taken over the frames after the first `skip`."""
    import torch
    s = L.Session(ctx, cfg)
    ctx.enable_timing(True)
    st, poses, mesh_ms, verts, lost = [], [], [], [], 0
    error = None
    for k in range(len(frames)):
        try:
            ok, p = s.process(frames[k], colors[k] if colors is not None else None)
        except L.NuiError as e:  # e.g. a full hash pool: the stream stops there
            error = {"frame": k, "status": e.status, "message": str(e)}
            break
        lost += 0 if ok else 1
        if k >= skip:
            st.append([ctx.stage_ms(i) for i in range(7)])
        poses.append(p[9:12].copy())
        if mesh_every and (k + 1) % mesh_every == 0:
            pos = np.zeros((mesh_cap, 3), np.float32)  # host buffers made outside the timing
            n = 0
            for rep in range(2):  # the first call also loads the kernels and tables
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                n = s.mesh_into(pos)
                torch.cuda.synchronize()
                if rep == 1:
                    mesh_ms.append((time.perf_counter() - t0) * 1e3)
            verts.append(int(n))
    ctx.enable_timing(False)
    hs = s.hash_stats() if cfg.volume_kind == 1 else None
    s.close()
    st = np.array(st)
    med = np.median(st, 0)
    out = {"frames": len(poses), "tracking_lost": lost, "frames_per_s": round(1e3 / float(med[6]), 1),
           "stage_ms_median": {n: round(float(v), 4) for n, v in zip(STAGE_NAMES, med)},
           "ate_mm": _ate(poses, gt)}
    if mesh_every:
        out["mesh_ms"] = [round(x, 2) for x in mesh_ms]
        out["mesh_vertices"] = verts
    if hs is not None:
        out["hash_visible_blocks_last"] = int(hs[0])
    if error is not None:
        out["error"] = error
    return out, np.array(poses)


def _render(L, kind, seed, n, color, W=W_IMG, H=H_IMG, radius=1.5, deg=2.0, extent=3.0):
    sc = L.SynthScene(kind, seed=seed, extent=extent)
    fr, co, gt = [], [], []
    for k in range(n):
        R, t = sc.pose(k, radius=radius, deg_per_frame=deg)
        d, c = sc.render(R, t, W, H, frame=k, noise_seed=seed * 7 + 1, color=color)
        fr.append(d)
        co.append(np.ascontiguousarray(c) if color else None)
        gt.append((np.asarray(R, np.float64), np.asarray(t, np.float64)))
    return fr, (co if color else None), gt


def _cpu_stages(frames, cfg_ns, nframes):
    """The reference's kernels compiled for the host (oracle/_ref), per stage, on the first
    nframes tracked frames of a sequence: ms per frame of preprocessing, ICP, integration and
    raycast (all host threads)."""
    from oracle.ref_engine import RefEngine
    eng = RefEngine(cfg_ns)
    spent = {"preprocess": 0.0, "icp": 0.0, "integrate": 0.0, "raycast": 0.0}
    pre, integ, ray = eng._preprocess, eng._integrate, eng._raycast

    def timed(name, f):
        def g(*a):
            t0 = time.perf_counter()
            r = f(*a)
            spent[name] += time.perf_counter() - t0
            return r
        return g
    eng._preprocess, eng._integrate, eng._raycast = timed("preprocess", pre), timed("integrate", integ), \
        timed("raycast", ray)
    eng.frame(frames[0])
    for k in spent:
        spent[k] = 0.0
    t0 = time.perf_counter()
    for k in range(1, nframes + 1):
        eng.frame(frames[k])
    total = time.perf_counter() - t0
    spent["icp"] = total - spent["preprocess"] - spent["integrate"] - spent["raycast"]
    return {"frames": nframes, "threads": os.cpu_count(), "frames_per_s": round(nframes / total, 3),
            "stage_ms": {k: round(v / nframes * 1e3, 1) for k, v in spent.items()},
            "format": "int16 (the reference's short2 volume)"}


def run_configs(args):
    """The workload's other configurations, each through the public per-frame or batched
    call on one GPU (synthetic scenes rendered first, not timed):
      1. dense 256^3 FP32 TSDF + weight over 3 m, 100 frames, ICP 10/5/4, marching cubes at
         the end; the reference's kernels on the host cores beside it, per stage;
      2. dense 512^3 over 4 m with colour ICP (photometric weight 0.1), FP32 against FP16 +
         u8, 100 frames;
      3. voxel hashing at 5 mm (2^20 buckets, 2^21-block pool), room-scale scene walked at
         1.2 m/s, colour ICP, raycast every frame, marching cubes every 100 frames;
      4. 32 batched sessions of mixed volume and image sizes (as in the main line).
    Prints one JSON line."""
    import types

    import torch
    from natureuserinterfacestudio_b200 import _lib as L
    torch.cuda.set_device(0)
    ctx = L.Context(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    out = {}
    # 1. plain dense 256^3
    fr, _, gt = _render(L, L.SYNTH_TABLETOP, 11, args.config_frames, False)
    cfg = L.default_cfg(res=(256, 256, 256), dim=(3.0, 3.0, 3.0), tsdf_format=L.TSDF_F32, trunc_dist=0.046875,
                        iterations=[10, 5, 4, 0], integration_threshold=0.0)
    r1, _ = _run_stream(L, ctx, cfg, fr, None, gt, mesh_every=len(fr))
    cpu_cfg = types.SimpleNamespace(width=W_IMG, height=H_IMG, fx=FOCAL, fy=FOCAL, cx=(W_IMG - 1) / 2.0,
                                    cy=(H_IMG - 1) / 2.0, depth_min=0.5, depth_max=4.5, res=(256, 256, 256),
                                    dim=(3.0, 3.0, 3.0), trunc_dist=0.046875, filter_radius=3,
                                    sigma_space2_inv_half=0.08, sigma_depth2_inv_half=50.0, depth_threshold=0.3,
                                    dist_threshold=0.1, levels=3, iterations=[10, 5, 4, 0])
    r1["cpu_reference"] = _cpu_stages(fr, cpu_cfg, args.config_cpu_frames)
    out["1_dense_256_fp32"] = r1
    # 2. dense 512^3 with colour ICP, FP32 and FP16 + u8
    fr, co, gt = _render(L, L.SYNTH_TABLETOP, 12, args.config_frames, True, extent=3.0)
    res2 = {}
    poses2 = {}
    for name, fmt in (("fp32", L.TSDF_F32), ("fp16_u8", L.TSDF_F16_U8)):
        cfg = L.default_cfg(res=(512, 512, 512), dim=(4.0, 4.0, 4.0), tsdf_format=fmt, trunc_dist=0.03,
                            iterations=[10, 5, 4, 0], integration_threshold=0.0, color_volume=1,
                            photometric_weight=0.1)
        res2[name], poses2[name] = _run_stream(L, ctx, cfg, fr, co, gt)
    res2["traj_rms_diff_mm"] = round(float(np.sqrt(np.mean(np.sum((poses2["fp32"] - poses2["fp16_u8"]) ** 2, 1))))
                                     * 1e3, 3)
    out["2_dense_512_color_fp32_vs_fp16"] = res2
    torch.cuda.empty_cache()
    ctx.trim()
    # 3. room-scale voxel hashing
    sc = L.SynthScene(L.SYNTH_ROOM, seed=13)
    fr, co, gt = [], [], []
    for k in range(args.room_frames):
        R, t = sc.pose(k)
        d, c = sc.render(R, t, W_IMG, H_IMG, frame=k, noise_seed=91, color=True)
        fr.append(d)
        co.append(np.ascontiguousarray(c))
        gt.append((np.asarray(R, np.float64), np.asarray(t, np.float64)))
    cfg = L.default_cfg(volume_kind=L.VOLUME_HASH, tsdf_format=L.TSDF_F16_U8, voxel_size=0.005, trunc_scale=0.02,
                        hash_buckets=1 << 20, hash_excess=1 << 20, hash_pool_blocks=1 << 21,
                        iterations=[10, 5, 4, 0], integration_threshold=0.0, depth_min=0.4, color_volume=1,
                        photometric_weight=0.1)
    out["3_hash_room_5mm"], _ = _run_stream(L, ctx, cfg, fr, co, gt, mesh_every=100, mesh_cap=1 << 24)
    out["3_hash_room_5mm"]["walk"] = "1.2 m/s at 30 Hz, %d frames" % args.room_frames
    torch.cuda.empty_cache()
    ctx.trim()
    # 4. batched mixed sizes
    out["4_batched_32_mixed"] = mixed_batch(L, ctx, torch, args.steps, args.warmup)
    print(json.dumps({"impl": "ours", "configs": out, "n_gpus": 1, "data": "synthetic: seeded analytic scenes, "
                      "Kinect noise model", "dtype": "f32 / f16"}))
    return 0


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    cpu = cpu_baseline(args, seconds=max(5.0, min(60.0, 3.0 * args.steps)))
    n_hash = sum(1 for i in range(args.sessions) if i % 5 >= 3)
    line = {"impl": "reference", "metric": METRIC,
            "value": cpu["value"], "unit": "frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": "serving-%dx640x480-dense%d-hash%d"
                                                        % (args.sessions, args.sessions - n_hash, n_hash),
                                            "sample": cpu["sample"]},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sessions", type=int, default=64)
    ap.add_argument("--sequences", type=int, default=8)
    ap.add_argument("--serve-seconds", dest="serve_seconds", type=float, default=12.0)
    ap.add_argument("--no-plain", dest="plain", action="store_false")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ate-frames", dest="ate_frames", type=int, default=100,
                    help="frames of the FP16-vs-plain-FP32 trajectory comparison (0: skip)")
    ap.add_argument("--ate-streams", dest="ate_streams", type=int, default=8)
    ap.add_argument("--no-mixed", dest="mixed", action="store_false",
                    help="skip the batched run of 32 sessions of mixed volume and image sizes")
    ap.add_argument("--no-autotune", dest="no_autotune", action="store_true",
                    help="keep the default launch shapes instead of timing the candidates first")
    ap.add_argument("--configs", action="store_true",
                    help="measure the other configurations (dense 256^3 with the reference's kernels on the host, "
                         "512^3 colour FP32 vs FP16, room-scale hash, batched) instead of the serving line")
    ap.add_argument("--config-frames", dest="config_frames", type=int, default=100)
    ap.add_argument("--config-cpu-frames", dest="config_cpu_frames", type=int, default=4)
    ap.add_argument("--room-frames", dest="room_frames", type=int, default=300)
    ap.add_argument("--tuning", default="",
                    help="launch shapes to use instead of autotuning: integration threads log2, ICP pixels "
                         "per thread, dense and hash ray tile widths, ICP blocks per session (e.g. 16,8,8,4,8)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.configs:
        return run_configs(args)
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
