#!/usr/bin/env python3
"""Benchmark of the frame-aligner non-rigid registration path on B200.

Workload: the 512x512x16 z-stack with nD = 32 control points and three displacement components,
50 frames per step (seeded synthetic acquisition: blob reference, random-walk displacement,
Poisson noise; see frame-aligner_b200/fa_synth.py). One step = FrameWarpAligner::addFrame for all
50 frames: +1 offset, phase-correlation rigid start (cuFFT FP64 + hand-written normalise / argmax),
starting-point choice and the trust-region solve, batched (one fused warp + error + J^T e pass and
one solve launch per iteration, captured in a CUDA graph).

  value  frames aligned per second with the frames already in HBM (device timing: CUDA events
         on the library's streams, summed over the K timed steps; max over ranks)
  e2e    the same through fa_aligner_add_frames with raw uint16 frames in pinned host memory,
         host->device copies and the D readback inside the timed region (wall clock)

Extra keys: `plain_fp32` (the FP32 single-frame path, host-driven iterations, one frame at a time,
timed both with frames resident in HBM and from host memory, so that each ratio compares like with
like), `serving` (the served stream: eight acquisitions of different sizes, Poisson arrivals at
2000 frames/s, 40 GB admission budget, warm start; p50/p99 latency and throughput), `roofline`
(the fused evaluation kernel against the measured HBM copy bandwidth), `cpu_baseline` (the
reference's CPU warper, compiled from its own sources, on a bounded sample), `clocks`.

--impl reference times the reference CPU path on this host's cores (rank 0 only).
"""
import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "frame-aligner_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import fa_synth as S  # noqa: E402

METRIC = "aligned frames/s at \u22640.01px RMS vs CPU ref; warp+J\u1d40J HBM GB/s; p99 frame latency"
UNIT = "frames/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=50)
    ap.add_argument("--plain-frames", type=int, default=8)
    ap.add_argument("--cpu-frames", type=int, default=0, help="CPU baseline sample size (0 = one per thread)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-uneven", action="store_true")
    ap.add_argument("--no-large", action="store_true", help="skip the 1024x1024x64 volume")
    ap.add_argument("--large-frames", type=int, default=200)
    ap.add_argument("--large-pool", type=int, default=2)
    ap.add_argument("--large-cpu", type=int, default=1, help="frames of the large volume solved on the CPU")
    ap.add_argument("--uneven-pool", type=int, default=4, help="distinct frames per size in the uneven batch")
    ap.add_argument("--only", choices=["roofline", "aligner"], default=None,
                    help="roofline: only the fused-pass probe on --frames FP16 frames; aligner: one aligner call "
                         "on --frames raw uint16 frames in HBM (both for ncu captures)")
    ap.add_argument("--tuning", default=None,
                    help="TILE_VOXELS,CTAS_PER_SM: the roofline probe's fused-pass tuning instead of the autotuner's "
                         "(under ncu the autotuner's timings do not represent a plain run; pass the plain run's choice)")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="length of the Poisson arrival stream")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="total arrivals per second")
    ap.add_argument("--serve-pool", type=int, default=6, help="distinct frames per served acquisition")
    ap.add_argument("--serve-slots", type=int, default=24, help="frame slots reserved per served acquisition")
    ap.add_argument("--serve-iters", type=int, default=4, help="trust-region iterations per serving graph launch")
    ap.add_argument("--serve-lags", type=int, nargs="+", default=[1, 4],
                    help="warm-start lags to serve with (1 = the previous frame's solution)")
    ap.add_argument("--capacity-rates", type=float, nargs="*", default=[4000.0, 8000.0, 16000.0],
                    help="offered rates of the saturation sweep (lag 4, --capacity-seconds each)")
    ap.add_argument("--capacity-seconds", type=float, default=1.0)
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def config_dict(n_frames, world):
    return {"workload": "z-stack 512x512x16, nD=32, 3 displacement components, %d frames per GPU per step" % n_frames,
            "volume": [16, 512, 512], "nD": 32, "frames_per_step": n_frames, "precision": "bf16 ref/grad, fp16 frames, fp32 sums, fp64 solve",
            "parallelism": "frames sharded over %d GPU(s), no collective on the data path" % world,
            "l2": "inputs exceed L2: %d frames x 8.4 MB fp16 + 33.6 MB reference/gradient per step" % n_frames}


def make_data(n_frames, rank, cfg=None):
    """Rank `rank`'s frames: its own seeded acquisition of the workload (weak scaling: every rank
    aligns n_frames of its own; no frame is shared, so the data path needs no collective)."""
    c = dict(cfg or S.CONFIG1)
    c["seed"] = c["seed"] + 7919 * rank
    return S.make_config(c, n_frames=n_frames)


def max_over_ranks(x, dist=None, device="cpu"):
    """The slowest rank's value (timings are reported as the max over ranks)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, polled every 100 ms on a thread while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()

    def _poll(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except (OSError, subprocess.SubprocessError):
                return
            self._stop.wait(0.1)

    def __enter__(self):
        self.thread = threading.Thread(target=self._poll, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self.thread.join(timeout=10)

    def summary(self):
        def num(s):
            try:
                return float(s)
            except ValueError:
                return None

        sm = [num(r[0]) for r in self.rows if r and num(r[0]) is not None]
        mx = [num(r[1]) for r in self.rows if len(r) > 1 and num(r[1]) is not None]
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 3 + i and r[3 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or "unknown"


def cpu_baseline(acq, n_threads, n_frames, what="the 512x512x16 nD=32 workload"):
    """The reference CPU warper (oracle/_ref, compiled from the reference's FrameWarper.cpp,
    OptimisationModel.cpp et al.) driving the trust-region solve, one frame per worker thread
    (FrameAlignerMex.cpp:24-25,120). The timing build uses the reference's own release flags
    (-msse3 -O3 -ffast-math -ftree-vectorize, CMakeLists.txt:17-21); without it the parity build
    (-O2), without either the C restatement. The trust region is the project's own statement of the
    algorithm: dlib, whose find_min_trust_region the reference calls, is not in the reference tree.
    Rigid shifts are computed before the timed region (numpy FP64 FFT), so the sample times the
    non-rigid solve only."""
    import oracle_py as O

    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    frames = acq.frames[:n_frames] + 1
    shifts = np.array([O.phase_shift(acq.reference, acq.frames[k]) for k in range(n_frames)])
    fast = O.ref_available(fast=True)
    if fast or O.ref_available():
        pool = O.RefPool(acq.reference + 1, acq.nD, line, il, ifr, n_threads, fast=fast)
        t0 = time.perf_counter()
        D, iters = pool.align(frames, shifts, 100)
        dt = time.perf_counter() - t0
        kind = "reference"
        build = ("reference sources, reference release flags -msse3 -O3 -ffast-math -ftree-vectorize" if fast
                 else "reference sources, -O2 parity build")
    else:
        ow = O.OracleWarper(acq.reference + 1, acq.nD, O.scan_init(line, il, ifr, nx, ny, nz))
        t0 = time.perf_counter()
        D, iters = ow.align_frames_mt(frames, shifts, n_threads, 100)
        dt = time.perf_counter() - t0
        kind = "port"
        build = "C restatement, -O2"
    return {"value": n_frames / dt, "unit": UNIT, "cores": n_threads, "kind": kind, "cpu_model": cpu_model(),
            "build": build,
            "sample": "%d frames of %s, non-rigid solve only (rigid shifts precomputed), %.1f s, %d threads "
                      "(one frame per thread); CpuFrameWarper + OptimisationModel from the reference's sources, "
                      "trust region = the project's statement of the algorithm (dlib absent from the reference "
                      "tree)" % (n_frames, what, dt, n_threads)}, D, shifts


def measure_plain(fa, ctx, acq, scan, pf, local):
    """The plain FP32 single-frame path: one frame at a time, the phase correlation and then the
    solve with the host driving every iteration (fa_align_frame). Timed two ways, like the batched
    figures: frames already in HBM (`value`), and from pinned host memory with the upload inside the
    timed region (`e2e`)."""
    import ctypes as C
    import torch

    ref32 = fa.Reference(ctx, acq.reference + 1, acq.nD, scan, fa.PREC_F32)
    corr = fa.Correlator(ctx, acq.reference)
    raw = torch.from_numpy(np.ascontiguousarray(acq.frames[:pf])).to(f"cuda:{local}")  # correlator input
    plus1 = raw + 1.0                                                                   # FrameWarpAligner's +1
    torch.cuda.synchronize()
    frs = [fa.Frame(ref32, device_ptr=plus1[k].data_ptr()) for k in range(pf)]
    frs[0].align(corr.compute_shift_device(raw[0].data_ptr()), 100)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(pf):
        frs[k].align(corr.compute_shift_device(raw[k].data_ptr()), 100)
    dev_fps = pf / (time.perf_counter() - t0)
    host_raw = torch.from_numpy(np.ascontiguousarray(acq.frames[:pf])).pin_memory()
    host_p1 = torch.from_numpy(np.ascontiguousarray(acq.frames[:pf] + 1)).pin_memory()
    shift = np.empty(3, np.float64)
    t0 = time.perf_counter()
    for k in range(pf):
        fa.check(fa.lib().fa_update_frame(frs[0]._h, C.c_void_p(host_p1[k].data_ptr()), fa.F32))
        fa.check(fa.lib().fa_correlator_shift(corr._h, host_raw[k].numpy(), shift))
        frs[0].align(shift, 100)
    e2e_fps = pf / (time.perf_counter() - t0)
    for f in frs:
        f.close()
    corr.close()
    ref32.close()
    return {"value": dev_fps, "e2e": e2e_fps, "unit": UNIT, "frames": pf,
            "note": "FP32 single-frame path (fa_align_frame: host-driven trust-region iterations) after the "
                    "device phase correlation; value with frames in HBM, e2e with each frame uploaded from "
                    "pinned host memory inside the timed region"}


def serving_data(args):
    """The served-stream acquisitions and their frames as raw uint16 in pinned host memory."""
    import torch

    acqs = S.config3_acquisitions(n_frames=args.serve_pool)
    pools = [torch.from_numpy(np.ascontiguousarray(a.frames.astype(np.uint16)).view(np.int16)).pin_memory()
             for a in acqs]
    return acqs, pools


def measure_capacity(fa, ctx, args, acqs, pools, lag=4):
    """Saturation sweep of the served stream: the same eight acquisitions at rising offered rates;
    the loop's capacity is the highest completed rate, reached where throughput stops tracking the
    offered rate."""
    import copy

    rows = []
    for rate in args.capacity_rates:
        a = copy.copy(args)
        a.serve_rate = rate
        a.serve_seconds = args.capacity_seconds
        r = measure_serving(fa, ctx, a, acqs, pools, lag)
        rows.append({"offered": rate, "arrival_rate_achieved": r["arrival_rate_achieved"],
                     "frames_per_s": r["frames_per_s"], "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
                     "peak_in_flight": r["peak_in_flight"]})
    return {"warm_start_lag": lag, "seconds_per_rate": args.capacity_seconds, "sweep": rows,
            "capacity_frames_per_s": max(r["frames_per_s"] for r in rows) if rows else None}


def measure_serving(fa, ctx, args, acqs, pools, lag):
    """The served stream: eight acquisitions (256x256x1 ... 1024x1024x4, nD 16-64), frames arriving as
    a Poisson process at args.serve_rate in total, each acquisition's frames drawn in order from a
    pool of args.serve_pool frames (raw uint16 in pinned host memory); warm start from the solution of
    the frame `lag` positions earlier in the same acquisition; 40 GB admission budget.
    Latency = submission -> result on the host."""
    srv = fa.Server(ctx, memory_budget=40 << 30, warm_start=lag, iterations_per_launch=args.serve_iters)
    ids = []
    for a in acqs:
        nz, ny, nx = a.reference.shape
        line, il, ifr = a.scan
        ids.append(srv.add_acquisition(a.reference, fa.scan_params(line, il, ifr, nx, ny, nz), frame_dtype=np.uint16,
                                       nD=a.nD, precision=fa.PREC_MIXED))
    n_acq = len(acqs)
    for i in ids:  # frame slots created before the stream (each admitted frame holds one)
        srv.reserve(i, args.serve_slots)
    # warm-up: every acquisition's pool once (graphs, cuFFT plans)
    warm = [srv.submit_ptr(ids[j], pools[j][k].data_ptr(), False) for k in range(args.serve_pool)
            for j in range(n_acq)]
    for t in warm:
        srv.wait(t, 300.0)
    srv.reset_stats()
    rng = np.random.Generator(np.random.PCG64(3333))
    n = max(1, int(args.serve_rate * args.serve_seconds))
    arrivals = np.cumsum(rng.exponential(1.0 / args.serve_rate, n))
    which = rng.integers(0, n_acq, n)
    nxt = [0] * n_acq
    tickets = []
    # The load generator must not pause: a collection of Python's cyclic garbage collector during
    # the stream holds the submitting thread back and then releases a burst of overdue arrivals.
    gc.collect()
    gc.disable()
    late_max = 0.0  # the latest submission behind its arrival time
    t0 = time.perf_counter()
    for i in range(n):
        target = t0 + arrivals[i]
        while True:
            d = target - time.perf_counter()
            if d <= 0:
                break
            if d > 2e-4:
                time.sleep(d - 1e-4)
        late_max = max(late_max, time.perf_counter() - target)
        j = int(which[i])
        tickets.append((j, srv.submit_ptr(ids[j], pools[j][nxt[j] % args.serve_pool].data_ptr(), False)))
        nxt[j] += 1
    t_sub = time.perf_counter() - t0
    gc.enable()
    iters = []
    lat = [[] for _ in range(n_acq)]
    for j, t in tickets:
        _, st, ms = srv.wait(t, 300.0)
        iters.append(st["iterations"])
        lat[j].append(ms)
    stats = srv.stats()
    srv.close()
    per_acq = []
    for j, a in enumerate(acqs):
        nz, ny, nx = a.reference.shape
        L = np.array(lat[j]) if lat[j] else np.zeros(1)
        per_acq.append({"acquisition": "%dx%dx%d nD=%d" % (nx, ny, nz, a.nD), "frames": len(lat[j]),
                        "p50_ms": float(np.percentile(L, 50)), "p99_ms": float(np.percentile(L, 99)),
                        "max_ms": float(L.max())})
    return {"warm_start_lag": lag, "iterations_per_launch": args.serve_iters, "arrival_rate": args.serve_rate, "arrival_rate_achieved": n / t_sub,
            "frames": n, "submit_late_max_ms": 1000.0 * late_max, "p50_ms": stats["p50_ms"], "p99_ms": stats["p99_ms"],
            "mean_ms": stats["mean_ms"],
            "max_ms": stats["max_ms"], "frames_per_s": stats["frames_per_s"],
            "peak_in_flight": stats["peak_in_flight"], "peak_slot_gb": stats["peak_slot_bytes"] / 1e9,
            "graph_launches": stats["graph_launches"], "iterations_mean": float(np.mean(iters)),
            "per_acquisition": per_acq}


def measure_uneven(fa, ctx, args):
    """The batched uneven-size workload: four single-plane acquisitions (128^2, 256^2, 512^2, 1024^2
    with nD 8 / 16 / 32 / 64), 64 frames each (drawn in order from args.uneven_pool distinct frames per
    size), BF16 reference / gradient, raw uint16 frames, all 256 frames submitted at once to a server
    whose acquisitions share one launch group: one persistent graph launch per iteration over frames
    of every size. Then, per size, each reduction of the mixed-precision pass at the solved D against
    the FP64 CPU statement (oracle): f, J^T e and the Hessian."""
    import oracle_py as O
    import torch

    acqs = S.config2_acquisitions(n_per_size=args.uneven_pool)
    pools = [torch.from_numpy(np.ascontiguousarray(a.frames.astype(np.uint16)).view(np.int16)).pin_memory()
             for a in acqs]
    srv = fa.Server(ctx, warm_start=False, shared_launches=True, max_in_flight=256)
    ids = []
    for a in acqs:
        nz, ny, nx = a.reference.shape
        line, il, ifr = a.scan
        ids.append(srv.add_acquisition(a.reference, fa.scan_params(line, il, ifr, nx, ny, nz), frame_dtype=np.uint16,
                                       nD=a.nD, precision=fa.PREC_MIXED))
        srv.reserve(ids[-1], 64)
    per = 64

    def burst():
        ts = [(j, k, srv.submit_ptr(ids[j], pools[j][k % args.uneven_pool].data_ptr(), False))
              for k in range(per) for j in range(len(acqs))]
        return [(j, k, srv.wait(t, 300.0)) for j, k, t in ts]

    burst()  # warm-up: graphs, slots, cuFFT plans
    srv.reset_stats()
    t0 = time.perf_counter()
    out = burst()
    wall = time.perf_counter() - t0
    stats = srv.stats()
    srv.close()
    errors = []
    for j, a in enumerate(acqs):
        nz, ny, nx = a.reference.shape
        line, il, ifr = a.scan
        D_sol = next(r[0] for jj, k, r in out if jj == j and k == 0)
        D_zero = np.zeros_like(D_sol)
        frame = a.frames[0] + 1
        ref = fa.Reference(ctx, a.reference + 1, a.nD, fa.scan_params(line, il, ifr, nx, ny, nz), fa.PREC_MIXED)
        fr = fa.Frame(ref, frame.astype(np.float16))
        ow = O.OracleWarper(a.reference + 1, a.nD, O.scan_init(line, il, ifr, nx, ny, nz))
        row = {"size": "%dx%d" % (ny, nx), "nD": a.nD}
        # f at the zero start and at the solution; J^T e at the zero start, where it is far from zero
        # (at the solution it is noise around zero and a relative error says nothing)
        for tag, D in (("start", D_zero), ("solution", D_sol)):
            f_gpu = fr.get_error(D)
            f_cpu, e = ow.get_error(frame, D, want_image=True)
            row["f_rel_" + tag] = abs(f_gpu - f_cpu) / abs(f_cpu)
            if tag == "start":
                g_gpu, g_cpu = fr.get_jacobian(D), ow.get_jacobian_from_error(e)
                row["jte_rel_max_start"] = float(np.max(np.abs(g_gpu - g_cpu)) / np.max(np.abs(g_cpu)))
        H_gpu, H_cpu = ref.hessian(), ow.hessian()
        row["hessian_rel_max"] = float(np.max(np.abs(H_gpu - H_cpu)) / np.max(np.abs(H_cpu)))
        # the served solve of frame 0 against the reference CPU solve of the same frame
        _, D_cpu, _ = cpu_baseline(a, 1, 1, "%dx%d" % (ny, nx))
        row["displacement_rms_vs_cpu_px"] = float(np.sqrt(((D_sol - D_cpu[0])[:, :2] ** 2).sum(-1).mean()))
        fr.close()
        ref.close()
        errors.append(row)
    return {"workload": "4 single-plane acquisitions 128^2 / 256^2 / 512^2 / 1024^2, nD 8 / 16 / 32 / 64, "
                        "64 raw uint16 frames each (%d distinct per size), one shared launch group" % args.uneven_pool,
            "frames": per * len(acqs), "wall_s": wall, "frames_per_s": per * len(acqs) / wall,
            "graph_launches": stats["graph_launches"],
            "reduction_error_vs_fp64_oracle": errors,
            "note": "errors of the mixed-precision pass (BF16 reference/gradient, FP16 frame, FP32 sums over "
                    "tiles of <= 2048 voxels, FP64 across tiles) against the FP64 CPU statement, each size's first "
                    "frame: f at the zero start and at the solved D, J^T e (max error / max |J^T e|) at the zero "
                    "start, the Hessian (FP64 from the FP32 gradient)"}


def measure_large(fa, ctx, args, local):
    """The large-volume workload: 1024x1024x64 reference (5000 blobs, mean 15 photons), nD = 64, three
    displacement components; args.large_frames frames (cycled from args.large_pool distinct ones)
    aligned through the full aligner pipeline -- 3-D FP64 phase correlation, then the batched solve --
    in calls of 50 raw uint16 frames resident in HBM; the fused pass's unique-byte rate on 8 frames;
    displacement RMS against the reference CPU solve of the first args.large_cpu frames."""
    import torch

    acq = S.make_config(S.CONFIG4, n_frames=args.large_pool)
    nz, ny, nx = acq.reference.shape
    N = nz * ny * nx
    line, il, ifr = acq.scan
    scan = fa.scan_params(line, il, ifr, nx, ny, nz)
    al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_MIXED, max_iterations=100)
    al.set_reference(acq.reference, scan)
    dev = torch.from_numpy(np.ascontiguousarray(acq.frames.astype(np.uint16)).view(np.int16)).to(f"cuda:{local}")
    batch = 50
    ptrs = [dev[k % args.large_pool].data_ptr() for k in range(batch)]
    D, _ = al.add_frames_device(ptrs, fa.U16, batch)  # warm-up
    ms, iters = 0.0, []
    done = 0
    while done < args.large_frames:
        m = min(batch, args.large_frames - done)
        D, st = al.add_frames_device(ptrs[:m], fa.U16, m)
        ms += al.last_device_ms()
        iters += [x["iterations"] for x in st]
        done += m
    al.close()
    del dev
    torch.cuda.empty_cache()
    ref = fa.Reference(ctx, acq.reference + 1, acq.nD, scan, fa.PREC_MIXED)
    frs = [fa.Frame(ref, (acq.frames[k % args.large_pool] + 1).astype(np.float16)) for k in range(8)]
    eval_ms = fa.profile_eval(frs, acq.D_true[0], 5)
    for f in frs:
        f.close()
    ref.close()
    algo = 8 * N * 2 + N * 8
    peak, _ = load_peaks()
    rms = None
    if args.large_cpu > 0:
        _, D_cpu, _ = cpu_baseline(acq, args.large_cpu, args.large_cpu, "the 1024x1024x64 nD=64 volume")
        rms = float(np.sqrt(((D[:args.large_cpu] - D_cpu) ** 2).sum(-1).mean()))
    return {"workload": "1024x1024x64 reference, nD = 64, 3 components, %d frames (%d distinct), raw uint16 in HBM, "
                        "calls of %d" % (args.large_frames, args.large_pool, batch),
            "frames_per_s": args.large_frames / (ms / 1000.0), "device_ms": ms,
            "iterations_mean": float(np.mean(iters)),
            "fused_pass_8_frames": {"ms_per_launch": eval_ms, "unique_bytes": algo,
                                    "achieved_gbs": algo / (eval_ms / 1000.0) / 1e9,
                                    "frac_of_measured_hbm": algo / (eval_ms / 1000.0) / 1e9 / peak},
            "displacement_rms_vs_cpu_px": rms, "cpu_frames": args.large_cpu}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    n_threads = os.cpu_count() or 1
    n = args.cpu_frames or n_threads
    acq = make_data(n, 0)
    times = []
    for step in range(args.warmup + args.steps):
        cb, _, _ = cpu_baseline(acq, n_threads, n)
        if step >= args.warmup:
            times.append(n / cb["value"])
    total = sum(times)
    value = n * args.steps / total
    cb["value"] = value
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic (seeded blob acquisition)",
            "config": config_dict(n, 1), "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_roofline_probe(args, local):
    """The fused-pass probe alone: one mixed-precision reference, args.frames FP16 frames, two timed
    launches of eval4_kernel (the command the DRAM-traffic captures in profiles/ run)."""
    import fa_b200 as fa

    acq = make_data(args.frames, 0)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    ctx = fa.Context(device=local, autotune=True)
    ref = fa.Reference(ctx, acq.reference + 1, acq.nD, fa.scan_params(line, il, ifr, nx, ny, nz), fa.PREC_MIXED)
    if args.tuning:
        tile_voxels, ctas_per_sm = (int(v) for v in args.tuning.split(","))
        ref.retune(tile_voxels, ctas_per_sm)
    frs = [fa.Frame(ref, (acq.frames[k] + 1).astype(np.float16)) for k in range(args.frames)]
    ms = fa.profile_eval(frs, acq.D_true[0], 2)
    print(json.dumps({"probe": "eval4_kernel<3, half, bf16>", "frames": args.frames, "ms_per_launch": ms,
                      "tuning": list(ref.tuning())}))
    return 0


def run_aligner_probe(args, local):
    """One aligner call alone: the mixed-precision aligner of the headline workload on args.frames raw
    uint16 frames already in HBM (phase correlation, conversion and batched solve), after one
    untimed call (the command the correlator captures in profiles/ run)."""
    import torch

    import fa_b200 as fa

    acq = make_data(args.frames, 0)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    ctx = fa.Context(device=local, autotune=True)
    al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_MIXED, max_iterations=100)
    al.set_reference(acq.reference, fa.scan_params(line, il, ifr, nx, ny, nz))
    dev = torch.from_numpy(np.ascontiguousarray(acq.frames.astype(np.uint16)).view(np.int16)).to(f"cuda:{local}")
    ptrs = [dev[k].data_ptr() for k in range(args.frames)]
    al.add_frames_device(ptrs, fa.U16, args.frames)
    al.add_frames_device(ptrs, fa.U16, args.frames)
    corr_ms, total_ms = al.last_phase_ms()
    print(json.dumps({"probe": "aligner", "frames": args.frames, "ms": total_ms, "ms_until_last_peak": corr_ms}))
    al.close()
    return 0


def run_ours(args, rank, world, local):
    import fa_b200 as fa

    if args.only == "roofline":
        return run_roofline_probe(args, local)
    if args.only == "aligner":
        return run_aligner_probe(args, local)

    pg = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist
    n = args.frames
    acq = make_data(n, rank)
    nz, ny, nx = acq.reference.shape
    line, il, ifr = acq.scan
    scan = fa.scan_params(line, il, ifr, nx, ny, nz)
    ctx = fa.Context(device=local, autotune=True)
    al = fa.Aligner(ctx, nD=acq.nD, precision=fa.PREC_MIXED, max_iterations=100)
    al.set_reference(acq.reference, scan)
    raw_u16 = np.ascontiguousarray(acq.frames.astype(np.uint16))
    N = nz * ny * nx

    import torch

    dev_frames = torch.from_numpy(raw_u16.view(np.int16)).to(f"cuda:{local}")  # raw counts, resident in HBM
    ptrs = [dev_frames[i].data_ptr() for i in range(n)]
    pinned = torch.from_numpy(raw_u16.view(np.int16)).pin_memory()
    host_ptrs = [pinned[i].data_ptr() for i in range(n)]

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    # warm-up (untimed)
    for _ in range(args.warmup):
        D, stats = al.add_frames_device(ptrs, fa.U16, n)
    barrier()
    launches0 = fa.kernel_launches()
    dev_ms = 0.0
    corr_ms = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            D, stats = al.add_frames_device(ptrs, fa.U16, n)
            c_ms, t_ms = al.last_phase_ms()
            dev_ms += t_ms
            corr_ms += c_ms
        barrier()
    launches = fa.kernel_launches() - launches0
    dev_ms = max_over_ranks(dev_ms, pg, f"cuda:{local}")
    value = n * world * args.steps / (dev_ms / 1000.0)
    iters = [s["iterations"] for s in stats]

    # end to end: raw uint16 frames from pinned host memory through the public API
    class HostFrames:
        pass

    import ctypes as C

    arr = (C.c_void_p * n)(*host_ptrs)
    Dh = np.empty((n, acq.nD, 3), np.float64)
    st = (fa.AlignStats * n)()
    for _ in range(max(1, args.warmup // 2)):
        fa.check(fa.lib().fa_aligner_add_frames(al._h, C.cast(arr, C.c_void_p), fa.U16, n, Dh, C.cast(st, C.c_void_p)))
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fa.check(fa.lib().fa_aligner_add_frames(al._h, C.cast(arr, C.c_void_p), fa.U16, n, Dh, C.cast(st, C.c_void_p)))
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0, pg, f"cuda:{local}")
    e2e = {"value": n * world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(n * N * 2),
           "d2h_bytes_per_step": int(n * acq.nD * 3 * 8 + n * C.sizeof(fa.AlignStats))}

    out = None
    if rank == 0:
        # roofline of the fused evaluation kernel: algorithmic bytes per launch / event-timed duration
        ref_m = fa.Reference(ctx, acq.reference + 1, acq.nD, scan, fa.PREC_MIXED)
        tile_voxels, ctas_per_sm = ref_m.tuning()
        frs = [fa.Frame(ref_m, (acq.frames[k] + 1).astype(np.float16)) for k in range(n)]
        ms = fa.profile_eval(frs, acq.D_true[0], 20)
        # Unique bytes one launch needs: each FP16 frame once, plus the BF16 reference and three
        # gradient planes once (the frames of a batch share them; after the first frame they are L2
        # hits, so counting them per frame would inflate the figure).
        algo_bytes = n * N * 2 + N * (2 + 3 * 2)
        achieved = algo_bytes / (ms / 1000.0) / 1e9
        peak, peak_kind = load_peaks()
        # DRAM bytes per launch from the ncu capture summarised in profiles/ (8- and 16-frame launches,
        # fitted per frame and shared, scaled to n frames), or null without it
        traffic = None
        tp = os.path.join(ROOT, "profiles", "eval_traffic.json")
        if os.path.exists(tp):
            t = json.load(open(tp))
            traffic = t["dram_bytes_shared"] + n * t["dram_bytes_per_frame"]
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "traffic_unit": "bytes per launch",
                    "kernel": "eval4_kernel<3, half, bf16> (fused warp + error + J^T e, grid form of the tile body "
                              "the aligner's persistent kernel runs)",
                    "algorithmic_bytes_per_launch": algo_bytes, "ms_per_launch": ms,
                    "bytes_per_unit": "2 B per voxel per frame + 8 B per voxel of the shared reference",
                    "tuning": {"tile_voxels": tile_voxels, "ctas_per_sm": ctas_per_sm},
                    "peak_source": "%s (MEASURED_PEAKS.json hbm_gbs)" % peak_kind if peak_kind == "measured" else "fallback 6.65 TB/s"}
        for f in frs:
            f.close()
        ref_m.close()
        plain = measure_plain(fa, ctx, acq, scan, min(args.plain_frames, n), local)
        serving = None
        if not args.no_serve:
            sacqs, spools = serving_data(args)
            serving = {"workload": "8 acquisitions " + ", ".join(
                           "%dx%dx%d nD=%d" % (a.reference.shape[2], a.reference.shape[1], a.reference.shape[0], a.nD)
                           for a in sacqs),
                       "memory_budget_gb": 40 * 2 ** 30 / 1e9,
                       "frames_from": "pinned host memory (raw uint16), %d distinct frames per acquisition"
                                      % args.serve_pool,
                       "runs": [measure_serving(fa, ctx, args, sacqs, spools, lag) for lag in args.serve_lags],
                       "capacity": measure_capacity(fa, ctx, args, sacqs, spools) if args.capacity_rates else None}
        large = None if args.no_large else measure_large(fa, ctx, args, local)
        uneven = None
        if not args.no_uneven:
            uneven = measure_uneven(fa, ctx, args)
        # The CPU baseline last: its 16 host threads and their multi-GB warpers change the host's
        # memory state, after which the latency-bound lag-1 served stream showed 30-50 ms stalls.
        cb = None
        D_cpu = None
        if not args.no_cpu:
            try:
                nt = os.cpu_count() or 1
                cb, D_cpu, _ = cpu_baseline(acq, nt, args.cpu_frames or min(nt, n))
            except Exception as ex:  # the baseline is reported, never required
                cb = {"value": None, "unit": UNIT, "cores": 0, "kind": "unavailable", "sample": str(ex)[:200]}
        rms_vs_cpu = None
        if D_cpu is not None:
            k = D_cpu.shape[0]
            rms_vs_cpu = float(np.sqrt(((D[:k] - D_cpu) ** 2).sum(-1).mean()))
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "bf16/fp16 storage, f32 accumulate, f64 solve",
               "data": "synthetic (seeded blob acquisition, Poisson noise)", "config": config_dict(n, world),
               "e2e": e2e, "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cb,
               "clocks": clk.summary(),
               "plain_fp32": plain,
               "batched_over_plain": value / world / plain["value"],
               "e2e_over_plain_e2e": e2e["value"] / world / plain["e2e"],
               "serving": serving,
               "batched_uneven": uneven,
               "large_volume": large,
               "displacement_rms_vs_cpu_px": rms_vs_cpu,
               "iterations": {"mean": float(np.mean(iters)), "max": int(np.max(iters))},
               "step_phases_ms": {"until_last_peak": corr_ms / args.steps, "total": dev_ms / args.steps,
                                  "note": "device time per step (rank 0) from the call's start until every "
                                          "frame was converted and phase-correlated, and in total; the first "
                                          "frames' solve overlaps the later frames' correlation"}}
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if out:
        print(json.dumps(out))
    return 0


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
