#!/usr/bin/env python
"""Benchmark of the B200 fractal-flame render path.

One step = one whole frame of the full forward workload: a synthetic flame of
8 transforms + 1 final (each 3-5 of the twelve variations), 1920x1080 with 2x
supersampling (3840x2160 internal), 1e9 plotted samples from 65,536 walkers,
density estimation radius 9 -> 0, log tone map fused with the firefly
downsample.  `value` is samples/s on the device (config already parsed into
a device table, output left in HBM); `e2e` is the same frame through the
reference's own boundary (`fae_call` render request -> RGBA8 in host memory).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank renders its own 65,536 walkers (weak scaling); the
ranks' histograms are summed with an NCCL reduce-scatter of row windows (the
path's one exchange step: a band of rows plus the density estimation's
reach), each rank finishes its band and the bands are gathered; the step
time is the max over ranks, and rank 0 prints one JSON line.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "fflame-rust_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

FULL_SEED = 6


def workload(name):
    from ffb200 import synthetic
    if name == "full_1080p_ss2":
        return dict(cfg=synthetic.full_flame(FULL_SEED), width=1920, height=1080, supersample=2,
                    iterations=1_000_000_000, walkers=65536,
                    desc="8 xforms + final, 12 variations, 1920x1080 ss2 (3840x2160 internal), 1e9 samples, "
                         "65536 walkers, DE radius 9->0, u32 count + FP32 RGB histogram")
    if name == "stress_4k":
        return dict(cfg=synthetic.stress_flame(21), width=3840, height=2160, supersample=2,
                    iterations=10_000_000_000, walkers=0, count_bits=64,
                    desc="16 xforms (6 rotations by k*60 deg), 3840x2160 ss2 (7680x4320 internal), 1e10 samples, "
                         "exact u64 count + u64 fixed-point RGB, DE radius 12->0")
    if name == "plain_256":
        return dict(cfg=synthetic.plain_flame(1), width=256, height=256, supersample=1, iterations=10_000_000,
                    walkers=16384, desc="3 xforms {linear,sinusoidal,spherical}, 256x256 ss1, 1e7 samples, no DE")
    raise SystemExit(f"unknown workload {name}")


# ----------------------------------------------------------------- clocks --
class ClockSampler:
    """nvidia-smi samples during the timed region (clocks, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        load = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_traffic(name):
    """dram bytes per launch of the chaos kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"ffb_chaos_{name}.txt")
    try:
        for line in open(path, encoding="utf-8"):
            if line.startswith("dram_bytes_per_launch_full:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


# ------------------------------------------------------------ CPU baseline --
def host_info():
    """The host threads this process may use and the CPU model."""
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    model = None
    try:
        for line in open("/proc/cpuinfo", encoding="utf-8"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return cores, model


def cpu_threads(wl):
    """All host threads, fewer if their private histograms (28 B a pixel
    each) would not fit in a quarter of the free memory."""
    cores, _ = host_info()
    W, H = wl["width"] * wl["supersample"], wl["height"] * wl["supersample"]
    per_thread = 28.0 * W * H
    try:
        import psutil
        free = psutil.virtual_memory().available
        cores = max(1, min(cores, int(free / 4 / per_thread)))
    except Exception:
        pass
    return max(1, min(cores, 128))


def cpu_rate(wl, steps, warmup, min_samples=1e7, min_s=2.0):
    """The oracle port of the render path on the host cores: a frame of the
    workload's flame at its internal size, built over steps.  Each step
    renders a fresh range of walkers (its own burn-in) into per-thread
    histograms made once before the first step; only the steps are timed,
    each at least `min_samples` samples and about `min_s` seconds (sized from
    the warm-up steps' rate).  Returns samples/s over the timed steps."""
    from oracle import oracle as O
    O.build()
    threads = cpu_threads(wl)
    W, H = wl["width"] * wl["supersample"], wl["height"] * wl["supersample"]
    fl = O.Flame(wl["cfg"], W, H)
    t0 = time.perf_counter()
    ctx = fl.cpu_render(threads)
    setup_s = time.perf_counter() - t0
    walkers = threads * 256
    per = max(64, int(min_samples) // walkers + 1)
    w0 = 0
    rate = None
    for _ in range(max(1, warmup)):
        t0 = time.perf_counter()
        plotted = ctx.run(w0, walkers, per + 20, seed=0x5EED)
        rate = plotted / max(time.perf_counter() - t0, 1e-9)
        w0 += walkers
    per = max(per, int(rate * min_s / walkers) + 1)
    times, samples = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        plotted = ctx.run(w0, walkers, per + 20, seed=0x5EED)
        times.append(time.perf_counter() - t0)
        samples.append(plotted)
        w0 += walkers
    t0 = time.perf_counter()
    inframe, _, _ = ctx.merge()
    merge_s = time.perf_counter() - t0
    ctx.close()
    _, model = host_info()
    return {
        "value": sum(samples) / sum(times), "unit": "samples/s", "cores": threads, "cpu_model": model,
        "per_core": sum(samples) / sum(times) / threads, "ms_per_step": 1e3 * sum(times) / len(times),
        "samples_per_step": sum(samples) / len(samples), "steps": steps,
        "setup_s": setup_s, "merge_s": merge_s, "inframe": int(inframe),
        "sample": f"{steps} steps of {walkers} walkers x {per} iterations after burn-in 20 "
                  f"({sum(samples) / len(samples):.3g} samples a step) of the same flame at {W}x{H}, f32, "
                  f"{threads} threads with a private histogram each (made once, merged after the steps, neither timed)",
    }


def cpu_baseline(wl):
    r = cpu_rate(wl, steps=3, warmup=1)
    r["kind"] = "port"
    return r


# ------------------------------------------------------------------ ours --
def run_ours(args, rank, world, local_rank):
    import torch
    from ffb200 import Engine, _native

    torch.cuda.set_device(local_rank)
    wl = workload(args.workload)
    cfg = json.dumps(wl["cfg"])
    W, H, ss = wl["width"], wl["height"], wl["supersample"]
    r = _native.Renderer(local_rank)
    job = dict(iterations=wl["iterations"], walkers=wl["walkers"], supersample=ss, walker0=rank * wl["walkers"],
               seed=0x5EED + 0, schedule=args.schedule, math=args.math, count_bits=wl.get("count_bits", 32),
               accumulate=args.accumulate, plot=args.plot)
    d_rgba = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
    # The library's kernels and the timing events share one (non-default) stream.
    side = torch.cuda.Stream()
    torch.cuda.set_stream(side)
    stream = side.cuda_stream
    if world > 1:
        # Weak scaling: every rank renders its own 65,536 walkers x 1e9
        # samples; the frame sums all ranks' histograms (NCCL reduce-scatter of row windows),
        # each rank tone-maps a band of rows, the bands are gathered.
        from ffb200 import distributed as D
        backend = D.CudaBackend(r, torch.device("cuda", local_rank), side)
        djob = {k: v for k, v in job.items() if k not in ("iterations", "walkers", "supersample", "walker0")}

        def step():
            return D.render(backend, cfg, W, H, iterations=wl["iterations"] * world, walkers=wl["walkers"] * world,
                            supersample=ss, **djob)
    else:
        def step():
            return r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=stream, sync=False, **job)
    out = r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=stream, sync=True, **job)   # compile + first frame
    samples_per_step = out.total_iterations
    launches_per_step = out.kernel_launches + (2 if world > 1 else 0)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    clocks = ClockSampler(local_rank) if rank == 0 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t_start.record()
    for _ in range(args.steps):
        step()
    t_end.record()
    t_end.synchronize()
    torch.cuda.synchronize()
    ms = t_start.elapsed_time(t_end) / args.steps
    clk = clocks.stop() if clocks else None
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if rank != 0:
        return None

    # Dominant kernel: the chaos game alone (events around its launch).
    chaos_ms, inframe = [], []
    exact = wl.get("count_bits", 32) == 64
    for _ in range(3):
        if exact:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            _, _, o = r.histogram_u64(cfg, W, H, **job)
            chaos_ms.append(o.render_time_ms or 0.0)
        else:
            _, _, o = r.histogram(cfg, W, H, **job)
            chaos_ms.append(o.render_time_ms)
        inframe.append(o.inframe_samples)
    c_ms = statistics.median(chaos_ms) or ms
    # 4 read-modify-writes per splatted sample: 4 B each (u32 count + FP32
    # colour), or 8 B each in exact mode (u64 count + u64 fixed-point colour).
    bytes_per_launch = (32.0 if exact else 16.0) * statistics.median(inframe)
    peaks, peak_kind = measured_peaks()
    achieved = bytes_per_launch / (c_ms * 1e-3) / 1e9
    traffic = profile_traffic(args.workload)
    # The splat's own ceiling: random-address 4-atomic splats into a histogram
    # of the same size (microbenchmark in the same run).
    npx = W * ss * H * ss
    bench_ms = r.atomic_bench(npx, 400_000_000, 0)
    splat_peak = 400_000_000 / (bench_ms * 1e-3)
    splat_rate = statistics.median(inframe) / (c_ms * 1e-3)
    # The splat kernel alone: ffb_plot over the same frame's records, each
    # launch run after its chaos launch instead of beside the next one.
    plot_alone = None
    if not exact and args.plot in ("auto", "deferred"):
        try:
            p_ms, p_samples, p_in = r.plot_bench(cfg, W, H, **job)
            plot_alone = {"kernel": "ffb_plot (final chain, palette, world_to_pixel, warp-aggregated 4-atomic splat)",
                          "ms": p_ms, "records": p_samples, "splats": p_in,
                          "splats_per_s": p_in / (p_ms * 1e-3), "frac": p_in / (p_ms * 1e-3) / splat_peak}
        except Exception as e:  # noqa: BLE001
            plot_alone = {"error": f"{type(e).__name__}: {e}"}

    # End to end: the reference's boundary, host buffers, copies inside.
    eng = Engine()
    req_iters = wl["iterations"]
    e2e_times = []
    info = None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        image = eng.render(cfg, W, H, iterations=req_iters, supersample=ss, walkers=wl["walkers"], exact=exact,
                           accumulate=args.accumulate)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_times.append(dt)
        info = image.info
    e2e_s = statistics.mean(e2e_times)
    o_e2e = _native.Output()
    # bytes the library copies for one render request (h2d: tables; d2h: RGBA8)
    rr = r.render(cfg, W, H, **job)[1]
    line = {
        "metric": "samples/s", "value": samples_per_step * world / (ms * 1e-3), "unit": "samples/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded flame generator; no dataset)",
        "config": config_for(args, wl, world),
        "samples_per_step": samples_per_step * world,
        "ms_per_frame": ms,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "kernel": "chaos game: ffb_chaos_sorted, with ffb_plot beside it on a second stream (deferred plotting)",
                     "kernel_ms": c_ms, "algorithmic_bytes_per_launch": bytes_per_launch,
                     "peak_kind": peak_kind},
        "l2_atomic": {"achieved_splats_per_s": splat_rate, "peak_splats_per_s": splat_peak,
                      "frac": splat_rate / splat_peak, "peak_from": "ffb_atomic_bench kind 0, same histogram size",
                      "plot_kernel_alone": plot_alone},
        "e2e": {"value": samples_per_step / e2e_s, "unit": "samples/s", "ms_per_frame": e2e_s * 1e3,
                "h2d_bytes_per_step": rr.h2d_bytes, "d2h_bytes_per_step": W * H * 4,
                "path": "fae_call render request (JSON config in, RGBA8 host bytes out)",
                "info_ms": info.get("ms") if info else None},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(wl)
    if world == 1 and not args.no_extra and args.workload == "full_1080p_ss2":
        line["fused"] = leg(fused_leg, r, wl, args)
        line["parity"] = leg(parity_leg, r, wl)
        line["batched"] = leg(run_batched, args, local_rank, steps=3, serial_steps=2)
        line["diff"] = leg(run_diff, args, local_rank, steps=10, cpu=False)
        line["stress_4k"] = leg(stress_leg, r, args)
        line["tiles"] = leg(tiles_leg, r)
    r.close()
    return line


def leg(fn, *a, **k):
    """An extra measurement of the default line; its failure is reported in
    the line, not raised."""
    try:
        return fn(*a, **k)
    except Exception as e:          # noqa: BLE001
        return {"error": f"{type(e).__name__}: {e}"}


def fused_leg(r, wl, args, steps=10):
    """The same frame with fused plotting (plot warps beside the walkers in
    one block, samples handed over in shared memory): frame time and the
    chaos stage's DRAM traffic, which is the histogram's alone."""
    import torch
    cfg = json.dumps(wl["cfg"])
    W, H, ss = wl["width"], wl["height"], wl["supersample"]
    job = dict(iterations=wl["iterations"], walkers=wl["walkers"], supersample=ss, seed=0x5EED, plot="fused")
    d_rgba = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
    side = torch.cuda.Stream()
    out = r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=side.cuda_stream, sync=True, **job)
    for _ in range(3):
        r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=side.cuda_stream, sync=False, **job)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(side)
    for _ in range(steps):
        r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=side.cuda_stream, sync=False, **job)
    ev1.record(side)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    _, _, o = r.histogram(cfg, wl["width"], wl["height"], **job)
    return {"ms_per_frame": ms, "samples_per_s": out.total_iterations / (ms * 1e-3), "chaos_ms": o.render_time_ms,
            "splats_per_s": o.inframe_samples / (o.render_time_ms * 1e-3), "traffic": profile_traffic(args.workload + "_fused"),
            "kernel": "ffb_chaos_fused (448 walker threads + 576 plot threads a block, 8-iteration shared-memory ring)"}


def parity_leg(r, wl, size=(480, 270)):
    """The benchmarked path against the oracle at the benchmark's samples a
    pixel, at a reduced size (outside the timed region): normalised
    log-density L1 / p99, block z-scores and the tone-mapped image, each
    beside two oracle renders' own difference (oracle/parity.py)."""
    from oracle import parity
    ss = wl["supersample"]
    spp = wl["iterations"] / float(wl["width"] * ss * wl["height"] * ss)
    samples = int(spp * size[0] * size[1] * ss * ss)
    t0 = time.perf_counter()
    m = parity.render_parity(r, wl["cfg"], size[0], size[1], ss, samples, wl["walkers"])
    m["within_noise"] = parity.within_noise(m)
    m["flame"] = f"synthetic.full_flame({FULL_SEED}) (the benchmark's flame), density estimation radius 9"
    m["seconds"] = time.perf_counter() - t0
    return m


def stress_leg(r, args, steps=2):
    """The 4K stress frame (7680x4320 internal, exact u64 counts, 1e10
    samples, DE 12) through the same device path, timed with CUDA events."""
    import torch
    wl = workload("stress_4k")
    cfg = json.dumps(wl["cfg"])
    W, H, ss = wl["width"], wl["height"], wl["supersample"]
    job = dict(iterations=wl["iterations"], walkers=wl["walkers"], supersample=ss, seed=0x5EED,
               count_bits=64, accumulate=args.accumulate)
    d_rgba = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
    side = torch.cuda.Stream()
    out = r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=side.cuda_stream, sync=True, **job)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(side)
    for _ in range(steps):
        r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=side.cuda_stream, sync=False, **job)
    ev1.record(side)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / steps
    del d_rgba
    torch.cuda.empty_cache()
    return {"ms_per_frame": ms, "samples_per_s": out.total_iterations / (ms * 1e-3), "samples": out.total_iterations,
            "steps": steps, "desc": wl["desc"]}


def tiles_leg(r, steps=2):
    """Direct splat against tile-sorted accumulation for the u32-count /
    FP32-colour histogram: the stress flame at 7680x4320 internal (531 MB,
    4x the L2) and 3e9 samples, then the benchmark frame (133 MB), each
    timed both ways with CUDA events."""
    import torch
    out = {}
    for name, cfg, W, H, iters, walkers in (
            ("f32_7680x4320_3e9", synthetic_cfg("stress"), 3840, 2160, 3_000_000_000, 0),
            ("f32_3840x2160_1e9", synthetic_cfg("full"), 1920, 1080, 1_000_000_000, 65536)):
        d_rgba = torch.empty(W * H * 4, dtype=torch.uint8, device="cuda")
        side = torch.cuda.Stream()
        row = {"histogram_mb": W * 2 * H * 2 * 16 / 1e6}
        for acc in ("direct", "tiled"):
            job = dict(iterations=iters, walkers=walkers, supersample=2, seed=0x5EED, accumulate=acc)
            r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=side.cuda_stream, sync=True, **job)
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(side)
            for _ in range(steps):
                r.render_device(cfg, W, H, d_rgba.data_ptr(), stream=side.cuda_stream, sync=False, **job)
            ev1.record(side)
            ev1.synchronize()
            row[f"{acc}_ms"] = ev0.elapsed_time(ev1) / steps
        row["tiled_speedup"] = row["direct_ms"] / row["tiled_ms"]
        out[name] = row
        del d_rgba
        torch.cuda.empty_cache()
    return out


def synthetic_cfg(kind):
    from ffb200 import synthetic
    return json.dumps(synthetic.stress_flame(21) if kind == "stress" else synthetic.full_flame(FULL_SEED))


def config_for(args, wl, world):
    """The workload's description, the same for both arms."""
    W, H, ss = wl["width"], wl["height"], wl["supersample"]
    exact = wl.get("count_bits", 32) == 64
    return {"workload": args.workload, "desc": wl["desc"], "width": W, "height": H, "supersample": ss,
            "samples": wl["iterations"], "walkers": wl["walkers"], "rng": "philox",
            "schedule": args.schedule, "math": args.math, "accumulate": args.accumulate,
            "l2": f"histogram {W * ss * H * ss * (32 if exact else 16) / 1e6:.1f} MB > 126 MB L2, cleared every step",
            "parallelism": f"walker shards x{world}" + (" + NCCL histogram reduce-scatter + row bands" if world > 1 else "")}


def run_batched(args, local_rank, steps=None, serial_steps=None):
    """256 synthetic flames (transform counts 2-12, 128^2-1024^2, 50-2000
    samples a pixel): one batched, graph-captured render against the same
    flames rendered one after another.  flames/s, device-timed; then the
    same comparison within each resolution class (the class's flames as a
    batch of their own, tuned for themselves)."""
    import torch
    from ffb200 import Batch, _native, synthetic
    torch.cuda.set_device(local_rank)
    steps = steps or args.steps
    serial_steps = serial_steps or max(1, args.steps // 2)
    r = _native.Renderer(local_rank)
    items = synthetic.batch_flames(n=256, seed=3)
    texts = [json.dumps(it[0]) for it in items]
    side = torch.cuda.Stream()
    outs = [torch.empty(w * h * 4, dtype=torch.uint8, device="cuda") for _, w, h, _, _ in items]

    def time_batch(b):
        for _ in range(max(1, min(args.warmup, 2))):
            b.run()
        return statistics.median(b.run() for _ in range(steps))

    def time_serial(idx):
        def serial():
            for i in idx:
                _, w, h, samples, seed = items[i]
                r.render_device(texts[i], w, h, outs[i].data_ptr(), stream=side.cuda_stream, sync=False,
                                iterations=samples, seed=seed)
        serial()
        side.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for _ in range(serial_steps):
            ev0.record(side)
            serial()
            ev1.record(side)
            ev1.synchronize()
            ms.append(ev0.elapsed_time(ev1))
        return statistics.median(ms)

    t0 = time.perf_counter()
    b = Batch(r, items, tune=True)
    setup_s = time.perf_counter() - t0
    info = b.info()
    clocks = ClockSampler(local_rank)
    clocks.start()
    batched_ms = time_batch(b)
    clk = clocks.stop()
    b.close()
    serial_ms = time_serial(range(len(items)))
    classes = {}
    for size in sorted({w for _, w, _, _, _ in items}):
        idx = [i for i, it in enumerate(items) if it[1] == size]
        bc = Batch(r, [items[i] for i in idx], tune=True)
        bms = time_batch(bc)
        samples = bc.info()["samples"]
        bc.close()
        sms = time_serial(idx)
        classes[f"{size}x{size}"] = {"flames": len(idx), "samples": samples, "batched_ms": bms, "serial_ms": sms,
                                     "batched_flames_per_s": len(idx) / (bms * 1e-3),
                                     "serial_flames_per_s": len(idx) / (sms * 1e-3), "ratio": sms / bms}
    n = len(items)
    r.close()
    return {
        "metric": "flames/s (batched 256)", "value": n / (batched_ms * 1e-3), "unit": "flames/s", "n_gpus": 1,
        "steps": steps, "warmup": args.warmup, "ms_per_step": batched_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded flame generator)",
        "config": {"workload": "batched_256", "flames": n, "samples": info["samples"],
                   "desc": "256 flames, 2-12 transforms {linear,sinusoidal,spherical}, 128^2-1024^2, 50-2000 spp",
                   "tuned": {"threads": info["threads"], "iterations_per_walker": info["iterations_per_walker"]},
                   "groups": info["groups"], "setup_s": setup_s},
        "flames_per_s": n / (batched_ms * 1e-3), "serial_flames_per_s": n / (serial_ms * 1e-3),
        "samples_per_s": info["samples"] / (batched_ms * 1e-3),
        "serial": {"value": n / (serial_ms * 1e-3), "unit": "flames/s", "ms": serial_ms},
        "batched_over_serial": serial_ms / batched_ms, "ratio": serial_ms / batched_ms,
        "per_size_class": classes,
        "clocks": clk,
    }


def run_diff(args, local_rank, steps=None, cpu=True):
    """The differentiable configuration: 4 transforms at 512^2, bilinear
    splat, 2e8 samples, loss = L2 between the image and the image at
    theta + N(0, 0.05).  One step = forward (theta -> image), the loss's
    gradient with respect to the image, and the adjoint (-> dL/dtheta).
    `value` is the step's time over the forward's (fwd+bwd / fwd)."""
    import numpy as np
    import torch
    from ffb200 import _native, diff, synthetic
    torch.cuda.set_device(local_rank)
    side = torch.cuda.Stream()
    torch.cuda.set_stream(side)
    steps = steps or args.steps
    cfg = synthetic.diff_flame(4)
    W, samples, walkers = 512, 200_000_000, 65536
    r = _native.Renderer(local_rank)
    dr = diff.DiffRenderer(cfg, W, W, samples, walkers=walkers, seed=2024, renderer=r)
    th = dr.theta0()
    noisy = th + torch.from_numpy(np.random.default_rng(2).normal(0, 0.05, th.numel()).astype(np.float32)).cuda()
    target = dr.forward_raw(noisy).clone()

    def fwd():
        return dr.forward_raw(th)

    def step():
        img = dr.forward_raw(th)
        d = 2.0 * (img - target)
        d[..., 3] = 0.0
        return dr.backward_raw(d)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    for _ in range(steps):
        fwd()
    ev[1].record()
    for _ in range(steps):
        step()
    ev[2].record()
    ev[2].synchronize()
    clk = clocks.stop()
    fwd_ms = ev[0].elapsed_time(ev[1]) / steps
    step_ms = ev[1].elapsed_time(ev[2]) / steps
    plotted, inframe = dr.samples()
    # The adjoint kernel alone, and the forward kernel's splat against the
    # vector-reduction ceiling at the same histogram size.
    img = dr.forward_raw(th)
    d = 2.0 * (img - target)
    ev[0].record()
    dr.backward_raw(d)
    ev[1].record()
    ev[1].synchronize()
    bwd_ms = ev[0].elapsed_time(ev[1])
    bench_ms = r.atomic_bench(W * W, 400_000_000, 2)
    v4_peak = 400_000_000 / (bench_ms * 1e-3)
    peaks, peak_kind = measured_peaks()
    bytes_per_launch = 64.0 * inframe            # 4 corners x one 16-byte vector reduction
    achieved = bytes_per_launch / (fwd_ms * 1e-3) / 1e9
    # End to end through the autograd Function: theta from pinned host memory,
    # the scalar loss and dL/dtheta back to the host, every step.
    host_th = th.cpu().pin_memory()
    host_g = torch.empty(th.numel(), dtype=torch.float32).pin_memory()
    e2e = []
    for i in range(args.warmup + steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t = host_th.to("cuda", non_blocking=True).requires_grad_()
        loss = ((dr.render(t)[..., :3] - target[..., :3]) ** 2).sum()
        loss.backward()
        host_g.copy_(t.grad, non_blocking=True)
        lv = loss.item()
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e.append(time.perf_counter() - t0)
    e2e_ms = statistics.mean(e2e) * 1e3
    e2e_fwd = []
    for i in range(args.warmup + steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        t = host_th.to("cuda", non_blocking=True)
        lv = ((dr.forward_raw(t)[..., :3] - target[..., :3]) ** 2).sum().item()
        if i >= args.warmup:
            e2e_fwd.append(time.perf_counter() - t0)
    e2e_fwd_ms = statistics.mean(e2e_fwd) * 1e3
    cpu = None
    if cpu and not args.no_cpu:
        cpu = cpu_baseline_diff(cfg, W)
    dr.close()
    return {
        "metric": "fwd+bwd time / fwd time", "value": step_ms / fwd_ms, "unit": "x", "n_gpus": 1,
        "steps": steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded flame generator)",
        "config": {"workload": "diff_512", "desc": "4 xforms {linear,sinusoidal,spherical} (contractive), 512x512 ss1, "
                   "2e8 samples, 65536 walkers, bilinear splat, L2 loss vs image at theta+N(0,0.05); "
                   f"grads for {dr.n_params} parameters through the last 16 iterations, checkpoints every 64",
                   "l2": "histogram 4 MB (L2-resident), cleared every forward"},
        "fwd_ms": fwd_ms, "fwd_bwd_ms": step_ms, "bwd_kernel_ms": bwd_ms,
        "samples_per_s_fwd": plotted / (fwd_ms * 1e-3), "samples_per_s_fwd_bwd": plotted / (step_ms * 1e-3),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": None, "kernel": "ffb_diff_forward",
                     "kernel_ms": fwd_ms, "algorithmic_bytes_per_launch": bytes_per_launch, "peak_kind": peak_kind},
        "l2_atomic": {"achieved_v4_reductions_per_s": 4 * inframe / (fwd_ms * 1e-3), "peak_v4_reductions_per_s": v4_peak,
                      "frac": 4 * inframe / (fwd_ms * 1e-3) / v4_peak, "peak_from": "ffb_atomic_bench kind 2, 512^2 pixels"},
        "e2e": {"value": e2e_ms / e2e_fwd_ms, "unit": "x", "ms_fwd_bwd": e2e_ms, "ms_fwd": e2e_fwd_ms,
                "h2d_bytes_per_step": th.numel() * 4, "d2h_bytes_per_step": th.numel() * 4 + 8,
                "path": "ffb200.diff.DiffRenderer.render (torch.autograd.Function): theta from pinned host memory, "
                        "loss and dL/dtheta back to the host"},
        "gpu_launches": 5 * steps + 3 * steps,
        "clocks": clk,
        "cpu_baseline": cpu,
    }


def cpu_baseline_diff(cfg, W, budget_s=10.0):
    """The FP64 oracle's forward and gradient on the host cores, on a bounded
    sample of the same flame at 512^2: samples/s of fwd and of fwd+bwd."""
    import numpy as np
    from oracle import oracle as O
    O.build()
    threads = min(os.cpu_count() or 1, 64)
    fl = O.DiffFlame(cfg, W, W)
    walkers, iters = threads * 16, 20 + 64
    t0 = time.perf_counter()
    hist, n = fl.render(walkers, iters, threads=threads)
    t_f = time.perf_counter() - t0
    scale = max(1, int(budget_s / 2 / max(t_f, 1e-3)))
    walkers *= min(scale, 64)
    t0 = time.perf_counter()
    hist, n = fl.render(walkers, iters, threads=threads)
    t_f = time.perf_counter() - t0
    dh = np.random.default_rng(0).normal(0, 1e-3, hist.shape)
    t0 = time.perf_counter()
    fl.grad(dh, walkers, iters, threads=threads)
    t_b = time.perf_counter() - t0
    return {"value": n / (t_f + t_b), "unit": "samples/s (fwd+bwd)", "fwd_samples_per_s": n / t_f, "cores": threads,
            "kind": "port", "sample": f"{n} samples ({walkers} walkers x 64 after burn-in 20) of the same flame at {W}x{W}; "
                                      "gradient per sample walking its 16-iteration window, FD Jacobians, f64"}


def run_reference(args, rank, world):
    """The reference's CPU path: there is none (variations exist only as
    WGSL; benches/flame_bench.rs:1-10), so the oracle port of it runs on all
    host threads, each step a bounded sample of the same workload."""
    if rank != 0:
        return None
    if args.workload == "diff_512":
        from ffb200 import synthetic
        rates = [cpu_baseline_diff(synthetic.diff_flame(4), 512, budget_s=4.0) for _ in range(args.steps)]
        v = statistics.mean(r["value"] for r in rates)
        fwd = statistics.mean(r["fwd_samples_per_s"] for r in rates)
        return {
            "impl": "reference", "metric": "fwd+bwd time / fwd time", "value": fwd / v, "unit": "x", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 2e8 / v * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded flame generator)",
            "config": {"workload": "diff_512"},
            "cpu_baseline": dict(rates[-1], value=fwd / v, unit="x"),
            "e2e": {"value": fwd / v, "unit": "x", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference has no gradients; this is the oracle's FP64 restatement of this build's definition",
        }
    wl = workload(args.workload)
    c = cpu_rate(wl, steps=args.steps, warmup=args.warmup)
    v = c["value"]
    return {
        "impl": "reference", "metric": "samples/s", "value": v, "unit": "samples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": c["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded flame generator; no dataset)",
        "config": config_for(args, wl, world),
        "samples_per_step": c["samples_per_step"],
        "ms_per_frame_extrapolated": wl["iterations"] / v * 1e3,
        "cpu_baseline": dict(c, kind="port"),
        "e2e": {"value": v, "unit": "samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU render path (its variations exist only as WGSL); this is the oracle's "
                "restatement of it (oracle/), each step a timed bounded sample of the frame; ms_per_step is that "
                "sample's measured time, ms_per_frame_extrapolated the whole frame at the measured rate",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="full_1080p_ss2",
                    choices=["full_1080p_ss2", "plain_256", "batched_256", "stress_4k", "diff_512"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the default line's extra legs (parity, batched, diff, 4K stress)")
    ap.add_argument("--math", default="precise", choices=["precise", "sfu"],
                    help="precise: IEEE-accurate sin/cos (the parity-tested path); sfu: the hardware's, as the reference GPU")
    ap.add_argument("--schedule", default="auto", choices=["auto", "plain", "sorted"],
                    help="walker scheduling of the chaos kernel (same orbits either way)")
    ap.add_argument("--accumulate", default="auto", choices=["auto", "direct", "tiled"],
                    help="exact mode: direct atomics on the histogram or tile-sorted accumulation")
    ap.add_argument("--plot", default="auto", choices=["auto", "inline", "deferred", "fused"],
                    help="where the samples are plotted: by each walker, by a second kernel, or by plot warps "
                         "in the walkers' own block (the same histogram)")
    ap.add_argument("--profile", type=float, default=0.0,
                    help="profiling run for ncu: only the chaos kernel of the workload, at this many samples")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.profile and args.workload == "diff_512":
        import torch
        from ffb200 import diff, synthetic
        dr = diff.DiffRenderer(synthetic.diff_flame(4), 512, 512, int(args.profile), walkers=65536, seed=2024)
        th = dr.theta0()
        for _ in range(args.warmup + args.steps):
            img = dr.forward_raw(th)
            g = dr.backward_raw(img * 0.01)
        torch.cuda.synchronize()
        print(json.dumps({"profile": "diff_512", "samples": dr.samples()[0], "grad_norm": float(g.norm())}))
        dr.close()
        return
    if args.profile:
        from ffb200 import _native
        wl = workload(args.workload)
        r = _native.Renderer(local_rank)
        job = dict(iterations=int(args.profile), walkers=wl["walkers"], supersample=wl["supersample"], seed=0x5EED,
                   schedule=args.schedule, count_bits=wl.get("count_bits", 32), accumulate=args.accumulate, plot=args.plot)
        hist = r.histogram_u64 if wl.get("count_bits", 32) == 64 else r.histogram
        for _ in range(args.warmup + args.steps):
            _, _, o = hist(json.dumps(wl["cfg"]), wl["width"], wl["height"], **job)
        print(json.dumps({"profile": args.workload, "samples": o.total_iterations, "inframe": o.inframe_samples,
                          "ms": o.render_time_ms}))
        return
    if args.workload in ("batched_256", "diff_512") and args.impl == "ours":
        runner = run_batched if args.workload == "batched_256" else run_diff
        line = runner(args, local_rank) if rank == 0 else None
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        line = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
