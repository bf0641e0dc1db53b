#!/usr/bin/env python
"""NL-SAR benchmark: Mpix/s of the fused B200 path on one 4096x4096 InSAR scene.

Workload: the plain NL-SAR configuration on a single 4096 x 4096 float32
synthetic scene (search window 21, patches {3,5,7}, scales {1,3}, h 15, c 49,
per-pixel selection by the largest bias-reduced ENL), statistics trained on a
separate seeded 128 x 128 homogeneous area (reflectivity 1, coherence 0.6).
Seeded synthetic data stands in for real interferograms.

A step is one full filter of the scene (prep kernels + the fused kernel) with
inputs resident in HBM (201 MB of inputs, larger than the 126 MB L2, so every
step streams them from HBM).  `e2e` is the same metric through the public host
API with pinned host buffers, copies included.  Under torchrun each rank
filters its own scene (weak scaling, no collective on the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Other patch and scale sets (`--patches 3,5,7,9,11 --scales 1,3,5`, the
reference example's settings) are timed the same way; the roofline's
algorithmic flop count follows them.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "NL-SAR Mpix/s"
UNIT = "Mpix/s"
SWS, PATCHES, SCALES, H_PARAM, C_PARAM = 21, [3, 5, 7], [1, 3], 15.0, 49.0


def flop_per_pixel(mode, patches=None, scales=None):
    """Algorithmic FP32 work per output pixel (FMA = 2 flops) with S scales,
    P patch sizes, N = 441 window offsets and U = 220 of a half window:
    pixel similarity S U 14 + box sums S P U 4 + weights S P U 10 + ENL
    statistics S P N 11 + their finalisation S P 30 + selection S P +
    weighted mean N 9 + 15 + set-up/decompose 40.  ENL-argmax selection
    computes every (patch, scale) combination; reference selection only the
    last statistics key (S = P = 1).  At patches {3,5,7}, scales {1,3}:
    57,956 (argmax) and 15,066 (reference)."""
    p = len(patches if patches is not None else PATCHES)
    sc = len(scales if scales is not None else SCALES)
    if mode != "argmax_enl":
        p = sc = 1
    n = SWS * SWS
    u = (n - 1) // 2
    return sc * u * 14 + sc * p * u * 4 + sc * p * u * 10 + sc * p * n * 11 + sc * p * 30 + sc * p + n * 9 + 15 + 40


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--size", type=int, default=None, help="scene side (plain: 4096, secondary: 8192)")
    p.add_argument("--mode", default="argmax_enl", choices=["argmax_enl", "reference"])
    p.add_argument("--cpu-sample", type=int, default=1536,
                   help="side of the CPU-baseline crop (about 10-15 s of oracle work on 16 host cores)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--patches", default=None, help="patch sizes, comma separated (default 3,5,7)")
    p.add_argument("--scales", default=None, help="scale sizes, comma separated (default 1,3)")
    p.add_argument("--config", default="plain", choices=["plain", "batched", "serving", "secondary"],
                   help="plain: one 4096x4096 scene (the headline); batched: 48 scenes of uneven size; "
                        "serving: Poisson request streams through the request server; secondary: Goldstein, "
                        "boxcar and NL-InSAR on an 8192x8192 scene")
    p.add_argument("--nlinsar-size", type=int, default=2048, help="secondary: side of the NL-InSAR scene")
    p.add_argument("--polsar-size", type=int, default=1024, help="secondary: side of the 3x3 covariance scene")
    p.add_argument("--cov-size", type=int, default=2048, help="secondary: side of the 2x2 covariance scene")
    p.add_argument("--requests", type=int, default=96, help="serving: requests per stream")
    p.add_argument("--hbm-budget-gb", type=float, default=120.0, help="serving: admission budget")
    p.add_argument("--no-extras", action="store_true",
                   help="plain: skip the shortened batched and served measurements beside the headline")
    p.add_argument("--extra-requests", type=int, default=24, help="plain: requests of the served stream")
    return p.parse_args()


def max_over_ranks(value, dist, device):
    """The largest `value` over all ranks, returned on every rank (`value`
    itself without a process group).  Times of a multi-GPU run are reported
    as the maximum over ranks."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(rank):
    """Scene seed of a replica: each rank filters its own scene (weak scaling,
    no data exchanged between ranks)."""
    return 1 + rank


def aggregate_mpix(n_ranks, side, ms):
    """Whole-job Mpix/s: every rank filtered one side x side scene in `ms`
    (the slowest rank's time)."""
    return n_ranks * side * side / (ms * 1e-3) / 1e6


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        finally:
            os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_stats(dcl, synthetic):
    t1, t2, tp = synthetic.training_area(128, seed=7)
    return dcl.nlsar_train_insar(t1, t2, tp, PATCHES, SCALES)


def cpu_oracle_rate(a1, a2, ph, stats, side, mode, threads):
    """The oracle (FP32 restatement of the reference path) on a side x side
    crop, all host threads: Mpix/s and seconds."""
    from oracle import pyoracle

    y0 = (a1.shape[0] - side) // 2
    x0 = (a1.shape[1] - side) // 2
    crop = [x[y0:y0 + side, x0:x0 + side].copy() for x in (a1, a2, ph)]
    t = time.perf_counter()
    pyoracle.nlsar_insar(*crop, SWS, PATCHES, SCALES, stats, H_PARAM, C_PARAM,
                         select_mode=1 if mode == "argmax_enl" else 0, nthreads=threads)
    dt = time.perf_counter() - t
    return side * side / dt / 1e6, dt


def traffic_from_profiles(size):
    """DRAM bytes per fused launch from the committed ncu summary, scaled to
    `size`, or None."""
    path = os.path.join(ROOT, "profiles", "nlsar_fast_kernel.md")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_pixel:"):
                return float(line.split(":")[1]) * size * size
    except OSError:
        pass
    return None


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    import numpy as np  # noqa: F401

    import despeckcl_b200 as dcl  # noqa: F401  (stats container only)
    from despeckcl_b200 import synthetic
    from oracle import pyoracle

    threads = os.cpu_count() or 1
    t1, t2, tp = synthetic.training_area(128, seed=7)
    stats = pyoracle.training_insar(t1, t2, tp, PATCHES, SCALES)
    side = min(args.cpu_sample, args.size)
    a1, a2, ph = synthetic.insar_scene(args.size, args.size, 1)
    for _ in range(args.warmup):
        cpu_oracle_rate(a1, a2, ph, stats, min(side, 64), args.mode, threads)
    times = []
    for _ in range(args.steps):
        _, dt = cpu_oracle_rate(a1, a2, ph, stats, side, args.mode, threads)
        times.append(dt)
    ms = 1e3 * sum(times) / len(times)
    value = side * side / (ms * 1e-3) / 1e6
    sample = (f"{side}x{side} centre crop of the {args.size}x{args.size} scene per step, FP32 oracle "
              f"(CPU restatement of the reference path; the OpenCL reference cannot be built here)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"plain NL-SAR, {args.size}x{args.size} scene (CPU sample {side}x{side})",
                       "search_window": SWS, "patches": PATCHES, "scales": SCALES, "select_mode": args.mode},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import ctypes

    import numpy as np
    import torch

    import despeckcl_b200 as dcl
    from despeckcl_b200 import synthetic

    ws, rank, local = dist_env()
    if ws != args.gpus:
        args.gpus = ws
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    L = dcl.lib()
    S = args.size
    stats = make_stats(dcl, synthetic)
    a1, a2, ph = synthetic.insar_scene(S, S, replica_seed(rank))
    dev = [torch.from_numpy(x).cuda() for x in (a1, a2, ph)]
    out = tuple(torch.empty((S, S), dtype=torch.float32, device="cuda") for _ in range(3))
    stream = torch.cuda.current_stream()

    def step():
        dcl.nlsar_insar_device(*dev, SWS, PATCHES, SCALES, stats, H_PARAM, C_PARAM, select_mode=args.mode, out=out,
                               stream=stream)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clk:
        L.dcl_profile_begin()
        start.record(stream)
        for _ in range(args.steps):
            step()
        stop.record(stream)
        torch.cuda.synchronize()
        fused_ms = ctypes.c_double()
        fused_n = ctypes.c_long()
        all_n = ctypes.c_long()
        rc = L.dcl_profile_end(ctypes.byref(fused_ms), ctypes.byref(fused_n), ctypes.byref(all_n))
        if rc != 0:
            raise RuntimeError(L.dcl_last_error().decode())
    ms_step = max_over_ranks(start.elapsed_time(stop) / args.steps, dist, "cuda")
    if dist:
        dist.barrier()
    clocks = clk.summary()
    value = aggregate_mpix(args.gpus, S, ms_step)

    # end to end through the public host API, pinned host buffers
    pin = [torch.from_numpy(x).pin_memory() for x in (a1, a2, ph)]
    hout = [torch.empty((S, S), dtype=torch.float32).pin_memory() for _ in range(3)]
    hin = [p.numpy() for p in pin]
    hres = [o.numpy() for o in hout]

    def e2e_step():
        import despeckcl_b200.api as api

        pk, pp, npn = api._ints(PATCHES)
        sk, sp, nsn = api._ints(SCALES)
        arr, n, keep = api._entries(stats)
        api._check(L.dcl_nlsar_insar(api._fp(hin[0]), api._fp(hin[1]), api._fp(hin[2]), api._fp(hres[0]),
                                     api._fp(hres[1]), api._fp(hres[2]), S, S, SWS, pp, npn, sp, nsn, arr, n,
                                     ctypes.c_float(H_PARAM), ctypes.c_float(C_PARAM), api._mode(args.mode)))

    e2e_step()
    if dist:
        dist.barrier()
    ke = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(ke):
        e2e_step()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / ke, dist, "cuda")
    e2e_value = aggregate_mpix(args.gpus, S, e2e_ms)
    np.testing.assert_array_equal(hres[0], out[0].cpu().numpy())  # same result through both entry points

    peak = ctypes.c_double()
    if L.dcl_measure_fp32_tflops(ctypes.byref(peak)) != 0:
        raise RuntimeError(L.dcl_last_error().decode())
    kern_ms = fused_ms.value / max(1, fused_n.value)
    achieved = flop_per_pixel(args.mode) * S * S / (kern_ms * 1e-3) / 1e12
    # the committed ncu summary covers the headline configuration only
    headline = PATCHES == [3, 5, 7] and SCALES == [1, 3] and args.mode == "argmax_enl"
    traffic = traffic_from_profiles(S) if headline else None

    # the batched and served workloads, shortened, beside the headline (one
    # GPU only; the headline numbers above are already taken)
    batched = served = None
    if args.gpus == 1 and not args.no_extras and PATCHES == [3, 5, 7] and SCALES == [1, 3]:
        del dev, out
        torch.cuda.empty_cache()
        batched = batched_measure(args, stats, 3)
        served = serving_measure(args, stats, args.extra_requests, (1.1,))

    cpu = None
    if rank == 0 and args.gpus == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, dt = cpu_oracle_rate(a1, a2, ph, stats, min(args.cpu_sample, S), args.mode, threads)
        side = min(args.cpu_sample, S)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{side}x{side} centre crop of the scene, FP32 oracle (CPU restatement of the reference "
                         f"path), {dt:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator, 40 rectangles + fringes, "
                                                          "single-look speckle)",
            "config": {"workload": f"plain NL-SAR on one {S}x{S} scene per GPU", "search_window": SWS,
                       "patches": PATCHES, "scales": SCALES, "h": H_PARAM, "c": C_PARAM,
                       "select_mode": args.mode, "l2": "inputs 201 MB > L2 126 MB per step",
                       "parallelism": f"replica x{args.gpus}"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 3 * S * S * 4,
                    "d2h_bytes_per_step": 3 * S * S * 4, "ms_per_step": e2e_ms},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                         "frac": achieved / peak.value, "traffic": traffic,
                         "kernel": "nlsar_fast_kernel (specialised fused NL-SAR)", "kernel_ms": kern_ms,
                         "flop_per_pixel": flop_per_pixel(args.mode),
                         "peak_source": "measured in-process FP32 FMA probe (dcl_measure_fp32_tflops)"},
            "gpu_launches": int(all_n.value),
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if batched:
            line["batched"] = batched
        if served:
            line["serving"] = {k: v for k, v in served.items() if k != "rates"}
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def batched_scenes(n=48, lo=256, hi=2048, seed0=100):
    """The batched workload: n scenes with H, W uniform in [lo, hi] (seeded)."""
    import numpy as np

    rng = np.random.default_rng(2024)
    return [(int(rng.integers(lo, hi + 1)), int(rng.integers(lo, hi + 1)), seed0 + i) for i in range(n)]


def batched_measure(args, stats, k):
    """48 interferograms of uneven size: one persistent launch per run (eager
    and as a CUDA graph, kernel instantiation picked by the autotuner) against
    looping the plain one-scene-per-launch path over the same scenes; device
    times with CUDA events on the launching stream."""
    import torch

    import despeckcl_b200 as dcl
    from despeckcl_b200 import synthetic

    spec = batched_scenes()
    scenes = []
    for h, w, seed in spec:
        scenes.append(tuple(torch.from_numpy(x).cuda() for x in synthetic.insar_scene(h, w, seed)))
    mpix = sum(h * w for h, w, _ in spec) / 1e6
    stream = torch.cuda.current_stream()
    outs = [tuple(torch.empty((h, w), device="cuda") for _ in range(3)) for h, w, _ in spec]

    def loop():
        for s, o in zip(scenes, outs):
            dcl.nlsar_insar_device(*s, SWS, PATCHES, SCALES, stats, H_PARAM, C_PARAM, select_mode=args.mode, out=o,
                                   stream=stream)

    def timed(fn, k):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k

    ms_loop = timed(loop, k)
    eager = dcl.NlsarBatch(scenes, SWS, PATCHES, SCALES, stats, H_PARAM, C_PARAM, select_mode=args.mode, outs=outs,
                           graph=False, autotune=True)
    ms_eager = timed(lambda: eager.run(stream), k)
    graph = dcl.NlsarBatch(scenes, SWS, PATCHES, SCALES, stats, H_PARAM, C_PARAM, select_mode=args.mode, outs=outs,
                           graph=True, autotune=True)
    ms_graph = timed(lambda: graph.run(stream), k)
    res = {"workload": f"{len(spec)} scenes, H and W uniform in [256, 2048], {mpix:.1f} Mpix per step",
           "mpix_s": mpix / (ms_graph * 1e-3), "ms_per_step": ms_graph, "steps": k,
           "plain_loop": {"mpix_s": mpix / (ms_loop * 1e-3), "ms_per_step": ms_loop},
           "batched_eager": {"mpix_s": mpix / (ms_eager * 1e-3), "ms_per_step": ms_eager},
           "speedup_vs_plain_loop": ms_loop / ms_graph, "kernel_variant": graph.variant,
           "gpu_launches": graph.launches}
    eager.close()
    graph.close()
    del scenes, outs
    torch.cuda.empty_cache()
    return res


def run_batched(args):
    import torch

    import despeckcl_b200 as dcl
    from despeckcl_b200 import synthetic

    torch.cuda.set_device(0)
    stats = make_stats(dcl, synthetic)
    k = max(1, args.steps)
    with ClockSampler(torch.cuda.current_device()) as clk:
        r = batched_measure(args, stats, k)
    line = {
        "metric": "NL-SAR Mpix/s (batched)", "value": r["mpix_s"], "unit": UNIT, "n_gpus": 1,
        "steps": k, "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": r["workload"], "search_window": SWS, "patches": PATCHES, "scales": SCALES,
                   "select_mode": args.mode},
        "plain_loop": r["plain_loop"], "batched_eager": r["batched_eager"],
        "speedup_vs_plain_loop": r["speedup_vs_plain_loop"], "kernel_variant": r["kernel_variant"],
        "gpu_launches": r["gpu_launches"], "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def _pct(v, q):
    import numpy as np

    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def serving_measure(args, stats, n, factors):
    """Poisson request streams (`factors` times the plain path's request rate)
    of scenes with sides uniform in [256, 4096], each request seeded by its id,
    served by the request server (HBM-budget admission, continuous batching)
    and, under the same arrivals, by the plain path (one scene per call, one
    call at a time).  Inputs and outputs stay on the device; latency runs from
    a request's arrival to the end of its last launch."""
    import threading
    import time

    import numpy as np
    import torch

    import despeckcl_b200 as dcl
    from despeckcl_b200 import synthetic

    rng = np.random.default_rng(5)
    sizes = [(int(rng.integers(256, 4097)), int(rng.integers(256, 4097))) for _ in range(n)]
    scenes = [synthetic.insar_scene_device(h, w, i) for i, (h, w) in enumerate(sizes)]
    outs = [tuple(torch.empty((h, w), device="cuda") for _ in range(3)) for h, w in sizes]
    torch.cuda.synchronize()
    px = np.array([h * w for h, w in sizes], dtype=np.float64)
    stream = torch.cuda.current_stream()
    kw = dict(select_mode=args.mode)

    def plain_one(i):
        dcl.nlsar_insar_device(*scenes[i], SWS, PATCHES, SCALES, stats, H_PARAM, C_PARAM, out=outs[i], stream=stream,
                               **kw)

    # capacities: all requests queued at once
    for i in range(min(3, n)):
        plain_one(i)
    torch.cuda.synchronize()
    t = time.perf_counter()
    for i in range(n):
        plain_one(i)
        stream.synchronize()
    t_plain = time.perf_counter() - t
    mu = n / t_plain
    budget = int(args.hbm_budget_gb * (1 << 30))
    srv = dcl.NlsarServer(SWS, PATCHES, SCALES, stats, H_PARAM, C_PARAM, hbm_budget_bytes=budget, **kw)
    for rid in [srv.submit(*scenes[i], out=outs[i]) for i in range(min(3, n))]:
        srv.wait(rid, timeout=600)
    t = time.perf_counter()
    ids = [srv.submit(*scenes[i], out=outs[i]) for i in range(n)]
    for rid in ids:
        srv.wait(rid, timeout=600)
    t_served = time.perf_counter() - t

    def served_stream(arr):
        t0 = srv.now() + 0.01
        ids = [None] * n
        ready = threading.Semaphore(0)

        def client():
            for i in range(n):
                d = t0 + arr[i] - srv.now()
                if d > 0:
                    time.sleep(d)
                ids[i] = srv.submit(*scenes[i], out=outs[i])
                ready.release()

        th = threading.Thread(target=client)
        th.start()
        lat, done, chunks = [], [], []
        for i in range(n):
            ready.acquire()
            _, info = srv.wait(ids[i], timeout=600)
            lat.append(info["done_s"] - (t0 + arr[i]))
            done.append(info["done_s"] - t0)
            chunks.append(info["chunks"])
        th.join()
        span = max(done) - arr[0]
        return {"mpix_s": px.sum() / 1e6 / span, "p50_ms": 1e3 * _pct(lat, 50), "p99_ms": 1e3 * _pct(lat, 99),
                "mean_chunks": float(np.mean(chunks))}

    def plain_stream(arr):
        lat, done = [], []
        t0 = time.perf_counter() + 0.01
        for i in range(n):
            d = t0 + arr[i] - time.perf_counter()
            if d > 0:
                time.sleep(d)
            plain_one(i)
            stream.synchronize()
            e = time.perf_counter() - t0
            lat.append(e - arr[i])
            done.append(e)
        span = max(done) - arr[0]
        return {"mpix_s": px.sum() / 1e6 / span, "p50_ms": 1e3 * _pct(lat, 50), "p99_ms": 1e3 * _pct(lat, 99)}

    rates = []
    for k, f in enumerate(factors):
        lam = f * mu
        arr = np.cumsum(np.random.default_rng(1000 + k).exponential(1.0 / lam, n))
        arr -= arr[0]
        b0 = srv.stats()["batches"]
        served = served_stream(arr)
        served["batches"] = srv.stats()["batches"] - b0
        plain = plain_stream(arr)
        rates.append({"rate_factor": f, "offered_req_s": lam, "offered_mpix_s": lam * px.mean() / 1e6,
                      "served": served, "plain": plain})
    st = srv.stats()
    srv.close()
    top = rates[-1]["served"]
    res = {"workload": f"{n} requests per stream, sides uniform in [256, 4096], {px.sum() / 1e6:.0f} Mpix per stream",
           "hbm_budget_gb": args.hbm_budget_gb, "max_inflight": 2, "max_batch_tiles": 148 * 8,
           "rate_factor": factors[-1], "mpix_s": top["mpix_s"], "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"],
           "plain_p50_ms": rates[-1]["plain"]["p50_ms"], "plain_p99_ms": rates[-1]["plain"]["p99_ms"],
           "capacity": {"plain_mpix_s": px.sum() / 1e6 / t_plain, "served_mpix_s": px.sum() / 1e6 / t_served,
                        "plain_req_s": mu, "ratio": t_plain / t_served},
           "rates": rates,
           "server": {"batches": st["batches"], "kernel_launches": st["kernel_launches"],
                      "peak_admitted_gb": st["peak_admitted_bytes"] / 2 ** 30, "peak_inflight": st["peak_inflight"]}}
    del scenes, outs
    torch.cuda.empty_cache()
    return res


def run_serving(args):
    import torch

    import despeckcl_b200 as dcl
    from despeckcl_b200 import synthetic

    torch.cuda.set_device(0)
    stats = make_stats(dcl, synthetic)
    n = args.requests
    with ClockSampler(torch.cuda.current_device()) as clk:
        r = serving_measure(args, stats, n, (0.5, 0.8, 1.1))
    line = {
        "metric": "NL-SAR served Mpix/s (Poisson arrivals at 1.1x the plain request rate)",
        "value": r["mpix_s"], "unit": UNIT, "n_gpus": 1, "steps": n, "warmup": 3,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (generated on the device, seed = request id)",
        "config": {"workload": r["workload"], "search_window": SWS, "patches": PATCHES, "scales": SCALES,
                   "select_mode": args.mode, "hbm_budget_gb": args.hbm_budget_gb, "max_inflight": 2,
                   "max_batch_tiles": 148 * 8},
        "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"], "capacity": r["capacity"], "rates": r["rates"],
        "server": r["server"], "gpu_launches": r["server"]["kernel_launches"], "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def run_secondary(args):
    """The secondary filters on the precision-study scene (8192 x 8192 by
    default, --size): Goldstein (patch 32, overlap 4, alpha 0.5), boxcar
    (window 7) and NL-InSAR (search 21, patch 7, lmin 10; one pass per step,
    --nlinsar-size scene).  Each is timed with CUDA events on the launching
    stream over K steps with inputs resident in HBM, larger than L2."""
    import ctypes

    import torch

    import despeckcl_b200 as dcl
    from despeckcl_b200 import synthetic

    torch.cuda.set_device(0)
    L = dcl.lib()
    stream = torch.cuda.current_stream()
    S = args.size or 8192
    a1, a2, ph = synthetic.insar_scene_device(S, S, 4)
    k = max(1, args.steps)

    def timed(fn):
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        L.dcl_profile_begin()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        import ctypes
        n_all = ctypes.c_long()
        L.dcl_profile_end(None, None, ctypes.byref(n_all))
        return a.elapsed_time(b) / k, int(n_all.value)

    hbm = None
    try:
        hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        hbm_src = "MEASURED_PEAKS.json hbm_gbs (measured)"
    except (OSError, KeyError, ValueError):
        hbm, hbm_src = 6650.0, "fallback 6.65 TB/s"
    res = {}
    with ClockSampler(torch.cuda.current_device()) as clk:
        g_out = tuple(torch.empty((S, S), device="cuda") for _ in range(2))
        ms, n = timed(lambda: dcl.goldstein_device(a1, a2, ph, 32, 4, 0.5, out=g_out, stream=stream))
        # algorithmic bytes: three planes in, reflectivity and phase out
        res["goldstein"] = {"mpix_s": S * S / (ms * 1e-3) / 1e6, "ms": ms, "launches_per_step": n / k,
                            "roofline": {"bound": "hbm", "bytes_per_pixel": 20,
                                         "achieved_gbs": 20 * S * S / (ms * 1e-3) / 1e9, "peak_gbs": hbm,
                                         "frac": 20 * S * S / (ms * 1e-3) / 1e9 / hbm}}
        b_out = tuple(torch.empty((S, S), device="cuda") for _ in range(3))
        ms, n = timed(lambda: dcl.boxcar_device(a1, a2, ph, 7, out=b_out, stream=stream))
        res["boxcar"] = {"mpix_s": S * S / (ms * 1e-3) / 1e6, "ms": ms, "launches_per_step": n / k,
                         "roofline": {"bound": "hbm", "bytes_per_pixel": 24,
                                      "achieved_gbs": 24 * S * S / (ms * 1e-3) / 1e9, "peak_gbs": hbm,
                                      "frac": 24 * S * S / (ms * 1e-3) / 1e9 / hbm}}
        Sn = min(args.nlinsar_size, S)
        n1, n2, nph = (x[:Sn, :Sn].contiguous() for x in (a1, a2, ph))
        est = tuple(torch.zeros((Sn, Sn), device="cuda") for _ in range(3))
        ms, n = timed(lambda: dcl.nlinsar_device(n1, n2, nph, 21, 7, 1, 10, estimates=est, stream=stream))
        res["nlinsar"] = {"mpix_s_per_pass": Sn * Sn / (ms * 1e-3) / 1e6, "ms_per_pass": ms, "side": Sn,
                          "launches_per_step": n / k}
        # NL-SAR on a 3x3 (PolSAR) covariance image: single-look three-channel
        # speckle k = L x per pixel (one random covariance), planes [18][H][W];
        # statistics trained on a homogeneous 128 x 128 crop of it
        Sp = min(args.polsar_size, S)
        g = torch.Generator(device="cuda")
        g.manual_seed(7)
        z = torch.randn((3, 5), generator=g, device="cuda", dtype=torch.complex64)
        Lc = torch.linalg.cholesky(z @ z.conj().T / 5)
        x = torch.randn((3, Sp * Sp), generator=g, device="cuda", dtype=torch.complex64)
        kv = (Lc @ x).reshape(3, Sp, Sp)
        cov = kv[:, None] * kv[None, :].conj()
        planes = torch.empty((18, Sp, Sp), device="cuda")
        planes[0::2] = cov.real.reshape(9, Sp, Sp)
        planes[1::2] = cov.imag.reshape(9, Sp, Sp)
        tr = planes[:, :128, :128].cpu().numpy()
        cplx = (tr[0::2] + 1j * tr[1::2]).reshape(3, 3, 128, 128)
        st3 = dcl.nlsar_train(cplx, PATCHES, SCALES)
        out3 = torch.empty_like(planes)
        import despeckcl_b200.api as api
        pk, pp, npn = api._ints(PATCHES)
        sk, sp, nsn = api._ints(SCALES)
        arr, ns3, keep = api._entries(st3)

        def polsar():
            api._check(L.dcl_nlsar_covmat_device(api._dptr(planes), api._dptr(out3), Sp, Sp, 3, SWS, pp, npn, sp,
                                                 nsn, arr, ns3, ctypes.c_float(H_PARAM), ctypes.c_float(C_PARAM),
                                                 api._mode(args.mode), api._stream(stream)))

        ms, n = timed(polsar)
        res["nlsar_3x3"] = {"mpix_s": Sp * Sp / (ms * 1e-3) / 1e6, "ms": ms, "side": Sp, "select_mode": args.mode,
                            "launches_per_step": n / k}
        # NL-SAR on a 2x2 covariance image (the covariance overload, 8 planes
        # in and out) built from the InSAR scene: C00 = a1^2, C11 = a2^2,
        # C01 = a1 a2 e^{i phi}, C10 = conj(C01)
        Sc = min(args.cov_size, S)
        c1, c2, cph = (x[:Sc, :Sc] for x in (a1, a2, ph))
        m = c1 * c2
        cov8 = torch.stack([c1 * c1, torch.zeros_like(c1), m * torch.cos(cph), m * torch.sin(cph),
                            m * torch.cos(cph), -m * torch.sin(cph), c2 * c2, torch.zeros_like(c1)]).contiguous()
        tr = cov8[:, :128, :128].cpu().numpy()
        st2 = dcl.nlsar_train((tr[0::2] + 1j * tr[1::2]).reshape(2, 2, 128, 128), PATCHES, SCALES)
        outc = torch.empty_like(cov8)
        arr2, ns2, keep2 = api._entries(st2)

        def cov2x2():
            api._check(L.dcl_nlsar_covmat_device(api._dptr(cov8), api._dptr(outc), Sc, Sc, 2, SWS, pp, npn, sp,
                                                 nsn, arr2, ns2, ctypes.c_float(H_PARAM), ctypes.c_float(C_PARAM),
                                                 api._mode(args.mode), api._stream(stream)))

        ms, n = timed(cov2x2)
        res["nlsar_2x2_covariance"] = {"mpix_s": Sc * Sc / (ms * 1e-3) / 1e6, "ms": ms, "side": Sc,
                                       "select_mode": args.mode, "launches_per_step": n / k}
    line = {"metric": "secondary filters Mpix/s", "value": res["goldstein"]["mpix_s"], "unit": UNIT, "n_gpus": 1,
            "steps": k, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (generated on the device, seed 4)",
            "config": {"workload": f"{S}x{S} scene: Goldstein p32 ov4 a0.5, boxcar w7, NL-InSAR sws21 p7 lmin10 "
                                   f"one pass on {min(args.nlinsar_size, S)}^2, NL-SAR 3x3 covariances on "
                                   f"{min(args.polsar_size, S)}^2, NL-SAR 2x2 covariances on "
                                   f"{min(args.cov_size, S)}^2",
                       "l2": f"inputs {3 * S * S * 4 / 1e6:.0f} MB > L2 126 MB"},
            "hbm_peak_source": hbm_src, "filters": res, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    global PATCHES, SCALES
    args = parse()
    if args.patches:
        PATCHES = [int(x) for x in args.patches.split(",")]
    if args.scales:
        SCALES = [int(x) for x in args.scales.split(",")]
    if args.size is None and args.config != "secondary":
        args.size = 4096
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "batched":
        return run_batched(args)
    if args.config == "serving":
        return run_serving(args)
    if args.config == "secondary":
        return run_secondary(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
