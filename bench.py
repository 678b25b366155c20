"""X-engine benchmark: input Gb/s and int8 cGEMM TOPS on one B200 (or N replicas).

Workload (the larger plain array): 32 x 32 = 1024 elements, 256 channels, complex
int8, three point sources (amplitudes 4, 2, 1 at seeded random (l, m) with
|l|, |m| < 0.4) plus complex Gaussian noise sigma = 8, K = 1024 samples per
sub-integration, int64 long-term integration, lower-triangle tiles only.
Packets use the wire format (8256-byte heaps, 64-byte header, planar int8
payload; 256 channels x 16 samples per packet).  Inputs are synthetic, made
by the seeded packet source.

One step = `--batch` sub-integrations (default 32, 17.3 GB of packets) through
corner-turn -> tcgen05 triangle GEMM (int32 in TMEM over the whole step) ->
int64 integration.  `value` is device-resident throughput; `e2e` is the same
work through the public context API from pinned host packets (host->device
copies inside the timed region, overlapped with compute) with the live image
read back every step.  `plain` is the per-sub-integration launch form.

`--impl reference` times the CPU restatement of the reference path (OpenMP
int64 correlator over the same packets) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "daqiri-mixer_b200"))

NANT, SIDE, NCH, TPKT, KSUB, G = 1024, 32, 256, 16, 1024, 64
HDR, STRIDE = 64, 64 + 2 * NCH * TPKT          # 8256
HEAPS_PER_SUB = KSUB // TPKT                   # 64
SIGMA, SEED = 8.0, 20261203
METRIC = "int8 cGEMM TOPS & input Gb/s vs roofline (stream vs plain); p50/p99 dump latency"
L2_BYTES = 126 * 1024 * 1024
# DRAM bytes of one k_xcorr_tri launch over its algorithmic bytes (planes read
# once + int64 cube read and written), from the ncu capture at the benchmark's
# own K of 32 768 samples per launch on 1024 elements x 32 channels:
# 2.7684 + 0.2753 GB measured / 2.7514 GB algorithmic (13 % extra plane reads).
XCORR_TRAFFIC_RATIO = (2.7684 + 0.2753) / 2.7514


# The plain (one array) workloads.  nch x tpkt = 4096 keeps the 8192-byte payload.
PLAIN_CONFIGS = {
    # the reference's own array: 16 x 16, 128 ch, K 256, 64 sub-integrations per dump,
    # star A1 6 at (0.10, -0.05) + planet 1.5 c/128 at radius 0.2, noise sigma 16
    "small": dict(nant=256, side=16, nch=128, ksub=256, grid=32, sigma=16.0, noise=0, batch=64,
                  text="filled 16x16=256 elements, 128 ch, K=256, 64 sub-integrations per dump "
                       "(one step = one dump), star + planet + sigma 16 noise"),
    # the larger plain array (the headline)
    "plain": dict(nant=1024, side=32, nch=256, ksub=1024, grid=64, sigma=8.0, noise=0, batch=32,
                  text="plain array 32x32=1024 elements, 256 ch, K=1024 per sub-integration, "
                       "3 sources + sigma 8 noise, int64 integration"),
    # large-N stress: uniform int8 in [-127, 127], 128 x 128 imaging
    "large": dict(nant=4096, side=64, nch=64, ksub=2048, grid=128, sigma=0.0, noise=1, batch=16,
                  text="large-N stress 64x64=4096 elements, 64 ch, K=2048 per sub-integration, "
                       "uniform int8 in [-127, 127], int64 integration, 128x128 imaging"),
}
CFG = PLAIN_CONFIGS["plain"]


def configure(nch=None, name="plain"):
    """Select a plain workload; optionally override the channel count of the
    packets (the payload stays 8192 bytes: tpkt = 4096 / nch)."""
    global CFG, NANT, SIDE, NCH, TPKT, KSUB, G, SIGMA, STRIDE, HEAPS_PER_SUB
    CFG = PLAIN_CONFIGS[name]
    NANT, SIDE, KSUB, G, SIGMA = CFG["nant"], CFG["side"], CFG["ksub"], CFG["grid"], CFG["sigma"]
    nch = nch or CFG["nch"]
    if 4096 % nch or (4096 // nch) % 16 or KSUB % (4096 // nch):
        raise SystemExit("--nch must divide 4096 with 4096/nch a multiple of 16 dividing K")
    NCH, TPKT = nch, 4096 // nch
    STRIDE = HDR + 2 * NCH * TPKT
    HEAPS_PER_SUB = KSUB // TPKT


def sources(seed=SEED):
    import numpy as np
    if CFG is PLAIN_CONFIGS["small"]:
        return [(0.10, -0.05, 6.0, 0.0), (0.2, 0.0, 0.0, 1.5)]
    if CFG["noise"] == 1:
        return []
    rng = np.random.default_rng(seed)
    lm = rng.uniform(-0.4, 0.4, size=(3, 2))
    return [(float(lm[s, 0]), float(lm[s, 1]), amp, 0.0) for s, amp in enumerate((4.0, 2.0, 1.0))]


def tri_ops(nsamp):
    T = NANT * (NANT + 1) // 2
    return 8.0 * T * nsamp * NCH


def wire_gbps(npackets, seconds):
    return 8.0 * STRIDE * npackets / seconds / 1e9


def dist_setup(n_gpus):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


def barrier(pg, dev):
    if pg is not None:
        import torch
        t = torch.zeros(1, device=dev)
        pg.all_reduce(t)


def max_over_ranks(pg, value, dev):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, value, dev):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    pg.all_reduce(t)
    return float(t.item())


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        loaded = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f)
    except OSError:
        return {}


def make_packets(mixer, torch, dev, nheaps, heap0=0):
    src = sources()
    sky = torch.from_numpy(mixer.sky_table(NANT, NCH, SIDE, src)).to(dev) if src else None
    pk = torch.empty(nheaps * NANT * STRIDE, dtype=torch.uint8, device=dev)
    mixer.gen_packets(pk, STRIDE, HDR, NANT, NCH, TPKT, nheaps, heap0, heap0 * NANT, 4096, sky,
                      SIGMA, SEED, CFG["noise"])
    return pk


def cpu_correlator_sample(packets_host, nheaps, target_s=12.0, max_threads=0, max_out=2e9):
    """Time the oracle's OpenMP int64 correlator on a channel subset of one
    sub-integration; returns (gbps_equivalent, cores, sample_description,
    seconds, full-square int64 V of the sampled channels)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    if max_threads:
        os.environ["OMP_NUM_THREADS"] = str(max_threads)
    sub = packets_host[: HEAPS_PER_SUB * NANT * STRIDE]
    planes = oracle.corner_turn(np.ascontiguousarray(sub), NANT, NCH, TPKT, HEAPS_PER_SUB)
    cores = oracle.max_threads()
    out = np.zeros((1, 2, NANT, NANT), dtype=np.int64)
    t0 = time.perf_counter()
    oracle.correlate(planes, c0=0, nc=1, out=out, mirror=False)
    t1 = time.perf_counter() - t0
    nc = int(max(1, min(NCH, target_s / max(t1, 1e-3), max_out / (16.0 * NANT * NANT))))
    out = np.zeros((nc, 2, NANT, NANT), dtype=np.int64)
    t0 = time.perf_counter()
    oracle.correlate(planes, c0=0, nc=nc, out=out, mirror=False)
    dt = time.perf_counter() - t0
    reps = 1
    if dt < target_s / 4:                       # small arrays: repeat for a stable sample
        reps = int(min(200, max(1, target_s / 2 / max(dt, 1e-4))))
        scratch = np.zeros_like(out)
        t0 = time.perf_counter()
        for _ in range(reps):
            oracle.correlate(planes, c0=0, nc=nc, out=scratch, mirror=False)
        dt = (time.perf_counter() - t0) / reps
    frac = nc / NCH
    gbps = wire_gbps(HEAPS_PER_SUB * NANT * frac, dt)
    desc = (f"OpenMP int64 correlator on {nc}/{NCH} channels of one K={KSUB} sub-integration "
            f"({NANT} elements, lower triangle), {dt:.3f} s per pass over {reps} pass(es); "
            f"Gb/s scaled by channel fraction")
    return gbps, cores, desc, dt, out


def run_reference(args):
    """CPU arm: the oracle restatement of the reference path on the host cores."""
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    src = sources()
    sky = oracle.sky_table(NANT, NCH, SIDE, src) if src else None
    pk = oracle.gen_packets(NANT, NCH, TPKT, HEAPS_PER_SUB, sky=sky, sigma=SIGMA, seed=SEED,
                            mode=CFG["noise"])
    planes = oracle.corner_turn(pk, NANT, NCH, TPKT, HEAPS_PER_SUB)
    cores = oracle.max_threads()
    nc = args.ref_channels
    out = np.zeros((nc, 2, NANT, NANT), dtype=np.int64)
    for _ in range(args.warmup if args.warmup < 2 else 1):
        oracle.correlate(planes, c0=0, nc=nc, out=out, mirror=False)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.correlate(planes, c0=0, nc=nc, out=out, mirror=False)
        ts.append(time.perf_counter() - t0)
    tot = sum(ts)
    frac = nc / NCH
    value = wire_gbps(HEAPS_PER_SUB * NANT * frac * args.steps, tot)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gb/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8->int64", "data": "synthetic (seeded packet source)",
        "config": {"workload": CFG["text"], "nant": NANT, "nch": NCH, "ksub": KSUB,
                   "sample": f"{nc} of {NCH} channels per step"},
        "tops": tri_ops(KSUB) * frac * args.steps / tot / 1e12,
        "cpu_baseline": {"value": value, "unit": "Gb/s", "cores": cores, "kind": "port",
                         "sample": f"oracle OpenMP int64 correlator, {nc}/{NCH} channels of one "
                                   f"K={KSUB} sub-integration per step, Gb/s scaled by the "
                                   f"channel fraction"},
        "e2e": {"value": value, "unit": "Gb/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_sweep(args):
    """Per-launch time of k_xcorr_tri against K (samples per launch) and epilogue
    mode on device-resident random planes: separates per-tile overhead from the
    steady-state tensor rate.  One JSON line per point."""
    import torch
    import mixer
    dev = torch.device("cuda:0")
    # library reference: cuBLASLt int8 GEMM through torch._int_mm, 8192^3
    a = torch.randint(-128, 128, (8192, 8192), dtype=torch.int8, device=dev)
    bt = torch.randint(-128, 128, (8192, 8192), dtype=torch.int8, device=dev)
    for _ in range(3):
        torch._int_mm(a, bt.t())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(10):
        torch._int_mm(a, bt.t())
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 10
    print(json.dumps({"library": "torch._int_mm (cuBLASLt int8) 8192^3", "ms": ms,
                      "tops": 2.0 * 8192 ** 3 / ms / 1e9}), flush=True)
    del a, bt
    shapes = [(1024, 64), (4096, 8)] if args.sweep_quick else [(1024, 64), (4096, 8), (256, 128)]
    ks = [1024, 8192, 32768] if args.sweep_quick else [1024, 2048, 4096, 8192, 16384, 32768]
    for (N, C) in shapes:
        n = mixer.vis_elems(N, C)
        v64 = torch.zeros(n, dtype=torch.int64, device=dev)
        v32 = torch.zeros(n, dtype=torch.int32, device=dev)
        for K in ks:
            planes = torch.randint(-128, 128, (2 * C * N * K,), dtype=torch.int8, device=dev)
            for mode, vis in [(mixer.VIS_STORE_I32, v32), (mixer.VIS_ACC_I64, v64)]:
                for _ in range(2):
                    mixer.xcorr_tri(planes, N, C, K, 0, K, mode, vis)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                for _ in range(5):
                    mixer.xcorr_tri(planes, N, C, K, 0, K, mode, vis)
                e1.record()
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1) / 5
                nb = (N + 127) // 128
                tiles = C * nb * (nb + 1) // 2
                print(json.dumps({"N": N, "C": C, "K": K, "mode": mode, "ms": ms,
                                  "tri_tops": 8.0 * N * (N + 1) / 2 * K * C / ms / 1e9,
                                  "tile_tops": 8.0 * tiles * 128 * 128 * K / ms / 1e9}), flush=True)
            del planes
    return 0


def batched_arrays(seed=SEED + 2, small=False):
    """48 independent arrays: N from {64, 96, ..., 1024}, C from {16, 32, ..., 512},
    K from {256, 512, ..., 4096}, each with one point source plus sigma 12 noise.
    small=True draws N from {64..256}, C from {16..64}: arrays too small to fill
    the GPU in a launch of their own."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for q in range(48):
        n = int(rng.choice(np.arange(64, (257 if small else 1025), 32)))
        c = int(rng.choice(np.arange(16, (65 if small else 513), 16)))
        k = int(rng.choice(np.arange(256, 4097, 256)))
        l, m = rng.uniform(-0.4, 0.4, size=2)
        out.append((n, c, k, float(l), float(m)))
    return out


def vis_checksum(torch, v):
    w = torch.arange(v.numel(), dtype=torch.int64, device=v.device) * 2654435761 + 12345
    return int((v.view(torch.int64) * w).sum().item())


def run_batched(args):
    """Config 'batched': uneven arrays, one persistent launch, autotuned, graph-replayed,
    against one launch per array; per-array results compared by checksum."""
    import torch
    import mixer
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    arrays = batched_arrays(small=args.small_arrays)
    probs, total_ops, in_bytes = [], 0.0, 0
    for idx, (n, c, k, l, m) in enumerate(arrays):
        tp = 16
        stride = 64 + 2 * c * tp
        nh = k // tp
        sky = torch.from_numpy(mixer.sky_table(n, c, 32, [(l, m, 4.0, 0.0)])).to(dev)
        pk = torch.empty(nh * n * stride, dtype=torch.uint8, device=dev)
        mixer.gen_packets(pk, stride, 64, n, c, tp, nh, 0, 0, 4096 + idx, sky, 12.0, SEED + idx, 0)
        planes = torch.empty(2 * c * n * k, dtype=torch.int8, device=dev)
        mixer.corner_turn(pk, stride, 64, n, c, tp, nh, 0, planes, k, 0)
        del pk, sky
        vis = torch.zeros(mixer.vis_elems(n, c), dtype=torch.int64, device=dev)
        probs.append({"planes": planes, "nant": n, "nch": c, "kt": k, "kbeg": 0, "klen": k,
                      "mode": mixer.VIS_ACC_I64, "vis": vis})
        total_ops += 8.0 * n * (n + 1) / 2 * k * c
        in_bytes += 2 * n * k * c
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    reps = max(3, min(args.steps, 20))

    def timed(fn):
        with torch.cuda.stream(stream):
            fn()
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                fn()
            e1.record(stream)
            stream.synchronize()
        return e0.elapsed_time(e1) / reps

    def plain():
        for p in probs:
            mixer.xcorr_tri(p["planes"], p["nant"], p["nch"], p["kt"], 0, p["kt"],
                            mixer.VIS_ACC_I64, p["vis"], stream=stream)

    def zero():
        with torch.cuda.stream(stream):     # same stream as the launches
            for p in probs:
                p["vis"].zero_()
        stream.synchronize()

    zero()
    with torch.cuda.stream(stream):
        plain()
    stream.synchronize()
    with torch.cuda.stream(stream):
        sums_plain = [vis_checksum(torch, p["vis"]) for p in probs]
    b = mixer.Batch(probs)
    t_untuned = timed(lambda: b.run(stream))
    t0 = time.perf_counter()
    tuned_ms = b.autotune(reps=3, stream=stream)
    tune_s = time.perf_counter() - t0
    b.capture_graph(stream)
    # plain launches and the tuned graph alternate, so the clock drift under the
    # power cap does not favour either form; medians over the rounds
    rounds = []
    for _ in range(5):
        rounds.append((timed(plain), timed(lambda: b.run(stream)), timed(lambda: b.replay(stream))))
    t_plain = statistics.median(r[0] for r in rounds)
    t_tuned = statistics.median(r[1] for r in rounds)
    t_graph = statistics.median(r[2] for r in rounds)
    zero()
    with torch.cuda.stream(stream):
        b.replay(stream)
    stream.synchronize()
    with torch.cuda.stream(stream):
        sums_batch = [vis_checksum(torch, p["vis"]) for p in probs]
    info = b.info()
    exact = sums_plain == sums_batch and info["kernel_err"] == 0
    line = {
        "metric": "batched uneven arrays: int8 cGEMM TOPS (triangle basis), batched vs plain",
        "config": {"workload": ("48 small arrays, N in {64..256 step 32}, C in {16..64 step 16}"
                                if args.small_arrays else
                                "48 arrays, N in {64..1024 step 32}, C in {16..512 step 16}")
                   + ", K in {256..4096 step 256}, 1 source + sigma 12 noise each (seeded)",
                   "total_ops": total_ops, "plane_bytes": in_bytes},
        "plain_ms": t_plain, "plain_tops": total_ops / t_plain / 1e9,
        "batched_untuned_ms": t_untuned, "batched_tuned_ms": t_tuned, "graph_ms": t_graph,
        "graph_tops": total_ops / t_graph / 1e9, "batched_over_plain": t_plain / t_graph,
        "autotune_s": tune_s, "autotune_best_ms": tuned_ms,
        "plan": {"nwork": info["nwork"], "order": ["lpt", "channel"][info["order"]],
                 "split_per_class": {str(c): info["split"][c] for c in range(1, 9)}},
        "bit_exact_vs_plain": exact, "reps": reps, "rounds": len(rounds),
        "per_round_plain_over_graph": [round(r[0] / r[2], 3) for r in rounds],
    }
    print(json.dumps(line))
    b.close()
    return 0 if exact else 1


# Serving workload: (nant, nch, tpkt, ksub, nsub_dump, side) of the two stream types.
SERVE_TYPES = {"256x128": (256, 128, 32, 256, 64, 16), "1024x64": (1024, 64, 64, 256, 64, 32)}


def run_serve(args):
    """Config 'serve': 8 concurrent streams (4 x 256 elements x 128 ch, 4 x 1024 x 64 ch)
    of wire-format heaps from the seeded sky source, paced to an aggregate rate with
    Poisson-jittered start / stop, admitted by a device-memory budget; dumps every 64
    sub-integrations.  Reports sustained Gb/s and p50 / p99 dump latency; then an
    unpaced run with all streams open gives the sustainable ceiling."""
    import threading
    import numpy as np
    import torch
    import mixer
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(SEED + 3)
    kinds = ["256x128"] * 4 + ["1024x64"] * 4
    pools = []
    for i, kind in enumerate(kinds):
        nant, nch, tpkt, ksub, nsub, side = SERVE_TYPES[kind]
        hps = ksub // tpkt
        stride = 64 + 2 * nch * tpkt
        sky = torch.from_numpy(mixer.sky_table(
            nant, nch, side, [(0.10, -0.05, 6.0, 0.0), (0.2, 0.0, 0.0, 1.5)])).to(dev)
        pk = torch.empty(nsub * hps * nant * stride, dtype=torch.uint8, device=dev)
        mixer.gen_packets(pk, stride, 64, nant, nch, tpkt, nsub * hps, 0, 0, 4096 + i, sky, 16.0,
                          SEED + 100 + i, 0)
        pools.append(pk)
    torch.cuda.synchronize()

    def one_run(run_s, gbps, budget, jitter):
        srv = mixer.Server(budget_bytes=budget, max_streams=8, ring_subs=16, batch_subs=8)
        per_stream = gbps / 8 * 1e9 / 8 if gbps > 0 else 0.0          # bytes / s
        if jitter:
            starts = np.cumsum(rng.exponential(run_s * 0.04, size=8))
            stops = np.minimum(starts + rng.uniform(0.5, 0.9, size=8) * run_s, run_s)
        else:
            starts, stops = np.zeros(8), np.full(8, run_s)
        t0 = time.perf_counter()
        ids = [None] * 8
        waits = [0.0] * 8
        refusals = [0] * 8
        submitted = [0] * 8
        active = [0.0] * 8
        span = [(0.0, 0.0)] * 8                  # (first, last) accepted submit, s from t0
        stamps = [[] for _ in range(8)]          # accepted submit times, s from t0
        done = threading.Event()

        def feeder(i):
            kind = kinds[i]
            nant, nch, tpkt, ksub, nsub, side = SERVE_TYPES[kind]
            hps = ksub // tpkt
            stride = 64 + 2 * nch * tpkt
            sub_bytes = hps * nant * stride
            d = mixer.make_desc(nant=nant, nch=nch, tpkt=tpkt, ksub=ksub, nsub_dump=nsub, side_x=side,
                                grid=0, pkt_stride=stride, hdr_bytes=64, max_heaps=1)
            while time.perf_counter() - t0 < starts[i]:
                time.sleep(0.001)
            tw = time.perf_counter()
            while ids[i] is None and time.perf_counter() - t0 < stops[i]:
                ids[i] = srv.try_open(d)
                if ids[i] is None:
                    refusals[i] += 1
                    time.sleep(0.002)
            waits[i] = time.perf_counter() - tw
            if ids[i] is None:
                return
            interval = sub_bytes / per_stream if per_stream > 0 else 0.0
            nxt = time.perf_counter()
            ta = nxt
            j = 0
            own = torch.cuda.Stream()
            while time.perf_counter() - t0 < stops[i]:
                if j % nsub == 0:                      # new lap over the pool: re-stamp seqs
                    srv.sync_copies()                  # the previous lap has been copied
                    mixer.restamp_seq(pools[i], nsub * hps * nant, stride, j * hps * nant,
                                      stream=own)
                    own.synchronize()
                if interval > 0:
                    while time.perf_counter() < nxt:
                        time.sleep(min(0.0005, max(0.0, nxt - time.perf_counter())))
                src = pools[i][(j % nsub) * sub_bytes:]
                while not srv.submit(ids[i], src, hps, seq0=0):
                    if time.perf_counter() - t0 >= stops[i]:
                        break
                    time.sleep(0.0002)
                else:
                    submitted[i] += sub_bytes
                    stamps[i].append(time.perf_counter() - t0)
                    j += 1
                    nxt += interval
                    continue
                break
            active[i] = time.perf_counter() - ta
            if stamps[i]:
                span[i] = (stamps[i][0], stamps[i][-1])
            # let the last full dump finish, then leave
            time.sleep(0.05)
            srv.close_stream(ids[i])
            ids[i] = None

        def poller():
            while not done.is_set():
                for sid in list(ids):
                    if sid is not None:
                        try:
                            srv.poll(sid)
                        except mixer.MixerError:
                            pass
                time.sleep(0.001)

        th = [threading.Thread(target=feeder, args=(i,)) for i in range(8)]
        pt = threading.Thread(target=poller)
        pt.start()
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall = time.perf_counter() - t0
        done.set()
        pt.join()
        st = srv.stats()
        srv.close()
        period = {k: v[4] * (v[3] // v[2]) * v[0] * (64 + 2 * v[1] * v[2]) / per_stream
                  for k, v in SERVE_TYPES.items()} if per_stream > 0 else None
        # aggregate over the window in which every stream was submitting
        w0 = max(a for a, _ in span)
        w1 = min(b for _, b in span)
        all_bytes = 0
        for i in range(8):
            sub_b = submitted[i] / max(1, len(stamps[i]))
            all_bytes += sub_b * sum(1 for t in stamps[i] if w0 <= t < w1)
        all_active = ({"window_s": round(w1 - w0, 2), "gbps": 8 * all_bytes / (w1 - w0) / 1e9}
                      if w1 - w0 > 0.5 else None)
        return {"wall_s": wall, "offered_gbps": gbps, "submitted_gbps": 8 * sum(submitted) / wall / 1e9,
                "aggregate_while_all_streams_active": all_active,
                "processed_gbps": 8 * st["bytes_processed"] / wall / 1e9,
                "dumps": st["dumps"], "p50_dump_latency_ms": 1e3 * st["p50_latency_s"],
                "p99_dump_latency_ms": 1e3 * st["p99_latency_s"],
                "max_dump_latency_ms": 1e3 * st["max_latency_s"],
                "integration_period_ms": ({k: 1e3 * v for k, v in period.items()} if period else None),
                "per_stream_gbps": [round(8 * b / a / 1e9, 1) if a > 0 else 0.0
                                    for b, a in zip(submitted, active)],
                "per_stream_target_gbps": gbps / 8 if gbps > 0 else None,
                "admitted": st["admitted"], "refused_attempts": st["refused"],
                "streams_refused_at_least_once": int(sum(r > 0 for r in refusals)),
                "open_latency_s": [round(w, 3) for w in waits], "launches": st["launches"],
                "work_items": st["work_items"], "seq_errors": st["seq_errors"],
                "kernel_err": st["kernel_err"]}

    paced = one_run(args.serve_seconds, args.serve_gbps, int(args.serve_budget_full_gb * (1 << 30)),
                    True)
    tight = one_run(args.serve_seconds, args.serve_gbps, int(args.serve_budget_gb * (1 << 30)), True)
    ceiling = one_run(min(args.serve_seconds, 6.0), 0.0, 64 << 30, False)
    line = {"metric": "serving: sustained input Gb/s and p50/p99 dump latency",
            "config": {"workload": "8 streams: 4 x (256 elements x 128 ch, tpkt 32), "
                       "4 x (1024 elements x 64 ch, tpkt 64), K 256, 64 sub-integrations per dump, "
                       "8256-byte heaps from the seeded sky source (device pools)",
                       "paced_gbps": args.serve_gbps, "budget_gb": args.serve_budget_full_gb,
                       "tight_budget_gb": args.serve_budget_gb},
            "paced": paced, "paced_tight_budget": tight, "unpaced_ceiling": ceiling}
    print(json.dumps(line))
    ok = all(r["kernel_err"] == 0 and r["seq_errors"] == 0 for r in (paced, tight, ceiling))
    return 0 if ok else 1


def run_kernels(args):
    """The path's HBM-bound kernels besides the corner-turn, on the selected plain
    workload's cube: int32 -> int64 integration (k_vis_flush), the FP32 dump
    (k_vis_unpack), exact int64 gridding (k_grid_tiles) and the shared-memory FFT
    (k_image_fft).  Each launch is timed alone with CUDA events after an L2 flush
    (a 256 MiB write), on device-resident inputs; achieved GB/s counts the
    algorithmic bytes and is compared with the measured HBM copy bandwidth.
    One JSON line per kernel."""
    import torch
    import mixer
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    N, C, side, Gs = CFG["nant"], NCH, CFG["side"], CFG["grid"]
    nt = mixer.vis_tiles(N)
    n = mixer.vis_elems(N, C)
    T = N * (N + 1) // 2
    hbm = measured_peaks().get("hbm_gbs")
    gen = torch.Generator(device=dev)
    gen.manual_seed(SEED)
    v64 = torch.randint(-2 ** 40, 2 ** 40, (n,), dtype=torch.int64, device=dev, generator=gen)
    v32 = torch.randint(-2 ** 30, 2 ** 30, (n,), dtype=torch.int32, device=dev, generator=gen)
    cube = torch.empty(C * 2 * N * N, dtype=torch.float32, device=dev)
    grid = torch.empty(C * Gs * Gs * 2, dtype=torch.int64, device=dev)
    img = torch.empty(C * Gs * Gs, dtype=torch.float32, device=dev)
    vmax = torch.empty(C, dtype=torch.float32, device=dev)
    vmin = torch.empty(C, dtype=torch.float32, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    cases = [
        ("k_vis_flush", lambda: mixer.vis_flush(v32, v64, n), 24 * n,
         "int32 read + int64 read + int64 write + int32 zeroed, per tile-packed element"),
        ("k_vis_unpack", lambda: mixer.vis_dump_f32(v64, N, C, cube), 8 * n + 8 * C * N * N,
         "tile-packed int64 cube read + FP32 [C][2][N][N] written"),
        ("k_grid_tiles", lambda: mixer.grid(v64, N, C, side, Gs, grid), 16 * T * C + 16 * C * Gs * Gs,
         "lower-triangle int64 entries read + int64 [C][G][G][2] grid written"),
        ("k_image_fft", lambda: mixer.image_fft(grid, C, Gs, img, vmax, vmin),
         16 * C * Gs * Gs + 4 * C * Gs * Gs,
         "int64 grid read + FP32 image written"),
    ]
    for name, fn, nbytes, what in cases:
        for _ in range(max(3, args.warmup)):
            fn()
        torch.cuda.synchronize()
        times = []
        for _ in range(max(3, min(args.steps, 50))):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = statistics.median(times)
        gbs = nbytes / ms / 1e6
        print(json.dumps({"kernel": name, "workload": CFG["text"], "nant": N, "nch": C,
                          "grid": Gs, "ms": ms, "algorithmic_bytes": nbytes, "bytes": what,
                          "gbs": gbs, "hbm_frac": gbs / hbm if hbm else None,
                          "peak": f"of measured {hbm} GB/s" if hbm else None,
                          "launches": len(times)}), flush=True)
    return 0


def mma_probe(torch, mixer, dev, local=0, runs=(("burst", 20000, 5), ("sustained", 200000, 20))):
    """Dense int8 tensor-core rate of this GPU with the GEMM's own MMA stream
    (mixer_mma_peak: resident shared-memory operands, no loads), with the SM
    clock sampled: the measured int8 ceiling beside the 2 x bf16 figure."""
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mixer.mma_peak(1000, 0, err)
    torch.cuda.synchronize()
    out = []
    for label, iters, reps in runs:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            e0.record()
            for _ in range(reps):
                mixer.mma_peak(iters, 0, err)
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        ops = float(sms) * iters * reps * mixer.MMA_PEAK_OPS_PER_ITER
        c = clk.summary()
        tops = ops / ms / 1e9
        out.append({"probe": "int8 MMA peak (tcgen05 kind::i8, M128 N256 K32, smem operands)",
                    "run": label, "ms": ms, "tops": tops, "clocks": c,
                    "ops_per_sm_per_clock": (tops * 1e12 / (sms * c["sm_mhz"] * 1e6)
                                             if c.get("sm_mhz") else None),
                    "kernel_err": int(err.item())})
    return out


def run_mma_peak(args):
    import torch
    import mixer
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    for line in mma_probe(torch, mixer, dev):
        print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import mixer
    rank, world, local, pg = dist_setup(args.gpus)
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if mixer.lib().mixer_device_ok() != mixer.OK:
        raise RuntimeError("not an sm_100 device")
    S = args.batch
    nheaps = S * HEAPS_PER_SUB
    npk = nheaps * NANT
    kt = nheaps * TPKT
    stream = torch.cuda.current_stream()

    # ---- inputs (device resident), state and planes ------------------------
    pk = make_packets(mixer, torch, dev, nheaps)
    planes = torch.empty(2 * NCH * NANT * kt, dtype=torch.int8, device=dev)
    vis = torch.zeros(mixer.vis_elems(NANT, NCH), dtype=torch.int64, device=dev)
    seq_err = torch.zeros(1, dtype=torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        mixer.corner_turn(pk, STRIDE, HDR, NANT, NCH, TPKT, nheaps, 0, planes, kt, 0, seq_err, err)
        if ev is not None:
            ev[1].record(stream)
        mixer.xcorr_tri(planes, NANT, NCH, kt, 0, kt, mixer.VIS_ACC_I64, vis, err)
        if ev is not None:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(pg, dev)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        for s in range(args.steps):
            step(evs[s])
        stop.record(stream)
        torch.cuda.synchronize()
    barrier(pg, dev)
    ms_total = start.elapsed_time(stop)
    ct_ms = [e[0].elapsed_time(e[1]) for e in evs]
    gemm_ms = [e[1].elapsed_time(e[2]) for e in evs]
    if int(err.item()) != 0 or int(seq_err.item()) != 0:
        raise RuntimeError(f"kernel error word {int(err.item())}, seq errors {int(seq_err.item())}")
    t_max = max_over_ranks(pg, ms_total, dev) / 1e3
    packets_all = sum_over_ranks(pg, float(npk * args.steps), dev)
    value = wire_gbps(packets_all, t_max)
    tops = tri_ops(kt) * args.steps * world / t_max / 1e12

    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_case": True, "nch": NCH, "subints": S,
                              "ms_per_step": ms_total / args.steps,
                              "xcorr_ms": statistics.mean(gemm_ms),
                              "corner_turn_ms": statistics.mean(ct_ms)}))
        return 0

    # ---- plain form: one launch pair per sub-integration ------------------------
    plain_steps = max(1, min(args.steps, 5))

    def plain_step():
        for s in range(S):
            h0 = s * HEAPS_PER_SUB
            mixer.corner_turn(pk[h0 * NANT * STRIDE:], STRIDE, HDR, NANT, NCH, TPKT, HEAPS_PER_SUB,
                              h0 * NANT, planes, KSUB, 0, seq_err, err)
            mixer.xcorr_tri(planes, NANT, NCH, KSUB, 0, KSUB, mixer.VIS_ACC_I64, vis, err)

    plain_step()
    torch.cuda.synchronize()
    barrier(pg, dev)
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(plain_steps):
        plain_step()
    p1.record(stream)
    torch.cuda.synchronize()
    plain_t = max_over_ranks(pg, p0.elapsed_time(p1), dev) / 1e3
    plain_value = wire_gbps(sum_over_ranks(pg, float(npk * plain_steps), dev), plain_t)

    # ---- end to end through the context API from pinned host packets ------------
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    # the end-to-end step holds at most 8 sub-integrations of pinned host packets (4.3 GB at
    # the plain array): PCIe-bound either way, and N ranks pin N copies
    e2e_heaps = min(nheaps, 8 * HEAPS_PER_SUB)
    e2e_npk = e2e_heaps * NANT
    host = torch.empty(e2e_npk * STRIDE, dtype=torch.uint8, pin_memory=True)
    host.copy_(pk[: e2e_npk * STRIDE])
    del planes
    torch.cuda.empty_cache()
    e2e = None
    with mixer.ArrayContext(nant=NANT, nch=NCH, tpkt=TPKT, ksub=KSUB, nsub_dump=1, side_x=SIDE,
                            grid=G, pkt_stride=STRIDE, hdr_bytes=HDR,
                            max_heaps=args.e2e_chunk * HEAPS_PER_SUB) as ctx:
        img = torch.empty(NCH * G * G, dtype=torch.float32, pin_memory=True)
        vmax = torch.empty(NCH, dtype=torch.float32, pin_memory=True)
        vmin = torch.empty(NCH, dtype=torch.float32, pin_memory=True)

        def e2e_step():
            ctx.correlate(host, e2e_heaps, seq0=0, on_device=False)
            ctx.image(img, vmax, vmin, on_device=False)

        e2e_step()
        torch.cuda.synchronize()
        barrier(pg, dev)
        q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        q0.record(stream)
        for _ in range(e2e_steps):
            e2e_step()
        q1.record(stream)
        torch.cuda.synchronize()
        e2e_t = max_over_ranks(pg, q0.elapsed_time(q1), dev) / 1e3
        st = ctx.stats()
        if st["kernel_err"] or st["seq_errors"]:
            raise RuntimeError(f"e2e counters {st}")
        e2e = {"value": wire_gbps(sum_over_ranks(pg, float(e2e_npk * e2e_steps), dev), e2e_t),
               "unit": "Gb/s", "h2d_bytes_per_step": int(e2e_npk * STRIDE),
               "sub_integrations_per_step": e2e_heaps // HEAPS_PER_SUB,
               "d2h_bytes_per_step": int(NCH * G * G * 4 + 2 * NCH * 4),
               "ms_per_step": 1e3 * e2e_t / e2e_steps, "steps": e2e_steps,
               "path": "mixer_correlate(host pinned packets) + mixer_image(host) per step"}

    # ---- roofline of the dominant kernel (the GEMM) --------------------------------
    peaks = measured_peaks()
    sustained = ms_total > 500.0          # a long timed region runs under the power cap
    bf16 = peaks.get("bf16_tflops_sustained" if sustained else "bf16_tflops")
    kind = "sustained" if sustained else "burst"
    if bf16:
        peak = 2.0 * bf16
        peak_src = (f"of measured: 2 x cuBLAS bf16 {kind} ({bf16} TF/s, MEASURED_PEAKS.json); "
                    "B200 dense int8 rate = 2 x dense bf16 rate")
    else:
        peak = 2.0 * (1400.0 if sustained else 1590.0)
        peak_src = f"of fallback: 2 x bf16 {kind}"
    gemm_avg = statistics.mean(gemm_ms) / 1e3
    achieved = tri_ops(kt) / gemm_avg / 1e12
    ct_avg = statistics.mean(ct_ms) / 1e3
    ct_bytes = npk * STRIDE + 2 * NCH * NANT * kt
    hbm = peaks.get("hbm_gbs", 6650.0)

    line = {
        "metric": METRIC, "value": value, "unit": "Gb/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8->int32(TMEM)->int64",
        "data": "synthetic (seeded packet source, wire format)",
        "config": {"workload": CFG["text"],
                   "nant": NANT, "nch": NCH, "tpkt": TPKT, "ksub": KSUB,
                   "subints_per_step": S, "packets_per_step": npk,
                   "bytes_per_step": npk * STRIDE,
                   "l2": "inputs larger than L2 (%.1f GB per step)" % (npk * STRIDE / 1e9),
                   "parallelism": f"replicas x{world}"},
        "tops": tops,
        "tops_full_square_basis": tops * 2 * NANT / (NANT + 1),
        "plain": {"value": plain_value, "unit": "Gb/s", "steps": plain_steps,
                  "form": "one corner-turn + GEMM launch per K=1024 sub-integration",
                  "stream_over_plain": value / plain_value},
        "kernels": {"corner_turn_ms": 1e3 * ct_avg, "corner_turn_gbs": ct_bytes / ct_avg / 1e9,
                    "corner_turn_hbm_frac": ct_bytes / ct_avg / 1e9 / hbm,
                    "xcorr_ms": 1e3 * gemm_avg},
        "roofline": {"kernel": "k_xcorr_tri", "bound": "tensor", "achieved": achieved,
                     "peak": peak, "unit": "TOPS", "frac": achieved / peak,
                     "peak_source": peak_src,
                     "traffic": XCORR_TRAFFIC_RATIO * (2 * NCH * NANT * kt + 2 * 8 * mixer.vis_elems(NANT, NCH)),
                     "traffic_note": "bytes per launch: algorithmic x 1.106, the DRAM/algorithmic "
                                     "ratio of an ncu capture at the same K (1024 el., 32 ch)",
                     "ops_per_launch": tri_ops(kt)},
        "clocks": clk.summary(),
        "gpu_launches": 2 * args.steps,
        "e2e": e2e,
    }
    # ---- the GEMM against the measured int8 tensor-core rate --------------------
    # The probe runs the GEMM's MMA stream with no memory traffic: per clock it is
    # the rate the tensor cores can reach; under the power cap it also holds a
    # higher clock than the GEMM, whose operand and cube traffic draw power too.
    probe = {r["run"]: r for r in mma_probe(torch, mixer, dev, local)}
    gemm_tile_tops = achieved * (mixer.vis_tiles(NANT) * 128 * 128) / (NANT * (NANT + 1) / 2)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    gmhz = line["clocks"].get("sm_mhz")
    sus = probe["sustained"]
    line["int8_mma_probe"] = {
        "burst_tops": probe["burst"]["tops"], "burst_mhz": probe["burst"]["clocks"].get("sm_mhz"),
        "sustained_tops": sus["tops"], "sustained_mhz": sus["clocks"].get("sm_mhz"),
        "probe_ops_per_sm_per_clock": sus["ops_per_sm_per_clock"],
        "gemm_tile_basis_tops": gemm_tile_tops,
        "gemm_ops_per_sm_per_clock": gemm_tile_tops * 1e12 / (sms * gmhz * 1e6) if gmhz else None,
        "gemm_per_clock_frac": (gemm_tile_tops * 1e12 / (sms * gmhz * 1e6) / sus["ops_per_sm_per_clock"]
                                if gmhz and sus["ops_per_sm_per_clock"] else None),
        "gemm_frac_of_sustained_probe": gemm_tile_tops / sus["tops"],
        "what": "tile basis (every computed 128 x 128 tile); the probe is mixer_mma_peak"}
    # ---- imaging of the integrated cube (grid + FFT), device resident ------------
    with mixer.ArrayContext(nant=NANT, nch=NCH, tpkt=TPKT, ksub=KSUB, nsub_dump=1, side_x=SIDE,
                            grid=G, pkt_stride=STRIDE, hdr_bytes=HDR, max_heaps=HEAPS_PER_SUB) as ic:
        ic.correlate(pk, HEAPS_PER_SUB, seq0=0)
        dimg = torch.empty(NCH * G * G, dtype=torch.float32, device=dev)
        ic.image(dimg)
        torch.cuda.synchronize()
        i0, i1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        i0.record(stream)
        for _ in range(10):
            ic.image(dimg)
        i1.record(stream)
        torch.cuda.synchronize()
        line["image_ms"] = i0.elapsed_time(i1) / 10
        line["image_grid"] = G
        if rank == 0:
            # FP32 outputs against FP64 computed here from the exact int64 state:
            # the dump cube (one rounding of int64) and the image (FP64 FFT of the
            # exact int64 grid), on the first channels
            import numpy as np
            ne = min(4, NCH)
            ex = torch.empty(ne * 2 * NANT * NANT, dtype=torch.int64, device=dev)
            f32 = torch.empty(ne * 2 * NANT * NANT, dtype=torch.float32, device=dev)
            mixer.vis_unpack_i64(ic.state_ptr(), NANT, ne, ex)
            mixer.vis_dump_f32(ic.state_ptr(), NANT, ne, f32)
            gi = torch.empty(ne * G * G * 2, dtype=torch.int64, device=dev)
            mixer.grid(ic.state_ptr(), NANT, ne, SIDE, G, gi)
            im = torch.empty(ne * G * G, dtype=torch.float32, device=dev)
            mixer.image_fft(gi, ne, G, im)
            torch.cuda.synchronize()
            exn = ex.cpu().numpy().astype(np.float64)
            fn = f32.cpu().numpy().astype(np.float64)
            nz = exn != 0
            cube_rel = float(np.max(np.abs(fn[nz] - exn[nz]) / np.abs(exn[nz]))) if nz.any() else 0.0
            g4 = gi.cpu().numpy().reshape(ne, G, G, 2)
            z = g4[..., 0].astype(np.float64) + 1j * g4[..., 1].astype(np.float64)
            ref = np.fft.fftshift(np.fft.fft2(z, axes=(-2, -1)).real, axes=(-2, -1))
            got = im.cpu().numpy().reshape(ne, G, G).astype(np.float64)
            peak = np.maximum(np.max(np.abs(ref), axis=(1, 2)), 1e-30)
            img_rel = float(np.max(np.max(np.abs(got - ref), axis=(1, 2)) / peak))
            line["fp32_error_vs_fp64"] = {
                "channels": ne, "cube_max_rel": cube_rel, "cube_bound": 2.0 ** -24,
                "image_max_err_over_peak": img_rel, "image_target": 1e-5}
            del ex, f32, gi, im
        if rank == 0 and not args.no_cpu_baseline:
            # CPU baseline (the oracle's OpenMP correlator on a channel subset of the first
            # sub-integration); its output also checks the GPU's V for that sub-integration
            hp = host[: HEAPS_PER_SUB * NANT * STRIDE].numpy()
            gbps, cores, desc, _, ref = cpu_correlator_sample(hp, HEAPS_PER_SUB,
                                                              target_s=args.cpu_seconds)
            line["cpu_baseline"] = {"value": gbps, "unit": "Gb/s", "cores": cores, "kind": "port",
                                    "sample": desc}
            ncheck = min(4, ref.shape[0])
            got = torch.empty(ncheck * 2 * NANT * NANT, dtype=torch.int64, device=dev)
            mixer.vis_unpack_i64(ic.state_ptr(), NANT, ncheck, got)
            torch.cuda.synchronize()
            import numpy as np
            low = np.tril(np.ones((NANT, NANT), dtype=bool))   # the sample holds b <= a only
            g = got.cpu().numpy().reshape(ncheck, 2, NANT, NANT)
            line["bit_exact_vs_cpu"] = {
                "channels": ncheck, "subints": 1, "entries": "lower triangle incl. diagonal",
                "equal": bool(np.array_equal(g[:, :, low], ref[:ncheck][:, :, low]))}
        # dump latency: from enqueueing the dump's last heaps (its last sub-integration,
        # device-resident packets) to the FP32 cube [C][2][N][N] complete in pinned host
        # memory; the step's earlier sub-integrations are correlated before the clock starts
        cube = torch.empty(NCH * 2 * NANT * NANT, dtype=torch.float32, pin_memory=True)
        cycles = 20 if cube.numel() * 4 < 1e9 else (5 if cube.numel() * 4 < 4e9 else 2)
        h_last = nheaps - HEAPS_PER_SUB
        lat = []
        for _ in range(cycles + 1):
            if h_last > 0:
                ic.correlate(pk, h_last, seq0=0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ic.correlate(pk[h_last * NANT * STRIDE:], HEAPS_PER_SUB, seq0=h_last * NANT)
            ic.dump(cube, on_device=False)
            torch.cuda.synchronize()
            lat.append(1e3 * (time.perf_counter() - t0))
        lat = sorted(lat[1:])
        line["dump_latency_ms"] = {
            "p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * (len(lat) - 1) + 0.5))],
            "cycles": cycles, "dump_bytes": cube.numel() * 4,
            "what": "enqueue of the dump's last sub-integration (mixer_correlate of its heaps) "
                    "to the FP32 cube in pinned host memory (mixer_dump)"}
        del cube
    if rank == 0:
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=0,
                    help="sub-integrations per step (0: the workload's default)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-chunk", type=int, default=2, help="sub-integrations per H2D chunk")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-channels", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nch", type=int, default=0,
                    help="channels per packet, tpkt = 4096/nch (0: the workload's)")
    ap.add_argument("--serve-seconds", type=float, default=30.0)
    ap.add_argument("--serve-gbps", type=float, default=380.0)
    ap.add_argument("--serve-budget-gb", type=float, default=6.0,
                    help="device budget of the admission run (streams wait for memory)")
    ap.add_argument("--serve-budget-full-gb", type=float, default=16.0,
                    help="device budget of the main paced run (every stream fits)")
    ap.add_argument("--config", default="plain",
                    choices=["plain", "small", "large", "batched", "serve"],
                    help="plain: the 1024-element array (headline); small: the reference's "
                         "256-element array; large: 4096 elements; batched: 48 uneven arrays; "
                         "serve: 8 concurrent streams")
    ap.add_argument("--small-arrays", action="store_true",
                    help="batched config with arrays too small to fill the GPU alone")
    ap.add_argument("--sweep-quick", action="store_true", help="fewer sweep points")
    ap.add_argument("--sweep-xcorr", action="store_true",
                    help="time the GEMM kernel over K and epilogue mode (JSON lines)")
    ap.add_argument("--profile", action="store_true",
                    help="device-resident steps only (small case for ncu captures)")
    ap.add_argument("--mma-peak", action="store_true",
                    help="measure the dense int8 tensor-core rate (burst and sustained)")
    ap.add_argument("--kernels", action="store_true",
                    help="time the integration, dump, gridding and FFT kernels (JSON lines)")
    args = ap.parse_args()
    configure(args.nch, args.config if args.config in PLAIN_CONFIGS else "plain")
    if args.batch <= 0:
        args.batch = CFG["batch"]
    if args.warmup < 3 and args.impl == "ours" and not args.profile:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        return run_reference(args)
    if args.sweep_xcorr:
        return run_sweep(args)
    if args.kernels:
        return run_kernels(args)
    if args.mma_peak:
        return run_mma_peak(args)
    if args.config == "batched":
        return run_batched(args)
    if args.config == "serve":
        return run_serve(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
