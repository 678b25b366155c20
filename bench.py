"""X-engine benchmark: input Gb/s and int8 cGEMM TOPS on one B200 (or N replicas).

Workload (the larger plain array): 32 x 32 = 1024 elements, 256 channels, complex
int8, three point sources (amplitudes 4, 2, 1 at seeded random (l, m) with
|l|, |m| < 0.4) plus complex Gaussian noise sigma = 8, K = 1024 samples per
sub-integration, int64 long-term integration, lower-triangle tiles only.
Packets use the wire format (8256-byte heaps, 64-byte header, planar int8
payload; 256 channels x 16 samples per packet).  Inputs are synthetic, made
by the seeded packet source.

One step = `--batch` sub-integrations (default 8, 4.3 GB of packets) through
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
# once + int64 cube read and written), from the ncu capture of the N 1024,
# C 64, K 4096 case: 1.6957 GB measured / 1.7456 GB algorithmic.
XCORR_TRAFFIC_RATIO = 1.6957 / 1.7456


def configure(nch):
    """Channel count of the packets; the payload stays 8192 bytes (2 x nch x tpkt)."""
    global NCH, TPKT, STRIDE, HEAPS_PER_SUB
    if 4096 % nch or (4096 // nch) % 16:
        raise SystemExit("--nch must divide 4096 with 4096/nch a multiple of 16")
    NCH, TPKT = nch, 4096 // nch
    STRIDE = HDR + 2 * NCH * TPKT
    HEAPS_PER_SUB = KSUB // TPKT


def sources(seed=SEED):
    import numpy as np
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
    sky = torch.from_numpy(mixer.sky_table(NANT, NCH, SIDE, sources())).to(dev)
    pk = torch.empty(nheaps * NANT * STRIDE, dtype=torch.uint8, device=dev)
    mixer.gen_packets(pk, STRIDE, HDR, NANT, NCH, TPKT, nheaps, heap0, heap0 * NANT, 4096, sky,
                      SIGMA, SEED, 0)
    return pk


def cpu_correlator_sample(packets_host, nheaps, target_s=12.0, max_threads=0):
    """Time the oracle's OpenMP int64 correlator on a channel subset of one
    sub-integration; returns (gbps_equivalent, cores, sample_description)."""
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
    nc = int(max(1, min(NCH, target_s / max(t1, 1e-3))))
    out = np.zeros((nc, 2, NANT, NANT), dtype=np.int64)
    t0 = time.perf_counter()
    oracle.correlate(planes, c0=0, nc=nc, out=out, mirror=False)
    dt = time.perf_counter() - t0
    frac = nc / NCH
    gbps = wire_gbps(HEAPS_PER_SUB * NANT * frac, dt)
    desc = (f"OpenMP int64 correlator on {nc}/{NCH} channels of one K={KSUB} sub-integration "
            f"({NANT} elements, lower triangle), {dt:.2f} s; Gb/s scaled by channel fraction")
    return gbps, cores, desc, dt


def run_reference(args):
    """CPU arm: the oracle restatement of the reference path on the host cores."""
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    sky = oracle.sky_table(NANT, NCH, SIDE, sources())
    pk = oracle.gen_packets(NANT, NCH, TPKT, HEAPS_PER_SUB, sky=sky, sigma=SIGMA, seed=SEED)
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
        "config": {"workload": "plain array 32x32=1024 elements, 256 ch, K=1024, 3 sources + "
                   "sigma 8 noise", "nant": NANT, "nch": NCH, "ksub": KSUB,
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
    for (N, C) in [(1024, 64), (4096, 8), (256, 128)]:
        n = mixer.vis_elems(N, C)
        v64 = torch.zeros(n, dtype=torch.int64, device=dev)
        v32 = torch.zeros(n, dtype=torch.int32, device=dev)
        for K in [1024, 2048, 4096, 8192, 16384, 32768]:
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
    host = torch.empty(npk * STRIDE, dtype=torch.uint8, pin_memory=True)
    host.copy_(pk)
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
            ctx.correlate(host, nheaps, seq0=0, on_device=False)
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
        e2e = {"value": wire_gbps(sum_over_ranks(pg, float(npk * e2e_steps), dev), e2e_t),
               "unit": "Gb/s", "h2d_bytes_per_step": int(npk * STRIDE),
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
        "config": {"workload": "plain array 32x32=1024 elements, 256 ch, K=1024 per "
                   "sub-integration, 3 sources + sigma 8 noise, int64 integration",
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
                     "traffic_note": "bytes per launch, scaled from the ncu capture of a smaller case",
                     "ops_per_launch": tri_ops(kt)},
        "clocks": clk.summary(),
        "gpu_launches": 2 * args.steps,
        "e2e": e2e,
    }
    if rank == 0 and not args.no_cpu_baseline:
        hp = host[: HEAPS_PER_SUB * NANT * STRIDE].numpy()
        gbps, cores, desc, _ = cpu_correlator_sample(hp, HEAPS_PER_SUB, target_s=args.cpu_seconds)
        line["cpu_baseline"] = {"value": gbps, "unit": "Gb/s", "cores": cores, "kind": "port",
                                "sample": desc}
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
    ap.add_argument("--batch", type=int, default=8, help="sub-integrations per step")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-chunk", type=int, default=2, help="sub-integrations per H2D chunk")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-channels", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nch", type=int, default=256, help="channels per packet (tpkt = 4096/nch)")
    ap.add_argument("--sweep-xcorr", action="store_true",
                    help="time the GEMM kernel over K and epilogue mode (JSON lines)")
    ap.add_argument("--profile", action="store_true",
                    help="device-resident steps only (small case for ncu captures)")
    args = ap.parse_args()
    configure(args.nch)
    if args.warmup < 3 and args.impl == "ours" and not args.profile:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        return run_reference(args)
    if args.sweep_xcorr:
        return run_sweep(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
