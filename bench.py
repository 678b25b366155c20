"""X-engine benchmark: input Gb/s and int8 cGEMM TOPS on one B200 (or N replicas).

Headline workload (the larger plain array): 32 x 32 = 1024 elements, 256
channels, complex int8, three point sources (amplitudes 4, 2, 1 at seeded random
(l, m) with |l|, |m| < 0.4) plus complex Gaussian noise sigma = 8, K = 1024
samples per sub-integration, int64 long-term integration, lower-triangle tiles
only.  Packets use the wire format (8256-byte heaps, 64-byte header, planar
int8 payload; 256 channels x 16 samples per packet).  Inputs are synthetic,
made by the seeded packet source.

One step = `--batch` sub-integrations (default 32, 17.3 GB of packets) through
corner-turn -> tcgen05 triangle GEMM (int32 in TMEM over the whole step) ->
int64 integration.  `value` is device-resident throughput; `e2e` is the same
work through the public context API from pinned host packets (host->device
copies inside the timed region, overlapped with compute) with the live image
read back every step.  `plain` is the per-sub-integration launch form.

With one GPU the default line also carries the other workloads, each measured
in the same run: `small` (the reference's 256-element array), `large` (4096
elements), `batched` (48 uneven arrays in one persistent launch replayed from a
CUDA graph, against one launch per array and sub-integration) and `serve`
(8 concurrent streams paced at 380 Gb/s).  The CPU-baseline leg at the end
times the oracle's correlator and checks, against the oracle, the cubes the
timed launches produced.

`--impl reference` times the CPU restatement of the reference path (OpenMP
int64 correlator over the same packets) on the host cores, and the reference's
own GPU kernels compiled from its sources (when built) on the same GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import socket
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
# A timed region longer than this runs under the power cap: its roofline uses
# the sustained int8 rate, a shorter one the burst rate.
SUSTAINED_REGION_MS = 500.0


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
CFG_NAME = "plain"


def configure(nch=None, name="plain"):
    """Select a plain workload; optionally override the channel count of the
    packets (the payload stays 8192 bytes: tpkt = 4096 / nch)."""
    global CFG, CFG_NAME, NANT, SIDE, NCH, TPKT, KSUB, G, SIGMA, STRIDE, HEAPS_PER_SUB
    CFG, CFG_NAME = PLAIN_CONFIGS[name], name
    NANT, SIDE, KSUB, G, SIGMA = CFG["nant"], CFG["side"], CFG["ksub"], CFG["grid"], CFG["sigma"]
    nch = nch or CFG["nch"]
    if 4096 % nch or (4096 // nch) % 16 or KSUB % (4096 // nch):
        raise SystemExit("--nch must divide 4096 with 4096/nch a multiple of 16 dividing K")
    NCH, TPKT = nch, 4096 // nch
    STRIDE = HDR + 2 * NCH * TPKT
    HEAPS_PER_SUB = KSUB // TPKT


def sources(seed=SEED):
    import numpy as np
    if CFG_NAME == "small":
        return [(0.10, -0.05, 6.0, 0.0), (0.2, 0.0, 0.0, 1.5)]
    if CFG["noise"] == 1:
        return []
    rng = np.random.default_rng(seed)
    lm = rng.uniform(-0.4, 0.4, size=(3, 2))
    return [(float(lm[s, 0]), float(lm[s, 1]), amp, 0.0) for s, amp in enumerate((4.0, 2.0, 1.0))]


def tri_ops(nsamp, nant=None, nch=None):
    n = NANT if nant is None else nant
    c = NCH if nch is None else nch
    return 8.0 * n * (n + 1) / 2 * nsamp * c


def wire_gbps(npackets, seconds, stride=None):
    return 8.0 * (stride or STRIDE) * npackets / seconds / 1e9


def ev_pair(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


# ---------------------------------------------------------------- ranks ----

def dist_setup(n_gpus, backend=None):
    """Rank, world size, local rank and the process group (None for one rank).
    NCCL when CUDA is present, gloo otherwise; a short timeout so ranks that
    wait for one another end with an error."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != n_gpus and rank == 0:
        print(f"warning: --gpus {n_gpus} but WORLD_SIZE {world}; reporting n_gpus = {world}",
              file=sys.stderr)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
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


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def launch_replicas(n, argv):
    """`bench.py --gpus N` started without a rank environment: run this script
    as N ranks on this node (one per GPU, torch.distributed.run on 127.0.0.1)
    and return the launcher's exit status.  Rank 0 prints the line."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", f"--master-port={free_port()}",
           os.path.abspath(__file__)] + list(argv)
    return subprocess.call(cmd)


def run_launcher_check(args):
    """The replica plumbing without a GPU (gloo): every rank reports a step time
    of 10 + rank ms over 100 (rank + 1) packets; rank 0 prints the reductions the
    benchmark line uses (max-over-ranks time, summed work, world size)."""
    import torch
    rank, world, local, pg = dist_setup(args.gpus, backend="gloo")
    dev = torch.device("cpu")
    barrier(pg, dev)
    t = max_over_ranks(pg, 10.0 + rank, dev)
    work = sum_over_ranks(pg, 100.0 * (rank + 1), dev)
    seeds = sum_over_ranks(pg, float(SEED + rank), dev)
    barrier(pg, dev)
    if rank == 0:
        print(json.dumps({"launcher_check": True, "n_gpus": world, "max_ms": t, "packets": work,
                          "seed_sum": seeds}))
    if pg is not None:
        pg.destroy_process_group()
    return 0


# ---------------------------------------------------------------- clocks ----

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
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
                power.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        loaded = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_median": statistics.median(power) if power else None}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return json.load(f)
    except OSError:
        return {}


def hbm_peak():
    """(GB/s, source) for HBM-bound kernels: the measured copy rate, else the fallback."""
    hbm = measured_peaks().get("hbm_gbs")
    return (float(hbm), "of measured (MEASURED_PEAKS.json hbm_gbs)") if hbm else (6650.0, "of fallback")


def make_packets(mixer, torch, dev, nheaps, heap0=0, seed=SEED):
    src = sources()
    sky = torch.from_numpy(mixer.sky_table(NANT, NCH, SIDE, src)).to(dev) if src else None
    pk = torch.empty(nheaps * NANT * STRIDE, dtype=torch.uint8, device=dev)
    mixer.gen_packets(pk, STRIDE, HDR, NANT, NCH, TPKT, nheaps, heap0, heap0 * NANT, 4096, sky,
                      SIGMA, seed, CFG["noise"])
    return pk


def packet_subset(torch, pk, nheaps, chans, elems=None):
    """Host copy of the payload bytes of `chans` (and antennas `elems`, all when
    None) of device packets, as header-less packets [nheaps * n'][2 * nc * tpkt]:
    re bytes of the channels, then im bytes.  For the CPU check only."""
    p3 = pk.view(nheaps, NANT, STRIDE)
    if elems is not None:
        p3 = p3.index_select(1, torch.as_tensor(elems, device=pk.device))
    cols = []
    for plane in (0, 1):
        for c in chans:
            base = HDR + plane * NCH * TPKT + c * TPKT
            cols.extend(range(base, base + TPKT))
    idx = torch.as_tensor(cols, dtype=torch.int64, device=pk.device)
    sub = p3.reshape(-1, STRIDE).index_select(1, idx)
    return sub.cpu().numpy()


def unpack_channels(torch, mixer, vis, nant, chans, elems=None):
    """Exact full-square int64 V [nc][2][n'][n'] of the given channels of a
    tile-packed cube (principal submatrix on `elems` when given), on the host."""
    per = mixer.vis_elems(nant, 1)
    out = []
    full = torch.empty(2 * nant * nant, dtype=torch.int64, device=vis.device)
    for c in chans:
        mixer.vis_unpack_i64(vis[c * per:], nant, 1, full)
        f = full.view(2, nant, nant)
        if elems is not None:
            e = torch.as_tensor(elems, device=vis.device)
            f = f.index_select(1, e).index_select(2, e)
        out.append(f.cpu().numpy())
    import numpy as np
    return np.stack(out)


# ------------------------------------------------------- plain workloads ----

def plain_run(torch, mixer, dev, steps, warmup, pg=None, local=0, seed=SEED, check=None,
              plain_steps=5, keep=False):
    """Device-resident steps of the selected plain workload: per step, one
    corner-turn of S sub-integrations of packets and ONE triangle GEMM over all
    their samples (int32 in TMEM, int64 added once).  Then the plain form: one
    corner-turn + GEMM launch per sub-integration (the reference's per-V-update
    launch form) on the same packets.

    check = (channels, elements or None): after the timed loop, the host copy of
    those channels' packet bytes and of the timed cube's V on them is returned
    in r["check"] for the CPU-baseline leg, with the number of launches that
    integrated the same packets (warm-up + timed steps)."""
    S = CFG["batch"]
    nheaps = S * HEAPS_PER_SUB
    npk = nheaps * NANT
    kt = nheaps * TPKT
    stream = torch.cuda.current_stream()
    pk = make_packets(mixer, torch, dev, nheaps, seed=seed)
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

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
    start, stop = ev_pair(torch)
    barrier(pg, dev)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        start.record(stream)
        for s in range(steps):
            step(evs[s])
        stop.record(stream)
        torch.cuda.synchronize()
    barrier(pg, dev)
    ms_total = start.elapsed_time(stop)
    ct_ms = [e[0].elapsed_time(e[1]) for e in evs]
    gemm_ms = [e[1].elapsed_time(e[2]) for e in evs]
    if int(err.item()) != 0 or int(seq_err.item()) != 0:
        raise RuntimeError(f"kernel error word {int(err.item())}, seq errors {int(seq_err.item())}")
    r = {"S": S, "nheaps": nheaps, "npk": npk, "kt": kt, "ms_total": ms_total, "ct_ms": ct_ms,
         "gemm_ms": gemm_ms, "clocks": clk.summary(), "steps": steps, "warmup": warmup}
    if check is not None:
        chans, elems = check
        r["check"] = {"subpk": packet_subset(torch, pk, nheaps, chans, elems),
                      "got": unpack_channels(torch, mixer, vis, NANT, chans, elems),
                      "nant": NANT if elems is None else len(elems), "nch": len(chans),
                      "tpkt": TPKT, "nheaps": nheaps, "mult": warmup + steps,
                      "channels": list(chans), "elements": None if elems is None else
                      f"{len(elems)} of {NANT} (principal submatrix)"}
    if plain_steps > 0:
        def plain_step():
            for s in range(S):
                h0 = s * HEAPS_PER_SUB
                mixer.corner_turn(pk[h0 * NANT * STRIDE:], STRIDE, HDR, NANT, NCH, TPKT,
                                  HEAPS_PER_SUB, h0 * NANT, planes, KSUB, 0, seq_err, err)
                mixer.xcorr_tri(planes, NANT, NCH, KSUB, 0, KSUB, mixer.VIS_ACC_I64, vis, err)

        plain_step()
        torch.cuda.synchronize()
        barrier(pg, dev)
        p0, p1 = ev_pair(torch)
        p0.record(stream)
        for _ in range(plain_steps):
            plain_step()
        p1.record(stream)
        torch.cuda.synchronize()
        r["plain_ms_total"] = p0.elapsed_time(p1)
        r["plain_steps"] = plain_steps
        if int(err.item()) != 0 or int(seq_err.item()) != 0:
            raise RuntimeError("plain form: kernel or seq error")
    if keep:
        r["_bufs"] = {"pk": pk, "planes": planes, "vis": vis, "err": err, "seq_err": seq_err}
    else:
        del pk, planes, vis
        torch.cuda.empty_cache()
    return r


def gemm_only_window(torch, mixer, planes, vis, kt, err, local, min_ms=600.0):
    """The GEMM alone, back to back on the timed step's planes for at least
    `min_ms`, with the SM clock sampled: the clock the GEMM itself runs at
    (the step's median also covers the corner-turn phases, which hold a
    higher clock under the power cap)."""
    stream = torch.cuda.current_stream()
    e0, e1 = ev_pair(torch)
    e0.record(stream)
    mixer.xcorr_tri(planes, NANT, NCH, kt, 0, kt, mixer.VIS_ACC_I64, vis, err)
    e1.record(stream)
    torch.cuda.synchronize()
    n = max(3, int(min_ms / max(e0.elapsed_time(e1), 1e-3)) + 1)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(n):
            mixer.xcorr_tri(planes, NANT, NCH, kt, 0, kt, mixer.VIS_ACC_I64, vis, err)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    return {"launches": n, "ms_per_launch": ms, "tops": tri_ops(kt) / ms / 1e9,
            "clocks": clk.summary()}


def workload_summary(r, probe=None):
    """Compact block for one plain workload: throughput, stream/plain, GEMM and
    corner-turn rates."""
    value = wire_gbps(r["npk"] * r["steps"], r["ms_total"] / 1e3)
    gemm = statistics.mean(r["gemm_ms"]) / 1e3
    ct = statistics.mean(r["ct_ms"]) / 1e3
    ct_bytes = r["npk"] * STRIDE + 2 * NCH * NANT * r["kt"]
    hbm, _ = hbm_peak()
    tops = tri_ops(r["kt"]) / gemm / 1e12
    nb = (NANT + 127) // 128
    tile_tops = tops * (nb * (nb + 1) // 2 * 128 * 128) / (NANT * (NANT + 1) / 2)
    out = {"workload": CFG["text"], "nant": NANT, "nch": NCH, "tpkt": TPKT, "ksub": KSUB,
           "subints_per_step": r["S"], "steps": r["steps"], "warmup": r["warmup"],
           "bytes_per_step": r["npk"] * STRIDE,
           "value": value, "unit": "Gb/s", "ms_per_step": r["ms_total"] / r["steps"],
           "gemm_ms": 1e3 * gemm, "gemm_tops": tops, "gemm_tile_basis_tops": tile_tops,
           "corner_turn_ms": 1e3 * ct, "corner_turn_hbm_frac": ct_bytes / ct / 1e9 / hbm,
           "clocks": r["clocks"]}
    if "plain_ms_total" in r:
        pv = wire_gbps(r["npk"] * r["plain_steps"], r["plain_ms_total"] / 1e3)
        out["plain"] = {"value": pv, "unit": "Gb/s", "steps": r["plain_steps"],
                        "form": f"one corner-turn + GEMM launch per K={KSUB} sub-integration"}
        out["stream_over_plain"] = value / pv
    if probe:
        kind = "sustained" if r["ms_total"] > SUSTAINED_REGION_MS else "burst"
        out["gemm_frac_of_int8_peak"] = tops / probe[kind]["tops"]
        out["int8_peak_kind"] = kind
        # the GEMM's own roofline: its algorithmic bytes per launch (planes read once,
        # int64 cube read and written) against its ops; the bound is the lower of the
        # measured int8 rate and intensity x HBM bandwidth
        gbytes = 2 * NCH * NANT * r["kt"] + 2 * 8 * mixer_vis_elems_host(NANT, NCH)
        ai = tri_ops(r["kt"]) / gbytes
        mem_tops = ai * hbm / 1e3
        peak = min(probe[kind]["tops"], mem_tops)
        out["gemm_roofline"] = {"ops_per_byte": ai, "bound": "hbm" if mem_tops < probe[kind]["tops"]
                                else "tensor", "peak_tops": peak, "frac": tops / peak,
                                "basis": "triangle ops over planes + int64 cube RMW bytes"}
    return out


def mixer_vis_elems_host(nant, nch):
    """Tile-packed cube elements (re + im), as mixer_vis_elems computes them."""
    nb = (nant + 127) // 128
    return nch * nb * (nb + 1) // 2 * 2 * 128 * 128


# ---------------------------------------------------------------- batched ----

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


def batched_block(torch, mixer, dev, S=4, small=False, rounds=5, reps=2, tune_reps=1,
                  check_arrays=3, n_arrays=48):
    """48 uneven arrays, S sub-integrations of each per pass.  Plain form: one
    GEMM launch per array and sub-integration (K samples each, int64 added per
    launch), the reference's per-V-update launch form.  Batched form: ONE
    persistent launch over every array's tiles with each work item contracting
    the array's S sub-integrations (S*K samples, int32 in TMEM, one int64 add),
    plan autotuned, replayed from a CUDA graph.  Inputs are the arrays' int8 X
    planes (corner-turned from the seeded packet source before timing); both
    forms read the same bytes.  Results: plain == batched per array (checksum),
    and the sampled arrays' V go to the CPU leg for the oracle check."""
    stream = torch.cuda.Stream()
    arrays = batched_arrays(small=small)[:n_arrays]
    # the largest S up to the one asked for whose planes, cubes and packet buffer fit
    # in 90 % of the free device memory
    free, _ = torch.cuda.mem_get_info(dev)
    per_sub = sum(2 * n * c * k for n, c, k, _, _ in arrays)
    cubes = sum(8 * mixer.vis_elems(n, c) for n, c, _, _, _ in arrays)
    pk_max = max((k // 16) * n * (64 + 32 * c) for n, c, k, _, _ in arrays)
    S_asked = S
    while S > 1 and S * per_sub + cubes + pk_max > 0.9 * free:
        S -= 1
    probs, total_ops, plane_bytes = [], 0.0, 0
    t_gen = time.perf_counter()
    for idx, (n, c, k, l, m) in enumerate(arrays):
        tp = 16
        stride = 64 + 2 * c * tp
        nh = k // tp
        kt = S * k
        sky = torch.from_numpy(mixer.sky_table(n, c, 32, [(l, m, 4.0, 0.0)])).to(dev)
        pk = torch.empty(nh * n * stride, dtype=torch.uint8, device=dev)
        planes = torch.empty(2 * c * n * kt, dtype=torch.int8, device=dev)
        for s in range(S):                    # distinct samples per sub-integration
            mixer.gen_packets(pk, stride, 64, n, c, tp, nh, s * nh, s * nh * n, 4096 + idx, sky, 12.0,
                              SEED + idx, 0)
            mixer.corner_turn(pk, stride, 64, n, c, tp, nh, s * nh * n, planes, kt, s * k)
        del pk, sky
        vis = torch.zeros(mixer.vis_elems(n, c), dtype=torch.int64, device=dev)
        probs.append({"planes": planes, "nant": n, "nch": c, "kt": kt, "kbeg": 0, "klen": kt,
                      "ksub": k, "mode": mixer.VIS_ACC_I64, "vis": vis})
        total_ops += 8.0 * n * (n + 1) / 2 * kt * c
        plane_bytes += 2 * n * kt * c
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t_gen

    def timed(fn, r=reps):
        with torch.cuda.stream(stream):
            fn()
            stream.synchronize()
            e0, e1 = ev_pair(torch)
            e0.record(stream)
            for _ in range(r):
                fn()
            e1.record(stream)
            stream.synchronize()
        return e0.elapsed_time(e1) / r

    def plain():
        for s in range(S):
            for p in probs:
                mixer.xcorr_tri(p["planes"], p["nant"], p["nch"], p["kt"], s * p["ksub"], p["ksub"],
                                mixer.VIS_ACC_I64, p["vis"], stream=stream)

    def zero():
        with torch.cuda.stream(stream):
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
    t_untuned = timed(lambda: b.run(stream), 1)
    t0 = time.perf_counter()
    tuned_ms = b.autotune(reps=tune_reps, stream=stream) if tune_reps > 0 else None
    tune_s = time.perf_counter() - t0
    b.capture_graph(stream)
    # plain launches and the graph alternate, so the clock drift under the power
    # cap favours neither form; medians over the rounds
    res = []
    for _ in range(rounds):
        res.append((timed(plain), timed(lambda: b.replay(stream))))
    t_plain = statistics.median(x[0] for x in res)
    t_graph = statistics.median(x[1] for x in res)
    zero()
    with torch.cuda.stream(stream):
        b.replay(stream)
    stream.synchronize()
    with torch.cuda.stream(stream):
        sums_batch = [vis_checksum(torch, p["vis"]) for p in probs]
    info = b.info()
    # sampled arrays for the oracle: the smallest, a middle and the largest by work
    order = sorted(range(len(probs)), key=lambda q: total_ops_of(probs[q]))
    pick = sorted({order[0], order[len(order) // 2], order[-1]})[:check_arrays]
    samples = []
    for q in pick:
        p = probs[q]
        n, c, kt = p["nant"], p["nch"], p["kt"]
        chans = [0, c - 1]
        pl = p["planes"].view(2, c, n, kt)[:, chans].cpu().numpy()
        samples.append({"array": q, "nant": n, "nch": c, "kt": kt, "channels": chans, "planes": pl,
                        "got": unpack_channels(torch, mixer, p["vis"], n, chans)})
    exact_vs_plain = sums_plain == sums_batch and info["kernel_err"] == 0
    out = {
        "workload": (f"{len(arrays)} of 48 " if len(arrays) < 48 else "48 ")
        + ("small arrays, N in {64..256 step 32}, C in {16..64 step 16}" if small else
           "arrays, N in {64..1024 step 32}, C in {16..512 step 16}")
        + f", K in {{256..4096 step 256}} per sub-integration, {S} sub-integrations per pass, "
          "1 source + sigma 12 noise each (seeded)",
        "subints_per_pass": S, "subints_asked": S_asked, "total_ops": total_ops,
        "plane_bytes": plane_bytes,
        "plain_ms": t_plain, "plain_tops": total_ops / t_plain / 1e9,
        "plain_launches_per_pass": S * len(probs),
        "graph_ms": t_graph, "graph_tops": total_ops / t_graph / 1e9,
        "batched_untuned_ms": t_untuned, "batched_over_plain": t_plain / t_graph,
        "input_gbps_plain": 8 * plane_bytes / t_plain / 1e6,
        "input_gbps_batched": 8 * plane_bytes / t_graph / 1e6,
        "autotune_s": tune_s, "autotune_best_ms": tuned_ms, "setup_s": gen_s,
        "plan": {"nwork": info["nwork"], "order": ["lpt", "channel"][info["order"]],
                 "split_per_class": {str(c): info["split"][c] for c in range(1, 9)}},
        "bit_exact_vs_plain": exact_vs_plain, "rounds": rounds, "reps": reps,
        "per_round_plain_over_graph": [round(x[0] / x[1], 3) for x in res],
        "what": "TOPS on the triangle basis; input Gb/s counts the int8 X planes read",
    }
    b.close()
    del probs
    torch.cuda.empty_cache()
    return out, samples


def total_ops_of(p):
    return p["nant"] * (p["nant"] + 1) / 2 * p["kt"] * p["nch"]


# ----------------------------------------------------------------- serving ----

# Serving workload: (nant, nch, tpkt, ksub, nsub_dump, side) of the two stream types.
SERVE_TYPES = {"256x128": (256, 128, 32, 256, 64, 16), "1024x64": (1024, 64, 64, 256, 64, 32)}


def serve_pools(torch, mixer, dev, kinds):
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
    return pools


def serve_run(torch, mixer, kinds, pools, run_s, gbps, budget, jitter, rng):
    """One run of the server: 8 feeder threads (one per stream) submit their
    pool of heaps paced to gbps / 8 each (unpaced when gbps <= 0) between a
    Poisson-jittered start and stop; a poller copies dumps out."""
    import threading
    import numpy as np
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
                mixer.restamp_seq(pools[i], nsub * hps * nant, stride, j * hps * nant, stream=own)
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
        time.sleep(0.05)                           # let the last full dump finish
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
    w0 = max(a for a, _ in span)              # window in which every stream was submitting
    w1 = min(b for _, b in span)
    all_bytes = 0
    for i in range(8):
        sub_b = submitted[i] / max(1, len(stamps[i]))
        all_bytes += sub_b * sum(1 for t in stamps[i] if w0 <= t < w1)
    all_active = ({"window_s": round(w1 - w0, 2), "gbps": 8 * all_bytes / (w1 - w0) / 1e9}
                  if w1 - w0 > 0.5 else None)
    out = {"feeders": "python threads", "wall_s": wall, "offered_gbps": gbps,
           "submitted_gbps": 8 * sum(submitted) / wall / 1e9,
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
    if period:
        out["p99_under_integration_period"] = out["p99_dump_latency_ms"] < min(
            1e3 * v for v in period.values())
    return out


SERVE_BIN = os.path.join(ROOT, "daqiri-mixer_b200", "mixer_serve")


def serve_cpp(seconds, gbps, budget_gb, jitter, device=0, reserve=True):
    """One run of the C++ load generator (app/mixer_serve.cpp): eight feeder
    threads on the C-ABI, one JSON line of results.  reserve: the streams' state
    is allocated before the run (mixer_server_reserve), as a server that knows
    its stream shapes does at start-up."""
    if not os.path.exists(SERVE_BIN):
        raise RuntimeError(f"{SERVE_BIN} missing: build it with make -C daqiri-mixer_b200")
    cmd = [SERVE_BIN, "--seconds", str(seconds), "--gbps", str(gbps), "--budget-gb", str(budget_gb),
           "--jitter", "1" if jitter else "0", "--device", str(device), "--seed", str(SEED),
           "--reserve", "1" if reserve else "0"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=seconds + 300)
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    if not lines:
        raise RuntimeError(f"mixer_serve exited {p.returncode}: {p.stderr[-500:]}")
    out = json.loads(lines[-1])
    out["rc"] = p.returncode
    period = {k: 1e3 * v[4] * (v[3] // v[2]) * v[0] * (64 + 2 * v[1] * v[2]) / (gbps / 8 * 1e9 / 8)
              for k, v in SERVE_TYPES.items()} if gbps > 0 else None
    if period:
        out["integration_period_ms"] = period
        out["p99_under_integration_period"] = out["p99_dump_latency_ms"] < min(period.values())
    return out


def serve_block(torch, mixer, dev, args, paced_s, unpaced_s, tight=False, python_feeders=False,
                cold=True):
    """Serving: the paced run (every stream at 380 / 8 Gb/s, Poisson-jittered
    start / stop, budget for all eight, the streams' state reserved before the
    run), the same run without the reservation (every admission allocates its
    state while the other streams are served), optionally the admission run
    with a tight budget, and the unpaced run with all eight streams open from
    start to end (the server's own ceiling).  C++ feeders (mixer_serve) unless
    python_feeders."""
    out = {"workload": "8 streams: 4 x (256 elements x 128 ch, tpkt 32), 4 x (1024 elements x 64 ch, "
                       "tpkt 64), K 256, 64 sub-integrations per dump, 8256-byte heaps from the "
                       "seeded sky source (device pools), Poisson-jittered start / stop",
           "paced_gbps": args.serve_gbps, "budget_gb": args.serve_budget_full_gb}
    if python_feeders:
        import numpy as np
        rng = np.random.default_rng(SEED + 3)
        kinds = ["256x128"] * 4 + ["1024x64"] * 4
        pools = serve_pools(torch, mixer, dev, kinds)

        def run(s, g, b, j):
            return serve_run(torch, mixer, kinds, pools, s, g, int(b * (1 << 30)), j, rng)
    else:
        torch.cuda.empty_cache()

        def run(s, g, b, j, reserve=True):
            return serve_cpp(s, g, b, j, dev.index or 0, reserve)
    out["paced"] = run(paced_s, args.serve_gbps, args.serve_budget_full_gb, True)
    if cold and not python_feeders:
        out["paced_cold_admission"] = run(paced_s, args.serve_gbps, args.serve_budget_full_gb, True,
                                          reserve=False)
    if tight:
        out["tight_budget_gb"] = args.serve_budget_gb
        out["paced_tight_budget"] = run(paced_s, args.serve_gbps, args.serve_budget_gb, True)
    if unpaced_s > 0:
        out["unpaced_ceiling"] = run(unpaced_s, 0.0, 64.0, False)
    if python_feeders:
        del pools
        torch.cuda.empty_cache()
    runs = [v for k, v in out.items() if isinstance(v, dict) and "kernel_err" in v]
    out["ok"] = all(r["kernel_err"] == 0 and r["seq_errors"] == 0 and r.get("rc", 0) == 0
                    for r in runs)
    return out


# -------------------------------------------------------------- int8 probe ----

def mma_probe(torch, mixer, dev, local=0, runs=(("burst", 20000, 5), ("sustained", 200000, 20))):
    """Dense int8 tensor-core rate of this GPU with the GEMM's own MMA stream
    (mixer_mma_peak: resident shared-memory operands, no loads), with the SM
    clock sampled: the measured int8 ceiling the GEMM's roofline divides by."""
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mixer.mma_peak(1000, 0, err)
    torch.cuda.synchronize()
    out = []
    for label, iters, reps in runs:
        e0, e1 = ev_pair(torch)
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


# ------------------------------------------------------------ CPU-baseline leg ----

def cpu_leg(line, hp_sub, checks, batched_samples, args):
    """The CPU-baseline leg, the one place this script runs the oracle (the CPU
    restatement, as checker and baseline only): times the OpenMP int64
    correlator on a channel subset of one sub-integration of the headline
    packets, then checks every GPU cube handed in against it bit for bit."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    out = {}
    if hp_sub is not None and not args.no_cpu_baseline:
        configure(None, "plain")
        gbps, cores, desc, _, _ = cpu_correlator_sample(oracle, hp_sub, target_s=args.cpu_seconds)
        line["cpu_baseline"] = {"value": gbps, "unit": "Gb/s", "cores": cores, "kind": "port",
                                "sample": desc}
    for name, ck in checks:
        t0 = time.perf_counter()
        n, nc, tp, nh = ck["nant"], ck["nch"], ck["tpkt"], ck["nheaps"]
        planes = oracle.corner_turn(np.ascontiguousarray(ck["subpk"]).reshape(-1), n, nc, tp, nh,
                                    pkt_stride=2 * nc * tp, hdr=0)
        v = oracle.correlate(planes, mirror=False)
        low = np.tril(np.ones((n, n), dtype=bool))
        equal = bool(np.array_equal(ck["got"][:, :, low], ck["mult"] * v[:, :, low]))
        out[name] = {"equal": equal, "channels": ck["channels"], "elements": ck["elements"] or n,
                     "samples": nh * tp, "launches_integrated": ck["mult"],
                     "what": "timed cube == oracle V x launches (lower triangle incl. diagonal)",
                     "cpu_s": round(time.perf_counter() - t0, 2)}
    if batched_samples:
        res = []
        for s in batched_samples:
            v = oracle.correlate(np.ascontiguousarray(s["planes"]), mirror=False)
            n = s["nant"]
            low = np.tril(np.ones((n, n), dtype=bool))
            res.append({"array": s["array"], "nant": n, "nch": s["nch"], "samples": s["kt"],
                        "channels": s["channels"],
                        "equal": bool(np.array_equal(s["got"][:, :, low], v[:, :, low]))})
        out["batched"] = {"equal": all(r["equal"] for r in res), "arrays": res}
    return out


def cpu_correlator_sample(oracle, packets_host, target_s=12.0, max_out=2e9):
    """Time the oracle's OpenMP int64 correlator on a channel subset of one
    sub-integration; returns (gbps_equivalent, cores, sample_description,
    seconds, lower-triangle int64 V of the sampled channels)."""
    import numpy as np
    planes = oracle.corner_turn(np.ascontiguousarray(packets_host), NANT, NCH, TPKT, HEAPS_PER_SUB)
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


# ------------------------------------------------------------- reference arm ----

def run_reference(args):
    """Reference arm.  The reference's path is GPU code with no CPU
    implementation, so `value` is the oracle's OpenMP int64 correlator (the CPU
    restatement of that path) on the host cores, on a channel subset of the same
    workload per step.  `reference_gpu` times the reference's own kernels
    (k_packAB, cgemm_blk_t<true>, k_flush_cube, compiled from its sources into
    oracle/_ref/libref_gpu.so) on this GPU, as its gpu_thread launches them."""
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
    if not args.no_reference_gpu:
        try:
            line["reference_gpu"] = reference_gpu_block(oracle, pk, planes)
        except Exception as e:                      # reported, never fatal for the CPU arm
            line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
    print(json.dumps(line))
    return 0


def reference_gpu_block(oracle, pk_plain, planes_plain):
    """The reference's own GPU kernels on this GPU, timed with CUDA events on
    device-resident inputs (no H2D), as src/rx_host_corr.cu:159-170 launches
    them per V-update:
      own_shape: k_packAB + cgemm_blk_t<true> per V-update and k_flush_cube
                 every g_flush = 4 V-updates (its default, :113), at the shape
                 the reference is compiled for (256 elements, 128 channels,
                 K 1024 = 32 heaps per V-update); staged heaps cycle through 4
                 buffers (268 MB, larger than L2);
      headline:  cgemm_blk_t<true> per K=1024 V-update of the 1024-element,
                 256-channel array (its k_packAB and k_flush_cube are compiled
                 for the 256 x 128 shape only, so the corner-turn and flush are
                 not included: a lower bound on its V-update time)."""
    import numpy as np
    import torch
    if not torch.cuda.is_available():
        return {"unavailable": "no CUDA device"}
    if not oracle.ref_gpu_available():
        return {"unavailable": "oracle/_ref/libref_gpu.so not built (reference sources absent)"}
    ref = oracle.ref_gpu()
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    s = torch.cuda.current_stream()
    sp = s.cuda_stream
    n0, c0, tp0, hb, kp = (ref.ref_const(q) for q in range(5))
    out = {}

    # ---- own shape: pack + cgemm<true> (+ flush every 4) --------------------------
    nbuf = 4
    pk0 = oracle.gen_packets(n0, c0, tp0, hb * nbuf, sky=oracle.sky_table(
        n0, c0, 16, [(0.10, -0.05, 6.0, 0.0), (0.2, 0.0, 0.0, 1.5)]), sigma=16.0, seed=SEED)
    bb = torch.from_numpy(pk0.reshape(hb * nbuf * n0, 8256)[:, 64:].copy()).to(dev)   # header stripped
    per_bb = hb * n0 * 8192
    bbf = bb.view(-1)
    a = [torch.empty(c0 * n0 * kp, dtype=torch.int8, device=dev) for _ in range(4)]
    vre = torch.zeros(c0 * n0 * n0, dtype=torch.int32, device=dev)
    vim = torch.zeros_like(vre)
    cube = torch.zeros(c0 * 2 * n0 * n0, dtype=torch.float32, device=dev)

    def vupdate(i):
        rc = ref.ref_pack(bbf[(i % nbuf) * per_bb:].data_ptr(), a[0].data_ptr(), a[1].data_ptr(),
                          a[2].data_ptr(), a[3].data_ptr(), sp)
        rc |= ref.ref_cgemm(1, n0, n0, kp, c0, a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr(),
                            a[3].data_ptr(), vre.data_ptr(), vim.data_ptr(), sp)
        if i % 4 == 3:
            rc |= ref.ref_flush(cube.data_ptr(), vre.data_ptr(), vim.data_ptr(), sp)
        if rc:
            raise RuntimeError(f"reference kernel launch failed ({rc})")

    for i in range(8):
        vupdate(i)
    torch.cuda.synchronize()
    nv = 64
    e0, e1 = ev_pair(torch)
    e0.record(s)
    for i in range(nv):
        vupdate(i)
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / nv
    pkts = hb * n0
    ops = 8.0 * n0 * (n0 + 1) / 2 * kp * c0
    out["own_shape"] = {"kernels": "k_packAB + cgemm_blk_t<true> per V-update, k_flush_cube every 4",
                        "nant": n0, "nch": c0, "k_per_vupdate": kp, "vupdates": nv,
                        "ms_per_vupdate": ms, "value": 8.0 * 8256 * pkts / ms / 1e6, "unit": "Gb/s",
                        "tops_triangle_basis": ops / ms / 1e9,
                        "tops_full_square_basis": 8.0 * n0 * n0 * kp * c0 / ms / 1e9}
    del bb, bbf, a, vre, vim, cube
    torch.cuda.empty_cache()

    # ---- headline array: cgemm<true> per V-update ---------------------------------
    _, nch, nant, kt = planes_plain.shape
    xr = torch.from_numpy(np.ascontiguousarray(planes_plain[0])).to(dev).view(-1)
    xi = torch.from_numpy(np.ascontiguousarray(planes_plain[1])).to(dev).view(-1)
    nxi = torch.from_numpy(np.ascontiguousarray(-planes_plain[1].astype(np.int16)).astype(np.int8)).to(dev).view(-1)
    cre = torch.zeros(nch * nant * nant, dtype=torch.int32, device=dev)
    cim = torch.zeros_like(cre)

    def cg():
        rc = ref.ref_cgemm(1, nant, nant, kt, nch, xr.data_ptr(), xi.data_ptr(), xr.data_ptr(),
                           nxi.data_ptr(), cre.data_ptr(), cim.data_ptr(), sp)
        if rc:
            raise RuntimeError(f"reference cgemm launch failed ({rc})")

    for _ in range(2):
        cg()
    torch.cuda.synchronize()
    nv = 10
    e0.record(s)
    for _ in range(nv):
        cg()
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / nv
    npk = (kt // TPKT) * nant
    out["headline"] = {"kernels": "cgemm_blk_t<true> per V-update (corner-turn and flush not "
                                  "included: compiled for 256 x 128 only)",
                       "nant": nant, "nch": nch, "k_per_vupdate": kt, "vupdates": nv,
                       "ms_per_vupdate": ms, "value": 8.0 * STRIDE * npk / ms / 1e6, "unit": "Gb/s",
                       "tops_triangle_basis": tri_ops(kt, nant, nch) / ms / 1e9,
                       "tops_full_square_basis": 8.0 * nant * nant * kt * nch / ms / 1e9}
    return out


# --------------------------------------------------------------- other modes ----

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
    e0, e1 = ev_pair(torch)
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
                e0, e1 = ev_pair(torch)
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
    n = mixer.vis_elems(N, C)
    T = N * (N + 1) // 2
    hbm, hbm_src = hbm_peak()
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
            e0, e1 = ev_pair(torch)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = statistics.median(times)
        gbs = nbytes / ms / 1e6
        print(json.dumps({"kernel": name, "workload": CFG["text"], "nant": N, "nch": C,
                          "grid": Gs, "ms": ms, "algorithmic_bytes": nbytes, "bytes": what,
                          "gbs": gbs, "hbm_frac": gbs / hbm, "peak": f"{hbm_src}: {hbm} GB/s",
                          "launches": len(times)}), flush=True)
    return 0


def run_mma_peak(args):
    import torch
    import mixer
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    for line in mma_probe(torch, mixer, dev):
        print(json.dumps(line), flush=True)
    return 0


def run_batched(args):
    """`--config batched` alone: the batched block, with the oracle check of the
    sampled arrays."""
    import torch
    import mixer
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    out, samples = batched_block(torch, mixer, dev, S=args.batched_subints, small=args.small_arrays,
                                 rounds=5, reps=3, tune_reps=args.tune_reps, n_arrays=args.arrays)
    line = {"metric": "batched uneven arrays: int8 cGEMM TOPS (triangle basis), batched vs plain",
            "batched": out}
    if not args.no_cpu_baseline:
        line["bit_exact_vs_cpu"] = cpu_leg({}, None, [], samples, args)
    print(json.dumps(line))
    ok = out["bit_exact_vs_plain"] and line.get("bit_exact_vs_cpu", {}).get("batched", {}).get(
        "equal", True)
    return 0 if ok else 1


def run_serve(args):
    """`--config serve` alone: paced (full and tight budget) and unpaced runs."""
    import torch
    import mixer
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    out = serve_block(torch, mixer, dev, args, args.serve_seconds, min(args.serve_seconds, 10.0),
                      tight=True, python_feeders=args.serve_python)
    print(json.dumps({"metric": "serving: sustained input Gb/s and p50/p99 dump latency", **out}))
    return 0 if out["ok"] else 1


# ------------------------------------------------------------------ headline ----

def run_ours(args):
    import torch
    import mixer
    rank, world, local, pg = dist_setup(args.gpus)
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if mixer.lib().mixer_device_ok() != mixer.OK:
        raise RuntimeError("not an sm_100 device")
    seed = SEED + rank                      # independent replicas: each rank its own sky noise
    stream = torch.cuda.current_stream()
    want_check = rank == 0 and not args.no_cpu_baseline
    # the timed cube is checked on four channels (two, on a principal submatrix of
    # 512 elements, for arrays over 1024 elements: the CPU cost grows with N^2)
    chk = (([0, 1, NCH // 2, NCH - 1], None) if NANT <= 1024 else
           ([0, NCH - 1], list(range(256)) + list(range(NANT - 256, NANT))))
    r = plain_run(torch, mixer, dev, args.steps, args.warmup, pg, local, seed,
                  check=chk if want_check else None,
                  plain_steps=0 if args.profile else max(1, min(args.steps, 5)), keep=True)
    bufs = r.pop("_bufs")
    pk, planes, vis, err = bufs["pk"], bufs["planes"], bufs["vis"], bufs["err"]
    S, nheaps, npk, kt = r["S"], r["nheaps"], r["npk"], r["kt"]
    ms_total = r["ms_total"]
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_case": True, "nch": NCH, "subints": S,
                              "ms_per_step": ms_total / args.steps,
                              "xcorr_ms": statistics.mean(r["gemm_ms"]),
                              "corner_turn_ms": statistics.mean(r["ct_ms"])}))
        return 0
    t_max = max_over_ranks(pg, ms_total, dev) / 1e3
    packets_all = sum_over_ranks(pg, float(npk * args.steps), dev)
    value = wire_gbps(packets_all, t_max)
    tops = tri_ops(kt) * args.steps * world / t_max / 1e12
    plain_t = max_over_ranks(pg, r["plain_ms_total"], dev) / 1e3
    plain_value = wire_gbps(sum_over_ranks(pg, float(npk * r["plain_steps"]), dev), plain_t)

    # ---- the GEMM alone, with its own clock ---------------------------------------
    gemm_alone = gemm_only_window(torch, mixer, planes, vis, kt, err, local)

    # ---- host copy of one sub-integration for the CPU baseline -------------------
    hp_sub = pk[: HEAPS_PER_SUB * NANT * STRIDE].cpu().numpy() if want_check else None

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
        qe = [ev_pair(torch) for _ in range(e2e_steps)]
        for q in qe:
            q[0].record(stream)
            e2e_step()
            q[1].record(stream)
        torch.cuda.synchronize()
        per = [a.elapsed_time(b) for a, b in qe]
        e2e_t = max_over_ranks(pg, qe[0][0].elapsed_time(qe[-1][1]), dev) / 1e3
        st = ctx.stats()
        if st["kernel_err"] or st["seq_errors"]:
            raise RuntimeError(f"e2e counters {st}")
        e2e = {"value": wire_gbps(sum_over_ranks(pg, float(e2e_npk * e2e_steps), dev), e2e_t),
               "unit": "Gb/s", "h2d_bytes_per_step": int(e2e_npk * STRIDE),
               "sub_integrations_per_step": e2e_heaps // HEAPS_PER_SUB,
               "d2h_bytes_per_step": int(NCH * G * G * 4 + 2 * NCH * 4),
               "ms_per_step": 1e3 * e2e_t / e2e_steps, "steps": e2e_steps,
               "ms_per_step_min_max": [min(per), max(per)],
               "h2d_gbytes_per_s": e2e_npk * STRIDE * e2e_steps / e2e_t / 1e9,
               "bound": "PCIe host-to-device copy of the packets (Gen5 x16, ~55 GB/s in practice)",
               "path": "mixer_correlate(host pinned packets) + mixer_image(host) per step"}
    del host

    # ---- the GEMM against the measured int8 tensor-core rate --------------------
    # The probe runs the GEMM's MMA stream with no memory traffic: the dense int8
    # rate of this GPU (burst: a short region at boost clock; sustained: under
    # the power cap), the denominator of the GEMM's roofline.
    probe = {p["run"]: p for p in mma_probe(torch, mixer, dev, local)}
    peaks = measured_peaks()
    sustained = ms_total > SUSTAINED_REGION_MS
    kind = "sustained" if sustained else "burst"
    peak = probe[kind]["tops"]
    bf16 = peaks.get("bf16_tflops_sustained" if sustained else "bf16_tflops")
    gemm_avg = statistics.mean(r["gemm_ms"]) / 1e3
    achieved = tri_ops(kt) / gemm_avg / 1e12
    ct_avg = statistics.mean(r["ct_ms"]) / 1e3
    ct_bytes = npk * STRIDE + 2 * NCH * NANT * kt
    hbm, hbm_src = hbm_peak()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    nb = (NANT + 127) // 128
    tile_factor = (nb * (nb + 1) // 2 * 128 * 128) / (NANT * (NANT + 1) / 2)
    gmhz = gemm_alone["clocks"].get("sm_mhz")
    per_clk = probe["sustained"]["ops_per_sm_per_clock"]

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
        "plain": {"value": plain_value, "unit": "Gb/s", "steps": r["plain_steps"],
                  "form": "one corner-turn + GEMM launch per K=1024 sub-integration",
                  "stream_over_plain": value / plain_value},
        "kernels": {"corner_turn_ms": 1e3 * ct_avg, "corner_turn_gbs": ct_bytes / ct_avg / 1e9,
                    "corner_turn_hbm_frac": ct_bytes / ct_avg / 1e9 / hbm,
                    "corner_turn_peak": f"{hbm_src}: {hbm} GB/s", "xcorr_ms": 1e3 * gemm_avg},
        "roofline": {"kernel": "k_xcorr_tri", "bound": "tensor", "achieved": achieved,
                     "peak": peak, "unit": "TOPS", "frac": achieved / peak,
                     "peak_source": (f"of measured: the int8 tcgen05 MMA rate of this GPU, "
                                     f"mixer_mma_peak {kind} ({peak:.0f} TOPS), "
                                     f"{kind} because the timed region is "
                                     f"{'over' if sustained else 'under'} {SUSTAINED_REGION_MS:.0f} ms"),
                     "peak_bf16x2": 2.0 * bf16 if bf16 else None,
                     "frac_of_bf16x2": achieved / (2.0 * bf16) if bf16 else None,
                     "traffic": XCORR_TRAFFIC_RATIO * (2 * NCH * NANT * kt + 2 * 8 * mixer.vis_elems(NANT, NCH)),
                     "traffic_note": "bytes per launch: algorithmic x 1.106, the DRAM/algorithmic "
                                     "ratio of an ncu capture at the same K (1024 el., 32 ch)",
                     "ops_per_launch": tri_ops(kt),
                     "basis": "triangle: 8 ops per complex MAC over the N(N+1)/2 needed entries"},
        "clocks": r["clocks"],
        "gpu_launches": 2 * args.steps,
        "e2e": e2e,
    }
    line["int8_mma_probe"] = {
        "burst_tops": probe["burst"]["tops"], "burst_mhz": probe["burst"]["clocks"].get("sm_mhz"),
        "sustained_tops": probe["sustained"]["tops"],
        "sustained_mhz": probe["sustained"]["clocks"].get("sm_mhz"),
        "probe_ops_per_sm_per_clock": per_clk,
        "kernel_err": probe["burst"]["kernel_err"] | probe["sustained"]["kernel_err"]}
    line["gemm_alone"] = {
        "launches": gemm_alone["launches"], "ms_per_launch": gemm_alone["ms_per_launch"],
        "tops": gemm_alone["tops"], "tile_basis_tops": gemm_alone["tops"] * tile_factor,
        "clocks": gemm_alone["clocks"],
        "frac_of_sustained_probe": gemm_alone["tops"] / probe["sustained"]["tops"],
        "per_clock_frac": (gemm_alone["tops"] * tile_factor * 1e12 / (sms * gmhz * 1e6) / per_clk
                           if gmhz and per_clk else None),
        "what": "the GEMM back to back on the step's planes, clock sampled over the GEMM alone; "
                "per_clock_frac compares tile-basis ops per SM per clock with the probe's"}

    # ---- imaging of the integrated cube (grid + FFT), device resident ------------
    with mixer.ArrayContext(nant=NANT, nch=NCH, tpkt=TPKT, ksub=KSUB, nsub_dump=1, side_x=SIDE,
                            grid=G, pkt_stride=STRIDE, hdr_bytes=HDR, max_heaps=HEAPS_PER_SUB) as ic:
        ic.correlate(pk, HEAPS_PER_SUB, seq0=0)
        dimg = torch.empty(NCH * G * G, dtype=torch.float32, device=dev)
        ic.image(dimg)
        torch.cuda.synchronize()
        i0, i1 = ev_pair(torch)
        i0.record(stream)
        for _ in range(10):
            ic.image(dimg)
        i1.record(stream)
        torch.cuda.synchronize()
        line["image_ms"] = i0.elapsed_time(i1) / 10
        line["image_grid"] = G
        if rank == 0:
            line["fp32_error_vs_fp64"] = fp32_errors(torch, mixer, dev, ic)
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
    del pk, vis, bufs
    torch.cuda.empty_cache()
    checks = [("headline", r.pop("check"))] if want_check else []

    # ---- the other workloads, one GPU only ------------------------------------------
    batched_samples = []
    if world == 1 and not args.headline_only:
        # Each further workload is its own measurement: one that fails records its
        # error under block_errors instead of taking the headline line with it.
        def guarded(name, fn):
            try:
                return fn()
            except Exception as e:                      # noqa: BLE001 -- reported in the line
                line.setdefault("block_errors", {})[name] = f"{type(e).__name__}: {e}"
                torch.cuda.synchronize()
                torch.cuda.empty_cache()
                return None

        for name, chk in (("small", ([0, 1, 64, 127], None)),
                          ("large", ([0, 63], list(range(0, 256)) + list(range(3840, 4096))))):
            configure(None, name)
            rr = guarded(name, lambda: plain_run(torch, mixer, dev, min(args.steps, 10), 3, seed=SEED,
                                                 check=chk if want_check else None, plain_steps=3))
            if rr is not None:
                line[name] = workload_summary(rr, probe)
                if "check" in rr:
                    checks.append((name, rr.pop("check")))
        configure(None, "plain")
        bb = guarded("batched", lambda: batched_block(torch, mixer, dev, S=args.batched_subints,
                                                      tune_reps=args.tune_reps))
        if bb is not None:
            line["batched"], batched_samples = bb
        sv = guarded("serve", lambda: serve_block(torch, mixer, dev, args, args.serve_paced_seconds,
                                                  args.serve_unpaced_seconds))
        if sv is not None:
            line["serve"] = sv
    if rank == 0:
        ck = cpu_leg(line, hp_sub, checks, batched_samples if want_check else [], args)
        if ck:
            line["bit_exact_vs_cpu"] = ck
            line["bit_exact_timed"] = all(v["equal"] for v in ck.values())
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()
    # the headline's own cube must be exact; the other blocks report in the line
    return 0 if line.get("bit_exact_vs_cpu", {}).get("headline", {}).get("equal", True) else 1


def fp32_errors(torch, mixer, dev, ic):
    """FP32 outputs against FP64 computed here from the exact int64 state: the
    dump cube (one rounding of int64) and the image (FP64 FFT of the exact int64
    grid), on the first channels."""
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
    return {"channels": ne, "cube_max_rel": cube_rel, "cube_bound": 2.0 ** -24,
            "image_max_err_over_peak": img_rel, "image_target": 1e-5}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=0,
                    help="sub-integrations per step (0: the workload's default)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--e2e-chunk", type=int, default=2, help="sub-integrations per H2D chunk")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-channels", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip the reference's GPU kernels")
    ap.add_argument("--headline-only", action="store_true",
                    help="only the 1024-element workload (no small / large / batched / serve)")
    ap.add_argument("--batched-subints", type=int, default=4,
                    help="sub-integrations per array per batched pass")
    ap.add_argument("--arrays", type=int, default=48,
                    help="--config batched: the first N arrays of the seeded draw (small ncu cases)")
    ap.add_argument("--tune-reps", type=int, default=1,
                    help="launches per autotuner sample (0: no autotuning, the default plan)")
    ap.add_argument("--nch", type=int, default=0,
                    help="channels per packet, tpkt = 4096/nch (0: the workload's)")
    ap.add_argument("--serve-seconds", type=float, default=30.0)
    ap.add_argument("--serve-paced-seconds", type=float, default=12.0,
                    help="length of the paced serving run in the default line")
    ap.add_argument("--serve-unpaced-seconds", type=float, default=5.0,
                    help="length of the unpaced serving run in the default line")
    ap.add_argument("--serve-gbps", type=float, default=380.0)
    ap.add_argument("--serve-python", action="store_true",
                    help="--config serve with Python feeder threads instead of mixer_serve")
    ap.add_argument("--serve-budget-gb", type=float, default=6.0,
                    help="device budget of the admission run (streams wait for memory)")
    ap.add_argument("--serve-budget-full-gb", type=float, default=16.0,
                    help="device budget of the main paced run (every stream fits)")
    ap.add_argument("--config", default="plain",
                    choices=["plain", "small", "large", "batched", "serve"],
                    help="plain: the 1024-element array (headline, with every other workload "
                         "as a block of its line); small / large: that array alone; batched: "
                         "48 uneven arrays alone; serve: 8 concurrent streams alone")
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
    ap.add_argument("--launcher-check", action="store_true",
                    help="the replica launcher and reductions over gloo, no GPU work")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_replicas(args.gpus, sys.argv[1:])
    if args.launcher_check:
        return run_launcher_check(args)
    configure(args.nch, args.config if args.config in PLAIN_CONFIGS else "plain")
    if args.batch > 0:
        CFG["batch"] = args.batch
    if args.config in ("small", "large"):
        args.headline_only = True
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
