"""The benchmark's timed-cube check, on the CPU.

bench.py hands the CPU-baseline leg the packet bytes of a few channels (and,
for large arrays, a subset of the elements) plus the GPU cube's V on them; the
leg corner-turns and correlates those bytes with the oracle and compares the
lower triangle with `launches x V`.  Here the "GPU" cube is made by the oracle
itself, so the check must pass, and must fail once one entry is changed."""
import argparse

import numpy as np
import torch

import oracle


def _args():
    return argparse.Namespace(no_cpu_baseline=True, cpu_seconds=1.0)


def _case(elems):
    import bench
    bench.configure(None, "small")                       # 256 elements, 128 ch, tpkt 32
    nheaps = 3
    pk = oracle.gen_packets(bench.NANT, bench.NCH, bench.TPKT, nheaps, sigma=16.0, seed=3)
    chans = [0, 5, bench.NCH - 1]
    sub = bench.packet_subset(torch, torch.from_numpy(pk), nheaps, chans, elems)
    full = oracle.correlate(oracle.corner_turn(pk, bench.NANT, bench.NCH, bench.TPKT, nheaps))
    got = full[chans]
    if elems is not None:
        got = got[:, :, elems][:, :, :, elems]
    ck = {"subpk": sub, "got": 7 * got, "nant": bench.NANT if elems is None else len(elems),
          "nch": len(chans), "tpkt": bench.TPKT, "nheaps": nheaps, "mult": 7, "channels": chans,
          "elements": None if elems is None else f"{len(elems)} of {bench.NANT}"}
    return bench, ck


def test_timed_cube_check_passes_and_catches_a_change():
    for elems in (None, list(range(0, 40)) + list(range(200, 256))):
        bench, ck = _case(elems)
        out = bench.cpu_leg({}, None, [("t", ck)], [], _args())
        assert out["t"]["equal"], elems
        ck["got"] = ck["got"].copy()
        ck["got"][1, 1, 9, 4] += 1                       # one lower-triangle entry off by one
        out = bench.cpu_leg({}, None, [("t", ck)], [], _args())
        assert not out["t"]["equal"], elems
    bench.configure(None, "plain")


def test_batched_sample_check():
    import bench
    rng = np.random.default_rng(4)
    planes = rng.integers(-127, 128, size=(2, 2, 96, 512), dtype=np.int8)
    v = oracle.correlate(planes)
    s = {"array": 0, "nant": 96, "nch": 2, "kt": 512, "channels": [0, 1], "planes": planes,
         "got": v.copy()}
    assert bench.cpu_leg({}, None, [], [s], _args())["batched"]["equal"]
    s["got"][0, 0, 50, 49] -= 3
    assert not bench.cpu_leg({}, None, [], [s], _args())["batched"]["equal"]
