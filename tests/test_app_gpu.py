"""The receiver program (daqiri-mixer_b200/mixer_rx, the reference's
rx_host_corr command-line surface on the C-ABI): a deterministic run of N
V-updates writes a --dump record equal to the oracle's FP32-rounded V of the
same seeded packets and publishes Corr32 frames; a timed run at a paced rate
streams dumps about once a second."""
import os
import struct
import subprocess

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
APP = os.path.join(ROOT, "daqiri-mixer_b200", "mixer_rx")
REC = 128 * 2 * 256 * 256          # floats per --dump record


def _run(args, timeout=120):
    return subprocess.run([APP] + args, capture_output=True, text=True, timeout=timeout)


def test_deterministic_dump_matches_oracle(cuda, tmp_path):
    dump = str(tmp_path / "v.f32")
    name = "/corr32_app_%d" % os.getpid()
    r = _run(["rx.yaml", "--vupdates", "2", "--flush", "1", "--gbps", "0", "--dump", dump,
              "--shm", name, "--keep-shm", "--seed", "99"])
    assert r.returncode == 0, r.stderr
    rec = np.fromfile(dump, dtype=np.float32)
    assert rec.size % REC == 0 and rec.size >= REC
    last = rec[-REC:].reshape(128, 2, 256, 256)
    # the same packets from the CPU generator: 2 V-updates of the pool at orbit angle 0
    sky = oracle.sky_table(256, 128, 16, [(0.10, -0.05, 6.0, 0.0), (0.2, 0.0, 0.0, 1.5)])
    pk = oracle.gen_packets(256, 128, 32, 64, sky=sky, sigma=16.0, seed=99)
    full = oracle.correlate(oracle.corner_turn(pk, 256, 128, 32, 64))
    assert np.array_equal(last, full.astype(np.float32))
    with open("/dev/shm" + name, "rb") as f:
        magic, w, h, nch, seq = struct.unpack("<IIIIQ", f.read(24))
    os.unlink("/dev/shm" + name)
    assert (magic, w, h, nch) == (0x43523343, 32, 32, 128) and seq >= 1


def test_paced_run_streams_dumps(cuda, tmp_path):
    dump = str(tmp_path / "v.f32")
    r = _run(["--seconds", "3", "--fps", "10", "--gbps", "100", "--dump", dump,
              "--shm", "/corr32_app_paced_%d" % os.getpid()])
    assert r.returncode == 0, r.stderr
    assert "seq_errors=0" in r.stderr and "kernel_err=0" in r.stderr
    nrec = os.path.getsize(dump) // (4 * REC)
    assert 2 <= nrec <= 5, r.stderr


def test_serving_load_generator_runs_clean(cuda):
    """The streaming server driven by its C++ load generator (app/mixer_serve.cpp):
    eight concurrent streams paced to 96 Gb/s for 3 s with their state reserved
    ahead of serving.  Every stream keeps its rate, dumps arrive, the p99 dump
    latency stays under the shorter integration period (the 256-element streams'
    64 sub-integrations at 12 Gb/s each: 721 ms), and no sequence or kernel error
    is counted."""
    import json
    exe = os.path.join(ROOT, "daqiri-mixer_b200", "mixer_serve")
    r = subprocess.run([exe, "--seconds", "3", "--gbps", "96", "--budget-gb", "16", "--jitter", "0",
                        "--reserve", "1"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["status"] == "ok" and out["kernel_err"] == 0 and out["seq_errors"] == 0
    assert out["admitted"] == 8 and out["dumps"] > 0
    assert all(abs(g - 12.0) < 0.5 for g in out["per_stream_gbps"]), out["per_stream_gbps"]
    assert out["p99_dump_latency_ms"] < 721.0
