"""Host-side ingest pieces that need no GPU: heap alignment of a packet burst
(the reference's drain-thread logic, src/rx_host_corr.cu:127-141, with every
seq checked) under injected faults, and the Corr32 shared-memory publication
(src/rx_host_corr.cu:97-105) read back by layout and by the reference's own
viewer src/peek32.cpp built from its source."""
import mmap
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import mixer
import oracle

NANT, NCH, TPKT = 16, 4, 16
STRIDE = 64 + 2 * NCH * TPKT


def _burst(nheaps, seq0=0):
    return oracle.gen_packets(NANT, NCH, TPKT, nheaps, seq0=seq0, seed=3).reshape(-1, STRIDE)


def _align(pk):
    pk = np.ascontiguousarray(pk)
    return mixer.align_heaps(pk.reshape(-1), pk.shape[0], STRIDE, NANT)


def test_aligned_burst():
    r = _align(_burst(5))
    assert r == {"first": 0, "nheaps": 5, "next": 5 * NANT, "seq0": 0}


def test_misaligned_start_and_partial_tail():
    pk = _burst(5)[5:-3]                     # starts at seq 5, ends mid-heap
    r = _align(pk)
    assert r["first"] == NANT - 5 and r["seq0"] == NANT and r["nheaps"] == 3
    assert r["next"] == r["first"] + 3 * NANT


@pytest.mark.parametrize("fault", ["drop", "duplicate", "swap"])
def test_gap_ends_the_run(fault):
    pk = _burst(6)
    bad = 2 * NANT + 7                       # inside heap 2
    if fault == "drop":
        pk = np.delete(pk, bad, axis=0)
    elif fault == "duplicate":
        pk = np.insert(pk, bad, pk[bad], axis=0)
    else:
        pk[[bad, bad + 1]] = pk[[bad + 1, bad]]
    r = _align(pk)
    assert r["first"] == 0 and r["nheaps"] == 2          # heaps 0 and 1 are whole
    assert r["next"] == bad + (fault == "duplicate")      # resume where the seqs break
    rest = _align(pk[r["next"]:])                         # re-align after the gap
    assert rest["seq0"] % NANT == 0 and rest["seq0"] >= 3 * NANT


def test_no_aligned_packet():
    pk = _burst(1)[1:NANT]
    r = _align(pk)
    assert r["nheaps"] == 0 and r["first"] == pk.shape[0] and r["next"] == pk.shape[0]


def _publish(name, nch, G, img, seq):
    vmax = img.reshape(nch, -1).max(1).astype(np.float32)
    vmin = img.reshape(nch, -1).min(1).astype(np.float32)
    shm = mixer.Corr32Shm(name, nch, G)
    shm.publish(np.ascontiguousarray(img, dtype=np.float32), vmax, vmin, seq)
    return shm, vmax, vmin


def test_corr32_layout():
    nch, G = 3, 32
    img = np.random.default_rng(1).normal(size=(nch, G, G)).astype(np.float32)
    name = "/corr32_mixer_test_%d" % os.getpid()
    shm, vmax, vmin = _publish(name, nch, G, img, 7)
    try:
        with open("/dev/shm" + name, "rb") as f:
            buf = mmap.mmap(f.fileno(), 0, prot=mmap.PROT_READ)
            magic, w, h, n, seq = struct.unpack_from("<IIIIQ", buf, 0)
            assert (magic, w, h, n, seq) == (0x43523343, G, G, nch, 7)
            body = np.frombuffer(buf, dtype=np.float32, offset=24, count=nch * G * G + 2 * nch)
            assert np.array_equal(body[:nch * G * G].reshape(img.shape), img)
            assert np.array_equal(body[nch * G * G:nch * G * G + nch], vmax)
            assert np.array_equal(body[nch * G * G + nch:], vmin)
            del body
            buf.close()
    finally:
        shm.close()
    assert not os.path.exists("/dev/shm" + name)


def test_reference_viewer_reads_the_publication():
    peek = os.path.join(os.path.dirname(oracle.REF_GPU_PATH), "peek32")
    if not os.path.exists(peek):
        pytest.skip("oracle/_ref/peek32 not built")
    nch, G = 8, 32
    img = np.zeros((nch, G, G), dtype=np.float32)
    img[5, 9, 20] = 10.0                     # brightest pixel
    img[5, 25, 3] = 4.0                      # off-centre second source
    shm, _, _ = _publish("/corr32", nch, G, img, 1)
    try:
        out = subprocess.run([peek, "5"], capture_output=True, text=True, timeout=30).stdout
    finally:
        shm.close()
    assert "channel 5/8" in out
    assert re.search(r"star peak \(x=20,y=9\)", out), out


# ---- time-split multi-queue ingest (src/config.h:40-45, MIXER_NQ) -------------------

def _split(nheaps, nq, seq0=0):
    """One unsplit burst and its nq queues: heap tb goes to queue tb % nq, with the UDP
    destination port 4096 + q written into its packets as the sender steers them."""
    pk = _burst(nheaps, seq0=seq0).copy()
    tb0 = seq0 // NANT
    for h in range(nheaps):
        q = (tb0 + h) % nq
        rows = pk[h * NANT:(h + 1) * NANT]
        rows[:, 36] = (4096 + q) >> 8
        rows[:, 37] = (4096 + q) & 0xFF
    queues = [np.ascontiguousarray(pk.reshape(nheaps, NANT, STRIDE)[[h for h in range(nheaps)
                                                                      if (tb0 + h) % nq == q]])
              .reshape(-1) for q in range(nq)]
    return pk, queues


@pytest.mark.parametrize("nq,seq0", [(1, 0), (2, 0), (4, 3 * NANT), (3, 5 * NANT)])
def test_time_split_merge_restores_time_order(nq, seq0):
    pk, queues = _split(12, nq, seq0)
    out = np.zeros_like(pk).reshape(-1)
    r = mixer.merge_time_split(queues, STRIDE, NANT, 4096, 64, out)
    assert r["heaps"] == 12 and r["seq0"] == seq0
    assert np.array_equal(out.reshape(pk.shape), pk)
    assert r["consumed"] == [q.size // STRIDE for q in queues]


def test_time_split_merge_stops_at_a_lost_heap():
    nq = 3
    pk, queues = _split(12, nq)
    q1 = queues[1].reshape(-1, NANT, STRIDE)          # heaps 1, 4, 7, 10: lose heap 7
    queues[1] = np.ascontiguousarray(np.delete(q1, 2, axis=0)).reshape(-1)
    out = np.zeros_like(pk).reshape(-1)
    r = mixer.merge_time_split(queues, STRIDE, NANT, 4096, 64, out)
    assert r["heaps"] == 7                             # heaps 0..6, in order
    assert np.array_equal(out.reshape(pk.shape)[:7 * NANT], pk[:7 * NANT])
    assert r["consumed"] == [3 * NANT, 2 * NANT, 2 * NANT]


def test_time_split_merge_checks_seq_and_port():
    pk, queues = _split(8, 2)
    bad = [q.copy() for q in queues]
    bad[0].reshape(-1, STRIDE)[NANT + 3, 48:52] = 0xFF   # a corrupt seq inside heap 2 (queue 0)
    out = np.zeros_like(pk).reshape(-1)
    assert mixer.merge_time_split(bad, STRIDE, NANT, 4096, 64, out)["heaps"] == 2
    bad = [q.copy() for q in queues]
    bad[1].reshape(-1, STRIDE)[5, 37] ^= 1             # heap 1 arrived on another port
    assert mixer.merge_time_split(bad, STRIDE, NANT, 4096, 64, out)["heaps"] == 1
    assert mixer.merge_time_split(bad, STRIDE, NANT, 0, 64, out)["heaps"] == 8   # port unchecked
    assert mixer.merge_time_split(queues, STRIDE, NANT, 4096, 3, out)["heaps"] == 3   # room for 3
