"""Streaming server (mixer_server_*): continuous batching of concurrent array
streams.  Every dump equals the oracle's FP32-rounded exact int64 V of its
sub-integrations; a stream's dumps are bit-identical alone and in a mix of
other streams submitted in an interleaved order with ragged heap counts;
admission is refused over the memory budget and granted again once a stream
closes; a full staging ring pushes back with EBUSY."""
import time

import numpy as np
import pytest

import mixer
import oracle

pytestmark = pytest.mark.gpu

# (nant, nch, tpkt, ksub, nsub_dump, side)
STREAMS = {
    "A": (256, 128, 32, 256, 3, 16),
    "B": (128, 64, 64, 256, 2, 16),
    "C": (200, 32, 128, 512, 2, 10),
}


def _desc(nant, nch, tpkt, ksub, nsub, side):
    return mixer.make_desc(nant=nant, nch=nch, tpkt=tpkt, ksub=ksub, nsub_dump=nsub, side_x=side,
                           grid=0, pkt_stride=64 + 2 * nch * tpkt, hdr_bytes=64, max_heaps=1)


def _packets(name, ndumps, seed):
    nant, nch, tpkt, ksub, nsub, side = STREAMS[name]
    nheaps = ndumps * nsub * ksub // tpkt
    sky = oracle.sky_table(nant, nch, side, [(0.1, -0.05, 6.0, 0.0)])
    return oracle.gen_packets(nant, nch, tpkt, nheaps, seq0=1000, sky=sky, sigma=16.0, seed=seed)


def _expected_dumps(name, pk, ndumps):
    nant, nch, tpkt, ksub, nsub, side = STREAMS[name]
    hpd = nsub * ksub // tpkt
    stride = 64 + 2 * nch * tpkt
    out = []
    for d in range(ndumps):
        chunk = pk[d * hpd * nant * stride:(d + 1) * hpd * nant * stride]
        full = oracle.correlate(oracle.corner_turn(chunk, nant, nch, tpkt, hpd))
        out.append(full.astype(np.float32))
    return out


def _run(server, names, pks, ndumps, rng, cuda):
    import torch
    ids = {n: server.open(_desc(*STREAMS[n])) for n in names}
    dev = {n: torch.from_numpy(pks[n]).to(cuda) for n in names}
    torch.cuda.synchronize()
    pos = {n: 0 for n in names}
    total = {n: pks[n].size // ((64 + 2 * STREAMS[n][1] * STREAMS[n][2]) * STREAMS[n][0])
             for n in names}
    got = {n: [] for n in names}
    deadline = time.time() + 120
    while any(len(got[n]) < ndumps for n in names):
        assert time.time() < deadline, "server did not deliver the dumps"
        for n in names:
            nant, nch, tpkt = STREAMS[n][:3]
            hb = nant * (64 + 2 * nch * tpkt)
            if pos[n] < total[n]:
                k = int(min(total[n] - pos[n], rng.integers(1, 2 * (STREAMS[n][3] // tpkt) + 2)))
                if server.submit(ids[n], dev[n][pos[n] * hb:], k, seq0=1000, on_device=True):
                    pos[n] += k
            buf = np.empty((nch, 2, nant, nant), dtype=np.float32)
            info = server.poll(ids[n], buf)
            if info is not None:
                assert info["index"] == len(got[n])
                got[n].append(buf)
    for n in names:
        server.close_stream(ids[n])
    return got


def test_server_mix_equals_alone_and_oracle(cuda):
    rng = np.random.default_rng(0)
    ndumps = 2
    pks = {n: _packets(n, ndumps, seed=10 + i) for i, n in enumerate(STREAMS)}
    srv = mixer.Server(budget_bytes=8 << 30, max_streams=8, ring_subs=4, batch_subs=2)
    mixed = _run(srv, list(STREAMS), pks, ndumps, rng, cuda)
    st = srv.stats()
    assert st["kernel_err"] == 0 and st["seq_errors"] == 0
    assert st["dumps"] == ndumps * len(STREAMS)
    assert st["p50_latency_s"] > 0 and st["p99_latency_s"] >= st["p50_latency_s"]
    srv.close()
    exp = _expected_dumps("A", pks["A"], ndumps)
    for d in range(ndumps):
        assert np.array_equal(mixed["A"][d], exp[d])
    for n in ("B", "C"):
        exp = _expected_dumps(n, pks[n], 1)
        assert np.array_equal(mixed[n][0], exp[0])
    srv = mixer.Server(budget_bytes=8 << 30, max_streams=8, ring_subs=4, batch_subs=2)
    alone = _run(srv, ["A"], {"A": pks["A"]}, ndumps, np.random.default_rng(7), cuda)
    srv.close()
    for d in range(ndumps):
        assert np.array_equal(alone["A"][d], mixed["A"][d])


def test_server_admission_by_budget(cuda):
    d = _desc(*STREAMS["B"])
    probe = mixer.Server(budget_bytes=1 << 40, max_streams=8)
    need = probe.stream_bytes(d)
    probe.close()
    srv = mixer.Server(budget_bytes=2 * need + need // 2, max_streams=8)
    a = srv.open(d)
    b = srv.open(d)
    assert srv.try_open(d) is None                    # over budget
    srv.close_stream(a)
    c = srv.try_open(d)                               # memory came back
    assert c is not None
    st = srv.stats()
    assert st["admitted"] == 3 and st["refused"] == 1
    assert st["bytes_used"] == 2 * need
    srv.close_stream(b)
    srv.close_stream(c)
    srv.close()
    slots = mixer.Server(budget_bytes=1 << 40, max_streams=1)
    s0 = slots.open(d)
    assert slots.try_open(d) is None                  # out of slots
    slots.close_stream(s0)
    slots.close()


def test_server_backpressure(cuda):
    import torch
    nant, nch, tpkt, ksub, nsub, side = STREAMS["B"]
    d = _desc(nant, nch, tpkt, 256, 1, side)
    hps = ksub // tpkt
    pk = torch.from_numpy(_packets("B", 4, seed=3)[: 8 * hps * nant * (64 + 2 * nch * tpkt)]).to(cuda)
    hb = nant * (64 + 2 * nch * tpkt)
    srv = mixer.Server(budget_bytes=8 << 30, max_streams=2, ring_subs=2, batch_subs=1)
    sid = srv.open(d)
    accepted = 0
    t0 = time.time()
    # nobody polls: two dumps fill both dump slots, the worker stops, the ring fills
    while accepted < 8 and time.time() - t0 < 20:
        if srv.submit(sid, pk[accepted * hps * hb:], hps, seq0=1000):
            accepted += 1
        else:
            break
        time.sleep(0.05)
    assert accepted < 8                               # pushed back
    got = 0
    t0 = time.time()
    while got < 2 and time.time() - t0 < 20:
        if srv.poll(sid) is not None:
            got += 1
    assert got == 2
    srv.close_stream(sid)
    srv.close()


def test_server_poll_and_close_from_two_threads(cuda):
    """A poller thread copying dumps out while the owner closes the stream:
    close waits for the copy, nothing is freed under it, both calls succeed."""
    import threading
    import torch
    nant, nch, tpkt, ksub, nsub, side = STREAMS["A"]
    d = _desc(nant, nch, tpkt, ksub, 1, side)
    hps = ksub // tpkt
    hb = nant * (64 + 2 * nch * tpkt)
    pk = torch.from_numpy(_packets("A", 1, seed=5)).to(cuda)
    srv = mixer.Server(budget_bytes=8 << 30, max_streams=2, ring_subs=4, batch_subs=1)
    sid = srv.open(d)
    for q in range(2):                                # two dumps of one sub-integration each
        while not srv.submit(sid, pk[q * hps * hb:], hps, seq0=1000, on_device=True):
            time.sleep(0.01)
    errors, polled = [], []
    stop = threading.Event()

    def poller():
        buf = np.empty((nch, 2, nant, nant), dtype=np.float32)
        while not stop.is_set():
            try:
                info = srv.poll(sid, buf)
            except mixer.MixerError:                  # the stream is gone: expected at the end
                break
            except Exception as e:                    # anything else is a failure
                errors.append(e)
                break
            if info is not None:
                polled.append(info["index"])

    t0 = time.time()
    while srv.stats()["dumps"] < 1 and time.time() - t0 < 20:
        time.sleep(0.01)
    th = threading.Thread(target=poller)
    th.start()
    time.sleep(0.05)
    srv.close_stream(sid)
    stop.set()
    th.join()
    assert not errors
    assert polled == sorted(polled) and len(set(polled)) == len(polled)
    st = srv.stats()
    assert st["kernel_err"] == 0 and st["bytes_used"] == 0
    srv.close()


def test_server_refuses_oversize_descriptors(cuda):
    """Admission refuses shapes the work list cannot address (more than 65535
    lower-triangle tiles per channel, i.e. nant > 46208, or more than 65535
    channels) before reserving anything, and the server stays usable."""
    srv = mixer.Server(budget_bytes=1 << 40, max_streams=2, ring_subs=2, batch_subs=1)
    for nant, nch in ((46209, 16), (1024, 65536)):
        d = mixer.make_desc(nant=nant, nch=nch, tpkt=16, ksub=256, nsub_dump=1, side_x=16, grid=0,
                            pkt_stride=64 + 2 * nch * 16, hdr_bytes=64, max_heaps=1)
        with pytest.raises(mixer.MixerError) as e:
            srv.open(d)
        assert e.value.rc == mixer.EINVAL
    assert srv.stats()["bytes_used"] == 0 and srv.stats()["admitted"] == 0
    nant, nch, tpkt, ksub, nsub, side = STREAMS["B"]
    sid = srv.open(_desc(nant, nch, tpkt, ksub, nsub, side))      # a valid shape still opens
    srv.close_stream(sid)
    srv.close()


def test_server_reserve_then_admit(cuda):
    """mixer_server_reserve allocates streams' state ahead of serving; admissions
    of that shape then succeed and their dumps are still exact; a reservation
    for more streams than the server has slots is refused."""
    import torch
    nant, nch, tpkt, ksub, nsub, side = STREAMS["B"]
    d = _desc(nant, nch, tpkt, ksub, nsub, side)
    srv = mixer.Server(budget_bytes=8 << 30, max_streams=2, ring_subs=4, batch_subs=2)
    with pytest.raises(mixer.MixerError) as e:
        srv.reserve(d, 3)
    assert e.value.rc == mixer.EINVAL
    srv.reserve(d, 2)
    assert srv.stats()["bytes_used"] == 0                 # nothing counts until admitted
    pk = _packets("B", 1, seed=9)
    want = _expected_dumps("B", pk, 1)[0]
    dev = torch.from_numpy(pk).to(cuda)
    hps = ksub // tpkt
    hb = nant * (64 + 2 * nch * tpkt)
    sids = [srv.open(d), srv.open(d)]
    for sid in sids:
        for q in range(nsub):
            while not srv.submit(sid, dev[q * hps * hb:], hps, seq0=1000, on_device=True):
                time.sleep(0.005)
    buf = np.empty((nch, 2, nant, nant), dtype=np.float32)
    for sid in sids:
        t0 = time.time()
        while True:
            info = srv.poll(sid, buf)
            if info is not None:
                break
            assert time.time() - t0 < 30, "no dump"
            time.sleep(0.005)
        assert np.array_equal(buf, want)
        srv.close_stream(sid)
    st = srv.stats()
    assert st["kernel_err"] == 0 and st["seq_errors"] == 0 and st["bytes_used"] == 0
    srv.close()
