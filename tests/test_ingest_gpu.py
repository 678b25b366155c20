"""Checkpoint / resume of the int64 integration state: integrate, save, resume
in a fresh context, integrate the rest -- identical to one uninterrupted run
(the reference cannot resume: its float cube is zeroed once,
src/rx_host_corr.cu:188)."""
import numpy as np
import pytest

import mixer
import oracle

pytestmark = pytest.mark.gpu


def test_checkpoint_resume_is_exact(cuda, tmp_path):
    import torch
    nant, nch, tpkt = 256, 128, 32
    pk = oracle.gen_packets(nant, nch, tpkt, 16, sky=oracle.sky_table(nant, nch, 16, [(0.1, 0.0, 6.0, 0.0)]),
                            sigma=16.0, seed=77)
    hb = nant * (64 + 2 * nch * tpkt)
    dpk = torch.from_numpy(pk).to(cuda)
    full = oracle.correlate(oracle.corner_turn(pk, nant, nch, tpkt, 16))
    path = str(tmp_path / "state.ckpt")
    with mixer.ArrayContext(max_heaps=8) as a:
        a.correlate(dpk, 8, seq0=0)
        torch.cuda.synchronize()
        a.save(path)
    with mixer.ArrayContext(max_heaps=8) as b:
        b.load(path)
        assert b.stats()["samples"] == 8 * tpkt
        b.correlate(dpk[8 * hb:], 8, seq0=8 * nant)
        out = torch.zeros(full.size, dtype=torch.int64, device=cuda)
        b.read_vis_i64(out, full_square=True)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().reshape(full.shape), full)
        assert b.stats()["samples"] == 16 * tpkt
    with mixer.ArrayContext(nant=128, max_heaps=8) as c:   # other shape: refused
        with pytest.raises(mixer.MixerError) as e:
            c.load(path)
        assert e.value.rc == mixer.EINVAL


def test_time_split_queues_merge_and_correlate_exactly(cuda):
    """Four time-split RX queues (heap tb on queue tb % 4, UDP port 4096 + q) merged on
    the host and correlated from host memory: the same cube as the oracle's on the
    unsplit burst, with no sequence errors."""
    import torch
    nant, nch, tpkt, nheaps, nq = 256, 128, 32, 16, 4
    stride = 64 + 2 * nch * tpkt
    pk = oracle.gen_packets(nant, nch, tpkt, nheaps, sigma=16.0, seed=31).reshape(nheaps, nant, stride)
    for h in range(nheaps):
        pk[h, :, 36] = (4096 + h % nq) >> 8
        pk[h, :, 37] = (4096 + h % nq) & 0xFF
    queues = [np.ascontiguousarray(pk[q::nq]).reshape(-1) for q in range(nq)]
    merged = torch.empty(nheaps * nant * stride, dtype=torch.uint8, pin_memory=True)
    r = mixer.merge_time_split(queues, stride, nant, 4096, nheaps, merged.numpy())
    assert r["heaps"] == nheaps and r["seq0"] == 0
    full = oracle.correlate(oracle.corner_turn(pk.reshape(-1), nant, nch, tpkt, nheaps))
    with mixer.ArrayContext(max_heaps=8) as ctx:
        ctx.correlate(merged, nheaps, seq0=r["seq0"], on_device=False)
        out = torch.zeros(full.size, dtype=torch.int64, device=cuda)
        ctx.read_vis_i64(out, full_square=True)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().reshape(full.shape), full)
        st = ctx.stats()
        assert st["seq_errors"] == 0 and st["kernel_err"] == 0
