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
