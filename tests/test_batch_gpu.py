"""Batched persistent launch over uneven arrays (mixer_batch_*): every plan --
any K-split per size class, either item order, the autotuned plan and a CUDA
graph replay -- gives visibilities bit-identical to one mixer_xcorr_tri per
array and to the oracle."""
import numpy as np
import pytest

import mixer
import oracle

pytestmark = pytest.mark.gpu

SHAPES = [  # (N, C, K)
    (64, 3, 256), (96, 2, 512), (130, 2, 384), (200, 1, 1024), (256, 4, 256),
    (384, 1, 640), (40, 5, 128), (128, 2, 2048),
]


def _problems(cuda, mode=mixer.VIS_ACC_I64, shapes=SHAPES, seed=0):
    import torch
    rng = np.random.default_rng(seed)
    out = []
    for n, c, k in shapes:
        planes = rng.integers(-128, 128, size=(2, c, n, k), dtype=np.int8)
        dtype = torch.int64 if mode == mixer.VIS_ACC_I64 else torch.int32
        out.append({"planes_np": planes, "planes": torch.from_numpy(planes).to(cuda), "nant": n,
                    "nch": c, "kt": k, "kbeg": 0, "klen": k, "mode": mode,
                    "vis": torch.zeros(mixer.vis_elems(n, c), dtype=dtype, device=cuda)})
    return out


def _refs(probs):
    return [oracle.vis_tile_pack(oracle.correlate(p["planes_np"])).reshape(-1) for p in probs]


def _check(probs, refs, times=1):
    import torch
    torch.cuda.synchronize()
    for p, r in zip(probs, refs):
        assert np.array_equal(p["vis"].cpu().numpy().astype(np.int64), times * r), (p["nant"], p["nch"])


def _zero(probs):
    for p in probs:
        p["vis"].zero_()


@pytest.mark.parametrize("split,order", [
    ([1] * 65, mixer.ORDER_LPT), ([1] * 65, mixer.ORDER_CHANNEL),
    ([3] * 65, mixer.ORDER_LPT), ([1, 2, 4, 8, 16] + [1] * 60, mixer.ORDER_CHANNEL),
])
def test_batch_plans_bit_exact(cuda, split, order):
    probs = _problems(cuda)
    refs = _refs(probs)
    b = mixer.Batch(probs)
    b.plan(split, order)
    b.run()
    _check(probs, refs)
    info = b.info()
    assert info["kernel_err"] == 0 and info["order"] == order
    b.close()


def test_batch_equals_plain_launches(cuda):
    import torch
    probs = _problems(cuda, seed=3)
    plain = [torch.zeros_like(p["vis"]) for p in probs]
    for p, v in zip(probs, plain):
        mixer.xcorr_tri(p["planes"], p["nant"], p["nch"], p["kt"], 0, p["kt"], mixer.VIS_ACC_I64, v)
    b = mixer.Batch(probs)
    b.plan([2] * 65, mixer.ORDER_LPT)
    b.run()
    torch.cuda.synchronize()
    for p, v in zip(probs, plain):
        assert torch.equal(p["vis"], v)
    b.close()


def test_batch_autotune_then_graph_replay(cuda):
    import torch
    probs = _problems(cuda, seed=5)
    refs = _refs(probs)
    b = mixer.Batch(probs)
    ms = b.autotune(reps=1)
    assert ms > 0
    _zero(probs)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b.capture_graph(s)
        b.replay(s)
        b.replay(s)
    s.synchronize()
    _check(probs, refs, times=2)
    assert b.info()["kernel_err"] == 0
    b.close()


def test_batch_mixed_modes_and_long_k(cuda):
    import torch
    rng = np.random.default_rng(9)
    p32 = _problems(cuda, mode=mixer.VIS_STORE_I32, shapes=[(130, 2, 256)], seed=1)
    a32 = _problems(cuda, mode=mixer.VIS_ACC_I32, shapes=[(256, 1, 512)], seed=2)
    n, c, k = 128, 1, 65408 + 2048          # longer than one int32-safe item: forced split
    planes = rng.integers(-128, 128, size=(2, c, n, k), dtype=np.int8)
    big = [{"planes_np": planes, "planes": torch.from_numpy(planes).to(cuda), "nant": n, "nch": c,
            "kt": k, "kbeg": 0, "klen": k, "mode": mixer.VIS_ACC_I64,
            "vis": torch.zeros(mixer.vis_elems(n, c), dtype=torch.int64, device=cuda)}]
    probs = p32 + a32 + big
    refs = _refs(probs)
    b = mixer.Batch(probs)
    b.plan([4] * 65, mixer.ORDER_LPT)        # STORE item stays unsplit
    b.run()
    _check(probs, refs)
    b.close()


def test_batch_rejects_bad_problems(cuda):
    import torch
    v = torch.zeros(16, dtype=torch.int32, device=cuda)
    pl = torch.zeros(64, dtype=torch.int8, device=cuda)
    with pytest.raises(mixer.MixerError) as e:
        mixer.Batch([{"planes": pl, "nant": 128, "nch": 1, "kt": 100000, "klen": 100000,
                      "mode": mixer.VIS_ACC_I32, "vis": v}])
    assert e.value.rc == mixer.EOVERFLOW
    with pytest.raises(mixer.MixerError) as e:
        mixer.Batch([{"planes": pl, "nant": 128, "nch": 1, "kt": 100, "klen": 100,
                      "mode": mixer.VIS_ACC_I64, "vis": v}])
    assert e.value.rc == mixer.EINVAL


@pytest.mark.parametrize("split", [1, 3])
def test_batch_large_arrays_several_subintegrations(cuda, split):
    """Arrays of the 48-array workload's sizes (N up to 1024, C up to 512), each
    item contracting S = 4 sub-integrations of the array's K in one int32 TMEM
    accumulation, against one mixer_xcorr_tri per array and sub-integration and
    against the oracle on the first and last channel of every array.  With
    split 3 the items share tiles (atomic epilogue); with split 1 each owns its
    tile."""
    import torch
    S = 4
    shapes = [(992, 352, 1024), (1024, 48, 512), (160, 512, 256), (608, 16, 1280)]   # (N, C, K)
    g = torch.Generator(device=cuda).manual_seed(11)
    probs, plain = [], []
    for n, c, k in shapes:
        planes = torch.randint(-127, 128, (2 * c * n * S * k,), dtype=torch.int8, device=cuda,
                               generator=g)
        probs.append({"planes": planes, "nant": n, "nch": c, "kt": S * k, "kbeg": 0, "klen": S * k,
                      "mode": mixer.VIS_ACC_I64,
                      "vis": torch.zeros(mixer.vis_elems(n, c), dtype=torch.int64, device=cuda)})
        plain.append(torch.zeros(mixer.vis_elems(n, c), dtype=torch.int64, device=cuda))
    for p, v in zip(probs, plain):
        for s in range(S):
            mixer.xcorr_tri(p["planes"], p["nant"], p["nch"], p["kt"], s * p["klen"] // S,
                            p["klen"] // S, mixer.VIS_ACC_I64, v)
    b = mixer.Batch(probs)
    b.plan([split] * 65, mixer.ORDER_LPT)
    b.run()
    torch.cuda.synchronize()
    assert b.info()["kernel_err"] == 0
    for p, v in zip(probs, plain):
        assert torch.equal(p["vis"], v), (p["nant"], p["nch"])
        n, c = p["nant"], p["nch"]
        per = mixer.vis_elems(n, 1)
        for ch in (0, c - 1):
            pl = p["planes"].view(2, c, n, -1)[:, ch:ch + 1].cpu().numpy()
            want = oracle.vis_tile_pack(oracle.correlate(pl)).reshape(-1)
            got = p["vis"][ch * per:(ch + 1) * per].cpu().numpy()
            assert np.array_equal(got, want), (n, c, ch)
    b.close()
