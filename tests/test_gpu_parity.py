"""GPU parity: every kernel of the X-engine against the CPU oracle (bit-exact for
all integer work) and against the reference's own kernels compiled from its
sources (k_packAB + cgemm_blk_t, src/rx_host_corr.cu:61-72, src/cgemm.cuh:28-69).

Floating-point tolerances, stated here and used below:
  * FP32 dump cube vs exact int64: each entry is the single correctly rounded
    FP32 value (bit-exact against numpy's float32 cast).
  * FP32 image vs FP64 oracle: max |img - img64| <= 1e-5 * max |img64|.
"""
import numpy as np
import pytest

import mixer
import oracle

pytestmark = pytest.mark.gpu


def _t(arr, cuda):
    import torch
    return torch.from_numpy(np.ascontiguousarray(arr)).to(cuda)


def _zeros(n, dtype, cuda):
    import torch
    return torch.zeros(n, dtype=dtype, device=cuda)


def _sync():
    import torch
    torch.cuda.synchronize()


# ---------------------------------------------------------------- packet source

@pytest.mark.parametrize("nant,nch,tpkt,nheaps,mode,sigma", [
    (256, 128, 32, 4, 0, 16.0),
    (40, 64, 64, 3, 0, 12.0),
    (32, 256, 16, 2, 1, 0.0),
])
def test_gen_packets_match_oracle(cuda, nant, nch, tpkt, nheaps, mode, sigma):
    import torch
    sky = oracle.sky_table(nant, nch, 16, [(0.10, -0.05, 6.0, 0.0), (0.2, 0.0, 0.0, 1.5)])
    sky_m = mixer.sky_table(nant, nch, 16, [(0.10, -0.05, 6.0, 0.0), (0.2, 0.0, 0.0, 1.5)])
    assert np.array_equal(sky, sky_m)
    stride = 64 + 2 * nch * tpkt
    dev = _zeros(nheaps * nant * stride, torch.uint8, cuda)
    dsky = _t(sky, cuda)
    mixer.gen_packets(dev, stride, 64, nant, nch, tpkt, nheaps, 3, 77, 4096, dsky, sigma, 1234, mode)
    _sync()
    ref = oracle.gen_packets(nant, nch, tpkt, nheaps, heap0=3, seq0=77, sky=sky, sigma=sigma,
                             seed=1234, mode=mode)
    assert np.array_equal(dev.cpu().numpy(), ref)


# ------------------------------------------------------------------ corner-turn

@pytest.mark.parametrize("nant,nch,tpkt,nheaps,k0,extra", [
    (256, 128, 32, 8, 0, 0),      # wire default, one 256-sample sub-integration
    (96, 64, 64, 4, 128, 64),     # offset into a wider plane
    (128, 256, 16, 16, 0, 0),     # 256-channel packets
    (40, 16, 16, 3, 16, 32),      # heaps not a multiple of any group
])
def test_corner_turn_matches_oracle(cuda, nant, nch, tpkt, nheaps, k0, extra):
    import torch
    pk = oracle.gen_packets(nant, nch, tpkt, nheaps, seq0=9, seed=5, sigma=30.0)
    stride = 64 + 2 * nch * tpkt
    kt = k0 + nheaps * tpkt + extra
    dpk = _t(pk, cuda)
    planes = torch.full((2, nch, nant, kt), 7, dtype=torch.int8, device=cuda)
    seq_err = _zeros(1, torch.int32, cuda)
    err = _zeros(1, torch.int32, cuda)
    mixer.corner_turn(dpk, stride, 64, nant, nch, tpkt, nheaps, 9, planes, kt, k0, seq_err, err)
    _sync()
    got = planes.cpu().numpy()
    ref = oracle.corner_turn(pk, nant, nch, tpkt, nheaps)
    assert np.array_equal(got[:, :, :, k0:k0 + nheaps * tpkt], ref)
    assert np.all(got[:, :, :, :k0] == 7) and np.all(got[:, :, :, k0 + nheaps * tpkt:] == 7)
    assert int(seq_err.item()) == 0 and int(err.item()) == 0


def test_corner_turn_counts_seq_errors(cuda):
    import torch
    nant, nch, tpkt, nheaps = 64, 128, 32, 4
    stride = 64 + 2 * nch * tpkt
    pk = oracle.gen_packets(nant, nch, tpkt, nheaps, seq0=100)
    v = pk.reshape(-1, stride)
    v[5, 51] ^= 0x10          # one corrupted seq
    v[[70, 71]] = v[[71, 70]]  # two packets swapped
    planes = _zeros(2 * nch * nant * nheaps * tpkt, torch.int8, cuda)
    seq_err = _zeros(1, torch.int32, cuda)
    mixer.corner_turn(_t(pk, cuda), stride, 64, nant, nch, tpkt, nheaps, 100, planes,
                      nheaps * tpkt, 0, seq_err)
    _sync()
    assert int(seq_err.item()) == 3 == oracle.seq_errors(pk, nheaps * nant, 100, stride)


# --------------------------------------------------------- tensor-core triangle GEMM

def _rand_planes(rng, nch, nant, kt, lo=-128, hi=128):
    return rng.integers(lo, hi, size=(2, nch, nant, kt), dtype=np.int8)


@pytest.mark.parametrize("nant,nch,kt,kbeg,klen", [
    (128, 2, 128, 0, 128),
    (256, 3, 512, 0, 512),
    (200, 2, 384, 0, 384),      # N not a multiple of the tile
    (40, 5, 64, 0, 64),         # K shorter than one stage
    (384, 2, 256, 0, 256),      # 6 tiles per channel, 3 diagonal
    (256, 2, 512, 128, 256),    # sample sub-range
    (130, 1, 208, 16, 176),     # ragged: N = 128 + 2, K not a multiple of 128
])
def test_xcorr_store_i32_matches_oracle(cuda, nant, nch, kt, kbeg, klen):
    import torch
    rng = np.random.default_rng(nant * 7 + kt)
    planes = _rand_planes(rng, nch, nant, kt)
    vis = _zeros(mixer.vis_elems(nant, nch), torch.int32, cuda)
    err = _zeros(1, torch.int32, cuda)
    mixer.xcorr_tri(_t(planes, cuda), nant, nch, kt, kbeg, klen, mixer.VIS_STORE_I32, vis, err)
    _sync()
    assert int(err.item()) == 0
    full = oracle.correlate(planes, kbeg=kbeg, klen=klen)
    ref = oracle.vis_tile_pack(full).reshape(-1)
    got = vis.cpu().numpy().astype(np.int64)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("nant", [1, 15, 16, 17, 100, 129, 143, 160, 241, 255, 257, 300, 383, 1000])
@pytest.mark.parametrize("mode", ["store", "acc32", "acc64"])
def test_xcorr_ragged_last_block_matches_oracle(cuda, nant, mode):
    """N not a multiple of 128: the last block's tiles run with that block on
    the MMA's N side (N = 2 r16, r16 = rows rounded up to 16), the tiles left
    of the diagonal as conjugate transposes written back transposed.  Every
    rounding class of the last block, each mode, -128 rows in the ragged
    block; store mode rewrites the padding rows (the cube starts as junk),
    the accumulate modes add twice."""
    import torch
    rng = np.random.default_rng(nant * 3 + len(mode))
    nch, kt = 2, 384
    planes = _rand_planes(rng, nch, nant, kt)
    planes[:, :, -min(nant, 5):, ::3] = -128
    dpl = _t(planes, cuda)
    n = mixer.vis_elems(nant, nch)
    err = _zeros(1, torch.int32, cuda)
    ref = oracle.vis_tile_pack(oracle.correlate(planes)).reshape(-1)
    if mode == "store":
        vis = torch.full((n,), 0x5A5A5A5A, dtype=torch.int32, device=cuda)
        mixer.xcorr_tri(dpl, nant, nch, kt, 0, kt, mixer.VIS_STORE_I32, vis, err)
        times = 1
    else:
        dt = torch.int64 if mode == "acc64" else torch.int32
        md = mixer.VIS_ACC_I64 if mode == "acc64" else mixer.VIS_ACC_I32
        vis = _zeros(n, dt, cuda)
        for _ in range(2):
            mixer.xcorr_tri(dpl, nant, nch, kt, 0, kt, md, vis, err)
        times = 2
    _sync()
    assert int(err.item()) == 0
    assert np.array_equal(vis.cpu().numpy().astype(np.int64), times * ref)


def test_xcorr_accumulate_modes(cuda):
    import torch
    rng = np.random.default_rng(11)
    nant, nch, kt = 256, 4, 1024
    planes = _rand_planes(rng, nch, nant, kt)
    dpl = _t(planes, cuda)
    n = mixer.vis_elems(nant, nch)
    v32 = _zeros(n, torch.int32, cuda)
    v64 = _zeros(n, torch.int64, cuda)
    for k in range(0, kt, 256):
        mixer.xcorr_tri(dpl, nant, nch, kt, k, 256, mixer.VIS_ACC_I32, v32)
        mixer.xcorr_tri(dpl, nant, nch, kt, k, 256, mixer.VIS_ACC_I64, v64)
    _sync()
    ref = oracle.vis_tile_pack(oracle.correlate(planes)).reshape(-1)
    assert np.array_equal(v32.cpu().numpy().astype(np.int64), ref)
    assert np.array_equal(v64.cpu().numpy(), ref)
    # flush: v64 += v32, v32 = 0  (k_flush_cube, exact)
    mixer.vis_flush(v32, v64, n)
    _sync()
    assert np.array_equal(v64.cpu().numpy(), 2 * ref)
    assert int(v32.abs().max().item()) == 0


@pytest.mark.parametrize("pairs", ["0", "1"])
@pytest.mark.parametrize("max_ctas", [1, 7, 100000])
def test_xcorr_cta_cap_is_exact(cuda, monkeypatch, max_ctas, pairs):
    """mixer_xcorr_tri_ex: fewer persistent CTAs walk more items each, same cube
    (one-SM kernel, and the pair kernel with max_ctas / 2 clusters)."""
    import torch
    monkeypatch.setenv("MIXER_XCORR_PAIRS", pairs)
    rng = np.random.default_rng(31 + max_ctas)
    nant, nch, kt = 384, 3, 512
    planes = _rand_planes(rng, nch, nant, kt)
    v64 = _zeros(mixer.vis_elems(nant, nch), torch.int64, cuda)
    err = _zeros(1, torch.int32, cuda)
    mixer.xcorr_tri(_t(planes, cuda), nant, nch, kt, 0, kt, mixer.VIS_ACC_I64, v64, err,
                    max_ctas=max_ctas)
    _sync()
    assert int(err.item()) == 0
    ref = oracle.vis_tile_pack(oracle.correlate(planes)).reshape(-1)
    assert np.array_equal(v64.cpu().numpy(), ref)


@pytest.mark.parametrize("nant,nch,kt,kbeg,klen,mode", [
    (384, 3, 512, 0, 512, "store"),      # 3 row blocks: 3 pairs, one leftover pair
    (512, 2, 256, 0, 256, "acc64"),      # 4 blocks: 5 pairs
    (640, 2, 384, 128, 256, "store"),    # 5 blocks: last leftover pair has one tile
    (1000, 2, 208, 16, 176, "acc64"),    # 8 blocks, ragged N and K
    (1024, 4, 1024, 0, 1024, "acc32"),   # 8 blocks, 18 pairs per channel
])
def test_xcorr_pairs_match_oracle(cuda, monkeypatch, nant, nch, kt, kbeg, klen, mode):
    """MIXER_XCORR_PAIRS=1: from three 128-row blocks up the GEMM runs on pairs
    of SMs (tcgen05 cta_group::2): two tiles that share a column block per
    cluster, leftover tiles as conjugate-transposed products.  Every mode is
    exact."""
    import torch
    monkeypatch.setenv("MIXER_XCORR_PAIRS", "1")
    rng = np.random.default_rng(nant + kt + klen)
    planes = _rand_planes(rng, nch, nant, kt)
    dt = torch.int64 if mode == "acc64" else torch.int32
    vis = _zeros(mixer.vis_elems(nant, nch), dt, cuda)
    err = _zeros(1, torch.int32, cuda)
    md = {"store": mixer.VIS_STORE_I32, "acc32": mixer.VIS_ACC_I32, "acc64": mixer.VIS_ACC_I64}[mode]
    mixer.xcorr_tri(_t(planes, cuda), nant, nch, kt, kbeg, klen, md, vis, err)
    _sync()
    assert int(err.item()) == 0
    ref = oracle.vis_tile_pack(oracle.correlate(planes, kbeg=kbeg, klen=klen)).reshape(-1)
    assert np.array_equal(vis.cpu().numpy().astype(np.int64), ref)


def test_xcorr_pairs_equal_single_sm(cuda, monkeypatch):
    """The pair kernel (MIXER_XCORR_PAIRS=1) and the one-SM kernel give the same
    cube, including -128 inputs and the int32 bound of one launch."""
    import torch
    rng = np.random.default_rng(77)
    nant, nch, kt = 768, 2, 65408
    planes = rng.integers(-128, 128, size=(2, nch, nant, kt), dtype=np.int8)
    planes[:, :, :128] = -128                        # one row block at the extreme
    dpl = _t(planes, cuda)
    n = mixer.vis_elems(nant, nch)
    out = []
    for env in ("1", "0"):
        monkeypatch.setenv("MIXER_XCORR_PAIRS", env)
        v = _zeros(n, torch.int32, cuda)
        err = _zeros(1, torch.int32, cuda)
        mixer.xcorr_tri(dpl, nant, nch, kt, 0, kt, mixer.VIS_STORE_I32, v, err)
        _sync()
        assert int(err.item()) == 0
        out.append(v.cpu().numpy())
    assert np.array_equal(out[0], out[1])
    ref = oracle.vis_tile_pack(oracle.correlate(planes, nc=1)).reshape(-1)
    assert np.array_equal(out[0][:ref.size].astype(np.int64), ref)


def test_xcorr_partial_last_round_is_exact(cuda):
    """256 elements x 128 channels = 384 tile items on 148 persistent CTAs: the
    last round is partly empty and two thirds of the tiles are diagonal.  The
    int64 accumulate and int32 store launches give the same cube, equal to the
    oracle's exact sums on the first channels."""
    import torch
    rng = np.random.default_rng(41)
    nant, nch, kt = 256, 128, 16384
    planes = _rand_planes(rng, nch, nant, kt)
    dpl = _t(planes, cuda)
    n = mixer.vis_elems(nant, nch)
    v32 = _zeros(n, torch.int32, cuda)
    v64 = _zeros(n, torch.int64, cuda)
    err = _zeros(1, torch.int32, cuda)
    mixer.xcorr_tri(dpl, nant, nch, kt, 0, kt, mixer.VIS_STORE_I32, v32, err)
    mixer.xcorr_tri(dpl, nant, nch, kt, 0, kt, mixer.VIS_ACC_I64, v64, err)
    _sync()
    assert int(err.item()) == 0
    assert np.array_equal(v64.cpu().numpy(), v32.cpu().numpy().astype(np.int64))
    sub = 4                                                # oracle on the first channels
    ref = oracle.vis_tile_pack(oracle.correlate(planes, nc=sub)).reshape(-1)
    assert np.array_equal(v64[:ref.size].cpu().numpy(), ref)


@pytest.mark.parametrize("pairs", ["0", "1"])
def test_xcorr_large_array_matches_oracle(cuda, monkeypatch, pairs):
    """4096 elements (32 row blocks, 528 tiles per channel, tile indices past
    the float decode's easy range) and 4000 (ragged last block), int64 mode,
    one-SM and pair kernels."""
    import torch
    monkeypatch.setenv("MIXER_XCORR_PAIRS", pairs)
    for nant in (4096, 4000):
        rng = np.random.default_rng(nant)
        nch, kt = 1, 384
        planes = _rand_planes(rng, nch, nant, kt)
        v64 = _zeros(mixer.vis_elems(nant, nch), torch.int64, cuda)
        err = _zeros(1, torch.int32, cuda)
        mixer.xcorr_tri(_t(planes, cuda), nant, nch, kt, 0, kt, mixer.VIS_ACC_I64, v64, err)
        _sync()
        assert int(err.item()) == 0
        ref = oracle.vis_tile_pack(oracle.correlate(planes)).reshape(-1)
        assert np.array_equal(v64.cpu().numpy(), ref), nant


def test_mma_peak_probe(cuda):
    """The tensor-core rate probe runs its MMA stream to completion."""
    import torch
    err = _zeros(1, torch.int32, cuda)
    mixer.mma_peak(200, 0, err)
    mixer.mma_peak(50, 3, err)
    _sync()
    assert int(err.item()) == 0


def test_xcorr_extreme_inputs(cuda):
    """-128 everywhere: exact here; the reference's -A_im (src/cgemm.cuh:52) wraps."""
    import torch
    nant, nch, kt = 128, 1, 65408                      # largest int32-safe launch
    planes = np.full((2, nch, nant, kt), -128, dtype=np.int8)
    planes[1, 0, ::2] = 127
    vis = _zeros(mixer.vis_elems(nant, nch), torch.int32, cuda)
    mixer.xcorr_tri(_t(planes, cuda), nant, nch, kt, 0, kt, mixer.VIS_STORE_I32, vis)
    _sync()
    ref = oracle.vis_tile_pack(oracle.correlate(planes)).reshape(-1)
    assert np.array_equal(vis.cpu().numpy().astype(np.int64), ref)
    assert ref.max() == 2 * 128 * 128 * kt


def test_xcorr_long_integration_splits(cuda):
    """I64 mode over more samples than one int32-safe launch."""
    import torch
    rng = np.random.default_rng(2)
    nant, nch, kt = 128, 1, 65408 + 1024
    planes = rng.integers(-128, 128, size=(2, nch, nant, kt), dtype=np.int8)
    v64 = _zeros(mixer.vis_elems(nant, nch), torch.int64, cuda)
    mixer.xcorr_tri(_t(planes, cuda), nant, nch, kt, 0, kt, mixer.VIS_ACC_I64, v64)
    _sync()
    ref = oracle.vis_tile_pack(oracle.correlate(planes)).reshape(-1)
    assert np.array_equal(v64.cpu().numpy(), ref)


# ------------------------------------------------------------- cube outputs

def test_unpack_and_dump(cuda):
    import torch
    rng = np.random.default_rng(8)
    nant, nch, kt = 300, 3, 256
    planes = _rand_planes(rng, nch, nant, kt)
    full = oracle.correlate(planes) * 40000               # values beyond 2^24
    packed = _t(oracle.vis_tile_pack(full).reshape(-1), cuda)
    out64 = _zeros(nch * 2 * nant * nant, torch.int64, cuda)
    out32 = _zeros(nch * 2 * nant * nant, torch.float32, cuda)
    mixer.vis_unpack_i64(packed, nant, nch, out64)
    mixer.vis_dump_f32(packed, nant, nch, out32)
    _sync()
    assert np.array_equal(out64.cpu().numpy().reshape(full.shape), full)
    assert np.array_equal(out32.cpu().numpy().reshape(full.shape), full.astype(np.float32))


# ------------------------------------------------------------- context pipeline

def _config0_packets(nheaps, heap0=0, seed=99, nant=256, nch=128, tpkt=32, side=16):
    sky = oracle.sky_table(nant, nch, side, [(0.10, -0.05, 6.0, 0.0), (0.2, 0.0, 0.0, 1.5)])
    return oracle.gen_packets(nant, nch, tpkt, nheaps, heap0=heap0, seq0=heap0 * nant, sky=sky,
                              sigma=16.0, seed=seed)


def test_context_device_and_host_packets(cuda):
    import torch
    nheaps = 24
    pk = _config0_packets(nheaps)
    full = oracle.correlate(oracle.corner_turn(pk, 256, 128, 32, nheaps))
    with mixer.ArrayContext(max_heaps=8) as ctx:
        ctx.correlate(_t(pk, cuda), nheaps, seq0=0, on_device=True)       # 3 chunks
        out = _zeros(full.size, torch.int64, cuda)
        ctx.read_vis_i64(out, full_square=True)
        _sync()
        assert np.array_equal(out.cpu().numpy().reshape(full.shape), full)
        # same packets again from pageable and pinned host memory: doubles V
        ctx.correlate(pk, nheaps, seq0=0, on_device=False)
        pinned = torch.from_numpy(pk).pin_memory()
        ctx.correlate(pinned, nheaps, seq0=0, on_device=False)
        host = np.zeros(full.size, dtype=np.int64)
        ctx.read_vis_i64(host, full_square=True, on_device=False)
        _sync()
        assert np.array_equal(host.reshape(full.shape), 3 * full)
        st = ctx.stats()
        assert st["seq_errors"] == 0 and st["kernel_err"] == 0
        assert st["samples"] == 3 * nheaps * 32


def test_context_int32_split_and_dump(cuda, tmp_path):
    import torch
    nheaps = 16
    pk = _config0_packets(nheaps, seed=4)
    full = oracle.correlate(oracle.corner_turn(pk, 256, 128, 32, nheaps))
    with mixer.ArrayContext(max_heaps=16) as ctx:
        dpk = _t(pk, cuda)
        ctx.correlate_i32(dpk, 8, seq0=0)
        ctx.correlate_i32(dpk[8 * 256 * 8256:], 8, seq0=8 * 256)
        ctx.integrate()
        with pytest.raises(mixer.MixerError) as e:     # int32 headroom is enforced
            for _ in range(300):
                ctx.correlate_i32(dpk, 16, seq0=0)
        assert e.value.rc == mixer.EOVERFLOW
        ctx.reset()
        ctx.correlate_i32(dpk, 16, seq0=0)
        ctx.integrate()
        cube = torch.zeros(full.size, dtype=torch.float32, device=cuda)
        ctx.dump(cube)
        path = str(tmp_path / "v.f32")
        ctx.dump_to_file(path)
        ctx.dump_to_file(path)
        _sync()
        ref32 = full.astype(np.float32)
        assert np.array_equal(cube.cpu().numpy().reshape(full.shape), ref32)
        rec = np.fromfile(path, dtype=np.float32)
        assert rec.size == 2 * full.size
        assert np.array_equal(rec[:full.size].reshape(full.shape), ref32)


def test_context_detects_misordered_packets(cuda):
    nheaps = 8
    pk = _config0_packets(nheaps, seed=3).reshape(-1, 8256).copy()
    pk[[3, 4]] = pk[[4, 3]]
    with mixer.ArrayContext(max_heaps=8) as ctx:
        ctx.correlate(pk.reshape(-1), nheaps, seq0=0, on_device=False)
        assert ctx.stats()["seq_errors"] == 2


# ------------------------------------------------------------------- imaging

@pytest.mark.parametrize("nant,side,G,nch", [(256, 16, 32, 8), (1024, 32, 64, 2), (64, 8, 16, 3),
                                             (4096, 64, 128, 1)])
def test_grid_and_image(cuda, nant, side, G, nch):
    import torch
    rng = np.random.default_rng(nant)
    kt = 64
    planes = rng.integers(-100, 100, size=(2, nch, nant, kt), dtype=np.int8)
    full = oracle.correlate(planes)
    packed = _t(oracle.vis_tile_pack(full).reshape(-1), cuda)
    g = _zeros(nch * G * G * 2, torch.int64, cuda)
    mixer.grid(packed, nant, nch, side, G, g)
    img = _zeros(nch * G * G, torch.float32, cuda)
    vmax = _zeros(nch, torch.float32, cuda)
    vmin = _zeros(nch, torch.float32, cuda)
    mixer.image_fft(g, nch, G, img, vmax, vmin)
    _sync()
    gref = oracle.grid(full, side, G)
    assert np.array_equal(g.cpu().numpy().reshape(gref.shape), gref)
    i64 = oracle.image64(gref)
    got = img.cpu().numpy().reshape(i64.shape)
    for c in range(nch):
        err = np.abs(got[c] - i64[c]).max() / np.abs(i64[c]).max()
        assert err <= 1e-5, (c, err)
    assert np.array_equal(vmax.cpu().numpy(), got.reshape(nch, -1).max(1))
    assert np.array_equal(vmin.cpu().numpy(), got.reshape(nch, -1).min(1))


def test_delta_image_and_context_image(cuda):
    import torch
    pk = _config0_packets(8, seed=21)
    with mixer.ArrayContext(max_heaps=8) as ctx:
        img = torch.zeros(128 * 32 * 32, dtype=torch.float32, device=cuda)
        ctx.correlate(_t(pk, cuda), 8, seq0=0)
        ctx.image(img, delta=True)
        _sync()
        first = img.cpu().numpy().copy()
        ctx.correlate(_t(pk, cuda), 8, seq0=0)
        ctx.image(img, delta=True)                      # change since last image == first
        _sync()
        assert np.array_equal(img.cpu().numpy(), first)
        ctx.image(img, delta=False)                     # integrated == 2 x first
        _sync()
        full = 2 * oracle.correlate(oracle.corner_turn(pk, 256, 128, 32, 8))
        ref = oracle.image64(oracle.grid(full, 16, 32))
        got = img.cpu().numpy().reshape(ref.shape)
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


# ------------------------------------------------- the reference's own GPU kernels

def _ref_v_update(cuda, pk):
    """k_packAB + cgemm_blk_t<false> on one V-update (32 heaps x 256 antennas)."""
    import torch
    if not oracle.ref_gpu_available():
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    ref = oracle.ref_gpu()
    assert ref.ref_const(3) == 32 and ref.ref_const(4) == 1024
    bb = torch.from_numpy(pk.reshape(32 * 256, 8256)[:, 64:].copy()).to(cuda)   # header strip
    planes = [torch.zeros(128 * 256 * 1024, dtype=torch.int8, device=cuda) for _ in range(4)]
    cre = torch.zeros(128 * 256 * 256, dtype=torch.int32, device=cuda)
    cim = torch.zeros_like(cre)
    s = torch.cuda.current_stream().cuda_stream
    assert ref.ref_pack(bb.data_ptr(), *[p.data_ptr() for p in planes], s) == 0
    assert ref.ref_cgemm(0, 256, 256, 1024, 128, *[p.data_ptr() for p in planes], cre.data_ptr(),
                         cim.data_ptr(), s) == 0
    _sync()
    return planes, cre, cim


def test_matches_reference_gpu_kernels(cuda):
    import torch
    pk = _config0_packets(32, seed=2024)
    planes, cre, cim = _ref_v_update(cuda, pk)
    # corner-turn: our re / im planes equal the reference's A planes
    ours = torch.zeros(2 * 128 * 256 * 1024, dtype=torch.int8, device=cuda)
    mixer.corner_turn(_t(pk, cuda), 8256, 64, 256, 128, 32, 32, 0, ours, 1024, 0)
    _sync()
    o = ours.view(2, -1)
    assert torch.equal(o[0], planes[0]) and torch.equal(o[1], planes[1])
    # visibilities: bit-exact against cgemm_blk_t<false> (full square)
    with mixer.ArrayContext(max_heaps=32) as ctx:
        ctx.correlate(_t(pk, cuda), 32, seq0=0)
        v = torch.zeros(128 * 2 * 256 * 256, dtype=torch.int64, device=cuda)
        ctx.read_vis_i64(v, full_square=True)
        _sync()
        v = v.view(128, 2, 256, 256)
        assert torch.equal(v[:, 0], cre.view(128, 256, 256).to(torch.int64))
        assert torch.equal(v[:, 1], cim.view(128, 256, 256).to(torch.int64))


def test_image_matches_reference_publish_path(cuda):
    """k_flush_cube -> k_diff -> k_grid_cube -> cuFFT -> host fftshift (reference)
    against mixer_image on the same V; agreement to float rounding."""
    import torch
    pk = _config0_packets(32, seed=7)
    planes, cre, cim = _ref_v_update(cuda, pk)
    ref = oracle.ref_gpu()
    s = torch.cuda.current_stream().cuda_stream
    vcube = torch.zeros(128 * 2 * 256 * 256, dtype=torch.float32, device=cuda)
    vprev = torch.zeros_like(vcube)
    dv = torch.zeros_like(vcube)
    G = torch.zeros(128 * 32 * 32 * 2, dtype=torch.float32, device=cuda)
    im = torch.zeros_like(G)
    assert ref.ref_flush(vcube.data_ptr(), cre.data_ptr(), cim.data_ptr(), s) == 0
    assert ref.ref_diff(vcube.data_ptr(), vprev.data_ptr(), dv.data_ptr(), vcube.numel(), s) == 0
    assert ref.ref_grid(dv.data_ptr(), G.data_ptr(), s) == 0
    assert ref.ref_fft(G.data_ptr(), im.data_ptr(), s) == 0
    _sync()
    f = im.cpu().numpy().reshape(128, 32, 32, 2)[..., 0]
    ref_img = np.roll(f, (-16, -16), axis=(1, 2))            # host loop at :233
    with mixer.ArrayContext(max_heaps=32) as ctx:
        ctx.correlate(_t(pk, cuda), 32, seq0=0)
        img = torch.zeros(128 * 32 * 32, dtype=torch.float32, device=cuda)
        ctx.image(img)
        _sync()
        got = img.cpu().numpy().reshape(128, 32, 32)
    scale = np.abs(ref_img).max(axis=(1, 2), keepdims=True)
    assert np.all(np.abs(got - ref_img) <= 1e-4 * scale)
