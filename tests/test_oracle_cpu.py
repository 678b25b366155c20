"""CPU checks of the oracle restatement against direct numpy statements of the
reference formulas (src/cgemm.cuh:4-7, src/rx_host_corr.cu:63-71, :79-85)."""
import numpy as np
import pytest

import oracle


def _np_corner_turn(pk, nant, nch, tpkt, nheaps, hdr=64):
    stride = hdr + 2 * nch * tpkt
    p = pk.reshape(nheaps, nant, stride)[:, :, hdr:].view(np.int8)
    re = p[:, :, :nch * tpkt].reshape(nheaps, nant, nch, tpkt)
    im = p[:, :, nch * tpkt:].reshape(nheaps, nant, nch, tpkt)
    # [h][a][c][t] -> [c][a][h*tpkt + t]
    re = re.transpose(2, 1, 0, 3).reshape(nch, nant, nheaps * tpkt)
    im = im.transpose(2, 1, 0, 3).reshape(nch, nant, nheaps * tpkt)
    return np.stack([re, im])


def test_corner_turn_matches_index_map():
    nant, nch, tpkt, nheaps = 24, 8, 16, 5
    pk = oracle.gen_packets(nant, nch, tpkt, nheaps, seed=7, sigma=20.0)
    got = oracle.corner_turn(pk, nant, nch, tpkt, nheaps)
    assert np.array_equal(got, _np_corner_turn(pk, nant, nch, tpkt, nheaps))


def test_correlate_matches_complex_product():
    rng = np.random.default_rng(3)
    nch, nant, kt = 3, 37, 200
    planes = rng.integers(-128, 128, size=(2, nch, nant, kt), dtype=np.int8)
    got = oracle.correlate(planes)
    x = planes[0].astype(np.int64) + 1j * planes[1].astype(np.int64)
    v = np.einsum("cak,cbk->cab", x, np.conj(x))
    assert np.array_equal(got[:, 0], np.real(v).astype(np.int64))
    assert np.array_equal(got[:, 1], np.imag(v).astype(np.int64))


def test_correlate_range_and_subset():
    rng = np.random.default_rng(4)
    planes = rng.integers(-128, 128, size=(2, 6, 20, 96), dtype=np.int8)
    full = oracle.correlate(planes)
    part = oracle.correlate(planes, kbeg=0, klen=48, c0=2, nc=3)
    part = oracle.correlate(planes, kbeg=48, klen=48, c0=2, nc=3, out=part)
    assert np.array_equal(part, full[2:5])


def test_extreme_values_exact():
    # all -128: the reference's int8 negation (src/cgemm.cuh:52) wraps here
    planes = np.full((2, 1, 4, 64), -128, dtype=np.int8)
    v = oracle.correlate(planes)
    assert np.all(v[:, 0] == 2 * 128 * 128 * 64)
    assert np.all(v[:, 1] == 0)


def test_grid_matches_loop():
    rng = np.random.default_rng(5)
    nant, side, G = 16, 4, 8
    planes = rng.integers(-20, 20, size=(2, 2, nant, 32), dtype=np.int8)
    full = oracle.correlate(planes)
    g = oracle.grid(full, side, G)
    ref = np.zeros_like(g)
    for c in range(2):
        for a in range(nant):
            for b in range(nant):
                dy = (a // side - b // side) % G
                dx = (a % side - b % side) % G
                ref[c, dy, dx, 0] += full[c, 0, a, b]
                ref[c, dy, dx, 1] += full[c, 1, a, b]
    assert np.array_equal(g, ref)
    # Hermitian grid -> real image
    img = oracle.image64(g)
    z = g[..., 0] + 1j * g[..., 1]
    assert np.allclose(np.fft.fft2(z).imag, 0, atol=1e-6 * np.abs(z).sum())
    assert img.shape == (2, G, G)


def test_generator_statistics_and_headers():
    nant, nch, tpkt, nheaps = 64, 16, 32, 8
    pk = oracle.gen_packets(nant, nch, tpkt, nheaps, seq0=1000, seed=11, sigma=16.0)
    stride = 64 + 2 * nch * tpkt
    assert oracle.seq_errors(pk, nheaps * nant, 1000, stride) == 0
    p = pk.reshape(nheaps * nant, stride)
    seq = (p[:, 48].astype(np.uint32) << 24) | (p[:, 49].astype(np.uint32) << 16) | \
          (p[:, 50].astype(np.uint32) << 8) | p[:, 51]
    assert np.array_equal(seq, 1000 + np.arange(nheaps * nant, dtype=np.uint32))
    x = p[:, 64:].view(np.int8).astype(np.float64)
    assert abs(x.mean()) < 0.2
    assert 15.0 < x.std() < 17.0
    # uniform mode stays in [-127, 127]
    pu = oracle.gen_packets(nant, nch, tpkt, 2, seed=3, mode=1)
    u = pu.reshape(2 * nant, stride)[:, 64:].view(np.int8)
    assert u.min() >= -127 and u.max() <= 127 and u.min() < -120 and u.max() > 120


def test_sky_table_formula():
    tab = oracle.sky_table(4, 2, 2, [(0.1, -0.05, 6.0, 0.0)])
    a = 3
    x, y = a % 2, a // 2
    for c in range(2):
        fc = 1 + c / 2
        ph = -2 * np.pi * fc * (x * 0.1 + y * -0.05)
        assert np.isclose(tab[c, a, 0], 6 * np.cos(ph), rtol=0, atol=1e-12)
        assert np.isclose(tab[c, a, 1], 6 * np.sin(ph), rtol=0, atol=1e-12)


def test_seq_error_count():
    nant, nch, tpkt = 8, 4, 16
    pk = oracle.gen_packets(nant, nch, tpkt, 3, seq0=5)
    stride = 64 + 2 * nch * tpkt
    pk.reshape(-1, stride)[10, 51] ^= 1    # corrupt one seq
    assert oracle.seq_errors(pk, 3 * nant, 5, stride) == 1


@pytest.mark.parametrize("nant,nch,kt,kbeg,klen", [
    (37, 3, 256, 0, 256), (130, 2, 5000, 16, 4960), (256, 1, 4096, 0, 4096), (5, 4, 48, 16, 32),
])
def test_blocked_correlator_equals_pairwise(nant, nch, kt, kbeg, klen):
    """The blocked correlator (int16 pairs, 2 x 4 blocks, chunked int32 partial
    sums) against the pair-by-pair statement of the formula, on full-range int8
    including -128 and ragged shapes."""
    rng = np.random.default_rng(nant * 7 + kt)
    planes = rng.integers(-128, 128, size=(2, nch, nant, kt), dtype=np.int8)
    planes[:, :, 0, :] = -128                          # the extreme row
    got = oracle.correlate(planes, kbeg=kbeg, klen=klen, mirror=False)
    want = oracle.correlate_pairwise(planes, kbeg=kbeg, klen=klen)
    assert np.array_equal(got, want)
