"""ctypes access to the checkers (TEST INFRASTRUCTURE ONLY).

liboracle.so  -- CPU restatement of the reference path (mixer_oracle.c).
_ref/libref_gpu.so -- the reference's own kernels built from its sources
                      (ref_gpu.cu); present only where it was built.

Only tests/, the smoke check and the benchmark's CPU-baseline leg import
this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_PATH = os.path.join(_HERE, "liboracle.so")
REF_GPU_PATH = os.path.join(_HERE, "_ref", "libref_gpu.so")

_vp, _i32, _i64, _u32, _u16, _u64, _f64 = (C.c_void_p, C.c_int32, C.c_int64, C.c_uint32,
                                           C.c_uint16, C.c_uint64, C.c_double)
_orc = None
_ref = None


def _load():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_PATH):
            raise ImportError(f"{ORACLE_PATH} missing; run `make -C {_HERE} liboracle.so`")
        lib = C.CDLL(ORACLE_PATH)
        for name, res, args in [
            ("orc_philox4x32_10", None, [_vp, _u32, _u32, _vp]),
            ("orc_sky_table", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp]),
            ("orc_gen_packets", C.c_int, [_vp, _i64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          _i64, _u32, _u16, _vp, _f64, _u64, C.c_int]),
            ("orc_corner_turn", C.c_int, [_vp, _i64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          _vp, _i64, _i64]),
            ("orc_seq_errors", _i64, [_vp, _i64, _i64, _u32]),
            ("orc_correlate", C.c_int, [_vp, C.c_int, C.c_int, _i64, _i64, _i64, C.c_int, C.c_int,
                                        _vp, C.c_int, C.c_int]),
            ("orc_correlate_pairwise", C.c_int, [_vp, C.c_int, C.c_int, _i64, _i64, _i64, C.c_int,
                                                 C.c_int, _vp, C.c_int]),
            ("orc_grid", C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp]),
            ("orc_max_threads", C.c_int, []),
        ]:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _orc = lib
    return _orc


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    _load().orc_philox4x32_10(_p(c), key & 0xFFFFFFFF, (key >> 32) & 0xFFFFFFFF, _p(out))
    return out


def sky_table(nant, nch, side_x, sources):
    n = len(sources)
    arr = np.asarray(sources, dtype=np.float64).reshape(n, 4) if n else np.zeros((0, 4))
    l, m, a0, a1 = (np.ascontiguousarray(arr[:, q]) for q in range(4))
    out = np.zeros((nch, nant, 2), dtype=np.float64)
    _load().orc_sky_table(nant, nch, side_x, n, _p(l), _p(m), _p(a0), _p(a1), _p(out))
    return out


def gen_packets(nant, nch, tpkt, nheaps, heap0=0, seq0=0, port=4096, sky=None, sigma=16.0,
                seed=1, mode=0, pkt_stride=None, hdr=64):
    stride = pkt_stride or hdr + 2 * nch * tpkt
    buf = np.zeros(nheaps * nant * stride, dtype=np.uint8)
    skyp = None if sky is None else _p(np.ascontiguousarray(sky, dtype=np.float64))
    _load().orc_gen_packets(_p(buf), stride, hdr, nant, nch, tpkt, nheaps, heap0, seq0 & 0xFFFFFFFF,
                            port, skyp, float(sigma), seed & 0xFFFFFFFFFFFFFFFF, mode)
    return buf


def corner_turn(packets, nant, nch, tpkt, nheaps, kt=None, k0=0, pkt_stride=None, hdr=64):
    stride = pkt_stride or hdr + 2 * nch * tpkt
    kt = kt or nheaps * tpkt
    planes = np.zeros((2, nch, nant, kt), dtype=np.int8)
    _load().orc_corner_turn(_p(packets), stride, hdr, nant, nch, tpkt, nheaps, _p(planes), kt, k0)
    return planes


def seq_errors(packets, npk, seq0, pkt_stride):
    return int(_load().orc_seq_errors(_p(packets), pkt_stride, npk, seq0 & 0xFFFFFFFF))


def correlate(planes, kbeg=0, klen=None, c0=0, nc=None, out=None, mirror=True, nthreads=0):
    """Exact int64 V = X X^H, full square [nc][2][N][N] (added into `out`)."""
    _, nch, nant, kt = planes.shape
    klen = kt - kbeg if klen is None else klen
    nc = nch - c0 if nc is None else nc
    if out is None:
        out = np.zeros((nc, 2, nant, nant), dtype=np.int64)
    _load().orc_correlate(_p(planes), nant, nch, kt, kbeg, klen, c0, nc, _p(out),
                          1 if mirror else 0, nthreads)
    return out


def correlate_pairwise(planes, kbeg=0, klen=None, c0=0, nc=None, nthreads=0):
    """The same lower triangle as correlate(), one (a, b) pair at a time (the
    plain statement of the formula, the cross-check of the blocked form)."""
    _, nch, nant, kt = planes.shape
    klen = kt - kbeg if klen is None else klen
    nc = nch - c0 if nc is None else nc
    out = np.zeros((nc, 2, nant, nant), dtype=np.int64)
    _load().orc_correlate_pairwise(_p(planes), nant, nch, kt, kbeg, klen, c0, nc, _p(out), nthreads)
    return out


def grid(full, side_x, G):
    nch, _, nant, _ = full.shape
    g = np.zeros((nch, G, G, 2), dtype=np.int64)
    _load().orc_grid(_p(np.ascontiguousarray(full)), nant, nch, side_x, G, _p(g))
    return g


def image64(grid_i64):
    """FP64 image: Re(FFT2 forward(grid)), fftshifted; [nch][G][G]."""
    z = grid_i64[..., 0].astype(np.float64) + 1j * grid_i64[..., 1].astype(np.float64)
    f = np.fft.fft2(z, axes=(-2, -1))
    return np.fft.fftshift(f.real, axes=(-2, -1))


def vis_tile_pack(full):
    """Full square int64 [C][2][N][N] -> tile-packed lower triangle (product layout)."""
    nch, _, nant, _ = full.shape
    nb = (nant + 127) // 128
    nt = nb * (nb + 1) // 2
    out = np.zeros((nch, nt, 2, 128, 128), dtype=full.dtype)
    pad = np.zeros((nch, 2, nb * 128, nb * 128), dtype=full.dtype)
    pad[:, :, :nant, :nant] = full
    t = 0
    for i in range(nb):
        for j in range(i + 1):
            blk = pad[:, :, 128 * i:128 * i + 128, 128 * j:128 * j + 128]   # [c][p][m][n]
            out[:, t] = blk.transpose(0, 1, 3, 2)                             # [c][p][n][m]
            t += 1
    return out


def max_threads():
    return int(_load().orc_max_threads())


# ---- the reference's own GPU kernels ------------------------------------------

def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_PATH)


def ref_gpu():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_GPU_PATH)
        for name, res, args in [
            ("ref_const", C.c_int, [C.c_int]),
            ("ref_pack", C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
            ("ref_cgemm", C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp,
                                    _vp, _vp, _vp]),
            ("ref_flush", C.c_int, [_vp, _vp, _vp, _vp]),
            ("ref_diff", C.c_int, [_vp, _vp, _vp, C.c_size_t, _vp]),
            ("ref_grid", C.c_int, [_vp, _vp, _vp]),
            ("ref_fft", C.c_int, [_vp, _vp, _vp]),
        ]:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _ref = lib
    return _ref
