"""Python binding of the B200 X-engine C-ABI (libmixer_b200.so, include/mixer.h).

The library is the product; this module only loads it with ctypes and passes
pointers through.  Device buffers are torch tensors (or raw integer device
addresses); streams are torch.cuda.Stream objects or raw cudaStream_t ints.
If the shared library is missing the import fails: there is no fallback.

Entry points and the reference symbol each replaces:
    corner_turn      k_packAB            src/rx_host_corr.cu:61-72
    xcorr_tri        cgemm_blk_t<ACC>    src/cgemm.cuh:28-69
    vis_flush        k_flush_cube        src/rx_host_corr.cu:90-95
    vis_dump_f32     --dump record       src/rx_host_corr.cu:187,225-227
    grid             k_grid_cube (+k_diff) src/rx_host_corr.cu:74-85
    image_fft        cufftExecC2C + host fftshift src/rx_host_corr.cu:205-235
    gen_packets      tx_host k_sky + DAQIRI capture src/tx_host.cu:41-79
    ArrayContext     gpu_thread / publish loop src/rx_host_corr.cu:143-239
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MIXER_B200_LIB") or os.path.join(_HERE, "libmixer_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C {_HERE}` (or __graft_entry__.build()); "
        "the X-engine has no CPU fallback")
_lib = C.CDLL(LIB_PATH)

# ---- constants (include/mixer.h) ------------------------------------------
OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, EOVERFLOW, ENODEV, EBUSY = 0, -1, -2, -3, -4, -5, -6, -7
WIRE_NANT, WIRE_ACTIVE_NCH, WIRE_TPKT = 256, 128, 32
WIRE_PAYLOAD_BYTES, WIRE_HDR_BYTES, WIRE_BYTES, WIRE_SEQ_BYTE, WIRE_PPB = 8192, 64, 8256, 48, 256
WIRE_UDP_PORT = 4096
KMAX_I32 = 65408
NOALLOC_MAX_CELLS = 1 << 20
VIS_STORE_I32, VIS_ACC_I32, VIS_ACC_I64 = 0, 1, 2


class MixerError(RuntimeError):
    def __init__(self, rc: int, what: str):
        super().__init__(f"{what}: {_lib.mixer_strerror(rc).decode()} (status {rc})")
        self.rc = rc


def _check(rc: int, what: str) -> None:
    if rc != OK:
        raise MixerError(rc, what)


_vp, _i32, _i64, _u32, _u16, _u64, _f64 = (C.c_void_p, C.c_int32, C.c_int64, C.c_uint32,
                                           C.c_uint16, C.c_uint64, C.c_double)


class XcorrProblem(C.Structure):
    _fields_ = [("planes", _vp), ("nant", _i32), ("nch", _i32), ("kt", _i64), ("kbeg", _i64),
                ("klen", _i64), ("mode", _i32), ("vis", _vp)]


ORDER_LPT, ORDER_CHANNEL = 0, 1


class ServerCfg(C.Structure):
    _fields_ = [("budget_bytes", _i64), ("max_streams", _i32), ("ring_subs", _i32),
                ("batch_subs", _i32)]


class DumpInfo(C.Structure):
    _fields_ = [("available", _i32), ("nant", _i32), ("nch", _i32), ("pad_", _i32),
                ("index", _i64), ("latency_s", C.c_double)]


class ServerCounters(C.Structure):
    _fields_ = [("admitted", _i64), ("refused", _i64), ("launches", _i64), ("work_items", _i64),
                ("bytes_used", _i64), ("bytes_processed", _i64), ("dumps", _i64),
                ("seq_errors", _i64), ("p50_latency_s", C.c_double), ("p99_latency_s", C.c_double),
                ("max_latency_s", C.c_double), ("elapsed_s", C.c_double), ("kernel_err", _i32),
                ("pad_", _i32)]


class ArrayDesc(C.Structure):
    _fields_ = [("nant", _i32), ("nch", _i32), ("tpkt", _i32), ("ksub", _i32),
                ("nsub_dump", _i32), ("side_x", _i32), ("grid", _i32), ("pkt_stride", _i32),
                ("hdr_bytes", _i32), ("max_heaps", _i32)]


def _sig(name, res, *args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = list(args)
    return f


_sig("mixer_strerror", C.c_char_p, C.c_int)
_sig("mixer_device_ok", C.c_int)
_sig("mixer_vis_tiles", _i32, _i32)
_sig("mixer_vis_elems", _i64, _i32, _i32)
_sig("mixer_corner_turn", C.c_int, _vp, _i64, _i32, _i32, _i32, _i32, _i32, _u32, _vp, _i64, _i64,
     _vp, _vp, _vp)
_sig("mixer_xcorr_tri", C.c_int, _vp, _i32, _i32, _i64, _i64, _i64, _i32, _vp, _vp, _vp)
_sig("mixer_xcorr_tri_ex", C.c_int, _vp, _i32, _i32, _i64, _i64, _i64, _i32, _vp, _i32, _vp, _vp)
_sig("mixer_mma_peak", C.c_int, _i64, _i32, _vp, _vp)
_sig("mixer_vis_flush", C.c_int, _vp, _vp, _i64, _vp)
_sig("mixer_vis_dump_f32", C.c_int, _vp, _i32, _i32, _vp, _vp)
_sig("mixer_vis_unpack_i64", C.c_int, _vp, _i32, _i32, _vp, _vp)
_sig("mixer_grid", C.c_int, _vp, _i32, _i32, _i32, _i32, _vp, _vp, _vp)
_sig("mixer_image_fft", C.c_int, _vp, _i32, _i32, _vp, _vp, _vp, _vp)
_sig("mixer_image_noalloc", C.c_int, _vp, _i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp)
_sig("mixer_sky_table", C.c_int, _i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp)
_sig("mixer_gen_packets", C.c_int, _vp, _i64, _i32, _i32, _i32, _i32, _i32, _i64, _u32, _u16, _vp,
     _f64, _u64, _i32, _vp)
_sig("mixer_batch_create", C.c_int, C.POINTER(XcorrProblem), _i32, C.POINTER(_vp))
_sig("mixer_batch_plan", C.c_int, _vp, C.POINTER(_i32), _i32, _i32)
_sig("mixer_batch_autotune", C.c_int, _vp, _i32, _vp, C.POINTER(C.c_float))
_sig("mixer_batch_run", C.c_int, _vp, _vp)
_sig("mixer_batch_capture_graph", C.c_int, _vp, _vp)
_sig("mixer_batch_replay", C.c_int, _vp, _vp)
_sig("mixer_batch_info", C.c_int, _vp, C.POINTER(_i64), C.POINTER(_i32), C.POINTER(_i32),
     C.POINTER(_i32))
_sig("mixer_batch_destroy", C.c_int, _vp)
_sig("mixer_restamp_seq", C.c_int, _vp, _i64, _i64, _u32, _vp)
_sig("mixer_ctx_shape", C.c_int, _vp, C.POINTER(_i32), C.POINTER(_i32))
_sig("mixer_write_vis_i64", C.c_int, _vp, _vp, _i64)
_sig("mixer_state_save", C.c_int, _vp, C.c_char_p)
_sig("mixer_state_load", C.c_int, _vp, C.c_char_p)
_sig("mixer_merge_time_split", C.c_int, C.POINTER(_vp), C.POINTER(_i64), _i32, _i64, _i32, _u16,
     _i64, _vp, C.POINTER(_i64), C.POINTER(_u32), C.POINTER(_i64))
_sig("mixer_align_heaps", C.c_int, _vp, _i64, _i64, _i32, C.POINTER(_i64), C.POINTER(_i64),
     C.POINTER(_i64), C.POINTER(_u32))
_sig("mixer_desc_default", C.c_int, C.POINTER(ArrayDesc))
_sig("mixer_server_create", C.c_int, C.POINTER(ServerCfg), C.POINTER(_vp))
_sig("mixer_server_destroy", C.c_int, _vp)
_sig("mixer_server_stream_bytes", _i64, C.POINTER(ServerCfg), C.POINTER(ArrayDesc))
_sig("mixer_server_open", C.c_int, _vp, C.POINTER(ArrayDesc), C.POINTER(_i32))
_sig("mixer_server_reserve", C.c_int, _vp, C.POINTER(ArrayDesc), _i32)
_sig("mixer_server_close", C.c_int, _vp, _i32)
_sig("mixer_server_submit", C.c_int, _vp, _i32, _vp, _i64, _u32, _i32)
_sig("mixer_server_poll", C.c_int, _vp, _i32, C.POINTER(DumpInfo), _vp)
_sig("mixer_server_stats", C.c_int, _vp, C.POINTER(ServerCounters))
_sig("mixer_server_sync_copies", C.c_int, _vp)
_sig("mixer_create", C.c_int, C.POINTER(ArrayDesc), C.POINTER(_vp))
_sig("mixer_destroy", C.c_int, _vp)
_sig("mixer_reset", C.c_int, _vp, _vp)
_sig("mixer_correlate", C.c_int, _vp, _vp, _i64, _u32, _i32, _vp)
_sig("mixer_correlate_i32", C.c_int, _vp, _vp, _i64, _u32, _i32, _vp)
_sig("mixer_integrate", C.c_int, _vp, _vp)
_sig("mixer_dump", C.c_int, _vp, _vp, _i32, _vp)
_sig("mixer_dump_to_file", C.c_int, _vp, C.c_char_p, _vp)
_sig("mixer_read_vis_i64", C.c_int, _vp, _vp, _i32, _i32, _vp)
_sig("mixer_image", C.c_int, _vp, _vp, _vp, _vp, _i32, _i32, _vp)
_sig("mixer_stats", C.c_int, _vp, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i32))
_sig("mixer_state_ptr", _vp, _vp)
_sig("mixer_shm_open", C.c_int, C.c_char_p, _i32, _i32, C.POINTER(_vp))
_sig("mixer_shm_publish", C.c_int, _vp, _vp, _vp, _vp, _u64)
_sig("mixer_shm_close", C.c_int, _vp, _i32)

EXPORTED = [
    "mixer_vis_tiles", "mixer_vis_elems", "mixer_strerror", "mixer_device_ok",
    "mixer_corner_turn", "mixer_xcorr_tri", "mixer_xcorr_tri_ex", "mixer_mma_peak",
    "mixer_vis_flush", "mixer_vis_dump_f32",
    "mixer_vis_unpack_i64", "mixer_grid", "mixer_image_fft", "mixer_image_noalloc",
    "mixer_sky_table",
    "mixer_gen_packets", "mixer_desc_default", "mixer_create", "mixer_destroy", "mixer_reset",
    "mixer_correlate", "mixer_correlate_i32", "mixer_integrate", "mixer_dump",
    "mixer_dump_to_file", "mixer_read_vis_i64", "mixer_image", "mixer_stats", "mixer_state_ptr",
    "mixer_shm_open", "mixer_shm_publish", "mixer_shm_close",
    "mixer_batch_create", "mixer_batch_plan", "mixer_batch_autotune", "mixer_batch_run",
    "mixer_batch_capture_graph", "mixer_batch_replay", "mixer_batch_info", "mixer_batch_destroy",
    "mixer_server_create", "mixer_server_destroy", "mixer_server_stream_bytes", "mixer_server_open",
    "mixer_server_reserve",
    "mixer_server_close", "mixer_server_submit", "mixer_server_poll", "mixer_server_stats",
    "mixer_server_sync_copies",
    "mixer_restamp_seq", "mixer_ctx_shape", "mixer_write_vis_i64", "mixer_state_save",
    "mixer_state_load", "mixer_align_heaps", "mixer_merge_time_split",
]


def lib():
    return _lib


def _ptr(x) -> int | None:
    """Device / host address of a torch tensor, numpy array or raw int (None -> NULL)."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    raise TypeError(f"cannot take the address of {type(x)}")


def _stream(s) -> int | None:
    if s is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except ImportError:
            pass
        return None
    if isinstance(s, int):
        return s
    return s.cuda_stream


def vis_tiles(nant: int) -> int:
    return _lib.mixer_vis_tiles(nant)


def vis_elems(nant: int, nch: int) -> int:
    return _lib.mixer_vis_elems(nant, nch)


def device_ok() -> bool:
    return _lib.mixer_device_ok() == OK


# ---- stateless entry points ------------------------------------------------

def corner_turn(packets, pkt_stride, hdr_bytes, nant, nch, tpkt, nheaps, seq0, planes, kt, k0=0,
                seq_errors=None, err=None, stream=None):
    _check(_lib.mixer_corner_turn(_ptr(packets), pkt_stride, hdr_bytes, nant, nch, tpkt, nheaps,
                                  seq0 & 0xFFFFFFFF, _ptr(planes), kt, k0, _ptr(seq_errors),
                                  _ptr(err), _stream(stream)), "mixer_corner_turn")


def xcorr_tri(planes, nant, nch, kt, kbeg, klen, mode, vis, err=None, stream=None, max_ctas=0):
    if max_ctas:
        _check(_lib.mixer_xcorr_tri_ex(_ptr(planes), nant, nch, kt, kbeg, klen, mode, _ptr(vis),
                                       max_ctas, _ptr(err), _stream(stream)), "mixer_xcorr_tri_ex")
        return
    _check(_lib.mixer_xcorr_tri(_ptr(planes), nant, nch, kt, kbeg, klen, mode, _ptr(vis), _ptr(err),
                                _stream(stream)), "mixer_xcorr_tri")


def mma_peak(iters, ctas=0, err=None, stream=None):
    """One launch of the tensor-core rate probe: iters x 8 int8 MMAs per CTA."""
    _check(_lib.mixer_mma_peak(iters, ctas, _ptr(err), _stream(stream)), "mixer_mma_peak")


MMA_PEAK_OPS_PER_ITER = 8 * 2 * 128 * 256 * 32   # per CTA and iteration


def vis_flush(vis32, vis64, n, stream=None):
    _check(_lib.mixer_vis_flush(_ptr(vis32), _ptr(vis64), n, _stream(stream)), "mixer_vis_flush")


def vis_dump_f32(vis64, nant, nch, cube, stream=None):
    _check(_lib.mixer_vis_dump_f32(_ptr(vis64), nant, nch, _ptr(cube), _stream(stream)),
           "mixer_vis_dump_f32")


def vis_unpack_i64(vis64, nant, nch, cube, stream=None):
    _check(_lib.mixer_vis_unpack_i64(_ptr(vis64), nant, nch, _ptr(cube), _stream(stream)),
           "mixer_vis_unpack_i64")


def grid(vis64, nant, nch, side_x, G, out, prev=None, stream=None):
    _check(_lib.mixer_grid(_ptr(vis64), nant, nch, side_x, G, _ptr(out), _ptr(prev),
                           _stream(stream)), "mixer_grid")


def image_fft(grid_i64, nch, G, img, vmax=None, vmin=None, stream=None):
    _check(_lib.mixer_image_fft(_ptr(grid_i64), nch, G, _ptr(img), _ptr(vmax), _ptr(vmin),
                                _stream(stream)), "mixer_image_fft")


def image_noalloc(vis64, nant, nch, side_x, G, img, vmax=None, vmin=None, stream=None):
    """Grid + FFT image with the grid in the library's fixed device array (no
    allocation); nch * G * G <= NOALLOC_MAX_CELLS.  See include/mixer.h."""
    _check(_lib.mixer_image_noalloc(_ptr(vis64), nant, nch, side_x, G, _ptr(img), _ptr(vmax),
                                    _ptr(vmin), _stream(stream)), "mixer_image_noalloc")


def sky_table(nant, nch, side_x, sources):
    """sources: list of (l, m, amp0, amp1).  Returns numpy float64 [nch][nant][2]."""
    import numpy as np
    n = len(sources)
    arr = np.asarray(sources, dtype=np.float64).reshape(n, 4) if n else np.zeros((0, 4))
    l, m, a0, a1 = (np.ascontiguousarray(arr[:, q]) for q in range(4))
    out = np.zeros((nch, nant, 2), dtype=np.float64)
    _check(_lib.mixer_sky_table(nant, nch, side_x, n, _ptr(l), _ptr(m), _ptr(a0), _ptr(a1),
                                _ptr(out)), "mixer_sky_table")
    return out


def gen_packets(packets, pkt_stride, hdr_bytes, nant, nch, tpkt, nheaps, heap0, seq0, udp_port,
                sky, sigma, seed, noise_mode=0, stream=None):
    _check(_lib.mixer_gen_packets(_ptr(packets), pkt_stride, hdr_bytes, nant, nch, tpkt, nheaps,
                                  heap0, seq0 & 0xFFFFFFFF, udp_port, _ptr(sky), float(sigma),
                                  seed & 0xFFFFFFFFFFFFFFFF, noise_mode, _stream(stream)),
           "mixer_gen_packets")


def restamp_seq(packets, npk, pkt_stride, seq0, stream=None):
    _check(_lib.mixer_restamp_seq(_ptr(packets), npk, pkt_stride, seq0 & 0xFFFFFFFF, _stream(stream)),
           "mixer_restamp_seq")


def merge_time_split(queues, pkt_stride, nant, udp_port0, max_heaps, out):
    """Time-split multi-queue merge (host numpy buffers): queues = list of uint8
    arrays of whole packets, heap tb in queue tb % len(queues).  Returns dict(heaps,
    seq0, consumed=[packets used or skipped per queue])."""
    nq = len(queues)
    ptrs = (_vp * nq)(*[_ptr(q) for q in queues])
    npk = (_i64 * nq)(*[q.size // pkt_stride for q in queues])
    n, s0 = _i64(), _u32()
    used = (_i64 * nq)()
    _check(_lib.mixer_merge_time_split(ptrs, npk, nq, pkt_stride, nant, udp_port0, max_heaps,
                                       _ptr(out), C.byref(n), C.byref(s0), used),
           "mixer_merge_time_split")
    return {"heaps": n.value, "seq0": s0.value, "consumed": list(used)}


def align_heaps(packets, npk, pkt_stride, nant):
    """Host burst alignment: dict(first, nheaps, next, seq0)."""
    f, n, x, s = _i64(), _i64(), _i64(), _u32()
    _check(_lib.mixer_align_heaps(_ptr(packets), npk, pkt_stride, nant, C.byref(f), C.byref(n),
                                  C.byref(x), C.byref(s)), "mixer_align_heaps")
    return {"first": f.value, "nheaps": n.value, "next": x.value, "seq0": s.value}


# ---- array context ------------------------------------------------------------

def default_desc() -> ArrayDesc:
    d = ArrayDesc()
    _check(_lib.mixer_desc_default(C.byref(d)), "mixer_desc_default")
    return d


class ArrayContext:
    """One array's resident X-engine state (int64 cube, staging, imaging)."""

    def __init__(self, desc: ArrayDesc | None = None, **kw):
        d = desc if desc is not None else default_desc()
        for k, v in kw.items():
            setattr(d, k, v)
        self.desc = d
        h = _vp()
        _check(_lib.mixer_create(C.byref(d), C.byref(h)), "mixer_create")
        self._h = h.value

    def close(self):
        if self._h:
            _lib.mixer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def reset(self, stream=None):
        _check(_lib.mixer_reset(self._h, _stream(stream)), "mixer_reset")

    def correlate(self, packets, nheaps, seq0=0, on_device=True, stream=None):
        _check(_lib.mixer_correlate(self._h, _ptr(packets), nheaps, seq0 & 0xFFFFFFFF,
                                    1 if on_device else 0, _stream(stream)), "mixer_correlate")

    def correlate_i32(self, packets, nheaps, seq0=0, on_device=True, stream=None):
        _check(_lib.mixer_correlate_i32(self._h, _ptr(packets), nheaps, seq0 & 0xFFFFFFFF,
                                        1 if on_device else 0, _stream(stream)),
               "mixer_correlate_i32")

    def integrate(self, stream=None):
        _check(_lib.mixer_integrate(self._h, _stream(stream)), "mixer_integrate")

    def dump(self, out, on_device=True, stream=None):
        _check(_lib.mixer_dump(self._h, _ptr(out), 1 if on_device else 0, _stream(stream)),
               "mixer_dump")

    def dump_to_file(self, path: str, stream=None):
        _check(_lib.mixer_dump_to_file(self._h, path.encode(), _stream(stream)),
               "mixer_dump_to_file")

    def read_vis_i64(self, out, full_square=True, on_device=True, stream=None):
        _check(_lib.mixer_read_vis_i64(self._h, _ptr(out), 1 if full_square else 0,
                                       1 if on_device else 0, _stream(stream)),
               "mixer_read_vis_i64")

    def image(self, img, vmax=None, vmin=None, delta=False, on_device=True, stream=None):
        _check(_lib.mixer_image(self._h, _ptr(img), _ptr(vmax), _ptr(vmin), 1 if delta else 0,
                                1 if on_device else 0, _stream(stream)), "mixer_image")

    def stats(self):
        s, e, k = _i64(), _i64(), _i32()
        rc = _lib.mixer_stats(self._h, C.byref(s), C.byref(e), C.byref(k))
        if rc not in (OK, ETIMEOUT):
            _check(rc, "mixer_stats")
        return {"samples": s.value, "seq_errors": e.value, "kernel_err": k.value}

    def save(self, path: str):
        _check(_lib.mixer_state_save(self._h, path.encode()), "mixer_state_save")

    def load(self, path: str):
        _check(_lib.mixer_state_load(self._h, path.encode()), "mixer_state_load")

    def state_ptr(self) -> int:
        return _lib.mixer_state_ptr(self._h)


class Batch:
    """Uneven arrays in one persistent launch (plan, autotune, graph replay).

    problems: list of dicts with keys planes, nant, nch, kt, kbeg, klen, mode, vis.
    """

    def __init__(self, problems):
        arr = (XcorrProblem * len(problems))()
        for q, p in zip(arr, problems):
            q.planes, q.nant, q.nch = _ptr(p["planes"]), p["nant"], p["nch"]
            q.kt, q.kbeg, q.klen = p["kt"], p.get("kbeg", 0), p.get("klen", p["kt"])
            q.mode, q.vis = p.get("mode", VIS_ACC_I64), _ptr(p["vis"])
        self._keep = problems
        h = _vp()
        _check(_lib.mixer_batch_create(arr, len(problems), C.byref(h)), "mixer_batch_create")
        self._h = h.value

    def plan(self, split_per_class=(), order=ORDER_LPT):
        n = len(split_per_class)
        arr = (_i32 * max(n, 1))(*split_per_class)
        _check(_lib.mixer_batch_plan(self._h, arr, n, order), "mixer_batch_plan")

    def autotune(self, reps=2, stream=None) -> float:
        ms = C.c_float()
        _check(_lib.mixer_batch_autotune(self._h, reps, _stream(stream), C.byref(ms)),
               "mixer_batch_autotune")
        return ms.value

    def run(self, stream=None):
        _check(_lib.mixer_batch_run(self._h, _stream(stream)), "mixer_batch_run")

    def capture_graph(self, stream):
        _check(_lib.mixer_batch_capture_graph(self._h, _stream(stream)), "mixer_batch_capture_graph")

    def replay(self, stream=None):
        _check(_lib.mixer_batch_replay(self._h, _stream(stream)), "mixer_batch_replay")

    def info(self):
        n, o, e = _i64(), _i32(), _i32()
        sp = (_i32 * 65)()
        rc = _lib.mixer_batch_info(self._h, C.byref(n), C.byref(o), sp, C.byref(e))
        if rc not in (OK, ETIMEOUT):
            _check(rc, "mixer_batch_info")
        return {"nwork": n.value, "order": o.value, "split": list(sp), "kernel_err": e.value}

    def close(self):
        if self._h:
            _lib.mixer_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_desc(**kw) -> ArrayDesc:
    d = default_desc()
    for k, v in kw.items():
        setattr(d, k, v)
    return d


class Server:
    """Streaming X-engine: admission by memory budget, continuous batching, dumps."""

    def __init__(self, budget_bytes, max_streams=16, ring_subs=0, batch_subs=0):
        self.cfg = ServerCfg(budget_bytes, max_streams, ring_subs, batch_subs)
        h = _vp()
        _check(_lib.mixer_server_create(C.byref(self.cfg), C.byref(h)), "mixer_server_create")
        self._h = h.value

    def stream_bytes(self, desc: ArrayDesc) -> int:
        return _lib.mixer_server_stream_bytes(C.byref(self.cfg), C.byref(desc))

    def reserve(self, desc: ArrayDesc, count: int):
        """Allocate the device and pinned host state of `count` streams of this
        shape ahead of serving, so their admissions allocate nothing."""
        _check(_lib.mixer_server_reserve(self._h, C.byref(desc), count), "mixer_server_reserve")

    def open(self, desc: ArrayDesc) -> int:
        sid = _i32()
        _check(_lib.mixer_server_open(self._h, C.byref(desc), C.byref(sid)), "mixer_server_open")
        return sid.value

    def try_open(self, desc: ArrayDesc):
        sid = _i32()
        rc = _lib.mixer_server_open(self._h, C.byref(desc), C.byref(sid))
        if rc == EBUSY:
            return None
        _check(rc, "mixer_server_open")
        return sid.value

    def close_stream(self, sid: int):
        _check(_lib.mixer_server_close(self._h, sid), "mixer_server_close")

    def submit(self, sid, packets, nheaps, seq0=0, on_device=True) -> bool:
        """False when the stream's staging ring is full (retry later)."""
        rc = _lib.mixer_server_submit(self._h, sid, _ptr(packets), nheaps, seq0 & 0xFFFFFFFF,
                                      1 if on_device else 0)
        if rc == EBUSY:
            return False
        _check(rc, "mixer_server_submit")
        return True

    def sync_copies(self):
        _check(_lib.mixer_server_sync_copies(self._h), "mixer_server_sync_copies")

    def poll(self, sid, out=None):
        info = DumpInfo()
        _check(_lib.mixer_server_poll(self._h, sid, C.byref(info), _ptr(out)), "mixer_server_poll")
        if not info.available:
            return None
        return {"index": info.index, "latency_s": info.latency_s, "nant": info.nant,
                "nch": info.nch}

    def stats(self):
        st = ServerCounters()
        rc = _lib.mixer_server_stats(self._h, C.byref(st))
        if rc not in (OK, ETIMEOUT):
            _check(rc, "mixer_server_stats")
        return {f: getattr(st, f) for f, _ in ServerCounters._fields_ if f != "pad_"}

    def close(self):
        if self._h:
            _lib.mixer_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Corr32Shm:
    """Corr32 image publisher (src/rx_host_corr.cu:97-105)."""

    def __init__(self, name: str, nch: int, G: int):
        h = _vp()
        _check(_lib.mixer_shm_open(name.encode(), nch, G, C.byref(h)), "mixer_shm_open")
        self._h = h.value

    def publish(self, img, vmax, vmin, write_seq: int):
        _check(_lib.mixer_shm_publish(self._h, _ptr(img), _ptr(vmax), _ptr(vmin), write_seq),
               "mixer_shm_publish")

    def close(self, unlink=True):
        if self._h:
            _lib.mixer_shm_close(self._h, 1 if unlink else 0)
            self._h = None
