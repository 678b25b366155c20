// ctx.cu -- the array context: device state of one array and the host-side
// correlate -> integrate -> dump / image flow around the kernels.
//
// Mirrors the reference's gpu_thread / publish loop (src/rx_host_corr.cu:
// 143-175, 214-239) without its process globals (:108-118) or exit-on-error
// (:35): the context owns every device buffer, callers own inputs and
// outputs, and host packets are staged through two device buffers on a copy
// stream so the next copy overlaps the current corner-turn + GEMM (the
// reference's NBATCH ring and copy / compute streams, :44-45, :146-172).
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <string>
#include "common.cuh"

namespace mixer {

static thread_local std::string g_last_error;

int cuda_status(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) return MIXER_ENOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MIXER_ENODEV;
    return MIXER_ECUDA;
}

}  // namespace mixer

struct mixer_ctx {
    mixer_array_desc d;
    int dev;
    int64_t vis_elems;
    int64_t* vis64;
    int32_t* vis32;
    int8_t* planes;
    int64_t kt_max;
    uint8_t* stage[2];
    size_t stage_bytes;
    cudaEvent_t stage_free[2];
    cudaEvent_t stage_ready[2];
    bool stage_used[2];
    cudaStream_t copy_stream;
    int cur;
    int64_t* grid;
    int64_t* grid_prev;
    float* img;
    float* vmax;
    float* vmin;
    float* dump_dev;
    int64_t* unpack_dev;
    uint32_t* d_seq_err;
    int32_t* d_err;
    int64_t samples;
    int64_t i32_samples;
};

extern "C" const char* mixer_strerror(int status) {
    switch (status) {
        case MIXER_OK: return "ok";
        case MIXER_EINVAL: return "invalid argument or unsupported shape";
        case MIXER_ENOMEM: return "out of memory";
        case MIXER_ECUDA: return mixer::g_last_error.empty() ? "CUDA error" : mixer::g_last_error.c_str();
        case MIXER_ETIMEOUT: return "a bounded in-kernel wait timed out";
        case MIXER_EOVERFLOW: return "int32 headroom exceeded; integrate first";
        case MIXER_ENODEV: return "no sm_100 device";
        case MIXER_EBUSY: return "admission refused (memory budget or slots)";
        default: return "unknown status";
    }
}

extern "C" int mixer_device_ok(void) {
    int dev = 0;
    MIXER_CK(cudaGetDevice(&dev));
    cudaDeviceProp p;
    MIXER_CK(cudaGetDeviceProperties(&p, dev));
    return p.major == 10 ? MIXER_OK : MIXER_ENODEV;
}

extern "C" int mixer_desc_default(mixer_array_desc* d) {
    if (!d) return MIXER_EINVAL;
    d->nant = MIXER_WIRE_NANT;
    d->nch = MIXER_WIRE_ACTIVE_NCH;
    d->tpkt = MIXER_WIRE_TPKT;
    d->ksub = 32 * MIXER_WIRE_TPKT;   // HBATCH * TPKT = KPCH (src/rx_host_corr.cu:39-40)
    d->nsub_dump = 64;
    d->side_x = 16;
    d->grid = 32;
    d->pkt_stride = MIXER_WIRE_BYTES;
    d->hdr_bytes = MIXER_WIRE_HDR_BYTES;
    d->max_heaps = 32;
    return MIXER_OK;
}

static int desc_check(const mixer_array_desc* d) {
    if (!d || d->nant <= 0 || d->nch <= 0 || d->tpkt <= 0 || d->tpkt % 16 != 0) return MIXER_EINVAL;
    if (d->nant > 65536 || d->nch > 65535 || d->side_x <= 0 || d->grid < 0) return MIXER_EINVAL;
    if (d->pkt_stride % 16 != 0 || d->hdr_bytes % 16 != 0 || d->hdr_bytes < 64) return MIXER_EINVAL;
    if ((int64_t)d->hdr_bytes + 2LL * d->nch * d->tpkt > d->pkt_stride) return MIXER_EINVAL;
    if (d->max_heaps <= 0 || d->ksub <= 0 || d->ksub % d->tpkt != 0) return MIXER_EINVAL;
    return MIXER_OK;
}

static int grid_side(const mixer_array_desc* d) {
    if (d->grid > 0) return d->grid;
    const int sy = (d->nant + d->side_x - 1) / d->side_x;
    const int s = d->side_x > sy ? d->side_x : sy;
    int g = 1;
    while (g < 2 * s) g <<= 1;
    return g;
}

extern "C" int mixer_destroy(mixer_ctx* c) {
    if (!c) return MIXER_OK;
    cudaFree(c->vis64);
    cudaFree(c->vis32);
    cudaFree(c->planes);
    for (int s = 0; s < 2; ++s) {
        cudaFree(c->stage[s]);
        if (c->stage_free[s]) cudaEventDestroy(c->stage_free[s]);
        if (c->stage_ready[s]) cudaEventDestroy(c->stage_ready[s]);
    }
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    cudaFree(c->grid);
    cudaFree(c->grid_prev);
    cudaFree(c->img);
    cudaFree(c->vmax);
    cudaFree(c->vmin);
    cudaFree(c->dump_dev);
    cudaFree(c->unpack_dev);
    cudaFree(c->d_seq_err);
    cudaFree(c->d_err);
    free(c);
    return MIXER_OK;
}

extern "C" int mixer_create(const mixer_array_desc* d, mixer_ctx** out) {
    if (!out) return MIXER_EINVAL;
    *out = nullptr;
    int rc = desc_check(d);
    if (rc != MIXER_OK) return rc;
    mixer_ctx* c = static_cast<mixer_ctx*>(calloc(1, sizeof(mixer_ctx)));
    if (!c) return MIXER_ENOMEM;
    c->d = *d;
    c->d.grid = grid_side(d);
#define CK_OR_FREE(call)                                           \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) {                                   \
            int r_ = mixer::cuda_status(e_, #call);                \
            mixer_destroy(c);                                      \
            return r_;                                             \
        }                                                          \
    } while (0)
    CK_OR_FREE(cudaGetDevice(&c->dev));
    c->vis_elems = mixer_vis_elems(d->nant, d->nch);
    c->kt_max = (int64_t)d->max_heaps * d->tpkt;
    c->kt_max = (c->kt_max + 15) / 16 * 16;
    CK_OR_FREE(cudaMalloc(&c->vis64, (size_t)c->vis_elems * sizeof(int64_t)));
    CK_OR_FREE(cudaMemset(c->vis64, 0, (size_t)c->vis_elems * sizeof(int64_t)));
    CK_OR_FREE(cudaMalloc(&c->planes, (size_t)2 * d->nch * d->nant * c->kt_max));
    const int G = c->d.grid;
    CK_OR_FREE(cudaMalloc(&c->grid, (size_t)d->nch * G * G * 2 * sizeof(int64_t)));
    CK_OR_FREE(cudaMalloc(&c->grid_prev, (size_t)d->nch * G * G * 2 * sizeof(int64_t)));
    CK_OR_FREE(cudaMemset(c->grid_prev, 0, (size_t)d->nch * G * G * 2 * sizeof(int64_t)));
    CK_OR_FREE(cudaMalloc(&c->img, (size_t)d->nch * G * G * sizeof(float)));
    CK_OR_FREE(cudaMalloc(&c->vmax, (size_t)d->nch * sizeof(float)));
    CK_OR_FREE(cudaMalloc(&c->vmin, (size_t)d->nch * sizeof(float)));
    CK_OR_FREE(cudaMalloc(&c->d_seq_err, sizeof(uint32_t)));
    CK_OR_FREE(cudaMalloc(&c->d_err, sizeof(int32_t)));
    CK_OR_FREE(cudaMemset(c->d_seq_err, 0, sizeof(uint32_t)));
    CK_OR_FREE(cudaMemset(c->d_err, 0, sizeof(int32_t)));
    CK_OR_FREE(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    for (int s = 0; s < 2; ++s) {
        CK_OR_FREE(cudaEventCreateWithFlags(&c->stage_free[s], cudaEventDisableTiming));
        CK_OR_FREE(cudaEventCreateWithFlags(&c->stage_ready[s], cudaEventDisableTiming));
    }
    c->stage_bytes = (size_t)d->max_heaps * d->nant * d->pkt_stride;
#undef CK_OR_FREE
    *out = c;
    return MIXER_OK;
}

extern "C" int mixer_reset(mixer_ctx* c, void* stream) {
    if (!c) return MIXER_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    MIXER_CK(cudaMemsetAsync(c->vis64, 0, (size_t)c->vis_elems * sizeof(int64_t), st));
    if (c->vis32) MIXER_CK(cudaMemsetAsync(c->vis32, 0, (size_t)c->vis_elems * sizeof(int32_t), st));
    MIXER_CK(cudaMemsetAsync(c->grid_prev, 0,
                             (size_t)c->d.nch * c->d.grid * c->d.grid * 2 * sizeof(int64_t), st));
    MIXER_CK(cudaMemsetAsync(c->d_seq_err, 0, sizeof(uint32_t), st));
    MIXER_CK(cudaMemsetAsync(c->d_err, 0, sizeof(int32_t), st));
    c->samples = 0;
    c->i32_samples = 0;
    return MIXER_OK;
}

// Corner-turn + GEMM over nheaps heaps, staged in chunks of max_heaps.
static int correlate_impl(mixer_ctx* c, const void* packets, int64_t nheaps, uint32_t seq0,
                          int32_t on_device, void* stream, int32_t mode, void* vis) {
    if (!c || !packets || nheaps <= 0) return MIXER_EINVAL;
    const mixer_array_desc& d = c->d;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint8_t* src = static_cast<const uint8_t*>(packets);
    const int64_t heap_bytes = (int64_t)d.nant * d.pkt_stride;
    for (int64_t h0 = 0; h0 < nheaps; h0 += d.max_heaps) {
        const int32_t nh = (int32_t)((nheaps - h0) < d.max_heaps ? (nheaps - h0) : d.max_heaps);
        const uint8_t* chunk = src + h0 * heap_bytes;
        const uint8_t* dev_chunk = chunk;
        if (!on_device) {
            const int s = c->cur;
            if (!c->stage[s]) MIXER_CK(cudaMalloc(&c->stage[s], c->stage_bytes));
            if (c->stage_used[s]) MIXER_CK(cudaStreamWaitEvent(c->copy_stream, c->stage_free[s], 0));
            MIXER_CK(cudaMemcpyAsync(c->stage[s], chunk, (size_t)nh * heap_bytes,
                                     cudaMemcpyHostToDevice, c->copy_stream));
            MIXER_CK(cudaEventRecord(c->stage_ready[s], c->copy_stream));
            MIXER_CK(cudaStreamWaitEvent(st, c->stage_ready[s], 0));
            dev_chunk = c->stage[s];
        }
        const uint32_t sq = seq0 + (uint32_t)(h0 * d.nant);
        int rc = mixer_corner_turn(dev_chunk, d.pkt_stride, d.hdr_bytes, d.nant, d.nch, d.tpkt, nh,
                                   sq, c->planes, c->kt_max, 0, c->d_seq_err, c->d_err, stream);
        if (rc != MIXER_OK) return rc;
        rc = mixer_xcorr_tri(c->planes, d.nant, d.nch, c->kt_max, 0, (int64_t)nh * d.tpkt, mode, vis,
                             c->d_err, stream);
        if (rc != MIXER_OK) return rc;
        if (!on_device) {
            MIXER_CK(cudaEventRecord(c->stage_free[c->cur], st));
            c->stage_used[c->cur] = true;
            c->cur ^= 1;
        }
    }
    return MIXER_OK;
}

extern "C" int mixer_correlate(mixer_ctx* c, const void* packets, int64_t nheaps, uint32_t seq0,
                               int32_t on_device, void* stream) {
    const int rc = correlate_impl(c, packets, nheaps, seq0, on_device, stream, MIXER_VIS_ACC_I64,
                                  c ? c->vis64 : nullptr);
    if (rc == MIXER_OK) c->samples += nheaps * c->d.tpkt;
    return rc;
}

extern "C" int mixer_correlate_i32(mixer_ctx* c, const void* packets, int64_t nheaps, uint32_t seq0,
                                   int32_t on_device, void* stream) {
    if (!c || nheaps <= 0) return MIXER_EINVAL;
    if (c->i32_samples + nheaps * c->d.tpkt > MIXER_KMAX_I32) return MIXER_EOVERFLOW;
    if (!c->vis32) {
        MIXER_CK(cudaMalloc(&c->vis32, (size_t)c->vis_elems * sizeof(int32_t)));
        MIXER_CK(cudaMemsetAsync(c->vis32, 0, (size_t)c->vis_elems * sizeof(int32_t),
                                 static_cast<cudaStream_t>(stream)));
    }
    const int rc = correlate_impl(c, packets, nheaps, seq0, on_device, stream, MIXER_VIS_ACC_I32,
                                  c->vis32);
    if (rc == MIXER_OK) c->i32_samples += nheaps * c->d.tpkt;
    return rc;
}

extern "C" int mixer_integrate(mixer_ctx* c, void* stream) {
    if (!c) return MIXER_EINVAL;
    if (!c->vis32 || c->i32_samples == 0) return MIXER_OK;
    const int rc = mixer_vis_flush(c->vis32, c->vis64, c->vis_elems, stream);
    if (rc == MIXER_OK) {
        c->samples += c->i32_samples;
        c->i32_samples = 0;
    }
    return rc;
}

extern "C" int mixer_dump(mixer_ctx* c, float* out, int32_t out_on_device, void* stream) {
    if (!c || !out) return MIXER_EINVAL;
    const size_t n = (size_t)c->d.nch * 2 * c->d.nant * c->d.nant;
    if (out_on_device) return mixer_vis_dump_f32(c->vis64, c->d.nant, c->d.nch, out, stream);
    if (!c->dump_dev) MIXER_CK(cudaMalloc(&c->dump_dev, n * sizeof(float)));
    int rc = mixer_vis_dump_f32(c->vis64, c->d.nant, c->d.nch, c->dump_dev, stream);
    if (rc != MIXER_OK) return rc;
    MIXER_CK(cudaMemcpyAsync(out, c->dump_dev, n * sizeof(float), cudaMemcpyDeviceToHost,
                             static_cast<cudaStream_t>(stream)));
    return MIXER_OK;
}

extern "C" int mixer_dump_to_file(mixer_ctx* c, const char* path, void* stream) {
    if (!c || !path) return MIXER_EINVAL;
    const size_t n = (size_t)c->d.nch * 2 * c->d.nant * c->d.nant;
    float* host = nullptr;
    MIXER_CK(cudaMallocHost(&host, n * sizeof(float)));
    int rc = mixer_dump(c, host, 0, stream);
    if (rc == MIXER_OK) {
        cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) rc = mixer::cuda_status(e, "cudaStreamSynchronize");
    }
    if (rc == MIXER_OK) {
        FILE* f = fopen(path, "ab");
        if (!f) {
            rc = MIXER_EINVAL;
        } else {
            if (fwrite(host, sizeof(float), n, f) != n) rc = MIXER_EINVAL;
            fclose(f);
        }
    }
    cudaFreeHost(host);
    return rc;
}

extern "C" int mixer_read_vis_i64(mixer_ctx* c, int64_t* out, int32_t full_square,
                                  int32_t out_on_device, void* stream) {
    if (!c || !out) return MIXER_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!full_square) {
        MIXER_CK(cudaMemcpyAsync(out, c->vis64, (size_t)c->vis_elems * sizeof(int64_t),
                                 out_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
        return MIXER_OK;
    }
    const size_t n = (size_t)c->d.nch * 2 * c->d.nant * c->d.nant;
    if (out_on_device) return mixer_vis_unpack_i64(c->vis64, c->d.nant, c->d.nch, out, stream);
    if (!c->unpack_dev) MIXER_CK(cudaMalloc(&c->unpack_dev, n * sizeof(int64_t)));
    int rc = mixer_vis_unpack_i64(c->vis64, c->d.nant, c->d.nch, c->unpack_dev, stream);
    if (rc != MIXER_OK) return rc;
    MIXER_CK(cudaMemcpyAsync(out, c->unpack_dev, n * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    return MIXER_OK;
}

extern "C" int mixer_image(mixer_ctx* c, float* img, float* vmax, float* vmin, int32_t delta,
                           int32_t out_on_device, void* stream) {
    if (!c || !img) return MIXER_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int G = c->d.grid;
    int rc = mixer_grid(c->vis64, c->d.nant, c->d.nch, c->d.side_x, G, c->grid,
                        delta ? c->grid_prev : nullptr, stream);
    if (rc != MIXER_OK) return rc;
    if (out_on_device) return mixer_image_fft(c->grid, c->d.nch, G, img, vmax, vmin, stream);
    rc = mixer_image_fft(c->grid, c->d.nch, G, c->img, c->vmax, c->vmin, stream);
    if (rc != MIXER_OK) return rc;
    MIXER_CK(cudaMemcpyAsync(img, c->img, (size_t)c->d.nch * G * G * sizeof(float),
                             cudaMemcpyDeviceToHost, st));
    if (vmax)
        MIXER_CK(cudaMemcpyAsync(vmax, c->vmax, (size_t)c->d.nch * sizeof(float),
                                 cudaMemcpyDeviceToHost, st));
    if (vmin)
        MIXER_CK(cudaMemcpyAsync(vmin, c->vmin, (size_t)c->d.nch * sizeof(float),
                                 cudaMemcpyDeviceToHost, st));
    return MIXER_OK;
}

extern "C" int mixer_stats(mixer_ctx* c, int64_t* samples, int64_t* seq_errors, int32_t* kernel_err) {
    if (!c) return MIXER_EINVAL;
    if (samples) *samples = c->samples;
    if (seq_errors || kernel_err) {
        MIXER_CK(cudaDeviceSynchronize());
        uint32_t se = 0;
        int32_t ke = 0;
        MIXER_CK(cudaMemcpy(&se, c->d_seq_err, sizeof(se), cudaMemcpyDeviceToHost));
        MIXER_CK(cudaMemcpy(&ke, c->d_err, sizeof(ke), cudaMemcpyDeviceToHost));
        if (seq_errors) *seq_errors = se;
        if (kernel_err) *kernel_err = ke;
        if (ke) return MIXER_ETIMEOUT;
    }
    return MIXER_OK;
}

extern "C" int64_t* mixer_state_ptr(mixer_ctx* c) { return c ? c->vis64 : nullptr; }

extern "C" int mixer_ctx_shape(mixer_ctx* c, int32_t* nant, int32_t* nch) {
    if (!c) return MIXER_EINVAL;
    if (nant) *nant = c->d.nant;
    if (nch) *nch = c->d.nch;
    return MIXER_OK;
}

extern "C" int mixer_write_vis_i64(mixer_ctx* c, const int64_t* tile_packed, int64_t samples) {
    if (!c || !tile_packed || samples < 0) return MIXER_EINVAL;
    MIXER_CK(cudaDeviceSynchronize());
    MIXER_CK(cudaMemcpy(c->vis64, tile_packed, (size_t)c->vis_elems * sizeof(int64_t),
                        cudaMemcpyHostToDevice));
    c->samples = samples;
    return MIXER_OK;
}
