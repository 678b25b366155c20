// ingest.cpp -- host-side heap alignment of a packet burst, and checkpointing
// of the integration state.
//
// mixer_align_heaps does the job of the reference's drain thread
// (src/rx_host_corr.cu:127-141): it skips to the first packet whose
// big-endian seq (byte 48) is a multiple of nant and hands out whole heaps of
// nant consecutive packets.  The reference looks at the first packet of a
// burst only (:134), so one lost packet inside a group silently shifts every
// later antenna; here every seq is checked and a gap ends the run, so the
// caller resumes at the gap and re-aligns.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "mixer.h"

namespace {
inline uint32_t seq_at(const uint8_t* p) {
    return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3];
}
}  // namespace

extern "C" int mixer_align_heaps(const uint8_t* packets, int64_t npk, int64_t pkt_stride,
                                 int32_t nant, int64_t* first, int64_t* nheaps, int64_t* next,
                                 uint32_t* seq0) {
    if (!packets || npk < 0 || pkt_stride < MIXER_WIRE_SEQ_BYTE + 4 || nant <= 0 || !first ||
        !nheaps || !next)
        return MIXER_EINVAL;
    const uint8_t* s = packets + MIXER_WIRE_SEQ_BYTE;
    int64_t f = 0;
    while (f < npk && seq_at(s + f * pkt_stride) % (uint32_t)nant != 0) ++f;
    *first = f;
    *nheaps = 0;
    if (seq0) *seq0 = f < npk ? seq_at(s + f * pkt_stride) : 0;
    if (f >= npk) {
        *next = npk;
        return MIXER_OK;
    }
    const uint32_t base = seq_at(s + f * pkt_stride);
    int64_t p = f;
    while (p < npk) {
        if (seq_at(s + p * pkt_stride) != base + (uint32_t)(p - f)) break;   // gap or reorder
        ++p;
    }
    const int64_t whole = (p - f) / nant;
    *nheaps = whole;
    // resume at the gap if one ended the run, else right after the last whole heap
    *next = (p < npk) ? p : f + whole * nant;
    return MIXER_OK;
}

// ---- checkpoint of the integration state --------------------------------------
namespace {
struct CkptHeader {
    char magic[8];          // "MIXCKPT1"
    int32_t nant, nch;
    int64_t samples;
    int64_t elems;          // int64 values that follow (tile-packed re/im)
};
}  // namespace

extern "C" int mixer_state_save(mixer_ctx* ctx, const char* path) {
    if (!ctx || !path) return MIXER_EINVAL;
    int64_t samples = 0;
    int rc = mixer_stats(ctx, &samples, nullptr, nullptr);
    if (rc != MIXER_OK) return rc;
    int32_t nant = 0, nch = 0;
    rc = mixer_ctx_shape(ctx, &nant, &nch);
    if (rc != MIXER_OK) return rc;
    const int64_t n = mixer_vis_elems(nant, nch);
    std::vector<int64_t> host((size_t)n);
    if (cudaDeviceSynchronize() != cudaSuccess) return MIXER_ECUDA;
    rc = mixer_read_vis_i64(ctx, host.data(), 0, 0, nullptr);
    if (rc != MIXER_OK) return rc;
    if (cudaDeviceSynchronize() != cudaSuccess) return MIXER_ECUDA;
    CkptHeader h;
    memcpy(h.magic, "MIXCKPT1", 8);
    h.nant = nant;
    h.nch = nch;
    h.samples = samples;
    h.elems = n;
    FILE* f = fopen(path, "wb");
    if (!f) return MIXER_EINVAL;
    const bool ok = fwrite(&h, sizeof(h), 1, f) == 1 &&
                    fwrite(host.data(), sizeof(int64_t), (size_t)n, f) == (size_t)n;
    fclose(f);
    return ok ? MIXER_OK : MIXER_EINVAL;
}

extern "C" int mixer_state_load(mixer_ctx* ctx, const char* path) {
    if (!ctx || !path) return MIXER_EINVAL;
    int32_t nant = 0, nch = 0;
    int rc = mixer_ctx_shape(ctx, &nant, &nch);
    if (rc != MIXER_OK) return rc;
    FILE* f = fopen(path, "rb");
    if (!f) return MIXER_EINVAL;
    CkptHeader h;
    if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, "MIXCKPT1", 8) != 0 || h.nant != nant ||
        h.nch != nch || h.elems != mixer_vis_elems(nant, nch)) {
        fclose(f);
        return MIXER_EINVAL;
    }
    std::vector<int64_t> host((size_t)h.elems);
    const bool ok = fread(host.data(), sizeof(int64_t), (size_t)h.elems, f) == (size_t)h.elems;
    fclose(f);
    if (!ok) return MIXER_EINVAL;
    return mixer_write_vis_i64(ctx, host.data(), h.samples);
}

// ---- time-split multi-queue ingest ----------------------------------------------
// The reference's sender steers snapshot (heap) tb to RX queue tb % MIXER_NQ through
// the UDP destination port MIXER_UDP_PORT + q (src/config.h:40-45), so each queue
// carries every nq-th heap.  The merge below restores time order on the host: heap
// tb comes from queue tb % nq, must be the next heap at that queue's cursor, hold
// nant packets with seqs tb * nant + a (a = 0 .. nant-1) and, when udp_port0 != 0,
// carry destination port udp_port0 + q.  Heaps are copied to `out` until the first
// one that is missing, incomplete, misordered or on the wrong port; every packet a
// queue holds before its first aligned heap is skipped.  Integration is a sum over
// samples, so the merged heaps give the same visibilities as one unsplit queue.
extern "C" int mixer_merge_time_split(const uint8_t* const* queues, const int64_t* queue_npk,
                                      int32_t nq, int64_t pkt_stride, int32_t nant,
                                      uint16_t udp_port0, int64_t max_heaps, uint8_t* out,
                                      int64_t* out_heaps, uint32_t* seq0, int64_t* consumed) {
    if (!queues || !queue_npk || nq <= 0 || nq > 1024 || nant <= 0 ||
        pkt_stride < MIXER_WIRE_SEQ_BYTE + 4 || max_heaps < 0 || !out_heaps || !consumed ||
        (max_heaps > 0 && !out))
        return MIXER_EINVAL;
    for (int32_t q = 0; q < nq; ++q)
        if (queue_npk[q] < 0 || (queue_npk[q] > 0 && !queues[q])) return MIXER_EINVAL;
    auto seq = [&](int32_t q, int64_t p) { return seq_at(queues[q] + p * pkt_stride + MIXER_WIRE_SEQ_BYTE); };
    auto port = [&](int32_t q, int64_t p) {
        const uint8_t* h = queues[q] + p * pkt_stride;
        return (uint16_t)((h[36] << 8) | h[37]);     // UDP destination port (eth 14 + ipv4 20 + 2)
    };
    // each queue's cursor: its first packet that starts a heap
    std::vector<int64_t> cur(nq);
    int64_t start_tb = -1;
    for (int32_t q = 0; q < nq; ++q) {
        int64_t p = 0;
        while (p < queue_npk[q] && seq(q, p) % (uint32_t)nant != 0) ++p;
        cur[q] = p;
        if (p < queue_npk[q]) {
            const int64_t tb = seq(q, p) / (uint32_t)nant;
            if (start_tb < 0 || tb < start_tb) start_tb = tb;
        }
    }
    *out_heaps = 0;
    if (seq0) *seq0 = start_tb >= 0 ? (uint32_t)(start_tb * nant) : 0;
    int64_t n = 0;
    for (int64_t tb = start_tb; start_tb >= 0 && n < max_heaps; ++tb, ++n) {
        const int32_t q = (int32_t)(tb % nq);
        const int64_t p0 = cur[q];
        if (p0 + nant > queue_npk[q]) break;                     // not (yet) complete
        bool ok = true;
        for (int32_t a = 0; a < nant && ok; ++a) {
            ok = seq(q, p0 + a) == (uint32_t)(tb * nant + a) &&
                 (udp_port0 == 0 || port(q, p0 + a) == (uint16_t)(udp_port0 + q));
        }
        if (!ok) break;
        memcpy(out + n * nant * pkt_stride, queues[q] + p0 * pkt_stride, (size_t)(nant * pkt_stride));
        cur[q] = p0 + nant;
    }
    *out_heaps = n;
    for (int32_t q = 0; q < nq; ++q) consumed[q] = cur[q];
    return MIXER_OK;
}
