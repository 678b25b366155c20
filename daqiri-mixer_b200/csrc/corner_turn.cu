// corner_turn.cu -- packets (wire format) -> per-channel int8 planes.
//
// Replaces k_packAB (reference src/rx_host_corr.cu:61-72), which reads one
// byte per thread and writes four planes (A = X and B = conj(X), both
// [ch][ant][k]) one byte at a time.  Here one CTA owns one antenna and `hg`
// consecutive heaps of it, for a group of nchg channels:
//   1. one thread issues 2 x `hg` bulk TMA copies (cp.async.bulk) of the
//      group's re and im bytes of each payload into shared memory (heap stride
//      padded by tpkt bytes so the read-out below is free of bank conflicts);
//   2. all threads write the two planes re / im [C][N][kt] with 16-byte
//      stores, hg*tpkt contiguous bytes (whole cache lines) per (plane,
//      channel) row;
//   3. the first hg threads check each packet's big-endian seq at byte 48
//      against its position (the reference checks only the first packet of a
//      burst, src/rx_host_corr.cu:134).
// HBM-bound: algorithmic bytes = packets read + planes written.
#include "common.cuh"

namespace mixer {
namespace {

__global__ void __launch_bounds__(256)
    k_corner_turn(const uint8_t* __restrict__ pk, int64_t pkt_stride, int hdr, int nant, int nch,
                  int tpkt, int hg, int nchg, uint32_t seq0, int8_t* __restrict__ planes, int64_t kt,
                  int64_t k0, uint32_t* seq_err, int32_t* err) {
    extern __shared__ __align__(128) uint8_t sm[];
    __shared__ __align__(8) uint64_t bar_store;
    const int a = blockIdx.x;
    const int g = blockIdx.y;
    const int c0 = blockIdx.z * nchg;      // first channel of this CTA's group
    const int half = nch * tpkt;           // bytes per re or im plane of a payload
    const int part = nchg * tpkt;          // bytes of one plane staged per heap
    const int hstride = 2 * part + tpkt;   // padded heap stride in shared memory
    const uint32_t bar = smem_u32(&bar_store);

    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
        mbar_expect_tx(bar, (uint32_t)(hg * 2 * part));
        for (int hl = 0; hl < hg; ++hl) {
            const int64_t p = (int64_t)(g * hg + hl) * nant + a;
            const uint8_t* src = pk + p * pkt_stride + hdr + (int64_t)c0 * tpkt;
            bulk_g2s(smem_u32(sm + hl * hstride), src, (uint32_t)part, bar);                // re
            bulk_g2s(smem_u32(sm + hl * hstride + part), src + half, (uint32_t)part, bar);  // im
        }
    }
    if (seq_err && blockIdx.z == 0 && threadIdx.x < hg) {
        const int64_t p = (int64_t)(g * hg + threadIdx.x) * nant + a;
        const uint8_t* h = pk + p * pkt_stride + MIXER_WIRE_SEQ_BYTE;
        const uint32_t s = ((uint32_t)h[0] << 24) | ((uint32_t)h[1] << 16) |
                           ((uint32_t)h[2] << 8) | (uint32_t)h[3];
        if (s != seq0 + (uint32_t)p) atomicAdd(seq_err, 1u);
    }
    __syncthreads();   // barrier initialised before anyone polls it
    if (!mbar_wait(bar, 0)) {
        if (err) atomicOr(err, 8);
        mbar_wait(bar, 0);   // second bounded wait for the copies in flight
        return;
    }

    const int V = hg * tpkt / 16;              // 16-byte vectors per (plane, channel) row
    const int total = 2 * nchg * V;
    const int64_t kcol = k0 + (int64_t)g * hg * tpkt;
    if (blockDim.x % V == 0) {
        // Each thread keeps one column v of the rows and walks the channel rows
        // of each plane with pointer increments only (no multiply per store).
        const int v = threadIdx.x % V;
        const int rstep = blockDim.x / V;
        const int kb = v * 16;
        const int hl = kb / tpkt;
        const int64_t cstride = (int64_t)nant * kt;   // one channel row to the next
        const int64_t dstep = (int64_t)rstep * cstride;
        const int sstep = rstep * tpkt;
        const int cl0 = threadIdx.x / V;
#pragma unroll 1
        for (int plane = 0; plane < 2; ++plane) {
            const uint8_t* src = sm + hl * hstride + (kb - hl * tpkt) + plane * part + cl0 * tpkt;
            int8_t* dst = planes + ((int64_t)plane * nch + c0 + cl0) * cstride + (int64_t)a * kt +
                          kcol + kb;
#pragma unroll 4
            for (int cl = cl0; cl < nchg; cl += rstep) {
                *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(src);
                src += sstep;
                dst += dstep;
            }
        }
        return;
    }
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int v = idx % V;
        const int pc = idx / V;                // plane * nchg + local channel
        const int plane = pc / nchg;
        const int cl = pc - plane * nchg;
        const int kb = v * 16;
        const int hl = kb / tpkt;
        const int t0 = kb - hl * tpkt;
        const uint4 val =
            *reinterpret_cast<const uint4*>(sm + hl * hstride + plane * part + cl * tpkt + t0);
        int8_t* dst = planes + (((int64_t)plane * nch + c0 + cl) * nant + a) * kt + kcol + kb;
        *reinterpret_cast<uint4*>(dst) = val;
    }
}

// Heaps per CTA (hg): output row chunks of up to MIXER_CT_ROW_BYTES contiguous
// bytes (whole cache lines), a divisor of nheaps.  Channels per CTA (nchg): the
// largest divisor of nch whose staging fits MIXER_CT_SMEM_MAX, so several CTAs
// share an SM and overlap their loads and stores.
#ifndef MIXER_CT_ROW_BYTES
#define MIXER_CT_ROW_BYTES 256
#endif
#ifndef MIXER_CT_SMEM_MAX
#define MIXER_CT_SMEM_MAX (73 * 1024)
#endif
void pick_split(int nheaps, int nch, int tpkt, int& hg, int& nchg) {
    hg = 1;
    while (hg * tpkt < MIXER_CT_ROW_BYTES && nheaps % (hg * 2) == 0 &&
           (hg * 2) * (2 * tpkt + tpkt) <= MIXER_CT_SMEM_MAX)
        hg *= 2;
    nchg = nch;
    while ((int64_t)hg * (2LL * nchg * tpkt + tpkt) > MIXER_CT_SMEM_MAX) {
        int d = nchg - 1;
        while (d > 1 && nch % d != 0) --d;
        if (d < 1) d = 1;
        if (d == nchg) break;
        nchg = d;
    }
}

}  // namespace
}  // namespace mixer

extern "C" int mixer_corner_turn(const uint8_t* packets, int64_t pkt_stride, int32_t hdr_bytes,
                                 int32_t nant, int32_t nch, int32_t tpkt, int32_t nheaps,
                                 uint32_t seq0, int8_t* planes, int64_t kt, int64_t k0,
                                 uint32_t* seq_errors, int32_t* err, void* stream) {
    if (!packets || !planes || nant <= 0 || nch <= 0 || tpkt <= 0 || nheaps <= 0) return MIXER_EINVAL;
    if (tpkt % 16 != 0 || pkt_stride % 16 != 0 || hdr_bytes % 16 != 0 || kt % 16 != 0 ||
        k0 % 16 != 0 || k0 < 0)
        return MIXER_EINVAL;
    const int64_t P = 2LL * nch * tpkt;
    if (hdr_bytes < MIXER_WIRE_SEQ_BYTE + 4 || hdr_bytes + P > pkt_stride) return MIXER_EINVAL;
    if (P + tpkt > 200 * 1024) return MIXER_EINVAL;
    if (k0 + (int64_t)nheaps * tpkt > kt) return MIXER_EINVAL;
    if (reinterpret_cast<uintptr_t>(packets) % 16 || reinterpret_cast<uintptr_t>(planes) % 16)
        return MIXER_EINVAL;
    int hg, nchg;
    mixer::pick_split(nheaps, nch, tpkt, hg, nchg);
    if (nheaps / hg > 65535) return MIXER_EINVAL;   // grid.y limit
    const size_t smem = (size_t)hg * (size_t)(2 * nchg * tpkt + tpkt);
    if (smem > 48 * 1024)
        MIXER_CK(cudaFuncSetAttribute(mixer::k_corner_turn,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((unsigned)nant, (unsigned)(nheaps / hg), (unsigned)(nch / nchg));
    mixer::k_corner_turn<<<grid, 256, smem, static_cast<cudaStream_t>(stream)>>>(
        packets, pkt_stride, hdr_bytes, nant, nch, tpkt, hg, nchg, seq0, planes, kt, k0, seq_errors,
        err);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}
