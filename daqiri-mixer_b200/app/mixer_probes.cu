// mixer_probes -- micro-benchmarks behind the X-engine's kernel design choices.
//
//   mixer_probes mma   int8 tcgen05 MMA rate (MACs per SM per clock) for every
//                      M x N shape the triangle GEMM could use (M 64 / 128,
//                      N 64 / 128 / 256), operands resident in shared memory:
//                      tells whether M 64 MMAs (the only way to skip the unused
//                      quadrant of a diagonal tile) keep the per-row rate;
//   mixer_probes mix   the same with mixed shapes in one MMA stream (N 256 and
//                      N 128 interleaved or grouped, A == B, the diagonal-tile
//                      pattern): whether a shape change costs issue slots;
//   mixer_probes tma   TMA load rate (bytes per SM per clock) of 5-D boxes of
//                      16-byte rows taken straight from wire packets (1024
//                      elements x 256 channels x 16 samples per packet), against
//                      4-D boxes of 128-byte rows from corner-turned planes, each
//                      from DRAM-sized buffers and from an L2-resident footprint:
//                      whether the GEMM could read its operands from packets.
// One JSON line per measurement.  Every mbarrier wait is bounded, every TMA
// coordinate is inside its tensor, and every CTA lets its copies land before
// it exits.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "common.cuh"

using namespace mixer;

__global__ void __launch_bounds__(128, 1) k_mma_shape(int M, int N, int64_t iters, long long* cyc,
                                                        int* err) {
    extern __shared__ uint8_t sm[];
    const uint32_t raw = smem_u32(sm);
    const uint32_t base = (raw + 1023u) & ~1023u;
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(&slot), 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = slot;
    if (threadIdx.x == 0) {
        const uint32_t idesc = idesc_i8(M, N);
        const uint64_t a = sdesc_sw128(base), b = sdesc_sw128(base + 32768);
        const long long t0 = clock64();
        for (int64_t it = 0; it < iters; ++it) {
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t o = (uint64_t)((kk * 32) >> 4);
                mma_i8(tmem, a + o, b + o, idesc, (it > 0 || kk > 0) ? 1u : 0u);
            }
        }
        tc_commit(smem_u32(&bar));
        if (!mbar_wait(smem_u32(&bar), 0)) atomicOr(err, 1);
        const long long t1 = clock64();
        if (blockIdx.x == 0) *cyc = t1 - t0;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, 512);
    }
}

// Mixed shapes: mode 0 interleaved (N256 then N128 per K step), 1 grouped (4 x N256
// then 4 x N128), 2 N128 with A == B (same smem), 3 N128 with A != B,
// 4 N256 with B = [A ; next tile] (the diagonal D1 pattern)
__global__ void __launch_bounds__(128, 1) k_mma_mix(int mode, int64_t iters, long long* cyc, int* err) {
    extern __shared__ uint8_t sm[];
    const uint32_t raw = smem_u32(sm);
    const uint32_t base = (raw + 1023u) & ~1023u;
    __shared__ uint64_t bar;
    __shared__ uint32_t slot;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(&bar), 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(&slot), 512);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = slot;
    if (threadIdx.x == 0) {
        const uint32_t i256 = idesc_i8(128, 256), i128 = idesc_i8(128, 128);
        const uint64_t ar = sdesc_sw128(base), ai = sdesc_sw128(base + 16384);
        const long long t0 = clock64();
        for (int64_t it = 0; it < iters; ++it) {
            const uint32_t acc = it > 0 ? 1u : 0u;
            if (mode == 0) {
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const uint64_t o = (uint64_t)((kk * 32) >> 4);
                    mma_i8(tmem, ar + o, ar + o, i256, acc);
                    mma_i8(tmem + 256, ai + o, ai + o, i128, acc);
                }
            } else if (mode == 1) {
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                    mma_i8(tmem, ar + (uint64_t)((kk * 32) >> 4), ar + (uint64_t)((kk * 32) >> 4), i256, acc);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                    mma_i8(tmem + 256, ai + (uint64_t)((kk * 32) >> 4), ai + (uint64_t)((kk * 32) >> 4), i128,
                           acc);
            } else if (mode == 2 || mode == 3) {
                const uint64_t b = mode == 2 ? ai : sdesc_sw128(base + 32768);
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                    mma_i8(tmem + 256, ai + (uint64_t)((kk * 32) >> 4), b + (uint64_t)((kk * 32) >> 4), i128,
                           acc);
            } else {
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    const uint64_t o = (uint64_t)((kk * 32) >> 4);
                    mma_i8(tmem, ar + o, ar + o, i256, acc);
                    mma_i8(tmem + 256, ai + o, ar + o, i256, acc);
                }
            }
        }
        tc_commit(smem_u32(&bar));
        if (!mbar_wait(smem_u32(&bar), 0)) atomicOr(err, 1);
        const long long t1 = clock64();
        if (blockIdx.x == 0) *cyc = t1 - t0;
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, 512);
    }
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x,
                                            int y, int z, int w, int v) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y), "r"(z), "r"(w), "r"(v)
        : "memory");
}

// mode 0: 5-D packet map (t 16 B, channel 1, antenna 128, plane 2, heap hb)
// mode 1: 4-D plane map (k 128 B, antenna 128, channel 1, plane 1), 128-byte swizzle
__global__ void __launch_bounds__(32, 1) k_tma_rate(const __grid_constant__ CUtensorMap map, int mode,
                                                     int loads, int stages, int stage_bytes, int nch,
                                                     int nblk, int nkc, long long* cyc, int* err) {
    extern __shared__ uint8_t sm[];
    const uint32_t raw = smem_u32(sm);
    const uint32_t base = (raw + 1023u) & ~1023u;
    __shared__ uint64_t bars[16];
    if (threadIdx.x != 0) return;
    for (int s = 0; s < stages; ++s) mbar_init(smem_u32(&bars[s]), 1);
    fence_mbar_init();
    const long long t0 = clock64();
    uint32_t phase_bits = 0;
    int issued = 0;
    for (int i = 0; i < loads; ++i) {
        const int s = i % stages;
        if (i >= stages) {
            if (!mbar_wait(smem_u32(&bars[s]), (phase_bits >> s) & 1u)) {
                atomicOr(err, 1);
                break;
            }
            phase_bits ^= 1u << s;
        }
        ++issued;
        const uint32_t dst = base + s * stage_bytes;
        mbar_expect_tx(smem_u32(&bars[s]), stage_bytes);
        const int g = blockIdx.x * 7919 + i;
        const int c = g % nch, rb = (g / nch) % nblk, kc = (g / (nch * nblk)) % nkc;
        if (mode == 0)
            tma_load_5d(dst, &map, smem_u32(&bars[s]), 0, c, rb * 128, 0, kc * (stage_bytes / 4096));
        else
            tma_load_4d(dst, &map, smem_u32(&bars[s]), kc * 128, rb * 128, c, 0);
    }
    // every issued copy lands before the CTA exits (bounded waits)
    for (int q = issued - stages; q < issued; ++q) {
        if (q < 0) continue;
        const int s = q % stages;
        if (!mbar_wait(smem_u32(&bars[s]), (phase_bits >> s) & 1u)) atomicOr(err, 2);
        phase_bits ^= 1u << s;
    }
    const long long t1 = clock64();
    if (blockIdx.x == 0) *cyc = t1 - t0;
}

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                              CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                              CUtensorMapFloatOOBfill);
#define CK(x)                                                                           \
    do {                                                                                \
        cudaError_t e_ = (x);                                                           \
        if (e_ != cudaSuccess) {                                                        \
            fprintf(stderr, "%s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_)); \
            exit(1);                                                                    \
        }                                                                               \
    } while (0)

static void report(const char* what, const char* extra, double bytes_or_macs, long long c, float ms,
                   int sms, int er, bool mma) {
    if (mma)
        printf("{\"probe\":\"%s\",%s,\"macs_per_clk_per_sm\":%.1f,\"ms\":%.3f,\"tops\":%.1f,\"err\":%d}\n",
               what, extra, bytes_or_macs / c, ms, 2.0 * bytes_or_macs * sms / ms / 1e9, er);
    else
        printf("{\"probe\":\"%s\",%s,\"bytes_per_clk_per_sm\":%.1f,\"gbs_all_sms\":%.0f,\"err\":%d}\n",
               what, extra, bytes_or_macs / c, bytes_or_macs * sms / ms / 1e6, er);
}

int main(int argc, char** argv) {
    const char* what = argc > 1 ? argv[1] : "all";
    const bool do_mma = !strcmp(what, "mma") || !strcmp(what, "all");
    const bool do_mix = !strcmp(what, "mix") || !strcmp(what, "all");
    const bool do_tma = !strcmp(what, "tma") || !strcmp(what, "all");
    if (!do_mma && !do_mix && !do_tma) {
        fprintf(stderr, "usage: mixer_probes [mma|mix|tma|all]\n");
        return 2;
    }
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    long long* cyc;
    int* err;
    CK(cudaMalloc(&cyc, 8));
    CK(cudaMalloc(&err, 4));
    CK(cudaMemset(err, 0, 4));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto fetch = [&](long long& c, int& er, float& ms) {
        cudaMemcpy(&c, cyc, 8, cudaMemcpyDeviceToHost);
        cudaMemcpy(&er, err, 4, cudaMemcpyDeviceToHost);
        cudaEventElapsedTime(&ms, e0, e1);
    };
    const int smem1 = 65536 + 1024;
    CK(cudaFuncSetAttribute(k_mma_shape, cudaFuncAttributeMaxDynamicSharedMemorySize, smem1));
    const int shapes[][2] = {{128, 256}, {128, 128}, {128, 64}, {64, 256}, {64, 128}, {64, 64}};
    for (auto& sh : shapes) {
        if (!do_mma) break;
        const int64_t iters = 20000;
        k_mma_shape<<<sms, 128, smem1>>>(sh[0], sh[1], 1000, cyc, err);
        CK(cudaDeviceSynchronize());
        cudaEventRecord(e0);
        k_mma_shape<<<sms, 128, smem1>>>(sh[0], sh[1], iters, cyc, err);
        cudaEventRecord(e1);
        CK(cudaDeviceSynchronize());
        long long c = 0;
        int er = 0;
        float ms = 0;
        fetch(c, er, ms);
        char ex[64];
        snprintf(ex, sizeof ex, "\"M\":%d,\"N\":%d", sh[0], sh[1]);
        report("mma_i8", ex, (double)sh[0] * sh[1] * 32 * 4 * iters, c, ms, sms, er, true);
    }
    if (do_mix) {
        CK(cudaFuncSetAttribute(k_mma_mix, cudaFuncAttributeMaxDynamicSharedMemorySize, smem1));
        const double macs_per_iter[5] = {4.0 * (128 * 256 * 32 + 128 * 128 * 32),
                                         4.0 * (128 * 256 * 32 + 128 * 128 * 32), 4.0 * 128 * 128 * 32,
                                         4.0 * 128 * 128 * 32, 8.0 * 128 * 256 * 32};
        const char* names[5] = {"interleaved_n256_n128", "grouped_n256_n128", "n128_a_eq_b",
                                "n128_a_ne_b", "diag_d1_d2_n256"};
        for (int rep = 0; rep < 2; ++rep)
            for (int mode = 0; mode < 5; ++mode) {
                const int64_t iters = 20000;
                k_mma_mix<<<sms, 128, smem1>>>(mode, 500, cyc, err);
                CK(cudaDeviceSynchronize());
                cudaEventRecord(e0);
                k_mma_mix<<<sms, 128, smem1>>>(mode, iters, cyc, err);
                cudaEventRecord(e1);
                CK(cudaDeviceSynchronize());
                long long c = 0;
                int er = 0;
                float ms = 0;
                fetch(c, er, ms);
                char ex[64];
                snprintf(ex, sizeof ex, "\"mode\":\"%s\"", names[mode]);
                report("mma_mix", ex, macs_per_iter[mode] * iters, c, ms, sms, er, true);
            }
    }
    if (!do_tma) return 0;
    void* fp = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q));
    EncodeFn enc = (EncodeFn)fp;
    const int nant = 1024, nch = 256, tpkt = 16, stride = 8256, nheaps = 512;   // 4.3 GB
    const size_t pk_bytes = (size_t)nheaps * nant * stride;
    uint8_t *pk, *planes;
    CK(cudaMalloc(&pk, pk_bytes));
    CK(cudaMemset(pk, 1, pk_bytes));
    const int kt = nheaps * tpkt;
    CK(cudaMalloc(&planes, (size_t)2 * nch * nant * kt));
    CK(cudaMemset(planes, 1, (size_t)2 * nch * nant * kt));
    const int smem2 = 4 * 32768 + 1024;
    CK(cudaFuncSetAttribute(k_tma_rate, cudaFuncAttributeMaxDynamicSharedMemorySize, smem2));
    for (int l2res : {0, 1})
    for (int hb : {2, 4, 8}) {
        CUtensorMap map;
        const cuuint64_t dims[5] = {16, (cuuint64_t)nch, (cuuint64_t)nant, 2, (cuuint64_t)nheaps};
        const cuuint64_t strides[4] = {16, (cuuint64_t)stride, (cuuint64_t)nch * tpkt,
                                       (cuuint64_t)nant * stride};
        const cuuint32_t box[5] = {16, 1, 128, 2, (cuuint32_t)hb};
        const cuuint32_t es[5] = {1, 1, 1, 1, 1};
        CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 5, pk + 64, dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            printf("{\"probe\":\"tma_packets\",\"hb\":%d,\"encode_error\":%d}\n", hb, (int)r);
            continue;
        }
        // l2res: one 128-antenna block and 32 heaps (34 MB of packets), L2-resident
        const int sb = 2 * 128 * 16 * hb, loads = 4000, nkc = l2res ? 32 / hb : nheaps / hb;
        const int nb = l2res ? 1 : nant / 128;
        k_tma_rate<<<sms, 32, smem2>>>(map, 0, 200, 4, sb, nch, nb, nkc, cyc, err);
        CK(cudaDeviceSynchronize());
        cudaEventRecord(e0);
        k_tma_rate<<<sms, 32, smem2>>>(map, 0, loads, 4, sb, nch, nb, nkc, cyc, err);
        cudaEventRecord(e1);
        CK(cudaDeviceSynchronize());
        long long c = 0;
        int er = 0;
        float ms = 0;
        fetch(c, er, ms);
        char ex[64];
        snprintf(ex, sizeof ex, "\"heaps_per_box\":%d,\"box_bytes\":%d,\"l2_resident\":%d", hb, sb,
                 l2res);
        report("tma_packets_16B_rows", ex, (double)sb * loads, c, ms, sms, er, false);
    }
    {
        CUtensorMap map;
        const cuuint64_t dims[4] = {(cuuint64_t)kt, (cuuint64_t)nant, (cuuint64_t)nch, 2};
        const cuuint64_t strides[3] = {(cuuint64_t)kt, (cuuint64_t)kt * nant,
                                       (cuuint64_t)kt * nant * nch};
        const cuuint32_t box[4] = {128, 128, 1, 1};
        const cuuint32_t es[4] = {1, 1, 1, 1};
        CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, planes, dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        for (int l2res : {0, 1}) if (r == CUDA_SUCCESS) {
            // l2res: one 128-row block, 256 samples of every channel (8.4 MB), L2-resident
            const int sb = 16384, loads = 8000;
            const int nb = l2res ? 1 : nant / 128, nkc = l2res ? 2 : kt / 128;
            k_tma_rate<<<sms, 32, smem2>>>(map, 1, 200, 4, sb, nch, nb, nkc, cyc, err);
            CK(cudaDeviceSynchronize());
            cudaEventRecord(e0);
            k_tma_rate<<<sms, 32, smem2>>>(map, 1, loads, 4, sb, nch, nb, nkc, cyc, err);
            cudaEventRecord(e1);
            CK(cudaDeviceSynchronize());
            long long c = 0;
            int er = 0;
            float ms = 0;
            fetch(c, er, ms);
            report("tma_planes_sw128", l2res ? "\"box_bytes\":16384,\"l2_resident\":1"
                                             : "\"box_bytes\":16384,\"l2_resident\":0",
                   (double)sb * loads, c, ms, sms, er, false);
        }
        if (r != CUDA_SUCCESS) {
            printf("{\"probe\":\"tma_planes_sw128\",\"encode_error\":%d}\n", (int)r);
        }
    }
    return 0;
}
