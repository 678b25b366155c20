// vis.cu -- integration and output of the tile-packed visibility cube.
//
//  * mixer_vis_flush: vis64 += vis32, vis32 = 0.  Replaces k_flush_cube
//    (reference src/rx_host_corr.cu:90-95), which adds into a float cube and
//    stops being exact once an entry passes 2^24.
//  * mixer_vis_dump_f32 / mixer_vis_unpack_i64: the full-square cube
//    [C][2][N][N] of the --dump record (src/rx_host_corr.cu:187,225-227),
//    mirrored from the lower triangle by conjugation.  One CTA per 128 x 32
//    column group of a tile plane: coalesced loads along the tile's row
//    index, a shared-memory transpose for the lower half, direct stores for
//    the mirrored upper half.
#include "common.cuh"

namespace mixer {
namespace {

__global__ void __launch_bounds__(256)
    k_vis_flush(int4* __restrict__ v32, longlong2* __restrict__ v64, int64_t n4) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int4 a = v32[i];
        longlong2 lo = v64[2 * i], hi = v64[2 * i + 1];
        lo.x += a.x;
        lo.y += a.y;
        hi.x += a.z;
        hi.y += a.w;
        v64[2 * i] = lo;
        v64[2 * i + 1] = hi;
        v32[i] = make_int4(0, 0, 0, 0);
    }
}

__device__ __forceinline__ void decode_tile_v(int t, int& i, int& j) {
    int ii = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
    while ((ii + 1) * (ii + 2) / 2 <= t) ++ii;
    while (ii * (ii + 1) / 2 > t) --ii;
    i = ii;
    j = t - ii * (ii + 1) / 2;
}

template <typename T>
__device__ __forceinline__ T conv(long long v);
template <>
__device__ __forceinline__ float conv<float>(long long v) {
    return __ll2float_rn(v);
}
template <>
__device__ __forceinline__ long long conv<long long>(long long v) {
    return v;
}

// grid: x = 32-column group of a tile (4), y = tile * 2 + plane, z = channel.
// A CTA reads 128 rows x 32 columns of one tile plane (32 KB of int64, 16
// loads of 8 bytes a thread in flight, each warp instruction 256 contiguous
// bytes).  The mirrored upper entries V[b][a] = conj(V[a][b]) are the tile's
// columns, contiguous in the output too, so they are written straight from
// registers; the lower entries V[a][b] go through a shared-memory transpose
// (row stride 129: conflict-free both ways).
template <typename T>
__global__ void __launch_bounds__(256)
    k_vis_unpack(const long long* __restrict__ vis, int nant, int ntiles, T* __restrict__ out) {
    __shared__ T s[32][129];
    const int ng = blockIdx.x;
    const int t = blockIdx.y >> 1, p = blockIdx.y & 1;
    const int c = blockIdx.z;
    int i, j;
    decode_tile_v(t, i, j);
    const long long* src =
        vis + (((size_t)c * ntiles + t) * 2 + p) * 16384 + (size_t)(32 * ng) * 128;
    T* plane = out + ((size_t)c * 2 + p) * (size_t)nant * nant;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int a0 = 128 * i, b0 = 128 * j + 32 * ng;
    long long v[4][4];   // column w + 8 q, row lane + 32 r
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) v[q][r] = src[(w + 8 * q) * 128 + lane + 32 * r];
    if (i != j) {        // mirrored entry V[b][a]: a contiguous
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int b = b0 + w + 8 * q;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int a = a0 + lane + 32 * r;
                if (a < nant && b < nant)
                    plane[(size_t)b * nant + a] = p ? conv<T>(-v[q][r]) : conv<T>(v[q][r]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) s[w + 8 * q][lane + 32 * r] = conv<T>(v[q][r]);
    __syncthreads();
    // V[a][b], a = 128 i + m (row), b = 128 j + 32 ng + lane: b contiguous
    const int b = b0 + lane;
#pragma unroll 4
    for (int k = 0; k < 16; ++k) {
        const int m = 16 * w + k;
        const int a = a0 + m;
        if (a < nant && b < nant) plane[(size_t)a * nant + b] = s[lane][m];
    }
}

template <typename T>
int unpack(const int64_t* vis64, int32_t nant, int32_t nch, T* out, void* stream) {
    if (!vis64 || !out || nant <= 0 || nch <= 0 || nch > 65535) return MIXER_EINVAL;
    const int nt = mixer_vis_tiles(nant);
    if (2 * nt > 65535) return MIXER_EINVAL;
    dim3 grid(4, (unsigned)(2 * nt), (unsigned)nch);
    k_vis_unpack<T><<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const long long*>(vis64), nant, nt, out);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}

}  // namespace
}  // namespace mixer

extern "C" int mixer_vis_flush(int32_t* vis32, int64_t* vis64, int64_t n, void* stream) {
    if (!vis32 || !vis64 || n <= 0 || n % 4 != 0) return MIXER_EINVAL;
    if (reinterpret_cast<uintptr_t>(vis32) % 16 || reinterpret_cast<uintptr_t>(vis64) % 16)
        return MIXER_EINVAL;
    const int64_t n4 = n / 4;
    int64_t blocks = (n4 + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    mixer::k_vis_flush<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<int4*>(vis32), reinterpret_cast<longlong2*>(vis64), n4);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}

extern "C" int mixer_vis_dump_f32(const int64_t* vis64, int32_t nant, int32_t nch, float* cube,
                                  void* stream) {
    return mixer::unpack<float>(vis64, nant, nch, cube, stream);
}

extern "C" int mixer_vis_unpack_i64(const int64_t* vis64, int32_t nant, int32_t nch, int64_t* cube,
                                    void* stream) {
    return mixer::unpack<long long>(vis64, nant, nch, reinterpret_cast<long long*>(cube), stream);
}
