// vis.cu -- integration and output of the tile-packed visibility cube.
//
//  * mixer_vis_flush: vis64 += vis32, vis32 = 0.  Replaces k_flush_cube
//    (reference src/rx_host_corr.cu:90-95), which adds into a float cube and
//    stops being exact once an entry passes 2^24.
//  * mixer_vis_dump_f32 / mixer_vis_unpack_i64: the full-square cube
//    [C][2][N][N] of the --dump record (src/rx_host_corr.cu:187,225-227),
//    mirrored from the lower triangle by conjugation.  One CTA per 32 x 32
//    sub-block of a tile plane: coalesced loads along the tile's row index,
//    a shared-memory transpose for the lower half, direct stores for the
//    mirrored upper half.
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

// grid: x = 16 sub-blocks of a tile, y = tile * 2 + plane, z = channel
template <typename T>
__global__ void __launch_bounds__(256)
    k_vis_unpack(const long long* __restrict__ vis, int nant, int ntiles, T* __restrict__ out) {
    __shared__ long long s[32][33];
    const int sb = blockIdx.x;
    const int mi = sb >> 2, ni = sb & 3;
    const int t = blockIdx.y >> 1, p = blockIdx.y & 1;
    const int c = blockIdx.z;
    int i, j;
    decode_tile_v(t, i, j);
    const long long* src = vis + (((size_t)c * ntiles + t) * 2 + p) * 16384;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {
        const int n = 32 * ni + r, m = 32 * mi + tx;
        s[r][tx] = src[n * 128 + m];
    }
    __syncthreads();
    T* plane = out + ((size_t)c * 2 + p) * (size_t)nant * nant;
    // V[a][b], a = 128 i + m (row), b = 128 j + n (column): b contiguous
    for (int r = ty; r < 32; r += 8) {
        const int m = 32 * mi + r, n = 32 * ni + tx;
        const int a = 128 * i + m, b = 128 * j + n;
        if (a < nant && b < nant) plane[(size_t)a * nant + b] = conv<T>(s[tx][r]);
    }
    if (i != j) {   // mirrored entry V[b][a] = conj(V[a][b]): a contiguous
        for (int r = ty; r < 32; r += 8) {
            const int n = 32 * ni + r, m = 32 * mi + tx;
            const int a = 128 * i + m, b = 128 * j + n;
            if (a < nant && b < nant) {
                const long long v = s[r][tx];
                plane[(size_t)b * nant + a] = p ? conv<T>(-v) : conv<T>(v);
            }
        }
    }
}

template <typename T>
int unpack(const int64_t* vis64, int32_t nant, int32_t nch, T* out, void* stream) {
    if (!vis64 || !out || nant <= 0 || nch <= 0 || nch > 65535) return MIXER_EINVAL;
    const int nt = mixer_vis_tiles(nant);
    if (2 * nt > 65535) return MIXER_EINVAL;
    dim3 grid(16, (unsigned)(2 * nt), (unsigned)nch);
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
