// image.cu -- exact uv-gridding of the integrated cube and a batched
// shared-memory 2-D FFT.
//
// mixer_grid replaces k_grid_cube (reference src/rx_host_corr.cu:79-85): the
// reference scatters every ordered pair (a, b) of the FP32 cube with float
// atomicAdd, so its sum depends on the order of the atomics.  Here each CTA
// owns one (channel, lower-triangle tile), accumulates int64 sums in a small
// shared-memory window of the baseline offsets that tile can reach, and adds
// window cell S(d) to grid cell d and conj(S(d)) to cell -d with int64
// atomics: the pair (b, a) carries conj(V[a][b]), so this equals the
// full-square sum exactly, in any order.
//
// mixer_image_fft replaces cufftPlanMany/cufftExecC2C (src/rx_host_corr.cu:
// 205-206,222) plus the host fftshift / real part / min-max loop (:230-235):
// one CTA per channel loads the int64 grid as complex FP32 in bit-reversed
// order, runs radix-2 butterflies along rows then columns in shared memory
// with twiddles generated in FP64, and writes Re(F) shifted by G/2 in both
// axes together with the channel's max and min.
#include <mutex>
#include "common.cuh"

namespace mixer {
// Largest shared-memory window k_grid_tiles is launched with.
constexpr size_t kGridSmemMax = 200 * 1024;
size_t grid_smem_bytes(int nant, int side_x);

namespace {

__device__ __forceinline__ void decode_tile_g(int t, int& i, int& j) {
    int ii = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
    while ((ii + 1) * (ii + 2) / 2 <= t) ++ii;
    while (ii * (ii + 1) / 2 > t) --ii;
    i = ii;
    j = t - ii * (ii + 1) / 2;
}

__host__ __device__ inline int floordiv(int a, int b) { return a / b; }   // a >= 0

__host__ __device__ inline void tile_window(int i, int j, int nant, int sx, int& dylo, int& ny) {
    const int a0 = 128 * i, a1 = min(128 * i + 128, nant) - 1;
    const int b0 = 128 * j, b1 = min(128 * j + 128, nant) - 1;
    dylo = floordiv(a0, sx) - floordiv(b1, sx);
    const int dyhi = floordiv(a1, sx) - floordiv(b0, sx);
    ny = dyhi - dylo + 1;
}

__device__ __forceinline__ int pmod(int v, int g) {
    const int r = v % g;
    return r < 0 ? r + g : r;
}

// grid: x = tile, y = channel.  smem: windows re [ny][2 sx - 1] then im, int64.
// Launched with 256 threads: a thread keeps one tile row m (one element a) and
// walks every other column, four loads of each plane in flight before their
// adds, with the column element's array position advanced instead of divided.
__global__ void __launch_bounds__(256)
    k_grid_tiles(const long long* __restrict__ vis, int nant, int ntiles, int sx, int G,
                 unsigned long long* __restrict__ grid) {
    extern __shared__ unsigned long long win[];
    __shared__ unsigned long long diag[2];
    const int t = blockIdx.x, c = blockIdx.y;
    int i, j;
    decode_tile_g(t, i, j);
    int dylo, ny;
    tile_window(i, j, nant, sx, dylo, ny);
    const int nx = 2 * sx - 1;
    const int ncell = ny * nx;
    unsigned long long* win_re = win;
    unsigned long long* win_im = win + ncell;
    for (int q = threadIdx.x; q < 2 * ncell; q += blockDim.x) win[q] = 0ull;
    if (threadIdx.x < 2) diag[threadIdx.x] = 0ull;
    __syncthreads();

    const long long* re = vis + (((size_t)c * ntiles + t) * 2) * 16384;
    const long long* im = re + 16384;
    const int m = threadIdx.x & 127;             // this thread's tile row
    const int a = 128 * i + m;
    const int ya = a / sx, xa = a - ya * sx;
    // Columns n = n0, n0 + 2, ... below nlim: the array's last element and, on a
    // diagonal tile, the row itself (the upper half is the mirror image).
    int nlim = nant - 128 * j;
    if (nlim > 128) nlim = 128;
    if (i == j && nlim > m + 1) nlim = m + 1;
    if (a >= nant) nlim = 0;
    int n = threadIdx.x >> 7;
    int yb = (128 * j + n) / sx;                 // the column element's array position,
    int xb = 128 * j + n - yb * sx;              // advanced by two columns a step
    const int cbase = (ya - dylo) * nx + xa + sx - 1;   // cell = cbase - yb * nx - xb
#pragma unroll 1
    for (; n < nlim; n += 8) {
        long long vr[4], vi[4];
        int cell[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int nn = n + 2 * u;
            cell[u] = -2;
            vr[u] = 0;
            vi[u] = 0;
            if (nn < nlim) {
                vr[u] = re[nn * 128 + m];
                vi[u] = im[nn * 128 + m];
                cell[u] = (a == 128 * j + nn) ? -1 : cbase - yb * nx - xb;
            }
            xb += 2;
            while (xb >= sx) {
                xb -= sx;
                ++yb;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (cell[u] >= 0) {
                atomicAdd(&win_re[cell[u]], (unsigned long long)vr[u]);
                atomicAdd(&win_im[cell[u]], (unsigned long long)vi[u]);
            } else if (cell[u] == -1) {
                atomicAdd(&diag[0], (unsigned long long)vr[u]);
                atomicAdd(&diag[1], (unsigned long long)vi[u]);
            }
        }
    }
    __syncthreads();
    unsigned long long* gc = grid + (size_t)c * G * G * 2;
    for (int q = threadIdx.x; q < ncell; q += blockDim.x) {
        const unsigned long long sr = win_re[q], si = win_im[q];
        if (sr == 0ull && si == 0ull) continue;
        const int dy = q / nx + dylo, dx = q % nx - (sx - 1);
        const int f = pmod(dy, G) * G + pmod(dx, G);
        const int r = pmod(-dy, G) * G + pmod(-dx, G);
        atomicAdd(&gc[2 * f + 0], sr);
        atomicAdd(&gc[2 * f + 1], si);
        atomicAdd(&gc[2 * r + 0], sr);
        atomicAdd(&gc[2 * r + 1], (unsigned long long)(-(long long)si));
    }
    if (threadIdx.x == 0 && (diag[0] | diag[1])) {
        atomicAdd(&gc[0], diag[0]);
        atomicAdd(&gc[1], diag[1]);
    }
}

// grid = grid - prev, prev = old grid (delta imaging), n int64 values.
__global__ void k_grid_delta(long long* __restrict__ grid, long long* __restrict__ prev, int64_t n) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const long long g = grid[q];
        grid[q] = g - prev[q];
        prev[q] = g;
    }
}

__global__ void __launch_bounds__(512)
    k_image_fft(const long long* __restrict__ grid, int G, int logG, float* __restrict__ img,
                float* __restrict__ vmax, float* __restrict__ vmin) {
    extern __shared__ float2 S[];               // [G][G] then twiddles [G/2]
    float2* tw = S + G * G;
    __shared__ float red_max[16], red_min[16];
    const int c = blockIdx.x;
    const int GG = G * G, H = G / 2;
    // twiddles W_G^k = exp(-2 pi i k / G), generated in FP64
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * (double)k / (double)G, &sn, &cs);
        tw[k] = make_float2((float)cs, (float)(-sn));
    }
    const long long* g = grid + (size_t)c * GG * 2;
    const int sh = 32 - logG;
    for (int q = threadIdx.x; q < GG; q += blockDim.x) {
        const int y = q / G, x = q - y * G;
        const int yb = (int)(__brev((unsigned)y) >> sh), xb = (int)(__brev((unsigned)x) >> sh);
        S[yb * G + xb] = make_float2(__ll2float_rn(g[2 * q]), __ll2float_rn(g[2 * q + 1]));
    }
    __syncthreads();
    // pass 0: along x (within rows); pass 1: along y (within columns)
    for (int pass = 0; pass < 2; ++pass) {
        for (int s = 0; s < logG; ++s) {
            const int h = 1 << s;
            const int tstride = H >> s;          // twiddle index step
            for (int bf = threadIdx.x; bf < G * H; bf += blockDim.x) {
                const int line = bf / H, r = bf - line * H;
                const int jj = r & (h - 1), blk = r >> s;
                const int i0 = blk * 2 * h + jj, i1 = i0 + h;
                const int a0 = pass == 0 ? line * G + i0 : i0 * G + line;
                const int a1 = pass == 0 ? line * G + i1 : i1 * G + line;
                const float2 w = tw[jj * tstride];
                const float2 u = S[a0], v = S[a1];
                const float2 vw = make_float2(v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x);
                S[a0] = make_float2(u.x + vw.x, u.y + vw.y);
                S[a1] = make_float2(u.x - vw.x, u.y - vw.y);
            }
            __syncthreads();
        }
    }
    float mx = -3.4e38f, mn = 3.4e38f;
    float* out = img + (size_t)c * GG;
    for (int q = threadIdx.x; q < GG; q += blockDim.x) {
        const int y = q / G, x = q - y * G;
        const float v = S[((y + H) & (G - 1)) * G + ((x + H) & (G - 1))].x;
        out[q] = v;
        mx = fmaxf(mx, v);
        mn = fminf(mn, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    if ((threadIdx.x & 31) == 0) {
        red_max[threadIdx.x >> 5] = mx;
        red_min[threadIdx.x >> 5] = mn;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            mx = fmaxf(mx, red_max[w]);
            mn = fminf(mn, red_min[w]);
        }
        if (vmax) vmax[c] = mx;
        if (vmin) vmin[c] = mn;
    }
}

// Warp-level form for G = 32, 64 or 128 (E = G / 32 values a lane).  A
// length-G DIF FFT runs inside one warp: lane l holds elements x = l + 32 e;
// stages of span h >= 32 pair values of the same lane, stages of span h < 32
// pair lane l with lane l ^ h through shuffles, so no stage needs a block
// barrier.  Rows first (grid rows read from global memory, coalesced), then
// columns (from the padded shared-memory image, stride G + 1), both written
// back in natural order (DIF leaves element x holding frequency bitrev(x));
// then the shifted real part and the channel's max / min as above.
template <int G>
__device__ __forceinline__ void warp_fft(float2 (&v)[G / 32], const float2* __restrict__ tw, int lane) {
    constexpr int E = G / 32;
#pragma unroll
    for (int h = G / 2; h >= 32; h >>= 1) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
            if ((32 * e) & h) continue;                // upper element of its pair
            const int e2 = e + h / 32;
            const int j = (lane + 32 * e) & (2 * h - 1);
            const float2 w = tw[j * (G / (2 * h))];
            const float2 u = v[e], q = v[e2];
            const float2 d = make_float2(u.x - q.x, u.y - q.y);
            v[e] = make_float2(u.x + q.x, u.y + q.y);
            v[e2] = make_float2(d.x * w.x - d.y * w.y, d.x * w.y + d.y * w.x);
        }
    }
#pragma unroll
    for (int h = 16; h >= 1; h >>= 1) {
        const bool upper = (lane & h) != 0;
        const float2 w = tw[(lane & (h - 1)) * (G / (2 * h))];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const float qx = __shfl_xor_sync(0xffffffffu, v[e].x, h);
            const float qy = __shfl_xor_sync(0xffffffffu, v[e].y, h);
            if (!upper) {
                v[e] = make_float2(v[e].x + qx, v[e].y + qy);
            } else {
                const float2 d = make_float2(qx - v[e].x, qy - v[e].y);
                v[e] = make_float2(d.x * w.x - d.y * w.y, d.x * w.y + d.y * w.x);
            }
        }
    }
}

template <int G>
__global__ void __launch_bounds__(1024)
    k_image_fft_warp(const long long* __restrict__ grid, float* __restrict__ img,
                     float* __restrict__ vmax, float* __restrict__ vmin) {
    constexpr int E = G / 32, H = G / 2, P = G + 1, LOGG = G == 32 ? 5 : (G == 64 ? 6 : 7);
    extern __shared__ float2 S[];                      // [G][G + 1] then twiddles [G / 2]
    float2* tw = S + G * P;
    __shared__ float red_max[32], red_min[32];
    const int c = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    for (int k = threadIdx.x; k < H; k += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * (double)k / (double)G, &sn, &cs);   // W_G^k = exp(-2 pi i k / G), FP64
        tw[k] = make_float2((float)cs, (float)(-sn));
    }
    __syncthreads();
    const long long* g = grid + (size_t)c * G * G * 2;
    for (int y = warp; y < G; y += nwarps) {           // rows
        float2 v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) {
            const longlong2 gv = reinterpret_cast<const longlong2*>(g)[y * G + lane + 32 * e];
            v[e] = make_float2(__ll2float_rn(gv.x), __ll2float_rn(gv.y));
        }
        warp_fft<G>(v, tw, lane);
#pragma unroll
        for (int e = 0; e < E; ++e)
            S[y * P + (int)(__brev((unsigned)(lane + 32 * e)) >> (32 - LOGG))] = v[e];
    }
    __syncthreads();
    for (int x = warp; x < G; x += nwarps) {           // columns
        float2 v[E];
#pragma unroll
        for (int e = 0; e < E; ++e) v[e] = S[(lane + 32 * e) * P + x];
        warp_fft<G>(v, tw, lane);
        __syncwarp();
#pragma unroll
        for (int e = 0; e < E; ++e)
            S[(int)(__brev((unsigned)(lane + 32 * e)) >> (32 - LOGG)) * P + x] = v[e];
    }
    __syncthreads();
    float mx = -3.4e38f, mn = 3.4e38f;
    float* out = img + (size_t)c * G * G;
    for (int q = threadIdx.x; q < G * G; q += blockDim.x) {
        const int y = q / G, x = q - y * G;
        const float v = S[((y + H) & (G - 1)) * P + ((x + H) & (G - 1))].x;
        out[q] = v;
        mx = fmaxf(mx, v);
        mn = fminf(mn, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    if (lane == 0) {
        red_max[warp] = mx;
        red_min[warp] = mn;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < nwarps; ++w) {
            mx = fmaxf(mx, red_max[w]);
            mn = fminf(mn, red_min[w]);
        }
        if (vmax) vmax[c] = mx;
        if (vmin) vmin[c] = mn;
    }
}

template <int G>
int launch_fft_warp(const int64_t* grid, int32_t nch, float* img, float* vmax, float* vmin,
                    cudaStream_t st) {
    const size_t smem = (size_t)G * (G + 1) * sizeof(float2) + (size_t)(G / 2) * sizeof(float2);
    if (smem > 48 * 1024)
        MIXER_CK(cudaFuncSetAttribute(k_image_fft_warp<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
    k_image_fft_warp<G><<<(unsigned)nch, 1024, smem, st>>>(reinterpret_cast<const long long*>(grid),
                                                           img, vmax, vmin);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}

}  // namespace

// Shared memory of k_grid_tiles: the largest baseline window of any tile
// (16 bytes per int64 re / im cell).
size_t grid_smem_bytes(int nant, int side_x) {
    int maxcells = 0;
    for (int i = 0; i * 128 < nant; ++i)
        for (int j = 0; j <= i; ++j) {
            int dylo, ny;
            tile_window(i, j, nant, side_x, dylo, ny);
            const int cells = ny * (2 * side_x - 1);
            if (cells > maxcells) maxcells = cells;
        }
    return (size_t)maxcells * 16;
}
}  // namespace mixer

extern "C" int mixer_grid(const int64_t* vis64, int32_t nant, int32_t nch, int32_t side_x,
                          int32_t G, int64_t* grid, int64_t* prev, void* stream) {
    if (!vis64 || !grid || nant <= 0 || nch <= 0 || side_x <= 0 || G <= 0) return MIXER_EINVAL;
    if (nch > 65535 || G > 4096) return MIXER_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nt = mixer_vis_tiles(nant);
    const size_t smem = mixer::grid_smem_bytes(nant, side_x);
    if (smem > mixer::kGridSmemMax) return MIXER_EINVAL;
    if (smem > 48 * 1024)
        MIXER_CK(cudaFuncSetAttribute(mixer::k_grid_tiles,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const size_t gbytes = (size_t)nch * G * G * 2 * sizeof(int64_t);
    MIXER_CK(cudaMemsetAsync(grid, 0, gbytes, st));
    dim3 g((unsigned)nt, (unsigned)nch);
    mixer::k_grid_tiles<<<g, 256, smem, st>>>(reinterpret_cast<const long long*>(vis64), nant, nt,
                                              side_x, G,
                                              reinterpret_cast<unsigned long long*>(grid));
    MIXER_CK(cudaGetLastError());
    if (prev) {
        const int64_t n = (int64_t)nch * G * G * 2;
        int64_t blocks = (n + 255) / 256;
        if (blocks > 4096) blocks = 4096;
        mixer::k_grid_delta<<<(unsigned)blocks, 256, 0, st>>>(reinterpret_cast<long long*>(grid),
                                                              reinterpret_cast<long long*>(prev), n);
        MIXER_CK(cudaGetLastError());
    }
    return MIXER_OK;
}

extern "C" int mixer_image_fft(const int64_t* grid, int32_t nch, int32_t G, float* img, float* vmax,
                               float* vmin, void* stream) {
    if (!grid || !img || nch <= 0) return MIXER_EINVAL;
    int logG = 0;
    while ((1 << logG) < G) ++logG;
    if ((1 << logG) != G || G < 4 || G > 128) return MIXER_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (G == 32) return mixer::launch_fft_warp<32>(grid, nch, img, vmax, vmin, st);
    if (G == 64) return mixer::launch_fft_warp<64>(grid, nch, img, vmax, vmin, st);
    if (G == 128) return mixer::launch_fft_warp<128>(grid, nch, img, vmax, vmin, st);
    const size_t smem = (size_t)G * G * sizeof(float2) + (size_t)(G / 2) * sizeof(float2);
    if (smem > 48 * 1024)
        MIXER_CK(cudaFuncSetAttribute(mixer::k_image_fft,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    mixer::k_image_fft<<<(unsigned)nch, 512, smem, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const long long*>(grid), G, logG, img, vmax, vmin);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}

// ---- imaging without allocation ---------------------------------------------
// The grid scratch of mixer_image_noalloc: a fixed array in the library's
// device image (re, im int64 per cell), shared by every call on a device.
namespace mixer {
namespace {
__device__ __align__(256) long long g_noalloc_grid[2 * (size_t)MIXER_NOALLOC_MAX_CELLS];

// Device address of g_noalloc_grid on the current device, looked up once per
// device with that device current.
int noalloc_grid_address(int64_t** out) {
    static std::mutex mu;
    static int64_t* addr[64] = {};
    int dev = 0;
    MIXER_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return MIXER_EINVAL;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        MIXER_CK(cudaGetSymbolAddress(&p, g_noalloc_grid));
        addr[dev] = static_cast<int64_t*>(p);
    }
    *out = addr[dev];
    return MIXER_OK;
}
}  // namespace
}  // namespace mixer

extern "C" int mixer_image_noalloc(const int64_t* vis64, int32_t nant, int32_t nch, int32_t side_x,
                                   int32_t G, float* img, float* vmax, float* vmin, void* stream) {
    // Every check of mixer_grid and mixer_image_fft is made here first, so a
    // refused request enqueues nothing and leaves the shared array as it was.
    if (!vis64 || !img || nant <= 0 || nch <= 0 || side_x <= 0) return MIXER_EINVAL;
    if (G < 4 || G > 128 || (G & (G - 1)) != 0 || nch > 65535) return MIXER_EINVAL;
    if ((int64_t)nch * G * G > MIXER_NOALLOC_MAX_CELLS) return MIXER_EINVAL;
    if (mixer::grid_smem_bytes(nant, side_x) > mixer::kGridSmemMax) return MIXER_EINVAL;
    int64_t* grid = nullptr;
    int rc = mixer::noalloc_grid_address(&grid);
    if (rc != MIXER_OK) return rc;
    // mixer_grid clears the cells it uses on `stream` before adding into them.
    rc = mixer_grid(vis64, nant, nch, side_x, G, grid, nullptr, stream);
    if (rc != MIXER_OK) return rc;
    return mixer_image_fft(grid, nch, G, img, vmax, vmin, stream);
}
