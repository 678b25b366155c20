// xcorr.cu -- lower-triangle complex Hermitian GEMM V = X X^H per channel on
// tcgen05 int8 tensor cores (sm_100a).
//
// Replaces cgemm_blk_t<ACC> (reference src/cgemm.cuh:28-69).  The reference
// issues four wmma 16x16x16 products per tile from global memory, negates the
// A_im fragment (src/cgemm.cuh:52, wraps for -128) and computes the full
// square.  Here, per channel c and 128 x 128 tile (i, j) with j <= i, the B
// operand is the 256-row stack [Xr_j ; Xi_j] (the two plane tiles sit next to
// each other in shared memory), so two M=128, N=256 MMAs per 32-sample step
// produce all four real products:
//
//   D1 = Xr_i [Xr_j ; Xi_j]^T = [ R1 | P2 ]      (TMEM columns   0..255)
//   D2 = Xi_i [Xr_j ; Xi_j]^T = [ P1 | R2 ]      (TMEM columns 256..511)
//   Re V = R1 + R2,  Im V = P1 - P2              (epilogue)
//
// No operand is ever negated, so every int8 input, -128 included, is exact.
// Diagonal tiles (i == j) use the A tiles [Xr_i ; Xi_i] as B and load half
// the bytes.  When N is not a multiple of 128 the last block holds r < 128
// antennas; its tiles put that block on the N side with r16 = r rounded up to
// 16 rows per plane (N = 2 r16): tile (nb-1, j < nb-1) is computed as its
// conjugate transpose, A = block j and B = [Xr_nb-1 ; Xi_nb-1] (r16 rows
// each, one TMA box over both planes), and written back transposed; tile
// (nb-1, nb-1) keeps A = its own block.  Operands come from the corner-turned
// planes [2][C][N][kt] through 4-D TMA tensor loads (128-byte swizzle,
// 128 x 128-byte boxes)
// into a 3-deep shared-memory ring.  One elected thread issues all
// tcgen05.mma; the int32 accumulators stay in TMEM for the whole K range of
// the launch; eight epilogue warps read them back with tcgen05.ld and add
// them into the tile-packed int32 or int64 cube in HBM.
//
// Warp roles (320 threads with the default build, one CTA per SM, persistent
// over work items):
//   warp 0      TMA producer; picks the CTA's next item and passes its index
//               to the other roles through a shared-memory ring
//   warp 1      TMEM allocator + MMA issuer
//   warps 2..9  epilogue (TMEM lane quadrant = warp % 4, 64-column half =
//               (warp - 2) / 4)
// A single-array launch hands CTA b the items b, b + grid, ... (all items
// but the ragged block's cost the same); a table launch takes items in list
// order from a global counter, so CTAs stay on neighbouring items, which
// share operand blocks in L2, whatever each item costs.
#include "common.cuh"
#include "xcorr.cuh"
#include <cstdlib>
#include <cstring>

namespace mixer {

namespace {

// Pipeline geometry (build-time options): samples per stage (128 with the
// 128-byte swizzle or 64 with the 64-byte swizzle), stage count, and epilogue
// warps per TMEM lane quadrant.
#ifndef MIXER_XCORR_KC
#define MIXER_XCORR_KC 128
#endif
#ifndef MIXER_XCORR_STAGES
#define MIXER_XCORR_STAGES 3
#endif
#ifndef MIXER_XCORR_EPI_GROUPS
#define MIXER_XCORR_EPI_GROUPS 2
#endif
// int64 epilogue of an item that owns its tile: 1 = load, add, store; 0 = the
// 64-bit atomic add (fire and forget) that K-split items always use.  Measured
// on B200 the load-add-store form is 5 % faster at K 1024 per launch but 21 %
// slower at 256 elements and K 256 (its loads wait on DRAM latency), so the
// atomic add is the default.
#ifndef MIXER_XCORR_EXCL_RMW
#define MIXER_XCORR_EXCL_RMW 0
#endif
// Diagonal tiles (i == j) with three products instead of four: there
// P1 = Xi Xr^T = P2^T, so one M 128 x N 256 MMA gives [R1 | P2], one
// M 128 x N 128 MMA gives R2 = Xi Xi^T, and the epilogue forms
// Im = P2^T - P2 by exchanging 32 x 32 blocks of P2 through shared memory.
// 0: four products on every tile.
#ifndef MIXER_XCORR_DIAG3
#define MIXER_XCORR_DIAG3 0
#endif
// Tiles of a ragged last block (N not a multiple of 128) with the block on the
// MMA's N side, N = 2 r16 (1), or as full 128 x 128 tiles with zero rows (0).
#ifndef MIXER_XCORR_TAIL
#define MIXER_XCORR_TAIL 1
#endif
// Transposed ragged tiles: each warp passes its 32 x 16 blocks through shared
// memory so that a warp's adds cover two 128-byte lines per instruction (1),
// or adds straight from the TMEM rows, 32 lines per instruction (0).
#ifndef MIXER_XCORR_TAIL_XPOSE
#define MIXER_XCORR_TAIL_XPOSE 1
#endif
constexpr int kTile = 128;                       // tile rows = cols
constexpr int kWorkChunk = 128;                  // samples per work-list K unit
constexpr int kKc = MIXER_XCORR_KC;              // samples (bytes) per pipeline stage
constexpr int kSubPerChunk = kWorkChunk / kKc;
constexpr int kStages = MIXER_XCORR_STAGES;
constexpr int kTileBytes = kTile * kKc;
constexpr int kStageBytes = 4 * kTileBytes;      // Ar, Ai, Br, Bi
static_assert(kKc == 64 || kKc == 128, "stage of 64 or 128 samples");
constexpr int kEpiGroups = MIXER_XCORR_EPI_GROUPS;  // column groups per TMEM lane quadrant
constexpr int kEpiWarps = 4 * kEpiGroups;
constexpr int kEpiCols = kTile / kEpiGroups;     // 64 columns per warp
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr int kBarBytes = 512;
// Item ring (table launches take items from a global counter): the producer
// publishes each item index to the MMA and epilogue warps through kItemSlots
// slots after the pipeline barriers.
constexpr int kItemSlots = 8;
constexpr int kItemBar0 = 24;                    // first ring barrier (uint64 index)
static_assert(2 * MIXER_XCORR_STAGES + 5 <= kItemBar0, "barrier area");
static_assert((kItemBar0 + 3 * kItemSlots) * 8 <= kBarBytes, "barrier area");
// The diagonal-tile exchange needs the 2 x 4 layout of eight epilogue warps.
constexpr bool kDiag3 = MIXER_XCORR_DIAG3 != 0 && kEpiGroups == 2;
// Exchange area: one round's eight 32 x 32 int32 blocks of P2, rows padded to
// 33 words so that both the row-wise writes and the column-wise reads of a
// warp hit 32 different banks.
constexpr int kXchgStride = 33;
constexpr int kXchgBlock = 32 * kXchgStride;     // words per block
constexpr int kXchgBytes = kDiag3 ? 8 * kXchgBlock * 4 : 0;
// Transpose area of the ragged tiles: per epilogue warp 32 rows of 16 words,
// padded to 17 (row writes and the two-rows-per-read pattern are conflict-free).
// It shares the exchange area (the two serve different items).
constexpr int kXposeStride = 17;
constexpr int kXposeBytes =
    (MIXER_XCORR_TAIL && MIXER_XCORR_TAIL_XPOSE) ? kEpiWarps * 32 * kXposeStride * 4 : 0;
constexpr int kEpiSmemBytes = kXchgBytes > kXposeBytes ? kXchgBytes : kXposeBytes;
constexpr int kSmemBase = kStages * kStageBytes + 1024 + kBarBytes;
constexpr int kSmemBytes = kSmemBase + kEpiSmemBytes;   // the most a launch asks for
static_assert(kSmemBytes <= 232448, "shared memory");
constexpr uint32_t kTmemCols = 512;              // D1 (256) + D2 (256)
constexpr uint32_t kIdesc = idesc_i8(128, 256);
constexpr uint32_t kIdescN128 = idesc_i8(128, 128);
constexpr int kEpiBarrier = 1;                   // named barrier of the eight epilogue warps

struct XcorrArgs {
    int32_t nant, nch, nblk, ntiles;
    int32_t kbeg, nkc;   // first sample, number of 128-sample chunks
    int32_t mode;
    int32_t pad_;
    int64_t nwork;       // nch * ntiles, or the length of `work`
    void* vis;
    int32_t* err;
    // Item counter of a table launch, zero at its start (nullptr: CTA b takes
    // items b, b + grid, ...).
    unsigned long long* ctr;
    // Batched mode (work != nullptr): per-array tensor maps, problems, work list.
    // Two maps per array: [2p] the 128-row operand boxes, [2p + 1] the ragged
    // last block's box over both planes.
    const CUtensorMap* tmaps;
    const XcorrProblem* probs;
    const XcorrWork* work;
};

__device__ __forceinline__ void decode_tile(int t, int& i, int& j) {
    int ii = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
    while ((ii + 1) * (ii + 2) / 2 <= t) ++ii;
    while (ii * (ii + 1) / 2 > t) --ii;
    i = ii;
    j = t - ii * (ii + 1) / 2;
}

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    return kKc == 128 ? sdesc_sw128(saddr) : sdesc_sw64(saddr);
}

struct Item {
    const CUtensorMap* map;
    const CUtensorMap* map_tail;
    void* vis;
    int c, t, i, j, kbeg, kc0, nkc, mode, ntiles, excl;
    int tail;   // rows per plane of the ragged last block on the N side (0: full tile)
};

// Rows per plane of the last 128-row block rounded up to 16 (128 when full).
__host__ __device__ __forceinline__ int tail_rows(int nant) {
    const int r = nant - ((nant - 1) / kTile) * kTile;
    return (r + 15) & ~15;
}

__device__ __forceinline__ Item get_item(const XcorrArgs& a, const CUtensorMap* pmap,
                                         const CUtensorMap* pmap_tail, int64_t w) {
    Item it;
    int nant;
    if (a.work == nullptr) {
        it.c = (int)(w / a.ntiles);
        it.t = (int)(w - (int64_t)it.c * a.ntiles);
        it.map = pmap;
        it.map_tail = pmap_tail;
        nant = a.nant;
        it.vis = a.vis;
        it.kbeg = a.kbeg;
        it.kc0 = 0;
        it.nkc = a.nkc;
        it.mode = a.mode;
        it.ntiles = a.ntiles;
        it.excl = 1;          // one launch, one item per (channel, tile)
    } else {
        const XcorrWork wk = a.work[w];
        const XcorrProblem& pr = a.probs[wk.prob];
        it.c = (int)wk.chan;
        it.t = (int)wk.tile;
        it.map = a.tmaps + 2 * wk.prob;
        it.map_tail = it.map + 1;
        nant = pr.nant;
        it.vis = pr.vis;
        it.kbeg = pr.kbeg;
        it.kc0 = (int)wk.kc0;
        it.nkc = (int)wk.nkc;
        it.mode = pr.mode;
        it.ntiles = pr.ntiles;
        it.excl = pr.excl;
    }
    decode_tile(it.t, it.i, it.j);
    const int r16 = tail_rows(nant);
    it.tail = (MIXER_XCORR_TAIL && r16 < kTile && it.i == (nant - 1) / kTile) ? r16 : 0;
    return it;
}

// Four 32x32b.x16 TMEM loads (16 columns each) and the wait, in one asm
// statement so no use of the results can be scheduled before the wait.
__device__ __forceinline__ void tmem_ld4_x16(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                             uint32_t (&r)[4][16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%64];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%65];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47}, [%66];\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%67];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0][0]), "=r"(r[0][1]), "=r"(r[0][2]), "=r"(r[0][3]), "=r"(r[0][4]),
          "=r"(r[0][5]), "=r"(r[0][6]), "=r"(r[0][7]), "=r"(r[0][8]), "=r"(r[0][9]),
          "=r"(r[0][10]), "=r"(r[0][11]), "=r"(r[0][12]), "=r"(r[0][13]), "=r"(r[0][14]),
          "=r"(r[0][15]), "=r"(r[1][0]), "=r"(r[1][1]), "=r"(r[1][2]), "=r"(r[1][3]),
          "=r"(r[1][4]), "=r"(r[1][5]), "=r"(r[1][6]), "=r"(r[1][7]), "=r"(r[1][8]),
          "=r"(r[1][9]), "=r"(r[1][10]), "=r"(r[1][11]), "=r"(r[1][12]), "=r"(r[1][13]),
          "=r"(r[1][14]), "=r"(r[1][15]), "=r"(r[2][0]), "=r"(r[2][1]), "=r"(r[2][2]),
          "=r"(r[2][3]), "=r"(r[2][4]), "=r"(r[2][5]), "=r"(r[2][6]), "=r"(r[2][7]),
          "=r"(r[2][8]), "=r"(r[2][9]), "=r"(r[2][10]), "=r"(r[2][11]), "=r"(r[2][12]),
          "=r"(r[2][13]), "=r"(r[2][14]), "=r"(r[2][15]), "=r"(r[3][0]), "=r"(r[3][1]),
          "=r"(r[3][2]), "=r"(r[3][3]), "=r"(r[3][4]), "=r"(r[3][5]), "=r"(r[3][6]),
          "=r"(r[3][7]), "=r"(r[3][8]), "=r"(r[3][9]), "=r"(r[3][10]), "=r"(r[3][11]),
          "=r"(r[3][12]), "=r"(r[3][13]), "=r"(r[3][14]), "=r"(r[3][15])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3)
        : "memory");
}

// One and three 32x32b.x16 TMEM loads (16 columns each) with their wait.
__device__ __forceinline__ void tmem_ld_x16(uint32_t a, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(a)
        : "memory");
}

__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Adds (or stores) 16 elements of one row of TMEM into the cube: element e at
// e0 + e * kStride of the re plane and the im plane kTile * kTile further on
// (kStride 128: 16 columns of a tile row; 1: 16 rows of a tile column, for a
// tile computed as its conjugate transpose).
template <int kStride>
__device__ __forceinline__ void store16(const Item& it, size_t e0, const int32_t (&re)[16],
                                        const int32_t (&im)[16]) {
    if (it.mode == MIXER_VIS_ACC_I64 && MIXER_XCORR_EXCL_RMW && it.excl) {
        // the item owns the tile: a warp reads, adds and writes 256 contiguous
        // bytes per column and plane
        long long* v = reinterpret_cast<long long*>(it.vis) + e0;
        long long a[16], b[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            a[e] = v[e * kStride];
            b[e] = v[e * kStride + kTile * kTile];
        }
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            v[e * kStride] = a[e] + (long long)re[e];
            v[e * kStride + kTile * kTile] = b[e] + (long long)im[e];
        }
    } else if (it.mode == MIXER_VIS_ACC_I64) {
        unsigned long long* v = reinterpret_cast<unsigned long long*>(it.vis) + e0;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            atomicAdd(v + e * kStride, (unsigned long long)(long long)re[e]);
            atomicAdd(v + e * kStride + kTile * kTile, (unsigned long long)(long long)im[e]);
        }
    } else if (it.mode == MIXER_VIS_ACC_I32) {
        int* v = reinterpret_cast<int*>(it.vis) + e0;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            atomicAdd(v + e * kStride, re[e]);
            atomicAdd(v + e * kStride + kTile * kTile, im[e]);
        }
    } else {
        int* v = reinterpret_cast<int*>(it.vis) + e0;
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            v[e * kStride] = re[e];
            v[e * kStride + kTile * kTile] = im[e];
        }
    }
}

// Adds (or stores) one element of the cube, in the item's mode.
__device__ __forceinline__ void store1(const Item& it, size_t e, int32_t x) {
    if (it.mode == MIXER_VIS_ACC_I64 && MIXER_XCORR_EXCL_RMW && it.excl) {
        long long* v = reinterpret_cast<long long*>(it.vis) + e;
        *v += (long long)x;
    } else if (it.mode == MIXER_VIS_ACC_I64) {
        atomicAdd(reinterpret_cast<unsigned long long*>(it.vis) + e, (unsigned long long)(long long)x);
    } else if (it.mode == MIXER_VIS_ACC_I32) {
        atomicAdd(reinterpret_cast<int*>(it.vis) + e, x);
    } else {
        reinterpret_cast<int*>(it.vis)[e] = x;
    }
}

__global__ void __launch_bounds__(kThreads, 1)
    k_xcorr_tri(const __grid_constant__ CUtensorMap tmap,
                const __grid_constant__ CUtensorMap tmap_tail, const XcorrArgs args) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;           // 1 KiB aligned (swizzle atoms)
    uint8_t* gbase = smem_raw + (base - raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + kStages * kStageBytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kStages + 4);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    int32_t* xchg = reinterpret_cast<int32_t*>(gbase + kStages * kStageBytes + kBarBytes);
    volatile int64_t* witems = reinterpret_cast<volatile int64_t*>(bars + kItemBar0 + 2 * kItemSlots);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int FULL = 0, EMPTY = kStages, ACCF = 2 * kStages, ACCE = 2 * kStages + 1,
              DRAIN = 2 * kStages + 2, IFULL = kItemBar0, IEMPTY = kItemBar0 + kItemSlots;
    auto bar = [&](int k) { return smem_u32(&bars[k]); };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(bar(FULL + s), 1);
            mbar_init(bar(EMPTY + s), 1);
        }
        mbar_init(bar(ACCF), 1);
        mbar_init(bar(ACCE), 32 * kEpiWarps);
        mbar_init(bar(DRAIN), 1);
        for (int s = 0; s < kItemSlots; ++s) {
            mbar_init(bar(IFULL + s), 1);
            mbar_init(bar(IEMPTY + s), 1 + kEpiWarps);   // the MMA thread, one per epilogue warp
        }
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0 && args.work == nullptr) {
        prefetch_tmap(&tmap);
        prefetch_tmap(&tmap_tail);
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(tmem_slot), kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            int64_t issued = 0;
            bool ok = true;
            int islot = 0;
            uint32_t iphase = 0;
            int64_t w = blockIdx.x;
            while (ok) {
                // publish the item (or the end mark -1) to the MMA and epilogue warps
                if (w >= args.nwork) w = -1;
                if (!mbar_wait(bar(IEMPTY + islot), iphase ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                witems[islot] = w;
                mbar_arrive(bar(IFULL + islot));
                if (++islot == kItemSlots) {
                    islot = 0;
                    iphase ^= 1u;
                }
                if (w < 0) break;
                const Item it = get_item(args, &tmap, &tmap_tail, w);
                const bool diag = (it.i == it.j);
                const uint32_t bytes = it.tail ? 2 * kTileBytes + 2 * it.tail * kKc
                                               : (diag ? 2 * kTileBytes : 4 * kTileBytes);
                // A block: block j for a transposed ragged tile, else block i
                const int ia = (it.tail && !diag) ? it.j : it.i;
                for (int kc = 0; kc < it.nkc * kSubPerChunk; ++kc) {
                    if (!mbar_wait(bar(EMPTY + stage), phase ^ 1u, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t sb = base + stage * kStageBytes;
                    const uint32_t fb = bar(FULL + stage);
                    mbar_expect_tx(fb, bytes);
                    const int k = it.kbeg + it.kc0 * kWorkChunk + kc * kKc;
                    tma_load_4d(sb + 0 * kTileBytes, it.map, fb, k, ia * kTile, it.c, 0);
                    tma_load_4d(sb + 1 * kTileBytes, it.map, fb, k, ia * kTile, it.c, 1);
                    if (it.tail) {
                        // [Xr ; Xi] of the ragged block, it.tail rows each, one box
                        tma_load_4d(sb + 2 * kTileBytes, it.map_tail, fb, k, it.i * kTile, it.c, 0);
                    } else if (!diag) {
                        tma_load_4d(sb + 2 * kTileBytes, it.map, fb, k, it.j * kTile, it.c, 0);
                        tma_load_4d(sb + 3 * kTileBytes, it.map, fb, k, it.j * kTile, it.c, 1);
                    }
                    ++issued;
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                // next item: in list order from the launch's counter, or round robin
                w = args.ctr ? (int64_t)gridDim.x + (int64_t)atomicAdd(args.ctr, 1ull)
                             : w + gridDim.x;
            }
            if (!ok) {
                if (args.err) atomicOr(args.err, 1);
                *abort_flag = 1;
                // Let the copies already issued land before the CTA exits.
                for (int64_t q = issued - 1; q >= 0 && q >= issued - kStages; --q)
                    mbar_wait(bar(FULL + (int)(q % kStages)), (uint32_t)((q / kStages) & 1));
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0, acc_phase = 0;
            bool ok = true;
            const uint32_t t_d1 = tmem, t_d2 = tmem + 256;
            int islot = 0;
            uint32_t iphase = 0;
            while (true) {
                if (!mbar_wait(bar(IFULL + islot), iphase, abort_flag)) {
                    ok = false;
                    break;
                }
                const int64_t w = witems[islot];
                mbar_arrive(bar(IEMPTY + islot));
                if (++islot == kItemSlots) {
                    islot = 0;
                    iphase ^= 1u;
                }
                if (w < 0) break;
                const Item it = get_item(args, &tmap, &tmap_tail, w);
                const bool diag = (it.i == it.j);
                const uint32_t id1 = it.tail ? idesc_i8(128, 2 * it.tail) : kIdesc;
                if (!mbar_wait(bar(ACCE), acc_phase ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int kc = 0; kc < it.nkc * kSubPerChunk; ++kc) {
                    if (!mbar_wait(bar(FULL + stage), phase, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sb = base + stage * kStageBytes;
                    const uint64_t ar = sdesc(sb);
                    const uint64_t ai = sdesc(sb + kTileBytes);
                    // 256-row B operand [Xr_j ; Xi_j]: two adjacent tiles (2 it.tail
                    // rows for a ragged block)
                    const uint64_t b = (diag && !it.tail) ? ar : sdesc(sb + 2 * kTileBytes);
                    // diagonal tiles: D2 = Xi Xi^T (N 128) instead of Xi [Xr ; Xi]^T
                    const bool three = kDiag3 && diag && !it.tail;
                    const uint64_t b2 = three ? ai : b;
                    const uint32_t id2 = three ? kIdescN128 : id1;
#pragma unroll
                    for (int kk = 0; kk < kKc / 32; ++kk) {
                        const uint64_t o = (uint64_t)((kk * 32) >> 4);   // 32-byte K step
                        const uint32_t acc = (kc > 0 || kk > 0) ? 1u : 0u;
                        mma_i8(t_d1, ar + o, b + o, id1, acc);
                        mma_i8(t_d2, ai + o, b2 + o, id2, acc);
                    }
                    tc_commit(bar(EMPTY + stage));   // stage free once these MMAs finish
                    if (++stage == kStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                tc_commit(bar(ACCF));                // accumulators complete
                acc_phase ^= 1u;
            }
            if (!ok) {
                if (args.err) atomicOr(args.err, 2);
                *abort_flag = 1;
            }
            // No MMA may still be writing TMEM when it is released.
            tc_commit(bar(DRAIN));
            mbar_wait(bar(DRAIN), 0);
        }
    } else {
        // ------------------------------------------------------------ epilogue
        // Eight warps: TMEM lane quadrant warp % 4, column half (warp - 2) / 4.
        // Each warp reads its 64 columns 16 at a time and adds them into the
        // cube; TMEM is released once every warp has read its last chunk.
        const int q = warp & 3;
        const int col0 = kEpiCols * ((warp - 2) >> 2);
        const int m = q * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)col0;
        uint32_t acc_phase = 0;
        int islot = 0;
        uint32_t iphase = 0;
        while (true) {
            if (!mbar_wait(bar(IFULL + islot), iphase, abort_flag)) {
                if (args.err) atomicOr(args.err, 4);
                *abort_flag = 1;
                break;
            }
            const int64_t w = witems[islot];
            __syncwarp();
            if (lane == 0) mbar_arrive(bar(IEMPTY + islot));
            if (++islot == kItemSlots) {
                islot = 0;
                iphase ^= 1u;
            }
            if (w < 0) break;
            const Item it = get_item(args, &tmap, &tmap_tail, w);
            if (!mbar_wait(bar(ACCF), acc_phase, abort_flag)) {
                if (args.err) atomicOr(args.err, 4);
                *abort_flag = 1;
                break;
            }
            tc_fence_after();
            const size_t tb = ((size_t)it.c * it.ntiles + it.t) * (size_t)(2 * kTile * kTile);
            if (it.tail) {
                // Ragged last block on the N side: columns n < it.tail of each
                // product (R1 | P2 at 0 | it.tail, P1 | R2 at 256 | 256 + it.tail).
                // Transposed tile (i != j): TMEM row m is column m of tile (i, j)
                // and column n its row n, so Re = R1 + R2, Im = P2 - P1 and the
                // 16 values of a load belong to 16 consecutive rows.  Chunks of
                // 16 columns alternate between the column groups; in store mode
                // the rows past it.tail are written as zeros.
                const bool tr = it.i != it.j;
                const int g = (warp - 2) >> 2;
                const int nt = it.tail;
                const int ncols = it.mode == MIXER_VIS_STORE_I32 ? kTile : nt;
                const uint32_t tq = tmem + ((uint32_t)(q * 32) << 16);
                int last = -1;   // this warp's last chunk that reads TMEM
                for (int n0 = 16 * g; n0 < nt; n0 += 16 * kEpiGroups) last = n0;
                if (last < 0) {
                    tc_fence_before();
                    mbar_arrive(bar(ACCE));
                }
#pragma unroll 1
                for (int n0 = 16 * g; n0 < ncols; n0 += 16 * kEpiGroups) {
                    int32_t re[16], im[16];
                    if (n0 < nt) {
                        uint32_t r[4][16];   // R1, P2, P1, R2
                        tmem_ld4_x16(tq + n0, tq + nt + n0, tq + 256 + n0, tq + 256 + nt + n0, r);
                        if (n0 == last) {
                            tc_fence_before();
                            mbar_arrive(bar(ACCE));
                        }
#pragma unroll
                        for (int e = 0; e < 16; ++e) {
                            re[e] = (int32_t)(r[0][e] + r[3][e]);
                            im[e] = tr ? (int32_t)(r[1][e] - r[2][e]) : (int32_t)(r[2][e] - r[1][e]);
                        }
                    } else {
#pragma unroll
                        for (int e = 0; e < 16; ++e) re[e] = im[e] = 0;
                    }
                    if (tr && it.mode == MIXER_VIS_STORE_I32 &&
                        (reinterpret_cast<uintptr_t>(it.vis) & 15) == 0) {
                        // stores: a thread's 16 elements are contiguous, 4 x 16 bytes
                        int4* vr = reinterpret_cast<int4*>(reinterpret_cast<int*>(it.vis) + tb +
                                                           (size_t)m * kTile + n0);
                        int4* vi = vr + kTile * kTile / 4;
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            vr[e] = make_int4(re[4 * e], re[4 * e + 1], re[4 * e + 2], re[4 * e + 3]);
                            vi[e] = make_int4(im[4 * e], im[4 * e + 1], im[4 * e + 2], im[4 * e + 3]);
                        }
                    } else if (tr && kXposeBytes) {
                        // row `lane` of the warp's 32 x 16 block -> pairs of rows,
                        // 16 consecutive elements each, per instruction
                        int32_t* xs = xchg + (warp - 2) * 32 * kXposeStride;
                        const int rr = lane >> 4, cc = lane & 15;
#pragma unroll 1
                        for (int pl = 0; pl < 2; ++pl) {
#pragma unroll
                            for (int e = 0; e < 16; ++e) xs[lane * kXposeStride + e] = pl ? im[e] : re[e];
                            __syncwarp();
                            const size_t pb = tb + (size_t)pl * kTile * kTile + n0 + cc;
#pragma unroll 4
                            for (int s2 = 0; s2 < 16; ++s2) {
                                const int row = 2 * s2 + rr;
                                store1(it, pb + (size_t)(q * 32 + row) * kTile,
                                       xs[row * kXposeStride + cc]);
                            }
                            __syncwarp();
                        }
                    } else if (tr) {
                        store16<1>(it, tb + (size_t)m * kTile + n0, re, im);
                    } else {
                        store16<kTile>(it, tb + (size_t)n0 * kTile + m, re, im);
                    }
                }
            } else if (!(kDiag3 && it.i == it.j)) {
#pragma unroll 1
                for (int n0 = 0; n0 < kEpiCols; n0 += 16) {
                    uint32_t r[4][16];   // R1, P2, P1, R2
                    tmem_ld4_x16(trow + n0, trow + 128 + n0, trow + 256 + n0, trow + 384 + n0, r);
                    if (n0 == kEpiCols - 16) {           // this warp's TMEM reads are done
                        tc_fence_before();
                        mbar_arrive(bar(ACCE));
                    }
                    int32_t re[16], im[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        re[e] = (int32_t)(r[0][e] + r[3][e]);
                        im[e] = (int32_t)(r[2][e] - r[1][e]);
                    }
                    store16<kTile>(it, tb + (size_t)(col0 + n0) * kTile + m, re, im);
                }
            } else {
                // Diagonal tile: TMEM holds R1 (columns 0-127), P2 (128-255) and
                // R2 (256-383); Im[m][n] = P2[n][m] - P2[m][n].  Warp (q, h) owns
                // rows 32q.. and columns 64h..; it needs P2[n][m] for n in its
                // columns, i.e. the 32 x 32 blocks of P2 at rows of quadrants
                // 2h, 2h+1 and columns 32q.., which the warps of those quadrants
                // read from TMEM and pass through shared memory.  Round rho: the
                // warps of quadrants 2rho, 2rho+1 write their blocks (slot =
                // (quadrant - 2rho) * 4 + consumer quadrant), then the warps of
                // column half rho read them transposed and write their rows.
                const int hq = (warp - 2) >> 2;
#pragma unroll 1
                for (int rho = 0; rho < 2; ++rho) {
                    if ((q >> 1) == rho) {
#pragma unroll 1
                        for (int g = 0; g < 4; ++g) {
                            uint32_t p[16];
                            tmem_ld_x16(trow + 128 + 16 * g, p);
                            const int qc = 2 * hq + (g >> 1);
                            int32_t* dst = xchg + ((q - 2 * rho) * 4 + qc) * kXchgBlock +
                                           lane * kXchgStride + 16 * (g & 1);
#pragma unroll
                            for (int e = 0; e < 16; ++e) dst[e] = (int32_t)p[e];
                        }
                    }
                    named_bar_sync(kEpiBarrier, 32 * kEpiWarps);
                    if (hq == rho) {
#pragma unroll 1
                        for (int n0 = 0; n0 < kEpiCols; n0 += 16) {
                            uint32_t r1[16], p2[16], r2[16];
                            tmem_ld_x16(trow + n0, r1);
                            tmem_ld_x16(trow + 128 + n0, p2);
                            tmem_ld_x16(trow + 256 + n0, r2);
                            int32_t re[16], im[16];
#pragma unroll
                            for (int e = 0; e < 16; ++e) {
                                const int ep = n0 + e;     // column within this warp's 64
                                const int32_t p2t = xchg[((ep >> 5) * 4 + q) * kXchgBlock +
                                                         (ep & 31) * kXchgStride + lane];
                                re[e] = (int32_t)(r1[e] + r2[e]);
                                im[e] = (int32_t)((uint32_t)p2t - p2[e]);
                            }
                            store16<kTile>(it, tb + (size_t)(col0 + n0) * kTile + m, re, im);
                        }
                    }
                    named_bar_sync(kEpiBarrier, 32 * kEpiWarps);   // blocks consumed
                }
                tc_fence_before();
                mbar_arrive(bar(ACCE));                 // every TMEM read of the tile done
            }
            acc_phase ^= 1u;
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

// =============================================================================
// Pair kernel: one work item per cluster of two CTAs on two SMs.
//
// tcgen05 cta_group::2.  The pair's leader (cluster rank 0) issues M 256 x
// N 256 MMAs: A's 256 rows are 128 from each CTA's shared memory, and the
// 256-row B operand [Xr_j ; Xi_j] is split with Xr_j in the leader and Xi_j
// in the peer (same offsets).  Each CTA's TMEM then holds the four products
// of its own 128-row block against column block j,
//   D1 = Xr_a [Xr_j ; Xi_j]^T = [R1 | P2],  D2 = Xi_a [Xr_j ; Xi_j]^T = [P1 | R2],
// so one item computes two tiles (a0, j), (a1, j) that share column block j.
// Per SM and 32-sample step the tensor cores read 16 KB of shared memory
// instead of 24 KB and TMA writes 12 KB instead of 16 KB: 112 instead of 160
// bytes per clock at the full MMA rate.  Stages are 48 KB, four of them.
//
// Pairing.  Column block j holds tiles (i, j), i = j .. nb-1.  Consecutive
// rows pair up; a column with an odd count leaves its last tile (nb-1, j).
// Those leftovers share ROW block nb-1, so they pair as the products
// X_j X_{nb-1}^H against B = block nb-1, and the epilogue writes tile element
// (m, n) = conj(D[n][m]) (for the diagonal tile this is D itself).  Per
// channel: f(nb) = floor(nb^2/4) regular pairs, column j's first at
// f(nb) - f(nb - j), then ceil(ceil(nb/2)/2) leftover pairs; when ceil(nb/2)
// is odd the last leftover pair has no second tile and its peer half is
// computed and discarded.
// =============================================================================
constexpr int kPairStages = 4;
constexpr int kPairStageBytes = 3 * kTileBytes;   // A_re, A_im, this CTA's half of B
constexpr int kPairSmemBytes = kPairStages * kPairStageBytes + 1024 + kBarBytes;
constexpr uint32_t kIdescPair = idesc_i8(256, 256);
static_assert(kPairSmemBytes <= 232448, "shared memory");

struct PairArgs {
    int32_t nant, nch, nblk, ntiles;
    int32_t kbeg, nkc;   // first sample, number of 128-sample chunks
    int32_t mode;
    int32_t nreg;        // regular pairs per channel
    int32_t npairs;      // pairs per channel
    int32_t pad_;
    int64_t nwork;       // nch * npairs
    void* vis;
    int32_t* err;
};

// This CTA's half of pair item w.
struct PairHalf {
    int c, a, j, t;      // channel, A row block, B column block, stored tile
    bool valid, transposed;
};

__device__ __forceinline__ int quarter_sq(int n) { return (n * n) >> 2; }

__device__ __forceinline__ PairHalf pair_half(const PairArgs& g, int64_t w, int rank) {
    PairHalf h;
    h.c = (int)(w / g.npairs);
    const int p = (int)(w - (int64_t)h.c * g.npairs);
    const int nb = g.nblk;
    if (p < g.nreg) {
        // column j = nb - n with n the smallest count whose f(n) >= q
        const int q = g.nreg - p;
        int n = (int)(2.0f * sqrtf((float)q));
        if (n < 2) n = 2;
        while (quarter_sq(n) < q) ++n;
        while (n > 2 && quarter_sq(n - 1) >= q) --n;
        h.j = nb - n;
        h.a = h.j + 2 * (quarter_sq(n) - q) + rank;
        h.t = h.a * (h.a + 1) / 2 + h.j;
        h.valid = true;
        h.transposed = false;
    } else {
        const int s = 2 * (p - g.nreg) + rank;          // leftover of column nb-1-2s
        h.j = nb - 1;
        h.valid = s < ((nb + 1) >> 1);
        h.a = h.valid ? nb - 1 - 2 * s : nb - 1;
        h.t = (nb - 1) * nb / 2 + h.a;                  // tile (nb-1, a)
        h.transposed = true;
    }
    return h;
}

__global__ void __launch_bounds__(kThreads, 1)
    k_xcorr_pair(const __grid_constant__ CUtensorMap tmap, const PairArgs args) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;            // same offset in both CTAs
    uint8_t* gbase = smem_raw + (base - raw);
    uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + kPairStages * kPairStageBytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * kPairStages + 4);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const bool leader = (rank == 0);
    const int64_t cid = blockIdx.x >> 1, ncl = gridDim.x >> 1;
    const int FULL = 0, EMPTY = kPairStages, ACCF = 2 * kPairStages, ACCE = 2 * kPairStages + 1,
              DRAIN = 2 * kPairStages + 2;
    auto bar = [&](int k) { return smem_u32(&bars[k]); };
    // A wait that gives up stops both CTAs of the pair.
    auto raise_abort = [&]() {
        *abort_flag = 1;
        st_cluster_u32(mapa_shared(smem_u32((const void*)abort_flag), rank ^ 1u), 1u);
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < kPairStages; ++s) {
            mbar_init(bar(FULL + s), 1);      // leader: its expect_tx + both CTAs' bytes
            mbar_init(bar(EMPTY + s), 1);     // the leader's multicast commit
        }
        mbar_init(bar(ACCF), 1);
        mbar_init(bar(ACCE), 2 * 32 * kEpiWarps);   // leader: every epilogue thread of both
        mbar_init(bar(DRAIN), 1);
        *abort_flag = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) prefetch_tmap(&tmap);
    if (warp == 1) {
        tmem_alloc_pair(smem_u32(tmem_slot), kTmemCols);
        tmem_relinquish_pair();
    }
    tc_fence_before();
    cluster_sync_all();                       // barriers and TMEM ready in both CTAs
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------------------------------------------ producer (both)
        if (lane == 0) {
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true;
            for (int64_t w = cid; w < args.nwork && ok; w += ncl) {
                const PairHalf h = pair_half(args, w, (int)rank);
                for (int kc = 0; kc < args.nkc; ++kc) {
                    if (!mbar_wait(bar(EMPTY + stage), phase ^ 1u, abort_flag)) {
                        ok = false;
                        break;
                    }
                    const uint32_t sb = base + stage * kPairStageBytes;
                    const uint32_t fb = mapa_shared(bar(FULL + stage), 0);
                    if (leader) mbar_expect_tx(bar(FULL + stage), 2 * kPairStageBytes);
                    const int k = args.kbeg + kc * kKc;
                    tma_load_4d_pair(sb, &tmap, fb, k, h.a * kTile, h.c, 0);
                    tma_load_4d_pair(sb + kTileBytes, &tmap, fb, k, h.a * kTile, h.c, 1);
                    tma_load_4d_pair(sb + 2 * kTileBytes, &tmap, fb, k, h.j * kTile, h.c, (int)rank);
                    if (++stage == kPairStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            if (!ok) {
                if (args.err) atomicOr(args.err, 1);
                raise_abort();
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer (leader)
        if (lane == 0 && leader) {
            int stage = 0;
            uint32_t phase = 0, acc_phase = 0;
            bool ok = true;
            int64_t consumed = 0;
            const uint32_t t_d1 = tmem, t_d2 = tmem + 256;
            for (int64_t w = cid; w < args.nwork; w += ncl) {
                if (!mbar_wait(bar(ACCE), acc_phase ^ 1u, abort_flag)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                for (int kc = 0; kc < args.nkc; ++kc) {
                    if (!mbar_wait(bar(FULL + stage), phase, abort_flag)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sb = base + stage * kPairStageBytes;
                    const uint64_t ar = sdesc(sb);
                    const uint64_t ai = sdesc(sb + kTileBytes);
                    const uint64_t b = sdesc(sb + 2 * kTileBytes);
#pragma unroll
                    for (int kk = 0; kk < kKc / 32; ++kk) {
                        const uint64_t o = (uint64_t)((kk * 32) >> 4);   // 32-byte K step
                        const uint32_t acc = (kc > 0 || kk > 0) ? 1u : 0u;
                        mma_i8_pair(t_d1, ar + o, b + o, kIdescPair, acc);
                        mma_i8_pair(t_d2, ai + o, b + o, kIdescPair, acc);
                    }
                    tc_commit_pair(bar(EMPTY + stage), 0x3);   // stage free in both CTAs
                    ++consumed;
                    if (++stage == kPairStages) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (!ok) break;
                tc_commit_pair(bar(ACCF), 0x3);               // both CTAs' accumulators
                acc_phase ^= 1u;
            }
            if (!ok) {
                if (args.err) atomicOr(args.err, 2);
                raise_abort();
                // Let loads already counted on this CTA's barriers land.
                for (int64_t q = consumed; q < consumed + kPairStages; ++q)
                    mbar_wait(bar(FULL + (int)(q % kPairStages)), (uint32_t)((q / kPairStages) & 1));
            }
            // No MMA may still be writing either CTA's TMEM when it is released:
            // the peer deallocates only after the closing cluster barrier,
            // which this thread reaches after the wait.
            tc_commit_pair(bar(DRAIN), 0x1);
            mbar_wait(bar(DRAIN), 0);
        }
    } else {
        // ------------------------------------------------------------ epilogue (both)
        const int q = warp & 3;
        const int col0 = kEpiCols * ((warp - 2) >> 2);
        const int m = q * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)col0;
        const uint32_t acce = mapa_shared(bar(ACCE), 0);
        uint32_t acc_phase = 0;
        for (int64_t w = cid; w < args.nwork; w += ncl) {
            const PairHalf h = pair_half(args, w, (int)rank);
            if (!mbar_wait(bar(ACCF), acc_phase, abort_flag)) {
                if (args.err) atomicOr(args.err, 4);
                raise_abort();
                break;
            }
            tc_fence_after();
            const size_t tb = ((size_t)h.c * args.ntiles + h.t) * (size_t)(2 * kTile * kTile);
#pragma unroll 1
            for (int n0 = 0; n0 < kEpiCols; n0 += 16) {
                uint32_t r[4][16];   // R1, P2, P1, R2
                tmem_ld4_x16(trow + n0, trow + 128 + n0, trow + 256 + n0, trow + 384 + n0, r);
                if (n0 == kEpiCols - 16) {           // this warp's TMEM reads are done
                    tc_fence_before();
                    mbar_arrive_cluster(acce);
                }
                if (!h.valid) continue;
                // plain tile: element (m, n) at n * 128 + m; conjugate transpose:
                // D[m][n] goes to element (n, m), at m * 128 + n, with Im negated
                const size_t e0 = h.transposed ? tb + (size_t)m * kTile + (col0 + n0)
                                               : tb + (size_t)(col0 + n0) * kTile + m;
                const int es = h.transposed ? 1 : kTile;
                const int sg = h.transposed ? -1 : 1;
                if (args.mode == MIXER_VIS_ACC_I64) {
                    unsigned long long* v = reinterpret_cast<unsigned long long*>(args.vis) + e0;
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        atomicAdd(v + e * es, (unsigned long long)(long long)(int32_t)(r[0][e] + r[3][e]));
                        atomicAdd(v + e * es + kTile * kTile,
                                  (unsigned long long)(long long)(sg * (int32_t)(r[2][e] - r[1][e])));
                    }
                } else if (args.mode == MIXER_VIS_ACC_I32) {
                    int* v = reinterpret_cast<int*>(args.vis) + e0;
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        atomicAdd(v + e * es, (int)(r[0][e] + r[3][e]));
                        atomicAdd(v + e * es + kTile * kTile, sg * (int)(r[2][e] - r[1][e]));
                    }
                } else {
                    int* v = reinterpret_cast<int*>(args.vis) + e0;
#pragma unroll
                    for (int e = 0; e < 16; ++e) {
                        v[e * es] = (int)(r[0][e] + r[3][e]);
                        v[e * es + kTile * kTile] = sg * (int)(r[2][e] - r[1][e]);
                    }
                }
            }
            acc_phase ^= 1u;
        }
    }

    // Neither CTA leaves while the pair may still use its shared memory or TMEM.
    tc_fence_before();
    cluster_sync_all();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc_pair(tmem, kTmemCols);
    }
}


// Dense int8 tensor-core rate with the GEMM's own instruction stream: one CTA
// per SM issues `iters` times the k_xcorr_tri K-step (two M 128 x N 256 x K 32
// kind::i8 MMAs per 32 samples, four steps per 128-byte stage) from one
// resident shared-memory stage, with no loads, into the same 512 TMEM columns.
// The operand bytes are pseudo-random so the tensor cores draw realistic power.
__global__ void __launch_bounds__(128, 1) k_mma_peak(int64_t iters, int32_t* err) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(gbase + kStageBytes);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int warp = threadIdx.x >> 5;
    for (int q = threadIdx.x; q < kStageBytes / 4; q += blockDim.x)
        reinterpret_cast<uint32_t*>(gbase)[q] = (uint32_t)q * 2654435761u ^ 0x9e3779b9u;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x == 0) {
        mbar_init(smem_u32(bar), 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(smem_u32(tmem_slot), kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (threadIdx.x == 0) {
        const uint64_t ar = sdesc(base), ai = sdesc(base + kTileBytes), b = sdesc(base + 2 * kTileBytes);
        for (int64_t it = 0; it < iters; ++it) {
#pragma unroll
            for (int kk = 0; kk < kKc / 32; ++kk) {
                const uint64_t o = (uint64_t)((kk * 32) >> 4);
                const uint32_t acc = (it > 0 || kk > 0) ? 1u : 0u;
                mma_i8(tmem, ar + o, b + o, kIdesc, acc);
                mma_i8(tmem + 256, ai + o, b + o, kIdesc, acc);
            }
        }
        tc_commit(smem_u32(bar));
        if (!mbar_wait(smem_u32(bar), 0) && err) atomicOr(err, 2);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                              const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                              const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn get_encode() {
    static EncodeFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    }
    return fn;
}

int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return n > 0 ? n : 148;
}

}  // namespace

int xcorr_encode_map(CUtensorMap* map, const int8_t* planes, int32_t nant, int32_t nch, int64_t kt,
                     int64_t kend) {
    EncodeFn enc = get_encode();
    if (!enc) return MIXER_ECUDA;
    // dim 0 ends at kend so the last chunk of a range reads zeros past it.
    const cuuint64_t dims[4] = {(cuuint64_t)kend, (cuuint64_t)nant, (cuuint64_t)nch, 2};
    const cuuint64_t strides[3] = {(cuuint64_t)kt, (cuuint64_t)kt * nant,
                                   (cuuint64_t)kt * nant * nch};
    const cuuint32_t box[4] = {kKc, kTile, 1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<int8_t*>(planes), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     kKc == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? MIXER_OK : MIXER_EINVAL;
}

int xcorr_encode_maps(CUtensorMap* maps, const int8_t* planes, int32_t nant, int32_t nch, int64_t kt,
                      int64_t kend) {
    int rc = xcorr_encode_map(&maps[0], planes, nant, nch, kt, kend);
    if (rc != MIXER_OK) return rc;
    EncodeFn enc = get_encode();
    if (!enc) return MIXER_ECUDA;
    // The ragged last block: tail_rows(nant) rows of both planes in one box,
    // landing as [Xr rows ; Xi rows] (the 2 r16-row B operand).  Encoded for
    // every array; unused when N is a multiple of 128.
    const cuuint64_t dims[4] = {(cuuint64_t)kend, (cuuint64_t)nant, (cuuint64_t)nch, 2};
    const cuuint64_t strides[3] = {(cuuint64_t)kt, (cuuint64_t)kt * nant,
                                   (cuuint64_t)kt * nant * nch};
    const cuuint32_t box[4] = {kKc, (cuuint32_t)tail_rows(nant), 1, 2};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = enc(&maps[1], CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<int8_t*>(planes), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     kKc == 128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? MIXER_OK : MIXER_EINVAL;
}

// Dynamic shared memory of a launch: the transpose area only when it holds
// ragged-block tiles (measured: the larger carve-out slows the int64
// epilogue of other launches by up to 5 %).
static int launch_smem(bool ragged) {
    if (kDiag3) return kSmemBytes;
    return kSmemBase + ((MIXER_XCORR_TAIL && ragged) ? kXposeBytes : 0);
}

static int set_smem_attr() {
    static uint64_t attr_set = 0;   // one bit per device ordinal
    int dev = 0;
    MIXER_CK(cudaGetDevice(&dev));
    if (dev < 64 && !(attr_set & (1ull << dev))) {
        MIXER_CK(cudaFuncSetAttribute(k_xcorr_tri, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      kSmemBytes));
        attr_set |= 1ull << dev;
    }
    return MIXER_OK;
}

int xcorr_sm_count() { return sm_count(); }

// Pair kernel set-up, once per device: its shared-memory attribute and how
// many clusters of two CTAs can be resident at once (0: pairs unusable).
static int pair_clusters() {
    static int clusters[64];
    static uint64_t done = 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64) return 0;
    if (!(done & (1ull << dev))) {
        int n = 0;
        if (cudaFuncSetAttribute(k_xcorr_pair, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kPairSmemBytes) == cudaSuccess) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = 2;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(2 * 74);
            cfg.blockDim = dim3(kThreads);
            cfg.dynamicSmemBytes = kPairSmemBytes;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            if (cudaOccupancyMaxActiveClusters(&n, k_xcorr_pair, &cfg) != cudaSuccess) n = 0;
        }
        cudaGetLastError();   // a refused query leaves no error behind
        clusters[dev] = n;
        done |= 1ull << dev;
    }
    return clusters[dev];
}

// The pair kernel is opt-in (MIXER_XCORR_PAIRS=1 in the environment), from
// three 128-row blocks up (at most one discarded half per channel).  Measured
// on one B200 it is no faster than the one-SM kernel at boost clock and
// slower under the power cap (the clock settles lower: each SM still needs
// all of B, half of it from the peer), so the one-SM kernel is the default.
static bool pairs_wanted(int nblk) {
    if (kKc != 128 || nblk < 3) return false;
    const char* e = getenv("MIXER_XCORR_PAIRS");
    return e && e[0] == '1';
}

static int pair_launch(const CUtensorMap& map, int32_t nant, int32_t nch, int64_t kbeg,
                       int64_t klen, int32_t mode, void* vis, int32_t max_ctas, int32_t* err,
                       int clusters, cudaStream_t st) {
    PairArgs a;
    memset(&a, 0, sizeof(a));
    a.nant = nant;
    a.nch = nch;
    a.nblk = (nant + kTile - 1) / kTile;
    a.ntiles = a.nblk * (a.nblk + 1) / 2;
    a.kbeg = (int32_t)kbeg;
    a.nkc = (int32_t)((klen + kKc - 1) / kKc);
    a.mode = mode;
    a.nreg = a.nblk * a.nblk / 4;
    a.npairs = a.nreg + ((a.nblk + 1) / 2 + 1) / 2;
    a.nwork = (int64_t)nch * a.npairs;
    a.vis = vis;
    a.err = err;
    int64_t ncl = clusters;
    if (max_ctas > 0 && max_ctas / 2 < ncl) ncl = max_ctas / 2;
    if (a.nwork < ncl) ncl = a.nwork;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(2 * ncl));
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = kPairSmemBytes;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    MIXER_CK(cudaLaunchKernelEx(&cfg, k_xcorr_pair, map, a));
    return MIXER_OK;
}

// Launch over samples [kbeg, kbeg + klen) with klen <= MIXER_KMAX_I32.
// At most max_ctas persistent CTAs (<= 0: one per SM).
static int xcorr_launch(const int8_t* planes, int32_t nant, int32_t nch, int64_t kt, int64_t kbeg,
                        int64_t klen, int32_t mode, void* vis, int32_t max_ctas, int32_t* err,
                        cudaStream_t st) {
    CUtensorMap maps[2];
    int rc = xcorr_encode_maps(maps, planes, nant, nch, kt, kbeg + klen);
    if (rc != MIXER_OK) return rc;
    if (max_ctas != 1 && pairs_wanted((nant + kTile - 1) / kTile)) {
        const int clusters = pair_clusters();
        if (clusters > 0)
            return pair_launch(maps[0], nant, nch, kbeg, klen, mode, vis, max_ctas, err, clusters, st);
    }
    rc = set_smem_attr();
    if (rc != MIXER_OK) return rc;
    XcorrArgs a;
    a.nant = nant;
    a.nch = nch;
    a.nblk = (nant + kTile - 1) / kTile;
    a.ntiles = a.nblk * (a.nblk + 1) / 2;
    a.kbeg = (int32_t)kbeg;
    a.nkc = (int32_t)((klen + kWorkChunk - 1) / kWorkChunk);
    a.mode = mode;
    a.pad_ = 0;
    a.nwork = (int64_t)nch * a.ntiles;
    a.vis = vis;
    a.err = err;
    a.ctr = nullptr;
    a.tmaps = nullptr;
    a.probs = nullptr;
    a.work = nullptr;
    int64_t grid = sm_count();
    if (max_ctas > 0 && max_ctas < grid) grid = max_ctas;
    if (a.nwork < grid) grid = a.nwork;
    k_xcorr_tri<<<(unsigned)grid, kThreads, launch_smem(nant % kTile != 0), st>>>(maps[0], maps[1],
                                                                                  a);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}

int xcorr_launch_table(const CUtensorMap* d_tmaps, const XcorrProblem* d_probs,
                       const XcorrWork* d_work, int64_t nwork, int grid, int32_t* err,
                       unsigned long long* ctr, bool ragged, cudaStream_t st) {
    if (nwork <= 0 || grid <= 0 || !ctr) return MIXER_EINVAL;
    int rc = set_smem_attr();
    if (rc != MIXER_OK) return rc;
    MIXER_CK(cudaMemsetAsync(ctr, 0, sizeof(*ctr), st));
    XcorrArgs a;
    memset(&a, 0, sizeof(a));
    a.nwork = nwork;
    a.err = err;
    a.ctr = ctr;
    a.tmaps = d_tmaps;
    a.probs = d_probs;
    a.work = d_work;
    CUtensorMap unused;
    memset(&unused, 0, sizeof(unused));
    k_xcorr_tri<<<(unsigned)(grid < nwork ? grid : nwork), kThreads, launch_smem(ragged), st>>>(
        unused, unused, a);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}

}  // namespace mixer

extern "C" int32_t mixer_vis_tiles(int32_t nant) {
    if (nant <= 0) return 0;
    const int32_t nb = (nant + 127) / 128;
    return nb * (nb + 1) / 2;
}

extern "C" int64_t mixer_vis_elems(int32_t nant, int32_t nch) {
    if (nant <= 0 || nch <= 0) return 0;
    return (int64_t)nch * mixer_vis_tiles(nant) * 2 * 128 * 128;
}

extern "C" int mixer_xcorr_tri_ex(const int8_t* planes, int32_t nant, int32_t nch, int64_t kt,
                                  int64_t kbeg, int64_t klen, int32_t mode, void* vis,
                                  int32_t max_ctas, int32_t* err, void* stream) {
    if (!planes || !vis || nant <= 0 || nch <= 0 || kt <= 0 || kt % 16 != 0) return MIXER_EINVAL;
    if (kbeg < 0 || kbeg % 16 != 0 || klen <= 0 || kbeg + klen > kt) return MIXER_EINVAL;
    if (mode != MIXER_VIS_STORE_I32 && mode != MIXER_VIS_ACC_I32 && mode != MIXER_VIS_ACC_I64)
        return MIXER_EINVAL;
    if (kt > (int64_t)INT32_MAX || nant > 65536 || nch > 65536) return MIXER_EINVAL;
    if (reinterpret_cast<uintptr_t>(planes) % 16 != 0) return MIXER_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (mode != MIXER_VIS_ACC_I64) {
        if (klen > MIXER_KMAX_I32) return MIXER_EOVERFLOW;
        return mixer::xcorr_launch(planes, nant, nch, kt, kbeg, klen, mode, vis, max_ctas, err, st);
    }
    for (int64_t k = 0; k < klen; k += MIXER_KMAX_I32) {
        const int64_t len = (klen - k) < MIXER_KMAX_I32 ? (klen - k) : MIXER_KMAX_I32;
        const int rc =
            mixer::xcorr_launch(planes, nant, nch, kt, kbeg + k, len, mode, vis, max_ctas, err, st);
        if (rc != MIXER_OK) return rc;
    }
    return MIXER_OK;
}

extern "C" int mixer_mma_peak(int64_t iters, int32_t ctas, int32_t* err, void* stream) {
    if (iters <= 0) return MIXER_EINVAL;
    const int64_t n = ctas > 0 ? ctas : mixer::sm_count();
    constexpr int smem = mixer::kStageBytes + 1024 + 64;
    static uint64_t attr_set = 0;
    int dev = 0;
    MIXER_CK(cudaGetDevice(&dev));
    if (dev < 64 && !(attr_set & (1ull << dev))) {
        MIXER_CK(cudaFuncSetAttribute(mixer::k_mma_peak, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      smem));
        attr_set |= 1ull << dev;
    }
    mixer::k_mma_peak<<<(unsigned)n, 128, smem, static_cast<cudaStream_t>(stream)>>>(iters, err);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}

extern "C" int mixer_xcorr_tri(const int8_t* planes, int32_t nant, int32_t nch, int64_t kt,
                               int64_t kbeg, int64_t klen, int32_t mode, void* vis, int32_t* err,
                               void* stream) {
    return mixer_xcorr_tri_ex(planes, nant, nch, kt, kbeg, klen, mode, vis, 0, err, stream);
}
