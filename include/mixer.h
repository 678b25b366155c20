/* mixer.h -- C-ABI of the B200 X-engine (libmixer_b200.so).
 *
 * Plain C: pointers, sizes and int status codes; no CUDA or torch types in any
 * signature (a stream is passed as `void*`, i.e. a cudaStream_t; NULL = legacy
 * default stream).  Every entry point returns MIXER_OK (0) or a negative
 * MIXER_E* code and never exits the process (the reference's CK() macro calls
 * exit(1) on any CUDA error, src/rx_host_corr.cu:35).
 *
 * Two layers:
 *  1. Stateless kernel entry points on caller-owned device buffers.  Each one
 *     replaces one reference kernel or library call and is cited below.
 *  2. A context (`mixer_ctx`) that owns the device state of one array: the
 *     int64 integration cube, staging planes and imaging buffers.  It mirrors
 *     the reference's correlate -> integrate -> dump / image flow
 *     (src/rx_host_corr.cu:159-170, :219-236).
 *
 * Visibility layout ("tile-packed lower triangle").  Per channel the N x N
 * matrix is cut into 128 x 128 tiles; only tiles (i, j) with j <= i are kept,
 * in order t = i*(i+1)/2 + j.  A tile holds two planes (re, im), and inside a
 * plane the element for row a = 128 i + m, column b = 128 j + n sits at
 * n * 128 + m.  Index = (((c * ntiles + t) * 2 + p) * 128 + n) * 128 + m.
 * Diagonal tiles hold the full 128 x 128 block.  Rows / columns >= N are zero.
 * V[a][b] = sum_k x_a[k] * conj(x_b[k])   (src/cgemm.cuh:4-7).
 */
#ifndef MIXER_B200_H
#define MIXER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define MIXER_OK            0
#define MIXER_EINVAL       -1   /* bad argument or unsupported shape          */
#define MIXER_ENOMEM       -2   /* device or host allocation failed           */
#define MIXER_ECUDA        -3   /* a CUDA runtime call failed                 */
#define MIXER_ETIMEOUT     -4   /* a bounded in-kernel wait gave up           */
#define MIXER_EOVERFLOW    -5   /* int32 headroom of the cube would be exceeded */
#define MIXER_ENODEV       -6   /* no usable sm_100 device                    */
#define MIXER_EBUSY        -7   /* admission refused: memory budget or slots  */

/* ---- wire format: reference src/config.h:26-38, kept byte for byte ------ */
#define MIXER_WIRE_NANT           256   /* MIXER_NANT                       */
#define MIXER_WIRE_ACTIVE_NCH     128   /* MIXER_ACTIVE_NCH                 */
#define MIXER_WIRE_TPKT            32   /* MIXER_TPKT                       */
#define MIXER_WIRE_PAYLOAD_BYTES 8192   /* MIXER_PAYLOAD_BYTES              */
#define MIXER_WIRE_HDR_BYTES       64   /* MIXER_HDR_BYTES                  */
#define MIXER_WIRE_BYTES         8256   /* MIXER_WIRE_BYTES                 */
#define MIXER_WIRE_SEQ_BYTE        48   /* MIXER_SEQ_BYTE (big-endian u32)  */
#define MIXER_WIRE_PPB            256   /* MIXER_PPB                        */
#define MIXER_WIRE_UDP_PORT      4096   /* MIXER_UDP_PORT                   */

/* Largest sample count one tensor-core launch accumulates in int32 without
 * any possibility of overflow for arbitrary int8 input: |Re V| <=
 * 2 * 128 * 128 * K < 2^31  =>  K <= 65535; rounded down to the 128-sample
 * K-chunk of the GEMM.  (The reference's "safe to ~127" comment,
 * src/rx_host_corr.cu:88, does not hold; its real bound is g_flush <= 64.) */
#define MIXER_KMAX_I32 65408

/* epilogue modes of mixer_xcorr_tri */
#define MIXER_VIS_STORE_I32 0   /* vis32  = X X^H   (cgemm_blk_t<false>)     */
#define MIXER_VIS_ACC_I32   1   /* vis32 += X X^H   (cgemm_blk_t<true>)      */
#define MIXER_VIS_ACC_I64   2   /* vis64 += X X^H   (GEMM fused with integrate) */

/* ---- layout helpers ----------------------------------------------------- */
int32_t mixer_vis_tiles(int32_t nant);                    /* nblk*(nblk+1)/2  */
int64_t mixer_vis_elems(int32_t nant, int32_t nch);       /* per re+im, all ch */
const char* mixer_strerror(int status);
int mixer_device_ok(void);       /* MIXER_OK when device 0.. is sm_100 class */

/* ---- layer 1: stateless entry points (device pointers, async on stream) - */

/* Corner-turn.  Replaces k_packAB (src/rx_host_corr.cu:61-72) and the header
 * strip of the staging copy (src/rx_host_corr.cu:159).
 * packets: nheaps * nant packets at `pkt_stride` bytes, packet p = h*nant + a
 *          (heap h, antenna a = seq % nant, src/config.h:19-22); payload at
 *          `hdr_bytes`, planar re[nch*tpkt] | im[nch*tpkt], index c*tpkt + t.
 * planes:  int8 [2][nch][nant][kt]: plane 0 = re, 1 = im; sample
 *          k = k0 + h*tpkt + t.  Only the written range is touched.
 * seq0:    expected seq of packet 0; every packet whose big-endian seq at
 *          byte 48 differs from seq0 + p is counted into *seq_errors (device
 *          u32, may be NULL).  The reference checks only the first packet of
 *          a burst (src/rx_host_corr.cu:134).
 * err:     device int32 (may be NULL) receiving a non-zero bit if the bounded
 *          wait for the staging copies ever gave up.
 * Requires tpkt % 16 == 0, pkt_stride % 16 == 0, hdr_bytes % 16 == 0,
 * kt % 16 == 0, k0 % 16 == 0, k0 + nheaps*tpkt <= kt. */
int mixer_corner_turn(const uint8_t* packets, int64_t pkt_stride, int32_t hdr_bytes,
                      int32_t nant, int32_t nch, int32_t tpkt, int32_t nheaps,
                      uint32_t seq0, int8_t* planes, int64_t kt, int64_t k0,
                      uint32_t* seq_errors, int32_t* err, void* stream);

/* Lower-triangle complex Hermitian GEMM on tcgen05 int8 tensor cores.
 * Replaces cgemm_blk_t<ACC> (src/cgemm.cuh:28-69), which computes the full
 * square.  planes as written by mixer_corner_turn ([2][nch][nant][kt]);
 * samples [kbeg, kbeg+klen) are contracted.  vis is tile-packed (see top),
 * int32 for the *_I32 modes, int64 for MIXER_VIS_ACC_I64.  For the I32 modes
 * klen <= MIXER_KMAX_I32; the I64 mode splits longer ranges itself.
 * err: device int32 (may be NULL) that receives MIXER_ETIMEOUT bits if a
 * bounded wait in the kernel ever gave up.  kt % 16 == 0.
 * With MIXER_XCORR_PAIRS=1 in the environment and nant > 256 (three 128-row
 * blocks) the work runs on pairs of SMs instead (clusters of two CTAs, tcgen05
 * cta_group::2); both kernels give the same cube.  The one-SM kernel is the
 * default: on B200 the pair kernel measured no faster at boost clock and
 * slower under the power cap. */
int mixer_xcorr_tri(const int8_t* planes, int32_t nant, int32_t nch, int64_t kt,
                    int64_t kbeg, int64_t klen, int32_t mode, void* vis,
                    int32_t* err, void* stream);

/* Same, with at most max_ctas persistent CTAs (<= 0: one per SM; the pair
 * kernel uses max_ctas / 2 clusters, and max_ctas == 1 selects the one-SM
 * kernel).  Leaving SMs free lets an HBM-bound kernel on another stream (the
 * next corner-turn) run beside the tensor-bound GEMM. */
int mixer_xcorr_tri_ex(const int8_t* planes, int32_t nant, int32_t nch, int64_t kt,
                       int64_t kbeg, int64_t klen, int32_t mode, void* vis,
                       int32_t max_ctas, int32_t* err, void* stream);

/* Tensor-core rate probe (no counterpart in the reference): `ctas` CTAs
 * (<= 0: one per SM) each issue `iters` times the triangle GEMM's K-step (two
 * M 128 x N 256 x K 32 int8 MMAs per 32 samples, four per 128-sample stage)
 * from one resident shared-memory stage without any loads.  Each iteration is
 * 8 MMAs of 2 x 128 x 256 x 32 ops: time it on `stream` for the dense int8
 * rate the GEMM can approach on this device and clock.  err as above. */
int mixer_mma_peak(int64_t iters, int32_t ctas, int32_t* err, void* stream);

/* int32 -> int64 integration: vis64 += vis32; vis32 = 0 over n elements.
 * Replaces k_flush_cube (src/rx_host_corr.cu:90-95), which promotes into a
 * float cube and loses exactness past 2^24. */
int mixer_vis_flush(int32_t* vis32, int64_t* vis64, int64_t n, void* stream);

/* FP32 visibility cube [nch][2][nant][nant] (re plane, im plane; full square
 * mirrored by conjugation), the --dump record layout of
 * src/rx_host_corr.cu:187,225-227.  One rounding from exact int64. */
int mixer_vis_dump_f32(const int64_t* vis64, int32_t nant, int32_t nch,
                       float* cube, void* stream);

/* Exact full-square int64 cube [nch][2][nant][nant] (for checks / export). */
int mixer_vis_unpack_i64(const int64_t* vis64, int32_t nant, int32_t nch,
                         int64_t* cube, void* stream);

/* Exact uv-gridding.  Replaces k_grid_cube (src/rx_host_corr.cu:79-85): every
 * ordered pair (a, b) adds V[a][b] to cell ((ya-yb) mod G, (xa-xb) mod G) with
 * antenna a at (x, y) = (a % side_x, a / side_x); the diagonal lands once at
 * (0, 0).  grid: int64 [nch][G][G][2] (re, im), overwritten.
 * If prev != NULL the gridded cube is also stored there after subtracting
 * the previous contents (delta imaging, the k_diff monitor of
 * src/rx_host_corr.cu:74-77 done on the grid). */
int mixer_grid(const int64_t* vis64, int32_t nant, int32_t nch, int32_t side_x,
               int32_t G, int64_t* grid, int64_t* prev, void* stream);

/* Image = Re(FFT2 forward(grid)), fftshifted, per channel, plus per-channel
 * max / min.  Replaces cufftExecC2C (src/rx_host_corr.cu:205-206,222) and
 * the host fftshift / real / min-max loop (:230-235).  Shared-memory FFT,
 * FP32 arithmetic, twiddles generated in FP64.  G in {16,32,64,128}.
 * img: float [nch][G][G]; vmax, vmin: float [nch] (may be NULL). */
int mixer_image_fft(const int64_t* grid, int32_t nch, int32_t G, float* img,
                    float* vmax, float* vmin, void* stream);

/* Imaging without any device allocation: the same gridding + FFT as
 * mixer_grid followed by mixer_image_fft, but the intermediate int64 grid
 * lives in a fixed array inside the library instead of a caller or context
 * buffer.  It has no counterpart in the reference.  It exists for callers
 * that must not allocate device memory once they are running: a capture
 * framework that hands out a fixed memory budget at start-up, a real-time
 * receive loop where cudaMalloc / cudaFree could stall or synchronise the
 * device, or a host whose allocator belongs to another runtime.
 *   - Capacity: nch * G * G <= MIXER_NOALLOC_MAX_CELLS (16 MiB of int64 re/im
 *     cells, e.g. 256 x 64 x 64 or 64 x 128 x 128).  Every request that
 *     mixer_grid or mixer_image_fft would refuse (G not a power of two in
 *     4..128, more than 65535 channels, an array too wide for the gridder's
 *     shared-memory window) or that exceeds the capacity returns MIXER_EINVAL
 *     before anything is enqueued: the shared array is left untouched.
 *   - The array is part of the library's device image, so every GPU that
 *     loads the library holds those 16 MiB until the process exits.
 *   - The first call on each device looks up the array's device address
 *     (cudaGetSymbolAddress) in that device's primary context, the one the
 *     CUDA runtime uses, and keeps it for the life of the process; make that
 *     first call before any stream capture.  Driving the device through
 *     another driver-API context, or calling again after cudaDeviceReset, is
 *     not supported: the kept address belongs to the first primary context.
 *   - All calls share the one array and it keeps the previous call's
 *     contents; each call clears it on `stream` before gridding.  Calls whose
 *     work overlaps on the GPU (different streams, or several host threads)
 *     race on the array and must be serialised by the caller.
 * vis64 / img / vmax / vmin as for mixer_grid and mixer_image_fft. */
#define MIXER_NOALLOC_MAX_CELLS (1 << 20)
int mixer_image_noalloc(const int64_t* vis64, int32_t nant, int32_t nch, int32_t side_x,
                        int32_t G, float* img, float* vmax, float* vmin, void* stream);

/* ---- seeded packet source (replaces the DAQIRI capture / tx_host) -------- */

/* Sky model of one source list, evaluated in FP64 on the host:
 * X[c][a] = sum_s amp_s(c) * exp(-2 pi i f_c (x_a l_s + y_a m_s)),
 * f_c = 1 + c / nch, amp_s(c) = amp0_s + amp1_s * c / nch, antenna a at
 * (a % side_x, a / side_x).  Output: double [nch][nant][2]. */
int mixer_sky_table(int32_t nant, int32_t nch, int32_t side_x, int32_t nsrc,
                    const double* l, const double* m, const double* amp0,
                    const double* amp1, double* table);

/* Writes nheaps * nant packets in the wire format: 64-byte header with the
 * UDP destination port `udp_port` and big-endian seq = seq0 + p at byte 48;
 * payload int8 planar, sample = clip(rint(sky[c][a] + sigma * n), -127, 127)
 * with n an Irwin-Hall(12) normal deviate from Philox4x32-10 keyed by `seed`
 * and counted by (antenna, global sample index heap0*tpkt + h*tpkt + t,
 * channel).  noise_mode 0: sky + noise; 1: uniform integers in [-127, 127]
 * (sky ignored).  sky: device double [nch][nant][2] or NULL (zero sky). */
int mixer_gen_packets(uint8_t* packets, int64_t pkt_stride, int32_t hdr_bytes,
                      int32_t nant, int32_t nch, int32_t tpkt, int32_t nheaps,
                      int64_t heap0, uint32_t seq0, uint16_t udp_port,
                      const double* sky, double sigma, uint64_t seed,
                      int32_t noise_mode, void* stream);

/* ---- batched persistent launch over uneven arrays ------------------------ */

/* One array of a batch: planes as for mixer_xcorr_tri, samples
 * [kbeg, kbeg + klen), accumulated into its own tile-packed cube `vis`. */
typedef struct mixer_xcorr_problem {
    const int8_t* planes;   /* int8 [2][nch][nant][kt] */
    int32_t nant, nch;
    int64_t kt, kbeg, klen;
    int32_t mode;           /* MIXER_VIS_*; STORE_I32 items are never K-split */
    void* vis;
} mixer_xcorr_problem;

typedef struct mixer_batch mixer_batch;

#define MIXER_ORDER_LPT     0   /* items longest first (longest-processing-time) */
#define MIXER_ORDER_CHANNEL 1   /* array, channel, tile order (L2 locality)       */

/* Many independent arrays of different N, C and K in ONE persistent launch of
 * the triangle cGEMM (no counterpart in the reference, which launches one
 * fixed-shape kernel per V-update, src/rx_host_corr.cu:167).  The plan is a
 * device work list of (array, channel, tile, K-chunk range) items; results
 * are bit-identical to one mixer_xcorr_tri per array for every plan.
 * The problem descriptors (planes, vis pointers) are captured at creation. */
int mixer_batch_create(const mixer_xcorr_problem* probs, int32_t nprob, mixer_batch** out);
/* Explicit plan: K-split factor per size class (class = ceil(nant / 128),
 * index 0..nclass-1) and item order. */
int mixer_batch_plan(mixer_batch* b, const int32_t* split_per_class, int32_t nclass, int32_t order);
/* Autotuner: times candidate plans on the caller's own buffers -- a greedy
 * per-class K-split with longest-first order, then channel-major order with
 * that split -- `reps` launches per sample, each candidate against the
 * incumbent in an A-B-B-A pairing (clock drift cancels); a change is kept only
 * when it is at least 2 % faster, and the result must beat the default plan
 * (longest-first, no split) by as much or the default is kept.  The ACC-mode
 * cubes accumulate every trial: zero them afterwards. */
int mixer_batch_autotune(mixer_batch* b, int32_t reps, void* stream, float* best_ms);
/* One launch of the current plan.  The launch's CTAs take the work items in
 * list order from an item counter the batch owns (zeroed on `stream` before
 * the launch, so a captured graph zeroes it too): runs or replays of ONE batch
 * must not overlap on the GPU (they would also add into the same cubes). */
int mixer_batch_run(mixer_batch* b, void* stream);
/* Capture one launch of the current plan into a CUDA graph (stream must not be
 * the legacy default stream); replay it with mixer_batch_replay.  Re-planning
 * drops the graph. */
int mixer_batch_capture_graph(mixer_batch* b, void* stream);
int mixer_batch_replay(mixer_batch* b, void* stream);
/* Plan and error word: nwork items, order, split_per_class[65]; kernel_err
 * synchronises and returns MIXER_ETIMEOUT if a bounded wait gave up. */
int mixer_batch_info(mixer_batch* b, int64_t* nwork, int32_t* order, int32_t* split_per_class,
                     int32_t* kernel_err);
int mixer_batch_destroy(mixer_batch* b);

/* Rewrites the big-endian seq at byte 48 of npk packets to seq0, seq0+1, ...
 * so a generated packet pool can be replayed as a continuing stream. */
int mixer_restamp_seq(uint8_t* packets, int64_t npk, int64_t pkt_stride, uint32_t seq0, void* stream);

/* ---- layer 2: array context --------------------------------------------- */

typedef struct mixer_array_desc {
    int32_t nant;        /* N antennas (elements)                             */
    int32_t nch;         /* C channels carried by each packet                 */
    int32_t tpkt;        /* time samples per packet                           */
    int32_t ksub;        /* samples per sub-integration (multiple of tpkt)    */
    int32_t nsub_dump;   /* sub-integrations per dump                         */
    int32_t side_x;      /* array width: antenna a at (a % side_x, a / side_x) */
    int32_t grid;        /* image grid side G (0: 2 * max(side_x, side_y))    */
    int32_t pkt_stride;  /* bytes between packets in input buffers            */
    int32_t hdr_bytes;   /* payload offset inside a packet                    */
    int32_t max_heaps;   /* most heaps per antenna given to one correlate call */
} mixer_array_desc;

typedef struct mixer_ctx mixer_ctx;

/* Fills the reference's wire defaults: N 256, C 128, tpkt 32, ksub 1024
 * (HBATCH*TPKT, src/rx_host_corr.cu:39-40), side 16, G 32, stride 8256,
 * header 64, max_heaps 32. */
int mixer_desc_default(mixer_array_desc* d);
int mixer_create(const mixer_array_desc* d, mixer_ctx** out);
int mixer_destroy(mixer_ctx* ctx);
/* Zeroes the integration state and counters (stream-ordered). */
int mixer_reset(mixer_ctx* ctx, void* stream);

/* Corner-turn + triangle GEMM over nheaps heaps per antenna (nheaps*nant
 * packets, h-major), accumulated straight into the int64 cube.  packets are
 * device memory if packets_on_device, else host memory (pinned for async
 * copies) which is staged through the context.  The gpu_thread body of
 * src/rx_host_corr.cu:159-170 with the flush fused. */
int mixer_correlate(mixer_ctx* ctx, const void* packets, int64_t nheaps, uint32_t seq0,
                    int32_t packets_on_device, void* stream);
/* Reference-style split: V32 += X X^H into the context's int32 cube
 * (cgemm_blk_t<true>) ... */
int mixer_correlate_i32(mixer_ctx* ctx, const void* packets, int64_t nheaps, uint32_t seq0,
                        int32_t packets_on_device, void* stream);
/* ... and V64 += V32, V32 = 0 (k_flush_cube, exact). */
int mixer_integrate(mixer_ctx* ctx, void* stream);

/* FP32 dump cube [C][2][N][N]; out is device or host memory. */
int mixer_dump(mixer_ctx* ctx, float* out, int32_t out_on_device, void* stream);
/* Appends one raw record (no header) to `path`, like --dump
 * (src/rx_host_corr.cu:210-227).  Synchronous. */
int mixer_dump_to_file(mixer_ctx* ctx, const char* path, void* stream);
/* Exact int64 cube [C][2][N][N] or the raw tile-packed state. */
int mixer_read_vis_i64(mixer_ctx* ctx, int64_t* out, int32_t full_square,
                       int32_t out_on_device, void* stream);
/* Grid + FFT image of the integrated cube (delta != 0: of the change since the
 * previous delta image).  img [C][G][G], vmax / vmin [C]; device or host. */
int mixer_image(mixer_ctx* ctx, float* img, float* vmax, float* vmin, int32_t delta,
                int32_t out_on_device, void* stream);
/* Counters: samples integrated per channel, seq mismatches, kernel errors. */
int mixer_stats(mixer_ctx* ctx, int64_t* samples, int64_t* seq_errors, int32_t* kernel_err);
/* Raw device pointer of the int64 state (tile-packed). */
int64_t* mixer_state_ptr(mixer_ctx* ctx);

/* ---- streaming server: concurrent array streams, continuous batching ---- */

typedef struct mixer_server_cfg {
    int64_t budget_bytes;   /* device memory all admitted streams may reserve  */
    int32_t max_streams;    /* stream slots                                    */
    int32_t ring_subs;      /* staging depth per stream, sub-integrations (0: 8) */
    int32_t batch_subs;     /* most sub-integrations of a stream per launch (0: 4) */
} mixer_server_cfg;

typedef struct mixer_dump_info {
    int32_t available;      /* 1 if a dump was returned                        */
    int32_t nant, nch;
    int32_t pad_;
    int64_t index;          /* dump number of that stream, from 0              */
    double latency_s;       /* submit of its last heap -> dump in host memory  */
} mixer_dump_info;

typedef struct mixer_server_counters {
    int64_t admitted, refused, launches, work_items;
    int64_t bytes_used, bytes_processed, dumps, seq_errors;
    double p50_latency_s, p99_latency_s, max_latency_s, elapsed_s;
    int32_t kernel_err;
    int32_t pad_;
} mixer_server_counters;

typedef struct mixer_server mixer_server;

/* A serving loop with no counterpart in the reference (which serves one array
 * from one NIC queue, src/rx_host_corr.cu:143-175).  Streams of different
 * sizes are admitted against a device-memory budget and a slot count; a
 * worker thread batches the complete sub-integrations of every stream into
 * one persistent tensor-core launch per iteration (continuous batching);
 * every nsub_dump sub-integrations a stream's FP32 dump cube [C][2][N][N]
 * lands in pinned host memory.  A stream's dumps equal those of
 * mixer_correlate + mixer_dump on the same packets, alone or in any mix.
 * Stream descriptors need ksub % 128 == 0.  Calls are made with the
 * server's device current.  Threads: different streams may be submitted to,
 * polled and closed from different host threads; one stream's submissions
 * come from one thread at a time.  poll and close of the same stream may run
 * concurrently (close waits for a poll that is copying a dump out). */
int mixer_server_create(const mixer_server_cfg* cfg, mixer_server** out);
int mixer_server_destroy(mixer_server* sv);
/* Device bytes one stream of `d` reserves under `cfg`. */
int64_t mixer_server_stream_bytes(const mixer_server_cfg* cfg, const mixer_array_desc* d);
/* Allocation ahead of serving (no counterpart in the reference): device
 * memory from the server's pool and the pinned host dump buffers for `count`
 * streams of descriptor `d`, returned to the server's caches so that later
 * admissions of that shape allocate nothing.  Pinning a dump cube takes on
 * the order of a second per GB and holds the driver meanwhile, which delays
 * the dumps of streams already being served; a server that knows its stream
 * shapes reserves them before it starts.  Nothing counts against the budget
 * until a stream is admitted.  Synchronous; count <= max_streams. */
int mixer_server_reserve(mixer_server* sv, const mixer_array_desc* d, int32_t count);
/* Admission: MIXER_EBUSY when the budget or the slots are exhausted. */
int mixer_server_open(mixer_server* sv, const mixer_array_desc* d, int32_t* stream_id);
/* Synchronises the server's streams, frees the stream's memory and slot. */
int mixer_server_close(mixer_server* sv, int32_t stream_id);
/* Queue nheaps heaps (nheaps * nant packets, h-major) of the stream, host or
 * device memory; seq0 of the stream's first submission sets its expected
 * sequence.  MIXER_EBUSY when its staging ring is full (retry later). */
int mixer_server_submit(mixer_server* sv, int32_t stream_id, const void* packets, int64_t nheaps,
                        uint32_t seq0, int32_t on_device);
/* Oldest completed dump of the stream, copied to `out` (host, may be NULL to
 * discard) and released; info->available = 0 when none is ready. */
int mixer_server_poll(mixer_server* sv, int32_t stream_id, mixer_dump_info* info, float* out);
/* Waits until every heap submitted so far (all streams) has been copied into
 * the server's staging rings, so the caller may reuse its packet buffers. */
int mixer_server_sync_copies(mixer_server* sv);
/* Counters and p50 / p99 dump latency over all dumps so far. */
int mixer_server_stats(mixer_server* sv, mixer_server_counters* st);

/* Shape of a context's array. */
int mixer_ctx_shape(mixer_ctx* ctx, int32_t* nant, int32_t* nch);
/* Replaces the integration state with a host copy of the tile-packed int64
 * cube and sets the integrated-sample counter (synchronous). */
int mixer_write_vis_i64(mixer_ctx* ctx, const int64_t* tile_packed, int64_t samples);
/* Checkpoint / resume of the int64 integration state (the reference zeroes
 * its cube once and cannot resume, src/rx_host_corr.cu:188): a 32-byte
 * header {"MIXCKPT1", nant, nch, samples, count} and the raw tile-packed
 * cube.  Load refuses a file of another shape.  Synchronous. */
int mixer_state_save(mixer_ctx* ctx, const char* path);
int mixer_state_load(mixer_ctx* ctx, const char* path);

/* Heap alignment of a packet burst in host memory, as the reference's drain
 * thread does (src/rx_host_corr.cu:127-141), but checking every packet:
 * *first = index of the first packet whose big-endian seq is a multiple of
 * nant (*seq0 its seq), *nheaps = complete heaps of consecutive seqs from
 * there, *next = where to resume (the first packet of a gap, or the packet
 * after the last whole heap). */
int mixer_align_heaps(const uint8_t* packets, int64_t npk, int64_t pkt_stride, int32_t nant,
                      int64_t* first, int64_t* nheaps, int64_t* next, uint32_t* seq0);

/* Time-split multi-queue ingest (src/config.h:40-45, MIXER_NQ): the sender
 * steers snapshot (heap) tb to RX queue q = tb % nq, UDP destination port
 * MIXER_WIRE_UDP_PORT + q, so each queue's burst holds every nq-th heap in
 * increasing tb.  Merges nq such bursts (host memory, `queue_npk[q]` packets
 * each at `pkt_stride`) back into time order in `out` (host, room for
 * max_heaps * nant packets): heap tb is taken from queue tb % nq and must be
 * that queue's next heap, with seqs tb * nant + a and, when udp_port0 != 0,
 * destination port udp_port0 + q.  The merge stops at the first heap that is
 * missing, incomplete, misordered or on the wrong port.  *out_heaps = heaps
 * written, *seq0 = seq of the first, consumed[q] = packets of queue q used or
 * skipped (resume there).  The merged heaps go to mixer_correlate as one burst. */
int mixer_merge_time_split(const uint8_t* const* queues, const int64_t* queue_npk, int32_t nq,
                           int64_t pkt_stride, int32_t nant, uint16_t udp_port0,
                           int64_t max_heaps, uint8_t* out, int64_t* out_heaps, uint32_t* seq0,
                           int64_t* consumed);

/* Corr32 shared-memory publisher (src/rx_host_corr.cu:97-105,236): header
 * {u32 magic 0x43523343, w, h, nch; u64 write_seq} then img[nch][G][G],
 * vmax[nch], vmin[nch].  name like "/corr32". */
typedef struct mixer_shm mixer_shm;
int mixer_shm_open(const char* name, int32_t nch, int32_t G, mixer_shm** out);
int mixer_shm_publish(mixer_shm* shm, const float* img, const float* vmax,
                      const float* vmin, uint64_t write_seq);
int mixer_shm_close(mixer_shm* shm, int32_t unlink_name);

#ifdef __cplusplus
}
#endif
#endif /* MIXER_B200_H */
