/* mixer_oracle.c -- CPU restatement of the reference X-engine path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/, the
 * smoke check and the CPU-baseline leg of the benchmark load it (as
 * oracle/liboracle.so).  The product library never links or calls it.
 *
 * Restates, from the reference (xzackli/DAQIRI-MIXER):
 *   - the wire format and antenna = seq % N addressing  src/config.h:10-38
 *   - the corner-turn index map of k_packAB            src/rx_host_corr.cu:63-71
 *       ant, heap, sl -> c = sl / TPKT, t = sl % TPKT, klocal = heap*TPKT + t
 *   - the correlator formula V = X X^H                   src/cgemm.cuh:4-7,58-63
 *       Re V[a][b] = sum xr_a xr_b + xi_a xi_b
 *       Im V[a][b] = sum xi_a xr_b - xr_a xi_b
 *     in exact int64 (int32 partial sums over chunks of samples that cannot
 *     overflow; the sum blocked over 2 x 4 pairs of rows widened to int16 in
 *     64 x 64 cache tiles, AVX-512 VNNI where the CPU has it, cross-checked
 *     against the pair-by-pair form orc_correlate_pairwise);
 *   - the gridding index map of k_grid_cube             src/rx_host_corr.cu:79-85
 *       every ordered pair (a, b): cell ((ya-yb) mod G, (xa-xb) mod G)
 *     summed exactly in int64;
 *   - the seeded packet source of the product (Philox4x32-10, Salmon et al.
 *     2011; Irwin-Hall(12) noise; FP64 sky; rint + clip to [-127, 127]) so
 *     test inputs can be regenerated bit for bit on the CPU.
 * Parity of this restatement is pinned against the reference's own GPU
 * kernels (cgemm_blk_t, k_packAB, k_grid_cube) compiled from the reference
 * sources into oracle/_ref/ (see oracle/Makefile) through the golden
 * fixtures in tests/golden/.
 */
#include <immintrin.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SEQ_BYTE 48

/* ---------------------------------------------------------------- Philox */
static inline void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += W0;
            k1 += W1;
        }
        const uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c[0] = n0;
        c[1] = n1;
        c[2] = n2;
        c[3] = n3;
    }
}

void orc_philox4x32_10(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    philox(c, k0, k1);
    memcpy(out, c, sizeof(c));
}

/* --------------------------------------------------------------- sky table */
int orc_sky_table(int nant, int nch, int side_x, int nsrc, const double* l, const double* m,
                  const double* amp0, const double* amp1, double* table) {
    const double two_pi = 6.283185307179586476925286766559;
    for (int c = 0; c < nch; ++c) {
        const double fc = 1.0 + (double)c / (double)nch;
        for (int a = 0; a < nant; ++a) {
            const double x = (double)(a % side_x), y = (double)(a / side_x);
            double re = 0.0, im = 0.0;
            for (int s = 0; s < nsrc; ++s) {
                const double amp = amp0[s] + amp1[s] * (double)c / (double)nch;
                const double ph = -two_pi * fc * (x * l[s] + y * m[s]);
                re += amp * cos(ph);
                im += amp * sin(ph);
            }
            table[((int64_t)c * nant + a) * 2 + 0] = re;
            table[((int64_t)c * nant + a) * 2 + 1] = im;
        }
    }
    return 0;
}

/* ------------------------------------------------------------ packet source */
static void header64(uint8_t* h, int wire_bytes, uint16_t port) {
    memset(h, 0, 64);
    const uint8_t dst[6] = {0xa0, 0x88, 0xc2, 0x0d, 0x5e, 0x28};
    memcpy(h, dst, 6);
    h[12] = 0x08;
    h[13] = 0x00;
    uint8_t* ip = h + 14;
    ip[0] = 0x45;
    ip[2] = (uint8_t)((wire_bytes - 14) >> 8);
    ip[3] = (uint8_t)(wire_bytes - 14);
    ip[8] = 64;
    ip[9] = 17;
    ip[12] = 10, ip[13] = 0, ip[14] = 0, ip[15] = 1;
    ip[16] = 10, ip[17] = 0, ip[18] = 0, ip[19] = 2;
    uint32_t sum = 0;
    for (int i = 0; i < 20; i += 2) sum += ((uint32_t)ip[i] << 8) | ip[i + 1];
    while (sum >> 16) sum = (sum & 0xFFFF) + (sum >> 16);
    ip[10] = (uint8_t)((~sum & 0xFFFF) >> 8);
    ip[11] = (uint8_t)(~sum & 0xFF);
    uint8_t* udp = h + 34;
    udp[0] = udp[2] = (uint8_t)(port >> 8);
    udp[1] = udp[3] = (uint8_t)port;
    udp[4] = (uint8_t)((wire_bytes - 34) >> 8);
    udp[5] = (uint8_t)(wire_bytes - 34);
}

static inline int8_t quant(double sky, double sigma, int32_t n) {
    volatile double prod = sigma * ((double)n * (1.0 / 65536.0));   /* no contraction */
    const double x = sky + prod;
    double r = rint(x);
    if (r < -127.0) r = -127.0;
    if (r > 127.0) r = 127.0;
    return (int8_t)(int)r;
}

int orc_gen_packets(uint8_t* pk, int64_t stride, int hdr, int nant, int nch, int tpkt, int nheaps,
                    int64_t heap0, uint32_t seq0, uint16_t port, const double* sky, double sigma,
                    uint64_t seed, int mode) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const int wire = hdr + 2 * nch * tpkt;
    uint8_t tmpl[64];
    header64(tmpl, wire, port);
    const int64_t npk = (int64_t)nheaps * nant;
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < npk; ++p) {
        const int a = (int)(p % nant);
        const int64_t h = p / nant;
        uint8_t* q = pk + p * stride;
        memcpy(q, tmpl, 64);
        const uint32_t s = seq0 + (uint32_t)p;
        q[SEQ_BYTE + 0] = (uint8_t)(s >> 24);
        q[SEQ_BYTE + 1] = (uint8_t)(s >> 16);
        q[SEQ_BYTE + 2] = (uint8_t)(s >> 8);
        q[SEQ_BYTE + 3] = (uint8_t)s;
        int8_t* re = (int8_t*)(q + hdr);
        int8_t* im = re + nch * tpkt;
        for (int sl = 0; sl < nch * tpkt; ++sl) {
            const int c = sl / tpkt, t = sl % tpkt;
            const uint64_t tau = (uint64_t)(heap0 + h) * (uint64_t)tpkt + (uint64_t)t;
            if (mode == 1) {
                uint32_t ctr[4] = {(uint32_t)a, (uint32_t)tau, (uint32_t)(tau >> 32), (uint32_t)c};
                philox(ctr, k0, k1);
                re[sl] = (int8_t)((int)(((uint64_t)ctr[0] * 255u) >> 32) - 127);
                im[sl] = (int8_t)((int)(((uint64_t)ctr[1] * 255u) >> 32) - 127);
            } else {
                uint32_t w[12];
                for (uint32_t d = 0; d < 3; ++d) {
                    uint32_t ctr[4] = {(uint32_t)a, (uint32_t)tau, (uint32_t)(tau >> 32),
                                       (uint32_t)c | (d << 24)};
                    philox(ctr, k0, k1);
                    memcpy(w + 4 * d, ctr, 16);
                }
                int32_t sr = 0, si = 0;
                for (int k = 0; k < 6; ++k) {
                    sr += (int32_t)(w[k] & 0xFFFFu) + (int32_t)(w[k] >> 16);
                    si += (int32_t)(w[6 + k] & 0xFFFFu) + (int32_t)(w[6 + k] >> 16);
                }
                const double skr = sky ? sky[((int64_t)c * nant + a) * 2 + 0] : 0.0;
                const double ski = sky ? sky[((int64_t)c * nant + a) * 2 + 1] : 0.0;
                re[sl] = quant(skr, sigma, sr - 393210);
                im[sl] = quant(ski, sigma, si - 393210);
            }
        }
    }
    return 0;
}

/* -------------------------------------------------------------- corner-turn */
/* planes [2][nch][nant][kt]; packet p = h*nant + a; k = k0 + h*tpkt + t. */
int orc_corner_turn(const uint8_t* pk, int64_t stride, int hdr, int nant, int nch, int tpkt,
                    int nheaps, int8_t* planes, int64_t kt, int64_t k0) {
    const int64_t half = (int64_t)nch * tpkt;
#pragma omp parallel for schedule(static)
    for (int a = 0; a < nant; ++a)
        for (int h = 0; h < nheaps; ++h) {
            const uint8_t* q = pk + ((int64_t)h * nant + a) * stride + hdr;
            for (int64_t sl = 0; sl < half; ++sl) {
                const int c = (int)(sl / tpkt), t = (int)(sl % tpkt);
                const int64_t k = k0 + (int64_t)h * tpkt + t;
                planes[(((int64_t)0 * nch + c) * nant + a) * kt + k] = (int8_t)q[sl];
                planes[(((int64_t)1 * nch + c) * nant + a) * kt + k] = (int8_t)q[half + sl];
            }
        }
    return 0;
}

/* seq check: number of packets whose big-endian seq differs from seq0 + p */
int64_t orc_seq_errors(const uint8_t* pk, int64_t stride, int64_t npk, uint32_t seq0) {
    int64_t bad = 0;
    for (int64_t p = 0; p < npk; ++p) {
        const uint8_t* h = pk + p * stride + SEQ_BYTE;
        const uint32_t s = ((uint32_t)h[0] << 24) | ((uint32_t)h[1] << 16) | ((uint32_t)h[2] << 8) | h[3];
        bad += (s != seq0 + (uint32_t)p);
    }
    return bad;
}

/* --------------------------------------------------------------- correlator */
/* Four int8 dot products of one (a, b) pair over n <= 32768 samples; built
 * for AVX-512 / AVX2 / baseline x86-64 and picked at load time. */
__attribute__((target_clones("arch=x86-64-v4", "arch=x86-64-v3", "default")))
static void dot4(const int8_t* xr_a, const int8_t* xi_a, const int8_t* xr_b, const int8_t* xi_b,
                 int64_t n, int32_t* r_out, int32_t* i_out) {
    int32_t rr = 0, ii = 0, ir = 0, ri = 0;
    for (int64_t k = 0; k < n; ++k) {
        rr += (int32_t)xr_a[k] * xr_b[k];
        ii += (int32_t)xi_a[k] * xi_b[k];
        ir += (int32_t)xi_a[k] * xr_b[k];
        ri += (int32_t)xr_a[k] * xi_b[k];
    }
    *r_out = rr + ii;
    *i_out = ir - ri;
}

/* The formula pair by pair, one (a, b) at a time: the plain statement of the
 * correlator, kept as the cross-check of the blocked one below. */
int orc_correlate_pairwise(const int8_t* planes, int nant, int nch, int64_t kt, int64_t kbeg,
                           int64_t klen, int c0, int nc, int64_t* out, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const int64_t NN = (int64_t)nant * nant;
    const int64_t KB = 32768;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
    for (int cc = 0; cc < nc; ++cc)
        for (int a = 0; a < nant; ++a) {
            const int c = c0 + cc;
            const int8_t* xr_a = planes + ((int64_t)(0 * nch + c) * nant + a) * kt;
            const int8_t* xi_a = planes + ((int64_t)(1 * nch + c) * nant + a) * kt;
            int64_t* ore = out + (int64_t)cc * 2 * NN + (int64_t)a * nant;
            int64_t* oim = ore + NN;
            for (int b = 0; b <= a; ++b) {
                const int8_t* xr_b = planes + ((int64_t)(0 * nch + c) * nant + b) * kt;
                const int8_t* xi_b = planes + ((int64_t)(1 * nch + c) * nant + b) * kt;
                int64_t sre = 0, sim = 0;
                for (int64_t k0 = kbeg; k0 < kbeg + klen; k0 += KB) {
                    const int64_t k1 = (k0 + KB < kbeg + klen) ? k0 + KB : kbeg + klen;
                    int32_t r, i;
                    dot4(xr_a + k0, xi_a + k0, xr_b + k0, xi_b + k0, k1 - k0, &r, &i);
                    sre += r;
                    sim += i;
                }
                ore[b] += sre;
                oim[b] += sim;
            }
        }
    return 0;
}

/* One 2 x 4 block of (a, b) pairs over n int16 values (n / 2 samples).  Rows
 * are (re, im) pairs, P_x = (xr, xi) and Q_x = (-xi, xr), so that
 *   P_a . P_b = xr_a xr_b + xi_a xi_b = Re,   P_a . Q_b = xi_a xr_b - xr_a xi_b = Im
 * and one widening multiply-add over adjacent int16 lanes gives a whole
 * complex product's real or imaginary part.  The eight pairs share their row
 * loads (2 + 8 rows for 16 sums instead of 4 rows per pair). */
__attribute__((target_clones("arch=x86-64-v4", "arch=x86-64-v3", "default")))
static void block2x4(const int16_t* restrict pa0, const int16_t* restrict pa1,
                     const int16_t* restrict pb0, const int16_t* restrict pb1,
                     const int16_t* restrict pb2, const int16_t* restrict pb3,
                     const int16_t* restrict qb0, const int16_t* restrict qb1,
                     const int16_t* restrict qb2, const int16_t* restrict qb3, int64_t n,
                     int32_t re[8], int32_t im[8]) {
    int32_t r0 = 0, r1 = 0, r2 = 0, r3 = 0, r4 = 0, r5 = 0, r6 = 0, r7 = 0;
    int32_t i0 = 0, i1 = 0, i2 = 0, i3 = 0, i4 = 0, i5 = 0, i6 = 0, i7 = 0;
    for (int64_t j = 0; j < n; ++j) {
        const int32_t a0 = pa0[j], a1 = pa1[j];
        const int32_t b0 = pb0[j], b1 = pb1[j], b2 = pb2[j], b3 = pb3[j];
        const int32_t q0 = qb0[j], q1 = qb1[j], q2 = qb2[j], q3 = qb3[j];
        r0 += a0 * b0; r1 += a0 * b1; r2 += a0 * b2; r3 += a0 * b3;
        r4 += a1 * b0; r5 += a1 * b1; r6 += a1 * b2; r7 += a1 * b3;
        i0 += a0 * q0; i1 += a0 * q1; i2 += a0 * q2; i3 += a0 * q3;
        i4 += a1 * q0; i5 += a1 * q1; i6 += a1 * q2; i7 += a1 * q3;
    }
    re[0] = r0; re[1] = r1; re[2] = r2; re[3] = r3; re[4] = r4; re[5] = r5; re[6] = r6; re[7] = r7;
    im[0] = i0; im[1] = i1; im[2] = i2; im[3] = i3; im[4] = i4; im[5] = i5; im[6] = i6; im[7] = i7;
}

/* The same block with AVX-512 VNNI (vpdpwssd: 32 int16 products summed in
 * pairs into 16 int32 lanes, accumulated without saturation); n a multiple of
 * 32 (rows are zero-padded to that).  Chosen at run time where the CPU has it. */
__attribute__((target("avx512f,avx512bw,avx512vnni")))
static void block2x4_vnni(const int16_t* restrict pa0, const int16_t* restrict pa1,
                          const int16_t* restrict pb0, const int16_t* restrict pb1,
                          const int16_t* restrict pb2, const int16_t* restrict pb3,
                          const int16_t* restrict qb0, const int16_t* restrict qb1,
                          const int16_t* restrict qb2, const int16_t* restrict qb3, int64_t n,
                          int32_t re[8], int32_t im[8]) {
    __m512i r0 = _mm512_setzero_si512(), r1 = r0, r2 = r0, r3 = r0, r4 = r0, r5 = r0, r6 = r0, r7 = r0;
    __m512i i0 = r0, i1 = r0, i2 = r0, i3 = r0, i4 = r0, i5 = r0, i6 = r0, i7 = r0;
    for (int64_t j = 0; j < n; j += 32) {
        const __m512i a0 = _mm512_loadu_si512(pa0 + j), a1 = _mm512_loadu_si512(pa1 + j);
        const __m512i b0 = _mm512_loadu_si512(pb0 + j), b1 = _mm512_loadu_si512(pb1 + j);
        const __m512i b2 = _mm512_loadu_si512(pb2 + j), b3 = _mm512_loadu_si512(pb3 + j);
        r0 = _mm512_dpwssd_epi32(r0, a0, b0); r1 = _mm512_dpwssd_epi32(r1, a0, b1);
        r2 = _mm512_dpwssd_epi32(r2, a0, b2); r3 = _mm512_dpwssd_epi32(r3, a0, b3);
        r4 = _mm512_dpwssd_epi32(r4, a1, b0); r5 = _mm512_dpwssd_epi32(r5, a1, b1);
        r6 = _mm512_dpwssd_epi32(r6, a1, b2); r7 = _mm512_dpwssd_epi32(r7, a1, b3);
        const __m512i q0 = _mm512_loadu_si512(qb0 + j), q1 = _mm512_loadu_si512(qb1 + j);
        const __m512i q2 = _mm512_loadu_si512(qb2 + j), q3 = _mm512_loadu_si512(qb3 + j);
        i0 = _mm512_dpwssd_epi32(i0, a0, q0); i1 = _mm512_dpwssd_epi32(i1, a0, q1);
        i2 = _mm512_dpwssd_epi32(i2, a0, q2); i3 = _mm512_dpwssd_epi32(i3, a0, q3);
        i4 = _mm512_dpwssd_epi32(i4, a1, q0); i5 = _mm512_dpwssd_epi32(i5, a1, q1);
        i6 = _mm512_dpwssd_epi32(i6, a1, q2); i7 = _mm512_dpwssd_epi32(i7, a1, q3);
    }
    re[0] = _mm512_reduce_add_epi32(r0); re[1] = _mm512_reduce_add_epi32(r1);
    re[2] = _mm512_reduce_add_epi32(r2); re[3] = _mm512_reduce_add_epi32(r3);
    re[4] = _mm512_reduce_add_epi32(r4); re[5] = _mm512_reduce_add_epi32(r5);
    re[6] = _mm512_reduce_add_epi32(r6); re[7] = _mm512_reduce_add_epi32(r7);
    im[0] = _mm512_reduce_add_epi32(i0); im[1] = _mm512_reduce_add_epi32(i1);
    im[2] = _mm512_reduce_add_epi32(i2); im[3] = _mm512_reduce_add_epi32(i3);
    im[4] = _mm512_reduce_add_epi32(i4); im[5] = _mm512_reduce_add_epi32(i5);
    im[6] = _mm512_reduce_add_epi32(i6); im[7] = _mm512_reduce_add_epi32(i7);
}

typedef void (*block_fn)(const int16_t*, const int16_t*, const int16_t*, const int16_t*,
                         const int16_t*, const int16_t*, const int16_t*, const int16_t*,
                         const int16_t*, const int16_t*, int64_t, int32_t*, int32_t*);

/* Lower triangle of V for channels [c0, c0+nc) over samples [kbeg, kbeg+klen)
 * of planes [2][nch][nant][kt], ADDED into out[c - c0][2][nant][nant] at (a, b)
 * with b <= a; if mirror != 0 the upper triangle is then filled by
 * conjugation.  nthreads <= 0: OpenMP default.
 * Blocked form of orc_correlate_pairwise (same sums, exactly): per channel and
 * chunk of KC samples the rows are widened into P / Q (int16 pairs, rows padded
 * with zeros to a multiple of 64) and the triangle is walked in 64 x 64 tiles of
 * 2 x 4 blocks of pairs; int32 partial sums per chunk (|sum| <= 2 * 128^2 * KC < 2^31) are
 * added into int64. */
int orc_correlate(const int8_t* planes, int nant, int nch, int64_t kt, int64_t kbeg, int64_t klen,
                  int c0, int nc, int64_t* out, int mirror, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const int64_t NN = (int64_t)nant * nant;
    const int64_t KC = 1024;
    const int TB = 64;                               /* rows per cache tile */
    const int npad = (nant + TB - 1) / TB * TB;
    const int64_t row = 2 * KC;                      /* int16 per row of a chunk */
    __builtin_cpu_init();
    const block_fn block = __builtin_cpu_supports("avx512vnni") ? block2x4_vnni : block2x4;
    int16_t* P = (int16_t*)calloc((size_t)npad * row, sizeof(int16_t));
    int16_t* Q = (int16_t*)calloc((size_t)npad * row, sizeof(int16_t));
    if (!P || !Q) {
        free(P);
        free(Q);
        return -1;
    }
    for (int cc = 0; cc < nc; ++cc) {
        const int c = c0 + cc;
        int64_t* ore = out + (int64_t)cc * 2 * NN;
        int64_t* oim = ore + NN;
        for (int64_t k0 = kbeg; k0 < kbeg + klen; k0 += KC) {
            const int64_t len = (k0 + KC < kbeg + klen) ? KC : kbeg + klen - k0;
#pragma omp parallel for schedule(static)
            for (int a = 0; a < npad; ++a) {
                int16_t* p = P + (int64_t)a * row;
                int16_t* q = Q + (int64_t)a * row;
                if (a < nant) {
                    const int8_t* xr = planes + ((int64_t)(0 * nch + c) * nant + a) * kt + k0;
                    const int8_t* xi = planes + ((int64_t)(1 * nch + c) * nant + a) * kt + k0;
                    for (int64_t k = 0; k < len; ++k) {
                        p[2 * k] = xr[k];
                        p[2 * k + 1] = xi[k];
                        q[2 * k] = (int16_t)(-xi[k]);
                        q[2 * k + 1] = xr[k];
                    }
                }
                for (int64_t k = 2 * len; k < row; ++k) p[k] = q[k] = 0;
            }
            /* 64 x 64 tiles of the triangle; in a tile the 4 b rows of a block (P and
             * Q, 32 KB) stay in L1 while the tile's a rows stream from L2 */
            const int nt = npad / TB;
#pragma omp parallel for schedule(dynamic, 1)
            for (int tt = 0; tt < nt * (nt + 1) / 2; ++tt) {
                int ta = 0;
                while ((ta + 1) * (ta + 2) / 2 <= tt) ++ta;
                const int tb = tt - ta * (ta + 1) / 2;
                for (int b0 = tb * TB; b0 < (tb + 1) * TB; b0 += 4) {
                    const int16_t* pb = P + (int64_t)b0 * row;
                    const int16_t* qb = Q + (int64_t)b0 * row;
                    for (int a0 = ta * TB; a0 < (ta + 1) * TB; a0 += 2) {
                        if (b0 > a0 + 1) continue;               /* above the diagonal */
                        const int16_t* pa0 = P + (int64_t)a0 * row;
                        int32_t re[8], im[8];
                        /* rows are zero beyond 2 * len: run to a multiple of 32 int16 */
                        block(pa0, pa0 + row, pb, pb + row, pb + 2 * row, pb + 3 * row, qb,
                              qb + row, qb + 2 * row, qb + 3 * row,
                              (2 * len + 31) & ~(int64_t)31, re, im);
                        for (int u = 0; u < 2; ++u)
                            for (int v = 0; v < 4; ++v) {
                                const int a = a0 + u, b = b0 + v;
                                if (a < nant && b <= a) {
                                    ore[(int64_t)a * nant + b] += re[4 * u + v];
                                    oim[(int64_t)a * nant + b] += im[4 * u + v];
                                }
                            }
                    }
                }
            }
        }
    }
    free(P);
    free(Q);
    if (mirror) {
#pragma omp parallel for schedule(static)
        for (int cc = 0; cc < nc; ++cc) {
            int64_t* re = out + (int64_t)cc * 2 * NN;
            int64_t* im = re + NN;
            for (int a = 0; a < nant; ++a)
                for (int b = a + 1; b < nant; ++b) {
                    re[(int64_t)a * nant + b] = re[(int64_t)b * nant + a];
                    im[(int64_t)a * nant + b] = -im[(int64_t)b * nant + a];
                }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------ gridding */
/* full: [nch][2][nant][nant] int64 (full square).  grid: [nch][G][G][2] int64,
 * overwritten: every ordered pair (a, b) adds V[a][b] at
 * ((ya - yb) mod G, (xa - xb) mod G), (x, y) = (a % side_x, a / side_x). */
int orc_grid(const int64_t* full, int nant, int nch, int side_x, int G, int64_t* grid) {
    const int64_t NN = (int64_t)nant * nant;
    memset(grid, 0, sizeof(int64_t) * (size_t)nch * G * G * 2);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nch; ++c) {
        const int64_t* re = full + (int64_t)c * 2 * NN;
        const int64_t* im = re + NN;
        int64_t* g = grid + (int64_t)c * G * G * 2;
        for (int a = 0; a < nant; ++a)
            for (int b = 0; b < nant; ++b) {
                int dy = (a / side_x - b / side_x) % G, dx = (a % side_x - b % side_x) % G;
                if (dy < 0) dy += G;
                if (dx < 0) dx += G;
                g[(dy * G + dx) * 2 + 0] += re[(int64_t)a * nant + b];
                g[(dy * G + dx) * 2 + 1] += im[(int64_t)a * nant + b];
            }
    }
    return 0;
}

int orc_max_threads(void) { return omp_get_max_threads(); }
