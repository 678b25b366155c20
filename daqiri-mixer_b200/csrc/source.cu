// source.cu -- seeded packet source in the reference wire format.
//
// Stands in for the DAQIRI capture and for the reference's TX sky generator
// (src/tx_host.cu:41-60 k_sky, :62-79 header template).  Packets carry the
// header layout of src/config.h:10-23 (eth/ip/udp, big-endian seq at byte 48)
// and a planar int8 payload re[c*tpkt + t] | im[...].  Samples are
//     clip(rint(sky[c][a] + sigma * n), -127, 127)
// with sky evaluated once on the host in FP64 and n an Irwin-Hall(12) deviate
// built from Philox4x32-10 (Salmon et al., SC'11) integer draws, so the device
// and any CPU restatement of the same formula produce identical bytes.
#include <cmath>
#include <cstring>
#include "common.cuh"

namespace mixer {

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw 2011) ------------------------
struct U4 {
    uint32_t x, y, z, w;
};
__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}
__host__ __device__ __forceinline__ U4 philox4x32_10(U4 ctr, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += W0;
            k1 += W1;
        }
        const uint32_t lo0 = M0 * ctr.x, hi0 = mulhi32(M0, ctr.x);
        const uint32_t lo1 = M1 * ctr.z, hi1 = mulhi32(M1, ctr.z);
        ctr = U4{hi1 ^ ctr.y ^ k0, lo1, hi0 ^ ctr.w ^ k1, lo0};
    }
    return ctr;
}

namespace {

struct Hdr64 {
    uint8_t b[64];
};

// Irwin-Hall sum of 12 16-bit uniforms, centred: integer in [-393210, 393210],
// standard deviation 65536 * (1 - 2^-32)^0.5 ~= 65536.
__device__ __forceinline__ void noise_pair(uint32_t a, uint64_t tau, uint32_t c, uint32_t k0,
                                           uint32_t k1, int32_t& nre, int32_t& nim) {
    uint32_t w[12];
#pragma unroll
    for (uint32_t d = 0; d < 3; ++d) {
        const U4 r = philox4x32_10(U4{a, (uint32_t)tau, (uint32_t)(tau >> 32), c | (d << 24)}, k0, k1);
        w[4 * d + 0] = r.x;
        w[4 * d + 1] = r.y;
        w[4 * d + 2] = r.z;
        w[4 * d + 3] = r.w;
    }
    int32_t sr = 0, si = 0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        sr += (int32_t)(w[q] & 0xFFFFu) + (int32_t)(w[q] >> 16);
        si += (int32_t)(w[6 + q] & 0xFFFFu) + (int32_t)(w[6 + q] >> 16);
    }
    nre = sr - 393210;
    nim = si - 393210;
}

__device__ __forceinline__ int8_t quantise(double sky, double sigma, int32_t n) {
    // one product, one sum, each correctly rounded (no contraction)
    const double x = __dadd_rn(sky, __dmul_rn(sigma, (double)n * (1.0 / 65536.0)));
    double r = rint(x);
    r = r < -127.0 ? -127.0 : (r > 127.0 ? 127.0 : r);
    return (int8_t)(int)r;
}

__global__ void __launch_bounds__(256)
    k_gen_packets(uint8_t* __restrict__ pk, int64_t pkt_stride, int hdr, int nant, int nch, int tpkt,
                  int64_t heap0, uint32_t seq0, const Hdr64 tmpl, const double* __restrict__ sky,
                  double sigma, uint32_t k0, uint32_t k1, int mode) {
    const int64_t p = blockIdx.x;   // packet index within the call
    const int a = (int)(p % nant);
    const int64_t h = p / nant;
    uint8_t* pkt = pk + p * pkt_stride;
    if (threadIdx.x < 16) {
        uint32_t word;
        memcpy(&word, tmpl.b + 4 * threadIdx.x, 4);
        if (threadIdx.x == MIXER_WIRE_SEQ_BYTE / 4) {
            const uint32_t s = seq0 + (uint32_t)p;
            word = (s >> 24) | ((s >> 8) & 0xFF00u) | ((s << 8) & 0xFF0000u) | (s << 24);
        }
        reinterpret_cast<uint32_t*>(pkt)[threadIdx.x] = word;   // bytes 0..63
    }
    const int half = nch * tpkt;
    int8_t* re = reinterpret_cast<int8_t*>(pkt + hdr);
    int8_t* im = re + half;
    for (int s = threadIdx.x; s < half; s += blockDim.x) {
        const int c = s / tpkt;
        const int t = s - c * tpkt;
        const uint64_t tau = (uint64_t)(heap0 + h) * (uint64_t)tpkt + (uint64_t)t;
        int8_t vr, vi;
        if (mode == 1) {
            const U4 r = philox4x32_10(U4{(uint32_t)a, (uint32_t)tau, (uint32_t)(tau >> 32), (uint32_t)c},
                                       k0, k1);
            vr = (int8_t)((int)(((uint64_t)r.x * 255u) >> 32) - 127);
            vi = (int8_t)((int)(((uint64_t)r.y * 255u) >> 32) - 127);
        } else {
            int32_t nr, ni;
            noise_pair((uint32_t)a, tau, (uint32_t)c, k0, k1, nr, ni);
            double sr = 0.0, si = 0.0;
            if (sky) {
                sr = sky[((int64_t)c * nant + a) * 2 + 0];
                si = sky[((int64_t)c * nant + a) * 2 + 1];
            }
            vr = quantise(sr, sigma, nr);
            vi = quantise(si, sigma, ni);
        }
        re[s] = vr;
        im[s] = vi;
    }
}

// eth(14) + ipv4(20) + udp(8) + reserved, seq slot at 48 (src/config.h:10-14).
Hdr64 make_header(int wire_bytes, uint16_t port) {
    Hdr64 h;
    memset(h.b, 0, sizeof(h.b));
    const uint8_t dst[6] = {0xa0, 0x88, 0xc2, 0x0d, 0x5e, 0x28};
    memcpy(h.b, dst, 6);
    h.b[12] = 0x08;
    h.b[13] = 0x00;                       // IPv4
    uint8_t* ip = h.b + 14;
    ip[0] = 0x45;                         // version 4, ihl 5
    const int ip_len = wire_bytes - 14;
    ip[2] = (uint8_t)(ip_len >> 8);
    ip[3] = (uint8_t)ip_len;
    ip[8] = 64;                           // ttl
    ip[9] = 17;                           // udp
    const uint8_t src_ip[4] = {10, 0, 0, 1}, dst_ip[4] = {10, 0, 0, 2};
    memcpy(ip + 12, src_ip, 4);
    memcpy(ip + 16, dst_ip, 4);
    uint32_t sum = 0;
    for (int i = 0; i < 20; i += 2) sum += ((uint32_t)ip[i] << 8) | ip[i + 1];
    while (sum >> 16) sum = (sum & 0xFFFF) + (sum >> 16);
    const uint16_t ck = (uint16_t)~sum;
    ip[10] = (uint8_t)(ck >> 8);
    ip[11] = (uint8_t)ck;
    uint8_t* udp = h.b + 34;
    udp[0] = udp[2] = (uint8_t)(port >> 8);
    udp[1] = udp[3] = (uint8_t)port;
    const int udp_len = wire_bytes - 34;
    udp[4] = (uint8_t)(udp_len >> 8);
    udp[5] = (uint8_t)udp_len;
    return h;
}

__global__ void k_restamp(uint8_t* __restrict__ pk, int64_t npk, int64_t stride, uint32_t seq0) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npk) return;
    const uint32_t s = seq0 + (uint32_t)p;
    uint8_t* h = pk + p * stride + MIXER_WIRE_SEQ_BYTE;
    h[0] = (uint8_t)(s >> 24);
    h[1] = (uint8_t)(s >> 16);
    h[2] = (uint8_t)(s >> 8);
    h[3] = (uint8_t)s;
}

}  // namespace
}  // namespace mixer

extern "C" int mixer_restamp_seq(uint8_t* packets, int64_t npk, int64_t pkt_stride, uint32_t seq0,
                                 void* stream) {
    if (!packets || npk <= 0 || pkt_stride < 64) return MIXER_EINVAL;
    const int64_t blocks = (npk + 255) / 256;
    if (blocks > 0x7FFFFFFFLL) return MIXER_EINVAL;
    mixer::k_restamp<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(packets, npk,
                                                                                      pkt_stride, seq0);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}

extern "C" int mixer_sky_table(int32_t nant, int32_t nch, int32_t side_x, int32_t nsrc,
                               const double* l, const double* m, const double* amp0,
                               const double* amp1, double* table) {
    if (nant <= 0 || nch <= 0 || side_x <= 0 || nsrc < 0 || !table) return MIXER_EINVAL;
    if (nsrc > 0 && (!l || !m || !amp0 || !amp1)) return MIXER_EINVAL;
    const double two_pi = 6.283185307179586476925286766559;
    for (int c = 0; c < nch; ++c) {
        const double fc = 1.0 + (double)c / (double)nch;
        for (int a = 0; a < nant; ++a) {
            const double x = (double)(a % side_x), y = (double)(a / side_x);
            double re = 0.0, im = 0.0;
            for (int s = 0; s < nsrc; ++s) {
                const double amp = amp0[s] + amp1[s] * (double)c / (double)nch;
                const double ph = -two_pi * fc * (x * l[s] + y * m[s]);
                re += amp * std::cos(ph);
                im += amp * std::sin(ph);
            }
            table[((int64_t)c * nant + a) * 2 + 0] = re;
            table[((int64_t)c * nant + a) * 2 + 1] = im;
        }
    }
    return MIXER_OK;
}

extern "C" int mixer_gen_packets(uint8_t* packets, int64_t pkt_stride, int32_t hdr_bytes,
                                 int32_t nant, int32_t nch, int32_t tpkt, int32_t nheaps,
                                 int64_t heap0, uint32_t seq0, uint16_t udp_port, const double* sky,
                                 double sigma, uint64_t seed, int32_t noise_mode, void* stream) {
    if (!packets || nant <= 0 || nch <= 0 || tpkt <= 0 || nheaps <= 0) return MIXER_EINVAL;
    if (hdr_bytes < 64 || pkt_stride < hdr_bytes + 2LL * nch * tpkt || pkt_stride % 4 != 0)
        return MIXER_EINVAL;
    if (noise_mode != 0 && noise_mode != 1) return MIXER_EINVAL;
    if (nch >= (1 << 24)) return MIXER_EINVAL;
    const int wire = hdr_bytes + 2 * nch * tpkt;
    const mixer::Hdr64 tmpl = mixer::make_header(wire, udp_port);
    const int64_t npk = (int64_t)nheaps * nant;
    if (npk > 0x7FFFFFFFLL) return MIXER_EINVAL;
    mixer::k_gen_packets<<<(unsigned)npk, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        packets, pkt_stride, hdr_bytes, nant, nch, tpkt, heap0, seq0, tmpl, sky, sigma,
        (uint32_t)seed, (uint32_t)(seed >> 32), noise_mode);
    MIXER_CK(cudaGetLastError());
    return MIXER_OK;
}
