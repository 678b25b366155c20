// mixer_rx -- the receiver program of the X-engine.
//
// Re-creates the command-line surface and the loops of the reference's
// receiver (src/rx_host_corr.cu:177-246) on top of the C-ABI:
//   GPU thread  : correlate + integrate V-updates as they arrive
//                 (gpu_thread, :143-175) -- here from the seeded packet source
//                 replayed at --gbps, since no NIC / DAQIRI exists on this box;
//   main loop   : at --fps, a delta image of the integrated cube is published
//                 to the Corr32 shared memory (:214-236) and, about once a
//                 second with --dump, the FP32 cube record is appended (:224-227);
//   status line : once a second, like :237-238.
// Usage: mixer_rx [yaml] [--seconds N] [--fps F] [--device D] [--noflop]
//                 [--flush N] [--dump PATH] [--gbps R] [--shm NAME] [--keep-shm]
//                 [--vupdates N] [--seed S]
// The YAML argument is accepted for command-line compatibility and ignored.
// --flush N: V-updates (32 heaps each) per correlate call; int32 partial sums
// stay in TMEM for the call and are added into the int64 cube at its end.
// --vupdates N: stop after N V-updates, write one dump, exit (deterministic).
#include <cuda_runtime.h>
#include <atomic>
#include <chrono>
#include <cmath>
#include <csignal>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "mixer.h"

namespace {

volatile std::sig_atomic_t g_stop = 0;
void on_sig(int) { g_stop = 1; }

#define CHECK(call)                                                                      \
    do {                                                                                 \
        int rc_ = (call);                                                                \
        if (rc_ != MIXER_OK) {                                                           \
            fprintf(stderr, "[mixer_rx] %s: %s\n", #call, mixer_strerror(rc_));          \
            return 1;                                                                    \
        }                                                                                \
    } while (0)

constexpr int kHbatch = 32;   // heaps per V-update (src/rx_host_corr.cu:39)

// Star A1 = 6 at (0.10, -0.05) and a planet of amplitude 1.5 c / C on a circle of
// radius 0.2 (angle `ang`), evaluated on the host in FP64.
int make_sky(const mixer_array_desc& d, double ang, double* d_sky, std::vector<double>& h) {
    const double l[2] = {0.10, 0.2 * std::cos(ang)}, m[2] = {-0.05, 0.2 * std::sin(ang)};
    const double a0[2] = {6.0, 0.0}, a1[2] = {0.0, 1.5};
    h.resize((size_t)d.nch * d.nant * 2);
    int rc = mixer_sky_table(d.nant, d.nch, d.side_x, 2, l, m, a0, a1, h.data());
    if (rc != MIXER_OK) return rc;
    return cudaMemcpy(d_sky, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess
               ? MIXER_OK
               : MIXER_ECUDA;
}

}  // namespace

int main(int argc, char** argv) {
    int seconds = 0, device = 0, flush = 4;
    double fps = 20.0, gbps = 380.0, torbit = 20.0;
    bool noflop = false, keep_shm = false;
    long long vupdates_max = 0;
    unsigned long long seed = 20261203ull;
    const char* dump_path = nullptr;
    std::string shm_name = "/corr32";
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&]() { return (i + 1 < argc) ? argv[++i] : (char*)"0"; };
        if (a == "--seconds") seconds = atoi(next());
        else if (a == "--fps") fps = atof(next());
        else if (a == "--device") device = atoi(next());
        else if (a == "--noflop") noflop = true;
        else if (a == "--flush") flush = atoi(next());
        else if (a == "--dump") dump_path = next();
        else if (a == "--gbps") gbps = atof(next());
        else if (a == "--shm") shm_name = next();
        else if (a == "--keep-shm") keep_shm = true;
        else if (a == "--vupdates") vupdates_max = atoll(next());
        else if (a == "--seed") seed = strtoull(next(), nullptr, 10);
        else if (a == "--orbit") torbit = atof(next());
        else if (a.size() > 2 && a[0] == '-' && a[1] == '-') {
            fprintf(stderr, "usage: %s [yaml] [--seconds N][--fps F][--device D][--noflop][--flush N]"
                            "[--dump PATH][--gbps R][--shm NAME][--keep-shm][--vupdates N][--seed S]\n",
                    argv[0]);
            return 1;
        }
    }
    if (flush < 1 || fps <= 0.0) {
        fprintf(stderr, "[mixer_rx] --flush >= 1 and --fps > 0 required\n");
        return 1;
    }
    std::signal(SIGINT, on_sig);
    std::signal(SIGTERM, on_sig);
    if (cudaSetDevice(device) != cudaSuccess) {
        fprintf(stderr, "[mixer_rx] no device %d\n", device);
        return 1;
    }
    mixer_array_desc d;
    mixer_desc_default(&d);
    d.max_heaps = kHbatch * flush;
    mixer_ctx* ctx = nullptr;
    CHECK(mixer_create(&d, &ctx));
    const int G = 32;
    // source pool: 16 V-updates of the seeded sky, replayed with fresh seqs
    const int pool_vu = 16;
    const size_t vu_bytes = (size_t)kHbatch * d.nant * d.pkt_stride;
    uint8_t* pool = nullptr;
    double* d_sky = nullptr;
    if (cudaMalloc(&pool, pool_vu * vu_bytes) != cudaSuccess ||
        cudaMalloc(&d_sky, (size_t)d.nch * d.nant * 2 * sizeof(double)) != cudaSuccess) {
        fprintf(stderr, "[mixer_rx] out of device memory\n");
        return 1;
    }
    std::vector<double> hsky;
    CHECK(make_sky(d, 0.0, d_sky, hsky));
    CHECK(mixer_gen_packets(pool, d.pkt_stride, d.hdr_bytes, d.nant, d.nch, d.tpkt, pool_vu * kHbatch, 0,
                            0, MIXER_WIRE_UDP_PORT, d_sky, 16.0, seed, 0, nullptr));
    cudaDeviceSynchronize();
    cudaStream_t comp;
    cudaStreamCreateWithFlags(&comp, cudaStreamNonBlocking);
    mixer_shm* shm = nullptr;
    CHECK(mixer_shm_open(shm_name.c_str(), d.nch, G, &shm));
    std::vector<float> img((size_t)d.nch * G * G), vmax(d.nch), vmin(d.nch);
    std::mutex mu;   // one host thread at a time on the context
    std::atomic<unsigned long long> vupd{0};
    std::atomic<bool> gpu_done{false};
    std::atomic<int> gpu_err{0};
    fprintf(stderr, "[mixer_rx] seeded source (no DAQIRI) -> %d-channel cube of %dx%d images, "
                    "%d V-updates per launch, %.0f Gb/s offered, %.0f Hz, shm %s\n",
            d.nch, G, G, flush, gbps, fps, shm_name.c_str());

    std::thread gpu([&]() {
        cudaSetDevice(device);
        const double period = gbps > 0 ? 8.0 * (double)vu_bytes * flush / (gbps * 1e9) : 0.0;
        auto t_next = std::chrono::steady_clock::now();
        unsigned long long v = 0;
        double last_orbit = 0.0;
        const auto t0 = std::chrono::steady_clock::now();
        while (!g_stop && (vupdates_max == 0 || (long long)v < vupdates_max)) {
            if (period > 0) {
                std::this_thread::sleep_until(t_next);
                t_next += std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                    std::chrono::duration<double>(period));
            }
            const long long n = vupdates_max ? std::min<long long>(flush, vupdates_max - (long long)v) : flush;
            const int p0 = (int)(v % pool_vu);
            const int run = (int)std::min<long long>(n, pool_vu - p0);
            std::lock_guard<std::mutex> lk(mu);
            if (noflop) {
                v += run;
                vupd.store(v);
                continue;
            }
            // planet moves with wall time; refresh the pool about once a second
            const double t = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (vupdates_max == 0 && t - last_orbit > 1.0) {
                last_orbit = t;
                if (make_sky(d, 2.0 * M_PI * t / torbit, d_sky, hsky) != MIXER_OK ||
                    mixer_gen_packets(pool, d.pkt_stride, d.hdr_bytes, d.nant, d.nch, d.tpkt,
                                      pool_vu * kHbatch, 0, 0, MIXER_WIRE_UDP_PORT, d_sky, 16.0,
                                      seed + (unsigned long long)t, 0, comp) != MIXER_OK) {
                    gpu_err.store(1);
                    break;
                }
            }
            uint8_t* src = pool + (size_t)p0 * vu_bytes;
            const uint32_t seq = (uint32_t)(v * kHbatch * d.nant);
            int rc = mixer_restamp_seq(src, (int64_t)run * kHbatch * d.nant, d.pkt_stride, seq, comp);
            if (rc == MIXER_OK) rc = mixer_correlate(ctx, src, (int64_t)run * kHbatch, seq, 1, comp);
            if (rc != MIXER_OK) {
                fprintf(stderr, "[mixer_rx] correlate: %s\n", mixer_strerror(rc));
                gpu_err.store(rc);
                break;
            }
            v += run;
            vupd.store(v);
        }
        gpu_done.store(true);
    });

    const auto t0 = std::chrono::steady_clock::now();
    auto next = t0;
    uint64_t frame = 0;
    const uint64_t per_s = (uint64_t)std::max(1.0, std::round(fps));
    int status = 0;
    while (!g_stop) {
        const bool last = gpu_done.load();
        if (seconds > 0 &&
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >= seconds)
            break;
        next += std::chrono::duration_cast<std::chrono::steady_clock::duration>(
            std::chrono::duration<double>(1.0 / fps));
        if (!last) std::this_thread::sleep_until(next);
        {
            std::lock_guard<std::mutex> lk(mu);
            if (mixer_image(ctx, img.data(), vmax.data(), vmin.data(), 1, 0, comp) != MIXER_OK ||
                cudaStreamSynchronize(comp) != cudaSuccess) {
                status = 1;
                break;
            }
            if (dump_path && (frame % per_s == 0 || last) && mixer_dump_to_file(ctx, dump_path, comp) != MIXER_OK) {
                status = 1;
                break;
            }
        }
        float gmax = -1e30f;
        int gch = 0;
        for (int c = 0; c < d.nch; ++c)
            if (vmax[c] > gmax) {
                gmax = vmax[c];
                gch = c;
            }
        mixer_shm_publish(shm, img.data(), vmax.data(), vmin.data(), frame + 1);
        if (frame % per_s == 0 || last) {
            int64_t samples = 0, seq_err = 0;
            int32_t kerr = 0;
            {
                std::lock_guard<std::mutex> lk(mu);
                mixer_stats(ctx, &samples, &seq_err, &kerr);
            }
            fprintf(stderr, "[mixer_rx] frame %llu vupdates=%llu samples=%lld peak-ch=%d vmax=%.3g "
                            "seq_errors=%lld kernel_err=%d\n",
                    (unsigned long long)frame, (unsigned long long)vupd.load(), (long long)samples, gch,
                    gmax, (long long)seq_err, kerr);
            if (seq_err || kerr) status = 1;
        }
        ++frame;
        if (last) break;
    }
    g_stop = 1;
    gpu.join();
    if (gpu_err.load()) status = 1;
    fprintf(stderr, "[mixer_rx] stop after %llu frames; V-updates=%llu\n", (unsigned long long)frame,
            (unsigned long long)vupd.load());
    mixer_shm_close(shm, keep_shm ? 0 : 1);
    cudaStreamDestroy(comp);
    cudaFree(pool);
    cudaFree(d_sky);
    mixer_destroy(ctx);
    return status;
}
