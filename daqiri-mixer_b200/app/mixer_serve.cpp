// mixer_serve -- load generator for the streaming server, on the C-ABI.
//
// Eight concurrent array streams (four of 256 elements x 128 channels with 32
// samples per packet, four of 1024 elements x 64 channels with 64 samples per
// packet; K 256 per sub-integration, a dump every 64 sub-integrations) are fed
// to one mixer_server from eight C++ feeder threads, one per stream, each
// replaying a device pool of 64 sub-integrations of wire-format heaps from the
// seeded packet source (the sequence numbers are re-stamped every lap so the
// stream continues).  A poller thread takes the dumps as they complete.
//
// With --gbps R each stream is paced to R / 8 (the reference's ingest rate is
// ~380 Gb/s, README.md:9); with --gbps 0 every feeder submits as fast as the
// server accepts, so the run measures the server itself (admission, the
// continuous-batching worker, corner-turn + one tensor-core launch per
// iteration, dumps) rather than the feeders.  --jitter 1 staggers the stream
// starts and stops (Poisson starts, each stream active for 50-90 % of the run).
//
// Prints one JSON line: offered / submitted / processed Gb/s (wire bytes), the
// aggregate over the window in which all eight streams were submitting, p50 /
// p99 / max dump latency and the server's counters.
// Usage: mixer_serve [--seconds S] [--gbps R] [--budget-gb B] [--device D]
//                    [--jitter 0|1] [--seed N] [--batch-subs N] [--ring-subs N]
//                    [--nsub-dump N] [--reserve 0|1]
// --nsub-dump N: sub-integrations per dump (default 64); the dump cubes cross
// PCIe to host memory, so a sparser cadence shows how much of the unpaced
// ceiling those copies take.
// --reserve 1: before the timed run, mixer_server_reserve allocates the state
// of the eight streams (device pool, pinned dump buffers), as a server that
// knows its stream shapes does at start-up; admissions then allocate nothing.
#include <cuda_runtime.h>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <thread>
#include <vector>
#include "mixer.h"

namespace {

struct StreamType {
    int nant, nch, tpkt, ksub, nsub, side;
};
constexpr StreamType kTypes[2] = {{256, 128, 32, 256, 64, 16}, {1024, 64, 64, 256, 64, 32}};
constexpr int kStreams = 8;
constexpr int kPoolSubs = 64;      // sub-integrations of heaps in each replayed device pool

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void sleep_s(double s) {
    if (s > 0) std::this_thread::sleep_for(std::chrono::duration<double>(s));
}

struct Feed {
    StreamType ty;
    int64_t hps = 0, stride = 0, sub_bytes = 0;
    uint8_t* pool = nullptr;       // kPoolSubs sub-integrations of heaps, device
    double start = 0, stop = 0;    // seconds from t0
    std::atomic<int> id{-1};
    int64_t submitted = 0, refusals = 0;
    double open_wait = 0, active = 0;
    std::vector<double> stamps;    // accepted submissions, seconds from t0
    std::atomic<int64_t> dumps{0};  // dumps taken by the poller
    int err = MIXER_OK;
};

}  // namespace

int main(int argc, char** argv) {
    double seconds = 10.0, gbps = 380.0, budget_gb = 16.0;
    int device = 0, jitter = 1, batch_subs = 8, ring_subs = 16, nsub_dump = 64, reserve = 0;
    uint64_t seed = 20261203;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() { return i + 1 < argc ? argv[++i] : (char*)"0"; };
        if (a == "--seconds") seconds = atof(next());
        else if (a == "--gbps") gbps = atof(next());
        else if (a == "--budget-gb") budget_gb = atof(next());
        else if (a == "--device") device = atoi(next());
        else if (a == "--jitter") jitter = atoi(next());
        else if (a == "--seed") seed = strtoull(next(), nullptr, 10);
        else if (a == "--batch-subs") batch_subs = atoi(next());
        else if (a == "--ring-subs") ring_subs = atoi(next());
        else if (a == "--nsub-dump") nsub_dump = atoi(next());
        else if (a == "--reserve") reserve = atoi(next());
        else {
            fprintf(stderr, "usage: mixer_serve [--seconds S] [--gbps R] [--budget-gb B] [--device D] "
                            "[--jitter 0|1] [--seed N] [--batch-subs N] [--ring-subs N] "
                            "[--nsub-dump N] [--reserve 0|1]\n");
            return 2;
        }
    }
    if (cudaSetDevice(device) != cudaSuccess || mixer_device_ok() != MIXER_OK) {
        fprintf(stderr, "[mixer_serve] no usable sm_100 device %d\n", device);
        return 1;
    }
    std::vector<Feed> feeds(kStreams);
    std::mt19937_64 rng(seed + 3);
    std::exponential_distribution<double> expo(1.0 / (seconds * 0.04));
    std::uniform_real_distribution<double> frac(0.5, 0.9);
    double t_start = 0;
    for (int i = 0; i < kStreams; ++i) {
        Feed& f = feeds[i];
        f.ty = kTypes[i < 4 ? 0 : 1];
        if (nsub_dump > 0) f.ty.nsub = nsub_dump;
        f.hps = f.ty.ksub / f.ty.tpkt;
        f.stride = 64 + 2LL * f.ty.nch * f.ty.tpkt;
        f.sub_bytes = f.hps * f.ty.nant * f.stride;
        if (jitter) {
            t_start += expo(rng);
            f.start = t_start;
            f.stop = std::min(seconds, f.start + frac(rng) * seconds);
        } else {
            f.start = 0;
            f.stop = seconds;
        }
        // the pool: 64 sub-integrations of heaps of the star + planet sky, sigma 16
        const int64_t nheaps = (int64_t)kPoolSubs * f.hps;
        if (cudaMalloc(&f.pool, (size_t)(nheaps * f.ty.nant * f.stride)) != cudaSuccess) {
            fprintf(stderr, "[mixer_serve] pool allocation failed\n");
            return 1;
        }
        const double l[2] = {0.10, 0.2}, m[2] = {-0.05, 0.0}, a0[2] = {6.0, 0.0}, a1[2] = {0.0, 1.5};
        std::vector<double> sky((size_t)f.ty.nch * f.ty.nant * 2);
        double* d_sky = nullptr;
        int rc = mixer_sky_table(f.ty.nant, f.ty.nch, f.ty.side, 2, l, m, a0, a1, sky.data());
        if (rc == MIXER_OK && (cudaMalloc(&d_sky, sky.size() * sizeof(double)) != cudaSuccess ||
                               cudaMemcpy(d_sky, sky.data(), sky.size() * sizeof(double),
                                          cudaMemcpyHostToDevice) != cudaSuccess))
            rc = MIXER_ECUDA;
        if (rc == MIXER_OK)
            rc = mixer_gen_packets(f.pool, f.stride, 64, f.ty.nant, f.ty.nch, f.ty.tpkt, (int32_t)nheaps,
                                   0, 0, (uint16_t)(4096 + i), d_sky, 16.0, seed + 100 + i, 0, nullptr);
        if (rc == MIXER_OK && cudaDeviceSynchronize() != cudaSuccess) rc = MIXER_ECUDA;
        cudaFree(d_sky);
        if (rc != MIXER_OK) {
            fprintf(stderr, "[mixer_serve] packet source: %s\n", mixer_strerror(rc));
            return 1;
        }
    }
    mixer_server_cfg cfg;
    cfg.budget_bytes = (int64_t)(budget_gb * (double)(1ull << 30));
    cfg.max_streams = kStreams;
    cfg.ring_subs = ring_subs;
    cfg.batch_subs = batch_subs;
    mixer_server* sv = nullptr;
    int rc = mixer_server_create(&cfg, &sv);
    if (rc != MIXER_OK) {
        fprintf(stderr, "[mixer_serve] mixer_server_create: %s\n", mixer_strerror(rc));
        return 1;
    }
    auto desc_of = [&](const Feed& f) {
        mixer_array_desc d;
        mixer_desc_default(&d);
        d.nant = f.ty.nant;
        d.nch = f.ty.nch;
        d.tpkt = f.ty.tpkt;
        d.ksub = f.ty.ksub;
        d.nsub_dump = f.ty.nsub;
        d.side_x = f.ty.side;
        d.grid = 0;
        d.pkt_stride = (int32_t)f.stride;
        d.hdr_bytes = 64;
        d.max_heaps = 1;
        return d;
    };
    if (reserve) {
        for (int t = 0; t < 2; ++t) {         // four streams of each of the two shapes
            const mixer_array_desc d = desc_of(feeds[4 * t]);
            rc = mixer_server_reserve(sv, &d, 4);
            if (rc != MIXER_OK) {
                fprintf(stderr, "[mixer_serve] mixer_server_reserve: %s\n", mixer_strerror(rc));
                return 1;
            }
        }
    }
    const double per_stream = gbps > 0 ? gbps / kStreams * 1e9 / 8 : 0.0;   // bytes / s
    std::atomic<bool> done{false};
    std::atomic<int64_t> polled{0};
    const double t0 = now_s();

    auto feeder = [&](int i) {
        Feed& f = feeds[i];
        const mixer_array_desc d = desc_of(f);
        cudaSetDevice(device);
        sleep_s(t0 + f.start - now_s());
        const double tw = now_s();
        int sid = -1;
        while (now_s() - t0 < f.stop) {
            const int r = mixer_server_open(sv, &d, &sid);
            if (r == MIXER_OK) break;
            sid = -1;
            if (r != MIXER_EBUSY) {
                f.err = r;
                return;
            }
            ++f.refusals;
            sleep_s(0.002);
        }
        f.open_wait = now_s() - tw;
        if (sid < 0) return;
        f.id.store(sid);
        cudaStream_t own;
        cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking);
        const double interval = per_stream > 0 ? (double)f.sub_bytes / per_stream : 0.0;
        double nxt = now_s();
        const double ta = nxt;
        int64_t j = 0;
        bool stop = false;
        while (!stop && now_s() - t0 < f.stop) {
            if (j % kPoolSubs == 0) {        // new lap over the pool: re-stamp the sequence numbers
                int r = mixer_server_sync_copies(sv);      // the previous lap has been copied out
                if (r == MIXER_OK)
                    r = mixer_restamp_seq(f.pool, (int64_t)kPoolSubs * f.hps * f.ty.nant, f.stride,
                                          (uint32_t)(j * f.hps * f.ty.nant), own);
                if (r == MIXER_OK && cudaStreamSynchronize(own) != cudaSuccess) r = MIXER_ECUDA;
                if (r != MIXER_OK) {
                    f.err = r;
                    break;
                }
            }
            if (interval > 0) sleep_s(nxt - now_s());
            const uint8_t* src = f.pool + (j % kPoolSubs) * f.sub_bytes;
            while (true) {
                const int r = mixer_server_submit(sv, sid, src, f.hps, 0, 1);
                if (r == MIXER_OK) break;
                if (r != MIXER_EBUSY) {
                    f.err = r;
                    stop = true;
                    break;
                }
                if (now_s() - t0 >= f.stop) {
                    stop = true;
                    break;
                }
                sleep_s(0.0002);
            }
            if (stop) break;
            f.submitted += f.sub_bytes;
            f.stamps.push_back(now_s() - t0);
            ++j;
            nxt += interval;
        }
        f.active = now_s() - ta;
        sleep_s(0.05);                       // let the last full dump finish
        f.id.store(-1);
        const int r = mixer_server_close(sv, sid);
        if (r != MIXER_OK && f.err == MIXER_OK) f.err = r;
        cudaStreamDestroy(own);
    };
    auto poller = [&]() {
        cudaSetDevice(device);
        while (!done.load()) {
            for (auto& f : feeds) {
                const int sid = f.id.load();
                if (sid < 0) continue;
                mixer_dump_info info;
                if (mixer_server_poll(sv, sid, &info, nullptr) == MIXER_OK && info.available) {
                    polled.fetch_add(1);
                    f.dumps.fetch_add(1);
                }
            }
            sleep_s(0.001);
        }
    };
    std::thread pt(poller);
    std::vector<std::thread> th;
    for (int i = 0; i < kStreams; ++i) th.emplace_back(feeder, i);
    for (auto& t : th) t.join();
    const double wall = now_s() - t0;
    done.store(true);
    pt.join();
    mixer_server_counters st;
    memset(&st, 0, sizeof(st));
    const int src = mixer_server_stats(sv, &st);
    mixer_server_destroy(sv);
    for (auto& f : feeds) cudaFree(f.pool);

    // aggregate over the window in which every stream was submitting
    double w0 = 0, w1 = 1e30, all_bytes = 0, total = 0;
    bool all_ran = true;
    for (auto& f : feeds) {
        total += (double)f.submitted;
        if (f.stamps.empty()) {
            all_ran = false;
            continue;
        }
        w0 = std::max(w0, f.stamps.front());
        w1 = std::min(w1, f.stamps.back());
    }
    for (auto& f : feeds)
        for (double t : f.stamps)
            if (t >= w0 && t < w1) all_bytes += (double)f.sub_bytes;
    double dump_bytes = 0;
    for (auto& f : feeds)
        dump_bytes += (double)f.dumps.load() * f.ty.nch * 2.0 * f.ty.nant * f.ty.nant * sizeof(float);
    int err = src;
    for (auto& f : feeds)
        if (f.err != MIXER_OK && err == MIXER_OK) err = f.err;
    printf("{\"feeders\": \"c++ threads (mixer_serve)\", \"reserved\": %s, \"wall_s\": %.3f, "
           "\"offered_gbps\": %.1f, \"submitted_gbps\": %.2f, \"processed_gbps\": %.2f, ",
           reserve ? "true" : "false", wall, gbps, 8.0 * total / wall / 1e9, 8.0 * (double)st.bytes_processed / wall / 1e9);
    if (all_ran && w1 - w0 > 0.5)
        printf("\"aggregate_while_all_streams_active\": {\"window_s\": %.2f, \"gbps\": %.2f}, ", w1 - w0,
               8.0 * all_bytes / (w1 - w0) / 1e9);
    else
        printf("\"aggregate_while_all_streams_active\": null, ");
    printf("\"dumps\": %lld, \"dumps_polled\": %lld, \"dump_d2h_gbytes_per_s\": %.2f, "
           "\"sub_integrations_per_dump\": %d, \"p50_dump_latency_ms\": %.3f, "
           "\"p99_dump_latency_ms\": %.3f, \"max_dump_latency_ms\": %.3f, ",
           (long long)st.dumps, (long long)polled.load(), dump_bytes / wall / 1e9, feeds[0].ty.nsub,
           1e3 * st.p50_latency_s, 1e3 * st.p99_latency_s, 1e3 * st.max_latency_s);
    printf("\"per_stream_gbps\": [");
    for (int i = 0; i < kStreams; ++i)
        printf("%s%.1f", i ? ", " : "",
               feeds[i].active > 0 ? 8.0 * (double)feeds[i].submitted / feeds[i].active / 1e9 : 0.0);
    printf("], \"open_latency_s\": [");
    for (int i = 0; i < kStreams; ++i) printf("%s%.3f", i ? ", " : "", feeds[i].open_wait);
    printf("], \"admitted\": %lld, \"refused_attempts\": %lld, \"launches\": %lld, "
           "\"work_items\": %lld, \"seq_errors\": %lld, \"kernel_err\": %d, \"status\": \"%s\"}\n",
           (long long)st.admitted, (long long)st.refused, (long long)st.launches,
           (long long)st.work_items, (long long)st.seq_errors, st.kernel_err, mixer_strerror(err));
    return err == MIXER_OK && st.kernel_err == 0 && st.seq_errors == 0 ? 0 : 1;
}
