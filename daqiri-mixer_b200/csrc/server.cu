// server.cu -- streaming X-engine: concurrent array streams, continuous batching.
//
// The reference serves exactly one array from one NIC queue with one GPU
// thread (src/rx_host_corr.cu:143-175).  This server keeps several array
// streams of different sizes resident on one GPU:
//   * admission (mixer_server_open) reserves a stream's device state -- its
//     packet staging ring, corner-turn planes, int64 integration cube and
//     FP32 dump cube -- against a device-memory budget and a slot count, and
//     refuses with MIXER_EBUSY when either is exhausted; closing a stream
//     returns both, so a later open is admitted;
//   * mixer_server_submit copies heaps (host or device packets) into the
//     stream's ring on a copy stream;
//   * one worker thread runs the continuous-batching loop: every iteration it
//     takes the complete sub-integrations of ALL streams that have any, runs
//     their corner-turns, and then a single persistent k_xcorr_tri launch whose
//     work list holds every ready stream's (channel, tile) items, so streams
//     that arrive while others are on the GPU join the next launch;
//   * after nsub_dump sub-integrations a stream's int64 cube is unpacked into
//     its FP32 dump cube, copied to pinned host memory on a separate stream,
//     and zeroed; a host callback stamps the completion time, giving the dump
//     latency from the submission of the dump's last heap.
// Every stream's arithmetic is exactly that of mixer_correlate on the same
// packets, so a stream's dumps are identical alone and in any mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>
#include "xcorr.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double now_s() {
    return std::chrono::duration<double>(Clock::now().time_since_epoch()).count();
}

constexpr int kDumpSlots = 2;

// Pinned host memory in parts of at most kPinPart bytes.  Pinning a dump cube
// (hundreds of MB) in one cudaMallocHost call keeps the driver busy long
// enough to stall the other streams' launches and copies when a stream is
// admitted; part by part, their calls get through in between.
constexpr size_t kPinPart = (size_t)32 << 20;

struct PinnedBuf {
    std::vector<char*> parts;
    size_t bytes = 0;
    bool empty() const { return parts.empty(); }
};

void pinned_free(PinnedBuf& b) {
    for (char* p : b.parts) cudaFreeHost(p);
    b.parts.clear();
    b.bytes = 0;
}

// All parts or none: a failed call leaves b empty.
cudaError_t pinned_alloc(PinnedBuf& b, size_t bytes) {
    b.bytes = bytes;
    for (size_t off = 0; off < bytes; off += kPinPart) {
        void* p = nullptr;
        const cudaError_t e = cudaMallocHost(&p, std::min(kPinPart, bytes - off));
        if (e != cudaSuccess) {
            pinned_free(b);
            return e;
        }
        b.parts.push_back(static_cast<char*>(p));
        std::this_thread::yield();
    }
    return cudaSuccess;
}

// Device -> pinned host copy of `bytes`, one cudaMemcpyAsync per part.
cudaError_t pinned_d2h(PinnedBuf& b, const void* src, size_t bytes, cudaStream_t st) {
    const char* s = static_cast<const char*>(src);
    for (size_t q = 0, off = 0; off < bytes; ++q, off += kPinPart) {
        const cudaError_t e = cudaMemcpyAsync(b.parts[q], s + off, std::min(kPinPart, bytes - off),
                                              cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

void pinned_read(const PinnedBuf& b, void* dst, size_t bytes) {
    char* d = static_cast<char*>(dst);
    for (size_t q = 0, off = 0; off < bytes; ++q, off += kPinPart)
        memcpy(d + off, b.parts[q], std::min(kPinPart, bytes - off));
}

struct DumpSlot {
    PinnedBuf host;                 // pinned FP32 cube
    int state = 0;                  // 0 free, 1 in flight, 2 ready, 3 being read by poll
    int64_t index = 0;
    double t_last_submit = 0.0;
    std::atomic<double> t_done{0.0};
};

struct Stream {
    bool used = false;
    bool closing = false;
    mixer_array_desc d;
    int64_t bytes = 0;
    int64_t hps = 0;                // heaps per sub-integration
    int64_t ring_subs = 0;
    int64_t batch_subs = 0;         // most sub-integrations per launch
    int64_t heap_bytes = 0;
    uint8_t* ring = nullptr;
    int8_t* planes = nullptr;
    int64_t kt = 0;
    int64_t* vis = nullptr;
    float* dump_dev = nullptr;
    uint32_t* d_seq_err = nullptr;
    CUtensorMap map;
    std::vector<cudaEvent_t> ev_ready;   // per ring slot: its heaps are on the device
    std::vector<cudaEvent_t> ev_free;    // per ring slot: its corner-turn is done
    std::vector<double> t_slot_done;     // per ring slot: host time its last heap arrived
    std::vector<bool> slot_free_valid;
    cudaEvent_t ev_dump_copied = nullptr;
    cudaEvent_t ev_dump_kernel = nullptr;
    bool dump_copy_pending = false;
    DumpSlot dump[kDumpSlots];
    int64_t heaps_in = 0;           // heaps submitted
    int64_t subs_done = 0;          // sub-integrations taken by the worker
    int64_t subs_in_dump = 0;
    int64_t dumps_emitted = 0;
    int64_t dumps_dropped = 0;
    int64_t bytes_in = 0;
    int readers = 0;                // mixer_server_poll copies in progress
    uint32_t seq_next = 0;
    bool seq_set = false;
};

}  // namespace

struct mixer_server {
    mixer_server_cfg cfg;
    int dev = 0;
    std::mutex mu;          // stream table, counters
    std::mutex serve_mu;    // held by the worker for a whole iteration
    std::condition_variable cv;
    std::unique_ptr<Stream[]> streams;
    int nstreams = 0;
    int64_t bytes_used = 0;
    int64_t admitted = 0, refused = 0, launches = 0, items = 0;
    std::vector<double> latencies;
    double t_first = 0.0, t_last = 0.0;
    int64_t bytes_processed = 0;
    cudaStream_t copy = nullptr, comp = nullptr, d2h = nullptr;
    // double-buffered launch tables
    CUtensorMap* d_maps[2] = {nullptr, nullptr};
    mixer::XcorrProblem* d_probs[2] = {nullptr, nullptr};
    mixer::XcorrWork* d_work[2] = {nullptr, nullptr};
    int64_t work_cap[2] = {0, 0};
    // pinned host copies of the tables, so the uploads are truly asynchronous
    CUtensorMap* h_maps[2] = {nullptr, nullptr};
    mixer::XcorrProblem* h_probs[2] = {nullptr, nullptr};
    mixer::XcorrWork* h_work[2] = {nullptr, nullptr};
    int64_t h_work_cap[2] = {0, 0};
    cudaEvent_t table_free[2] = {nullptr, nullptr};
    bool table_used[2] = {false, false};
    int tsel = 0;
    int32_t* d_err = nullptr;
    unsigned long long* d_ctr = nullptr;   // item counter of the GEMM launches (stream comp)
    // Stream state comes from a server-owned stream-ordered pool and pinned dump
    // buffers are recycled, so opening or closing a stream never runs the
    // device-wide synchronisation of cudaMalloc / cudaFree / cudaFreeHost while
    // other streams are being served.
    cudaMemPool_t pool = nullptr;
    cudaStream_t alloc = nullptr;
    std::multimap<size_t, PinnedBuf> pinned_cache;   // guarded by mu
    // Superseded pinned work tables, freed with the server: cudaFreeHost would
    // synchronise the device in the middle of serving.
    std::vector<mixer::XcorrWork*> retired_work;
    std::thread worker;
    std::atomic<bool> stop{false};
    std::atomic<int> error{0};
};

namespace {

struct DoneCtx {
    DumpSlot* slot;
};

void CUDART_CB mark_done(void* p) {
    DoneCtx* c = static_cast<DoneCtx*>(p);
    c->slot->t_done.store(now_s());
    delete c;
}

int64_t stream_bytes(const mixer_array_desc& d, int64_t ring_subs, int64_t batch_subs) {
    const int64_t hps = d.ksub / d.tpkt;
    const int64_t ring = ring_subs * hps * d.nant * (int64_t)d.pkt_stride;
    const int64_t planes = 2LL * d.nch * d.nant * batch_subs * d.ksub;
    const int64_t vis = mixer_vis_elems(d.nant, d.nch) * 8;
    const int64_t dump = (int64_t)d.nch * 2 * d.nant * d.nant * 4;
    return ring + planes + vis + dump + 4096;
}

// Caller holds sv->mu; the stream's GPU work has finished.
void free_stream(mixer_server* sv, Stream& s) {
    for (void* p : {(void*)s.ring, (void*)s.planes, (void*)s.vis, (void*)s.dump_dev,
                    (void*)s.d_seq_err})
        if (p) cudaFreeAsync(p, sv->alloc);
    for (auto e : s.ev_ready) cudaEventDestroy(e);
    for (auto e : s.ev_free) cudaEventDestroy(e);
    if (s.ev_dump_copied) cudaEventDestroy(s.ev_dump_copied);
    if (s.ev_dump_kernel) cudaEventDestroy(s.ev_dump_kernel);
    const size_t dump_bytes = (size_t)s.d.nch * 2 * s.d.nant * s.d.nant * sizeof(float);
    for (auto& d : s.dump)
        if (!d.host.empty()) sv->pinned_cache.emplace(dump_bytes, std::move(d.host));
    s.ring = nullptr;
    s.planes = nullptr;
    s.vis = nullptr;
    s.dump_dev = nullptr;
    s.d_seq_err = nullptr;
    s.ev_ready.clear();
    s.ev_free.clear();
    s.ev_dump_copied = nullptr;
    s.ev_dump_kernel = nullptr;
    for (auto& d : s.dump) {
        d.host = PinnedBuf();
        d.state = 0;
    }
    s.used = false;
    s.closing = false;
    s.readers = 0;
}

// One iteration of the continuous-batching loop.  Returns true if it did work.
bool serve_once(mixer_server* sv) {
    struct Ready {
        int sid;
        int64_t sub0, nsub;
    };
    std::vector<Ready> ready;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        for (int sid = 0; sid < sv->nstreams; ++sid) {
            Stream& s = sv->streams[sid];
            if (!s.used || s.closing) continue;
            const int64_t full = s.heaps_in / s.hps;
            int64_t n = full - s.subs_done;
            if (n <= 0) continue;
            n = std::min<int64_t>(n, s.batch_subs);
            n = std::min<int64_t>(n, s.d.nsub_dump - s.subs_in_dump);   // stop at the dump edge
            // a dump slot must be free before the edge is crossed
            if (s.subs_in_dump + n == s.d.nsub_dump) {
                bool free_slot = false;
                for (auto& d : s.dump) free_slot |= (d.state == 0);
                if (!free_slot) continue;
            }
            ready.push_back({sid, s.subs_done, n});
        }
    }
    if (ready.empty()) return false;
    cudaStream_t comp = sv->comp;
    std::vector<CUtensorMap> maps;
    std::vector<mixer::XcorrProblem> probs;
    std::vector<mixer::XcorrWork> work;
    bool ragged = false;
    for (size_t r = 0; r < ready.size(); ++r) {
        Stream& s = sv->streams[ready[r].sid];
        if (s.d.nant % 128) ragged = true;
        // corner-turn the ready sub-integrations, one launch per contiguous run of ring slots
        for (int64_t q = 0; q < ready[r].nsub;) {
            const int64_t sub = ready[r].sub0 + q;
            const int64_t slot = sub % s.ring_subs;
            const int64_t run = std::min<int64_t>(ready[r].nsub - q, s.ring_subs - slot);
            cudaStreamWaitEvent(comp, s.ev_ready[slot + run - 1], 0);   // copies complete in order
            const uint8_t* src = s.ring + slot * s.hps * s.heap_bytes;
            const uint32_t seq = s.seq_next + (uint32_t)(sub * s.hps * s.d.nant);
            const int crc = mixer_corner_turn(src, s.d.pkt_stride, s.d.hdr_bytes, s.d.nant,
                                              s.d.nch, s.d.tpkt, (int32_t)(run * s.hps), seq,
                                              s.planes, s.kt, q * s.d.ksub, s.d_seq_err, sv->d_err,
                                              comp);
            if (crc != MIXER_OK) sv->error.store(crc);
            for (int64_t u = 0; u < run; ++u) cudaEventRecord(s.ev_free[slot + u], comp);
            q += run;
        }
        const int nb = (s.d.nant + 127) / 128;
        const int ntiles = nb * (nb + 1) / 2;
        const int64_t klen = ready[r].nsub * s.d.ksub;
        const uint32_t nkc = (uint32_t)((klen + 127) / 128);
        CUtensorMap m[2];
        const int mrc = mixer::xcorr_encode_maps(m, s.planes, s.d.nant, s.d.nch, s.kt, klen);
        if (mrc != MIXER_OK) sv->error.store(mrc);
        maps.push_back(m[0]);
        maps.push_back(m[1]);
        // one item per (channel, tile) over all ready sub-integrations, and every
        // stream has a cube of its own: the items own their tiles
        probs.push_back(mixer::XcorrProblem{s.d.nant, s.d.nch, ntiles, 0, MIXER_VIS_ACC_I64, 1, s.vis});
        for (int32_t c = 0; c < s.d.nch; ++c)
            for (int t = 0; t < ntiles; ++t) {
                mixer::XcorrWork it;
                it.prob = (uint16_t)r;
                it.tile = (uint16_t)t;
                it.chan = (uint32_t)c;
                it.kc0 = 0;
                it.nkc = nkc;
                work.push_back(it);
            }
    }
    std::stable_sort(work.begin(), work.end(),
                     [](const mixer::XcorrWork& a, const mixer::XcorrWork& b) { return a.nkc > b.nkc; });
    // tables: reuse set tsel once its previous launch finished
    const int ts = sv->tsel;
    sv->tsel ^= 1;
    if (sv->table_used[ts]) cudaEventSynchronize(sv->table_free[ts]);
    const size_t np = probs.size();
    if ((int64_t)work.size() > sv->work_cap[ts]) {
        // grow without synchronising the device: the device table comes from the
        // server's stream-ordered pool (the old one is released in stream order
        // after its last launch), the old pinned table is kept until destroy
        if (sv->d_work[ts]) cudaFreeAsync(sv->d_work[ts], comp);
        if (sv->h_work[ts]) sv->retired_work.push_back(sv->h_work[ts]);
        sv->d_work[ts] = nullptr;
        sv->h_work[ts] = nullptr;
        sv->work_cap[ts] = 0;
        const size_t cap = work.size() + work.size() / 2;
        cudaError_t e = cudaMallocFromPoolAsync((void**)&sv->d_work[ts], cap * sizeof(mixer::XcorrWork),
                                                sv->pool, comp);
        if (e == cudaSuccess) e = cudaMallocHost(&sv->h_work[ts], cap * sizeof(mixer::XcorrWork));
        if (e != cudaSuccess) {
            sv->error.store(mixer::cuda_status(e, "server work list"));
            return false;
        }
        sv->work_cap[ts] = (int64_t)cap;
    }
    if (sv->error.load()) return false;
    memcpy(sv->h_maps[ts], maps.data(), maps.size() * sizeof(CUtensorMap));
    memcpy(sv->h_probs[ts], probs.data(), np * sizeof(mixer::XcorrProblem));
    memcpy(sv->h_work[ts], work.data(), work.size() * sizeof(mixer::XcorrWork));
    cudaMemcpyAsync(sv->d_maps[ts], sv->h_maps[ts], maps.size() * sizeof(CUtensorMap),
                    cudaMemcpyHostToDevice, comp);
    cudaMemcpyAsync(sv->d_probs[ts], sv->h_probs[ts], np * sizeof(mixer::XcorrProblem),
                    cudaMemcpyHostToDevice, comp);
    cudaMemcpyAsync(sv->d_work[ts], sv->h_work[ts], work.size() * sizeof(mixer::XcorrWork),
                    cudaMemcpyHostToDevice, comp);
    const int rc = mixer::xcorr_launch_table(sv->d_maps[ts], sv->d_probs[ts], sv->d_work[ts],
                                             (int64_t)work.size(), mixer::xcorr_sm_count(), sv->d_err,
                                             sv->d_ctr, ragged, comp);
    if (rc != MIXER_OK) sv->error.store(rc);
    cudaEventRecord(sv->table_free[ts], comp);
    sv->table_used[ts] = true;
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->launches += 1;
    sv->items += (int64_t)work.size();
    for (const Ready& r : ready) {
        Stream& s = sv->streams[r.sid];
        s.subs_done += r.nsub;
        s.subs_in_dump += r.nsub;
        sv->bytes_processed += r.nsub * s.hps * s.heap_bytes;
        if (s.subs_in_dump < s.d.nsub_dump) continue;
        // dump edge: FP32 cube, D2H, zero the cube
        int slot = -1;
        for (int q = 0; q < kDumpSlots; ++q)
            if (s.dump[q].state == 0) {
                slot = q;
                break;
            }
        if (slot < 0) {                     // cannot happen: checked before the launch
            sv->error.store(MIXER_EINVAL);
            continue;
        }
        DumpSlot& ds = s.dump[slot];
        s.subs_in_dump = 0;
        // Every call of the dump edge is checked: on a failure the error is
        // latched in sv->error (every later call reports it) and the slot stays
        // free, so no poll can hand out a stale or partial cube.
        const size_t nbytes = (size_t)s.d.nch * 2 * s.d.nant * s.d.nant * sizeof(float);
        cudaError_t e = cudaSuccess;
        if (s.dump_copy_pending) e = cudaStreamWaitEvent(comp, s.ev_dump_copied, 0);
        int drc = e == cudaSuccess ? mixer_vis_dump_f32(s.vis, s.d.nant, s.d.nch, s.dump_dev, comp)
                                   : mixer::cuda_status(e, "dump edge: wait for the previous copy");
        if (drc == MIXER_OK &&
            ((e = cudaMemsetAsync(s.vis, 0, (size_t)mixer_vis_elems(s.d.nant, s.d.nch) * 8, comp)) !=
                 cudaSuccess ||
             (e = cudaEventRecord(s.ev_dump_kernel, comp)) != cudaSuccess ||
             (e = cudaStreamWaitEvent(sv->d2h, s.ev_dump_kernel, 0)) != cudaSuccess ||
             (e = pinned_d2h(ds.host, s.dump_dev, nbytes, sv->d2h)) != cudaSuccess ||
             (e = cudaEventRecord(s.ev_dump_copied, sv->d2h)) != cudaSuccess))
            drc = mixer::cuda_status(e, "dump edge");
        if (drc != MIXER_OK) {
            sv->error.store(drc);
            continue;
        }
        s.dump_copy_pending = true;
        ds.t_done.store(0.0);
        DoneCtx* done = new DoneCtx{&ds};
        if ((e = cudaLaunchHostFunc(sv->d2h, mark_done, done)) != cudaSuccess) {
            delete done;
            sv->error.store(mixer::cuda_status(e, "dump edge: completion callback"));
            continue;
        }
        // sv->mu is held here and by collect_done, so the callback's time stamp
        // is read only once the slot is marked in flight.
        ds.state = 1;
        ds.index = s.dumps_emitted++;
        ds.t_last_submit = s.t_slot_done[(s.subs_done - 1) % s.ring_subs];
    }
    return true;
}

void collect_done(mixer_server* sv) {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (int q = 0; q < sv->nstreams; ++q) {
        Stream& s = sv->streams[q];
        if (!s.used) continue;
        for (auto& d : s.dump) {
            if (d.state == 1) {
                const double t = d.t_done.load();
                if (t > 0.0) {
                    d.state = 2;
                    sv->latencies.push_back(t - d.t_last_submit);
                    sv->t_last = std::max(sv->t_last, t);
                }
            }
        }
    }
}

void worker_main(mixer_server* sv) {
    cudaSetDevice(sv->dev);
    while (!sv->stop.load()) {
        bool did;
        {
            std::lock_guard<std::mutex> it(sv->serve_mu);
            did = serve_once(sv);
        }
        collect_done(sv);
        if (!did) {
            std::unique_lock<std::mutex> lk(sv->mu);
            sv->cv.wait_for(lk, std::chrono::microseconds(200));
        }
    }
}

}  // namespace

extern "C" int64_t mixer_server_stream_bytes(const mixer_server_cfg* cfg, const mixer_array_desc* d) {
    if (!cfg || !d || d->tpkt <= 0 || d->ksub <= 0) return -1;
    const int64_t batch_subs = std::max<int64_t>(
        1, std::min<int64_t>(cfg->batch_subs > 0 ? cfg->batch_subs : 4, MIXER_KMAX_I32 / d->ksub));
    const int64_t ring_subs = std::max<int64_t>(cfg->ring_subs > 0 ? cfg->ring_subs : 8, 2);
    return stream_bytes(*d, ring_subs, batch_subs);
}

extern "C" int mixer_server_reserve(mixer_server* sv, const mixer_array_desc* d, int32_t count) {
    if (!sv || !d || count < 0 || count > sv->nstreams) return MIXER_EINVAL;
    if (d->nant <= 0 || d->nch <= 0 || d->nant > 65536 || d->nch > 65535) return MIXER_EINVAL;
    const size_t dump_bytes = (size_t)d->nch * 2 * d->nant * d->nant * sizeof(float);
    // device: take the streams' state from the pool once, so the pool holds it
    const int64_t per = mixer_server_stream_bytes(&sv->cfg, d);
    if (per <= 0) return MIXER_EINVAL;
    std::vector<void*> blocks;
    cudaError_t e = cudaSuccess;
    for (int32_t i = 0; i < count && e == cudaSuccess; ++i) {
        void* p = nullptr;
        e = cudaMallocFromPoolAsync(&p, (size_t)per, sv->pool, sv->alloc);
        if (e == cudaSuccess) blocks.push_back(p);
    }
    for (void* p : blocks) cudaFreeAsync(p, sv->alloc);
    const cudaError_t es = cudaStreamSynchronize(sv->alloc);
    if (e != cudaSuccess) return mixer::cuda_status(e, "mixer_server_reserve (device)");
    if (es != cudaSuccess) return mixer::cuda_status(es, "mixer_server_reserve (device)");
    // host: pinned dump buffers into the cache the admissions draw from
    for (int32_t i = 0; i < count * kDumpSlots; ++i) {
        PinnedBuf b;
        if ((e = pinned_alloc(b, dump_bytes)) != cudaSuccess)
            return mixer::cuda_status(e, "mixer_server_reserve (pinned)");
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->pinned_cache.emplace(dump_bytes, std::move(b));
    }
    return MIXER_OK;
}

extern "C" int mixer_server_create(const mixer_server_cfg* cfg, mixer_server** out) {
    if (!cfg || !out || cfg->budget_bytes <= 0 || cfg->max_streams <= 0 || cfg->max_streams > 4096)
        return MIXER_EINVAL;
    *out = nullptr;
    mixer_server* sv = new mixer_server();
    sv->cfg = *cfg;
    if (sv->cfg.ring_subs <= 0) sv->cfg.ring_subs = 8;
    if (sv->cfg.batch_subs <= 0) sv->cfg.batch_subs = 4;
    sv->streams.reset(new Stream[cfg->max_streams]);
    sv->nstreams = cfg->max_streams;
    cudaError_t e;
    auto fail = [&](cudaError_t err, const char* what) {
        const int r = mixer::cuda_status(err, what);
        mixer_server_destroy(sv);
        return r;
    };
    if ((e = cudaGetDevice(&sv->dev)) != cudaSuccess) return fail(e, "cudaGetDevice");
    if ((e = cudaStreamCreateWithFlags(&sv->copy, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&sv->comp, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&sv->d2h, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&sv->alloc, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(e, "server streams");
    {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = sv->dev;
        if ((e = cudaMemPoolCreate(&sv->pool, &props)) != cudaSuccess) return fail(e, "server pool");
        uint64_t keep = UINT64_MAX;   // freed stream memory stays in the pool for the next open
        if ((e = cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep)) !=
            cudaSuccess)
            return fail(e, "server pool");
        // Back the whole budget with device memory now, when it fits easily
        // (at most half of the free memory): the first admissions then take it
        // from the pool instead of mapping new memory while other streams run.
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && cfg->budget_bytes > 0 &&
            (size_t)cfg->budget_bytes <= free_b / 2) {
            void* p = nullptr;
            if (cudaMallocFromPoolAsync(&p, (size_t)cfg->budget_bytes, sv->pool, sv->alloc) ==
                cudaSuccess)
                cudaFreeAsync(p, sv->alloc);
            cudaGetLastError();        // a refused reservation only leaves the pool empty
            if ((e = cudaStreamSynchronize(sv->alloc)) != cudaSuccess) return fail(e, "server pool");
        }
    }
    for (int t = 0; t < 2; ++t) {
        // two tensor maps per stream (xcorr_encode_maps)
        if ((e = cudaMalloc(&sv->d_maps[t], 2 * cfg->max_streams * sizeof(CUtensorMap))) != cudaSuccess ||
            (e = cudaMalloc(&sv->d_probs[t], cfg->max_streams * sizeof(mixer::XcorrProblem))) != cudaSuccess ||
            (e = cudaMallocHost(&sv->h_maps[t], 2 * cfg->max_streams * sizeof(CUtensorMap))) != cudaSuccess ||
            (e = cudaMallocHost(&sv->h_probs[t], cfg->max_streams * sizeof(mixer::XcorrProblem))) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sv->table_free[t], cudaEventDisableTiming)) != cudaSuccess)
            return fail(e, "server tables");
    }
    if ((e = cudaMalloc(&sv->d_err, sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMemset(sv->d_err, 0, sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMalloc(&sv->d_ctr, sizeof(unsigned long long))) != cudaSuccess)
        return fail(e, "server error word");
    sv->worker = std::thread(worker_main, sv);
    *out = sv;
    return MIXER_OK;
}

extern "C" int mixer_server_destroy(mixer_server* sv) {
    if (!sv) return MIXER_OK;
    sv->stop.store(true);
    sv->cv.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    if (sv->comp) cudaStreamSynchronize(sv->comp);
    if (sv->d2h) cudaStreamSynchronize(sv->d2h);
    if (sv->copy) cudaStreamSynchronize(sv->copy);
    for (int q = 0; q < sv->nstreams; ++q)
        if (sv->streams[q].used) free_stream(sv, sv->streams[q]);
    for (int t = 0; t < 2; ++t)
        if (sv->d_work[t] && sv->alloc) cudaFreeAsync(sv->d_work[t], sv->alloc);
    if (sv->alloc) cudaStreamSynchronize(sv->alloc);
    if (sv->pool) cudaMemPoolDestroy(sv->pool);
    for (auto& kv : sv->pinned_cache) pinned_free(kv.second);
    sv->pinned_cache.clear();
    for (auto* p : sv->retired_work) cudaFreeHost(p);
    sv->retired_work.clear();
    for (int t = 0; t < 2; ++t) {
        cudaFree(sv->d_maps[t]);
        cudaFree(sv->d_probs[t]);
        cudaFreeHost(sv->h_maps[t]);
        cudaFreeHost(sv->h_probs[t]);
        cudaFreeHost(sv->h_work[t]);
        if (sv->table_free[t]) cudaEventDestroy(sv->table_free[t]);
    }
    cudaFree(sv->d_err);
    cudaFree(sv->d_ctr);
    if (sv->copy) cudaStreamDestroy(sv->copy);
    if (sv->comp) cudaStreamDestroy(sv->comp);
    if (sv->d2h) cudaStreamDestroy(sv->d2h);
    if (sv->alloc) cudaStreamDestroy(sv->alloc);
    delete sv;
    return MIXER_OK;
}

extern "C" int mixer_server_open(mixer_server* sv, const mixer_array_desc* d, int32_t* id) {
    if (!sv || !d || !id) return MIXER_EINVAL;
    if (d->nant <= 0 || d->nch <= 0 || d->tpkt <= 0 || d->tpkt % 16 || d->ksub <= 0 ||
        d->ksub % d->tpkt || d->ksub % 128 || d->nsub_dump <= 0 || d->pkt_stride % 16 ||
        d->hdr_bytes % 16 || d->hdr_bytes < 64 ||
        (int64_t)d->hdr_bytes + 2LL * d->nch * d->tpkt > d->pkt_stride)
        return MIXER_EINVAL;
    // Work items carry the tile index in 16 bits (at most 65535 lower-triangle
    // tiles: nant <= 46208), and the channel limit of mixer_create holds here too.
    const int64_t nblk = (d->nant + 127) / 128;
    if (d->nant > 65536 || d->nch > 65535 || nblk * (nblk + 1) / 2 > 65535) return MIXER_EINVAL;
    const int64_t batch_subs = std::max<int64_t>(
        1, std::min<int64_t>(sv->cfg.batch_subs, MIXER_KMAX_I32 / d->ksub));
    const int64_t ring_subs = std::max<int64_t>(sv->cfg.ring_subs, 2);
    const int64_t need = stream_bytes(*d, ring_subs, batch_subs);
    int sid = -1;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        for (int q = 0; q < sv->nstreams; ++q)
            if (!sv->streams[q].used) {
                sid = q;
                break;
            }
        if (sid < 0 || sv->bytes_used + need > sv->cfg.budget_bytes) {
            sv->refused += 1;
            return MIXER_EBUSY;
        }
        sv->bytes_used += need;      // reserve before allocating
        sv->streams[sid].used = true;
        sv->streams[sid].closing = true;   // invisible to the worker until set up
    }
    Stream& s = sv->streams[sid];
    s.d = *d;
    s.bytes = need;
    s.hps = d->ksub / d->tpkt;
    s.ring_subs = ring_subs;
    s.batch_subs = batch_subs;
    s.heap_bytes = (int64_t)d->nant * d->pkt_stride;
    s.kt = batch_subs * d->ksub;
    s.heaps_in = s.subs_done = s.subs_in_dump = s.dumps_emitted = s.dumps_dropped = s.bytes_in = 0;
    s.seq_set = false;
    s.dump_copy_pending = false;
    cudaError_t e = cudaSuccess;
    const size_t dump_bytes = (size_t)d->nch * 2 * d->nant * d->nant * sizeof(float);
    auto palloc = [&](void** p, size_t n) {
        return cudaMallocFromPoolAsync(p, n, sv->pool, sv->alloc);
    };
    const size_t vis_bytes = (size_t)mixer_vis_elems(d->nant, d->nch) * 8;
    if ((e = palloc((void**)&s.ring, ring_subs * s.hps * s.heap_bytes)) == cudaSuccess &&
        (e = palloc((void**)&s.planes, 2 * (size_t)d->nch * d->nant * s.kt)) == cudaSuccess &&
        (e = palloc((void**)&s.vis, vis_bytes)) == cudaSuccess &&
        (e = cudaMemsetAsync(s.vis, 0, vis_bytes, sv->alloc)) == cudaSuccess &&
        (e = palloc((void**)&s.dump_dev, dump_bytes)) == cudaSuccess &&
        (e = palloc((void**)&s.d_seq_err, sizeof(uint32_t))) == cudaSuccess &&
        (e = cudaMemsetAsync(s.d_seq_err, 0, sizeof(uint32_t), sv->alloc)) == cudaSuccess &&
        (e = cudaStreamSynchronize(sv->alloc)) == cudaSuccess &&   // usable on every stream
        (e = cudaEventCreateWithFlags(&s.ev_dump_copied, cudaEventDisableTiming)) == cudaSuccess &&
        (e = cudaEventCreateWithFlags(&s.ev_dump_kernel, cudaEventDisableTiming)) == cudaSuccess) {
        for (int q = 0; q < kDumpSlots && e == cudaSuccess; ++q) {
            {
                std::lock_guard<std::mutex> lk(sv->mu);
                auto it = sv->pinned_cache.find(dump_bytes);
                if (it != sv->pinned_cache.end()) {
                    s.dump[q].host = std::move(it->second);
                    sv->pinned_cache.erase(it);
                }
            }
            if (s.dump[q].host.empty()) e = pinned_alloc(s.dump[q].host, dump_bytes);
        }
        s.ev_ready.assign(ring_subs, nullptr);
        s.ev_free.assign(ring_subs, nullptr);
        s.t_slot_done.assign(ring_subs, 0.0);
        s.slot_free_valid.assign(ring_subs, false);
        for (int64_t q = 0; q < ring_subs && e == cudaSuccess; ++q) {
            e = cudaEventCreateWithFlags(&s.ev_ready[q], cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.ev_free[q], cudaEventDisableTiming);
        }
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    if (e != cudaSuccess) {
        free_stream(sv, s);
        sv->bytes_used -= need;
        return mixer::cuda_status(e, "mixer_server_open");
    }
    s.closing = false;
    sv->admitted += 1;
    *id = sid;
    return MIXER_OK;
}

extern "C" int mixer_server_submit(mixer_server* sv, int32_t id, const void* packets, int64_t nheaps,
                                   uint32_t seq0, int32_t on_device) {
    if (!sv || !packets || nheaps <= 0 || id < 0 || id >= (int32_t)sv->nstreams) return MIXER_EINVAL;
    if (sv->error.load()) return sv->error.load();
    int64_t h0, ring_heaps, hps;
    Stream* sp;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        Stream& s = sv->streams[id];
        if (!s.used || s.closing) return MIXER_EINVAL;
        ring_heaps = s.ring_subs * s.hps;
        hps = s.hps;
        // heaps the worker has not taken yet occupy the ring
        if (s.heaps_in + nheaps - s.subs_done * s.hps > ring_heaps) return MIXER_EBUSY;
        if (!s.seq_set) {
            s.seq_next = seq0;
            s.seq_set = true;
        }
        h0 = s.heaps_in;
        sp = &s;
    }
    Stream& s = *sp;
    std::vector<int64_t> completed;     // ring slots this call completed
    const uint8_t* src = static_cast<const uint8_t*>(packets);
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    int64_t done = 0;
    while (done < nheaps) {
        const int64_t h = h0 + done;
        const int64_t pos = h % ring_heaps;
        const int64_t slot = pos / hps;
        // the slot may still be read by an earlier corner-turn
        if (pos % hps == 0 && s.slot_free_valid[slot]) cudaStreamWaitEvent(sv->copy, s.ev_free[slot], 0);
        const int64_t n = std::min<int64_t>(nheaps - done, hps - pos % hps);
        MIXER_CK(cudaMemcpyAsync(s.ring + pos * s.heap_bytes, src + done * s.heap_bytes,
                                 (size_t)(n * s.heap_bytes), kind, sv->copy));
        done += n;
        if ((h0 + done) % hps == 0) {   // slot complete
            MIXER_CK(cudaEventRecord(s.ev_ready[slot], sv->copy));
            s.slot_free_valid[slot] = true;
            completed.push_back(slot);
        }
    }
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        const double t = now_s();
        if (sv->t_first == 0.0) sv->t_first = t;
        for (int64_t slot : completed) s.t_slot_done[slot] = t;
        s.heaps_in += nheaps;
        s.bytes_in += nheaps * s.heap_bytes;
    }
    sv->cv.notify_one();
    return MIXER_OK;
}

extern "C" int mixer_server_poll(mixer_server* sv, int32_t id, mixer_dump_info* info, float* out) {
    if (!sv || !info || id < 0 || id >= (int32_t)sv->nstreams) return MIXER_EINVAL;
    collect_done(sv);
    DumpSlot* best = nullptr;
    size_t nbytes = 0;
    Stream* sp;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        Stream& s = sv->streams[id];
        memset(info, 0, sizeof(*info));
        if (!s.used) return MIXER_EINVAL;
        for (auto& d : s.dump)
            if (d.state == 2 && (!best || d.index < best->index)) best = &d;
        if (!best) return MIXER_OK;
        info->available = 1;
        info->index = best->index;
        info->latency_s = best->t_done.load() - best->t_last_submit;
        info->nch = s.d.nch;
        info->nant = s.d.nant;
        nbytes = (size_t)s.d.nch * 2 * s.d.nant * s.d.nant * sizeof(float);
        best->state = 3;                 // close waits for the copy below
        s.readers += 1;
        sp = &s;
    }
    // the copy (hundreds of MB for a large array) runs without the server lock,
    // so the worker and the submitters are not held up by it
    if (out) pinned_read(best->host, out, nbytes);
    std::lock_guard<std::mutex> lk(sv->mu);
    best->state = 0;
    sp->readers -= 1;
    return MIXER_OK;
}

extern "C" int mixer_server_close(mixer_server* sv, int32_t id) {
    if (!sv || id < 0 || id >= (int32_t)sv->nstreams) return MIXER_EINVAL;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        Stream& s = sv->streams[id];
        if (!s.used || s.closing) return MIXER_EINVAL;
        s.closing = true;   // the worker stops scheduling it
    }
    // the worker's current iteration may still enqueue work for this stream:
    // wait for it to end (later iterations skip a closing stream), then drain
    { std::lock_guard<std::mutex> it(sv->serve_mu); }
    cudaStreamSynchronize(sv->copy);
    cudaStreamSynchronize(sv->comp);
    cudaStreamSynchronize(sv->d2h);
    collect_done(sv);
    while (true) {                       // a poll may still be copying a dump out
        {
            std::lock_guard<std::mutex> lk(sv->mu);
            Stream& s = sv->streams[id];
            if (s.readers == 0) {
                sv->bytes_used -= s.bytes;
                free_stream(sv, s);
                return MIXER_OK;
            }
        }
        std::this_thread::sleep_for(std::chrono::microseconds(100));
    }
}

extern "C" int mixer_server_stats(mixer_server* sv, mixer_server_counters* st) {
    if (!sv || !st) return MIXER_EINVAL;
    collect_done(sv);
    std::lock_guard<std::mutex> lk(sv->mu);
    memset(st, 0, sizeof(*st));
    st->admitted = sv->admitted;
    st->refused = sv->refused;
    st->launches = sv->launches;
    st->work_items = sv->items;
    st->bytes_used = sv->bytes_used;
    st->bytes_processed = sv->bytes_processed;
    st->dumps = (int64_t)sv->latencies.size();
    if (!sv->latencies.empty()) {
        std::vector<double> l = sv->latencies;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) {
            const size_t i = (size_t)std::min<double>((double)l.size() - 1, p * (double)(l.size() - 1) + 0.5);
            return l[i];
        };
        st->p50_latency_s = pct(0.50);
        st->p99_latency_s = pct(0.99);
        st->max_latency_s = l.back();
    }
    st->elapsed_s = (sv->t_first > 0.0) ? now_s() - sv->t_first : 0.0;
    int32_t ke = 0;
    cudaMemcpy(&ke, sv->d_err, sizeof(ke), cudaMemcpyDeviceToHost);
    st->kernel_err = ke;
    int64_t se = 0;
    for (int q = 0; q < sv->nstreams; ++q) {
        Stream& s = sv->streams[q];
        if (s.used && s.d_seq_err) {
            uint32_t v = 0;
            cudaMemcpy(&v, s.d_seq_err, sizeof(v), cudaMemcpyDeviceToHost);
            se += v;
        }
    }
    st->seq_errors = se;
    return sv->error.load() ? sv->error.load() : (ke ? MIXER_ETIMEOUT : MIXER_OK);
}

extern "C" int mixer_server_sync_copies(mixer_server* sv) {
    if (!sv) return MIXER_EINVAL;
    MIXER_CK(cudaStreamSynchronize(sv->copy));
    return MIXER_OK;
}
