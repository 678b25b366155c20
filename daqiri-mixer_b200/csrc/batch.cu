// batch.cu -- many uneven arrays in one persistent tensor-core launch.
//
// A batch is a list of independent arrays (element count, channel count and
// sample range each their own).  The planner turns it into one device work
// list of (array, channel, lower-triangle tile, K-chunk range) items that the
// persistent k_xcorr_tri walks in table mode, so small arrays no longer leave
// most of the 148 SMs idle and the tail of one array overlaps the next.
//
// Tile shape: 128 x 128 antennas per item, with a K extent that the plan
// chooses per size class (the class is the number of 128-row blocks of the
// array).  Splitting an array's K range into s items multiplies its work
// items by s (better balance over the persistent grid) at the cost of s
// int64 read-modify-write epilogues per tile; integer sums are exact in any
// order, so every split gives bit-identical visibilities.
// Triangle schedule: items ordered longest-first (the static round-robin over
// CTAs then approximates longest-processing-time scheduling) or in natural
// array / channel / tile order (L2 locality of a channel's operands).
// The autotuner times candidate plans on the caller's own buffers, each in an
// A-B-B-A pairing with the incumbent, and keeps a change only for a clear gain;
// the chosen launch can be captured once into a CUDA graph and replayed.  This has no counterpart in the reference, which launches one
// fixed-shape kernel per V-update (src/rx_host_corr.cu:167).
#include <algorithm>
#include <cstring>
#include <vector>
#include "xcorr.cuh"

namespace {

constexpr int kMaxClass = 64;
constexpr int kChunk = 128;

int nblk_of(int nant) { return (nant + 127) / 128; }

}  // namespace

struct mixer_batch {
    int dev;
    std::vector<mixer_xcorr_problem> probs;
    std::vector<mixer::XcorrProblem> tprobs;
    std::vector<char> shared_cube;     // per problem: its cube overlaps another problem's
    CUtensorMap* d_maps;
    mixer::XcorrProblem* d_probs;
    mixer::XcorrWork* d_work;
    int64_t work_cap;
    int64_t nwork;
    int32_t split[kMaxClass + 1];
    int32_t order;
    int32_t grid;
    int32_t* d_err;
    unsigned long long* d_ctr;   // item counter of the launch
    bool ragged;                 // some array's N is not a multiple of 128
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

static int build_work(mixer_batch* b, std::vector<mixer::XcorrWork>& w) {
    w.clear();
    for (size_t p = 0; p < b->probs.size(); ++p) {
        const mixer_xcorr_problem& pr = b->probs[p];
        const int nb = nblk_of(pr.nant);
        const int ntiles = nb * (nb + 1) / 2;
        const int64_t nkc = (pr.klen + kChunk - 1) / kChunk;
        // an item may hold at most MIXER_KMAX_I32 samples in its int32 TMEM accumulators
        const int64_t smin = (nkc + (MIXER_KMAX_I32 / kChunk) - 1) / (MIXER_KMAX_I32 / kChunk);
        int64_t s = b->split[nb <= kMaxClass ? nb : kMaxClass];
        if (pr.mode == MIXER_VIS_STORE_I32) s = 1;   // stores would race across items
        s = std::max<int64_t>(std::min<int64_t>(s, nkc), smin);
        const int64_t cs = (nkc + s - 1) / s;
        // one item per (channel, tile) on a cube of its own: the epilogue may
        // read-add-write instead of adding atomically
        b->tprobs[p].excl = ((nkc + cs - 1) / cs == 1 && !b->shared_cube[p]) ? 1 : 0;
        for (int32_t c = 0; c < pr.nch; ++c)
            for (int t = 0; t < ntiles; ++t)
                for (int64_t k0 = 0; k0 < nkc; k0 += cs) {
                    mixer::XcorrWork it;
                    it.prob = (uint16_t)p;
                    it.tile = (uint16_t)t;
                    it.chan = (uint32_t)c;
                    it.kc0 = (uint32_t)k0;
                    it.nkc = (uint32_t)std::min<int64_t>(cs, nkc - k0);
                    w.push_back(it);
                }
    }
    // Longest first by K extent; the stable sort keeps each channel's tiles
    // (ragged-block tiles included) next to each other, so the CTAs that
    // share a channel's row blocks run together and read them from L2.
    if (b->order == MIXER_ORDER_LPT)
        std::stable_sort(w.begin(), w.end(), [](const mixer::XcorrWork& a, const mixer::XcorrWork& c) {
            return a.nkc > c.nkc;
        });

    return MIXER_OK;
}

static int upload_plan(mixer_batch* b) {
    std::vector<mixer::XcorrWork> w;
    int rc = build_work(b, w);
    if (rc != MIXER_OK) return rc;
    if ((int64_t)w.size() > b->work_cap) {
        cudaFree(b->d_work);
        b->d_work = nullptr;
        MIXER_CK(cudaMalloc(&b->d_work, w.size() * sizeof(mixer::XcorrWork)));
        b->work_cap = (int64_t)w.size();
    }
    MIXER_CK(cudaMemcpy(b->d_work, w.data(), w.size() * sizeof(mixer::XcorrWork),
                        cudaMemcpyHostToDevice));
    MIXER_CK(cudaMemcpy(b->d_probs, b->tprobs.data(), b->tprobs.size() * sizeof(mixer::XcorrProblem),
                        cudaMemcpyHostToDevice));
    b->nwork = (int64_t)w.size();
    if (b->exec) {   // a captured graph refers to the old list
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    return MIXER_OK;
}

extern "C" int mixer_batch_destroy(mixer_batch* b) {
    if (!b) return MIXER_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_maps);
    cudaFree(b->d_probs);
    cudaFree(b->d_work);
    cudaFree(b->d_err);
    cudaFree(b->d_ctr);
    delete b;
    return MIXER_OK;
}

extern "C" int mixer_batch_create(const mixer_xcorr_problem* probs, int32_t nprob, mixer_batch** out) {
    if (!out || !probs || nprob <= 0 || nprob > 65535) return MIXER_EINVAL;
    *out = nullptr;
    for (int p = 0; p < nprob; ++p) {
        const mixer_xcorr_problem& q = probs[p];
        if (!q.planes || !q.vis || q.nant <= 0 || q.nch <= 0 || q.kt <= 0 || q.kt % 16) return MIXER_EINVAL;
        if (q.kbeg < 0 || q.kbeg % 16 || q.klen <= 0 || q.kbeg + q.klen > q.kt) return MIXER_EINVAL;
        if (q.kt > INT32_MAX || q.nant > 65536 || nblk_of(q.nant) * (nblk_of(q.nant) + 1) / 2 > 65535)
            return MIXER_EINVAL;
        if (q.mode != MIXER_VIS_STORE_I32 && q.mode != MIXER_VIS_ACC_I32 && q.mode != MIXER_VIS_ACC_I64)
            return MIXER_EINVAL;
        if (q.mode != MIXER_VIS_ACC_I64 && q.klen > MIXER_KMAX_I32) return MIXER_EOVERFLOW;
        if (reinterpret_cast<uintptr_t>(q.planes) % 16) return MIXER_EINVAL;
    }
    mixer_batch* b = new mixer_batch();
    memset(b->split, 0, sizeof(b->split));
    for (int c = 0; c <= kMaxClass; ++c) b->split[c] = 1;
    b->order = MIXER_ORDER_LPT;
    b->probs.assign(probs, probs + nprob);
    int rc = MIXER_OK;
    std::vector<CUtensorMap> maps(2 * (size_t)nprob);   // two per problem
    b->tprobs.resize(nprob);
    // problems whose cubes overlap share tiles: their items always add atomically
    b->shared_cube.assign(nprob, 0);
    for (int p = 0; p < nprob; ++p) {
        const size_t es = probs[p].mode == MIXER_VIS_ACC_I64 ? 8 : 4;
        const uintptr_t a0 = reinterpret_cast<uintptr_t>(probs[p].vis);
        const uintptr_t a1 = a0 + (size_t)mixer_vis_elems(probs[p].nant, probs[p].nch) * es;
        for (int q = 0; q < nprob; ++q) {
            if (q == p) continue;
            const size_t eq = probs[q].mode == MIXER_VIS_ACC_I64 ? 8 : 4;
            const uintptr_t b0 = reinterpret_cast<uintptr_t>(probs[q].vis);
            const uintptr_t b1 = b0 + (size_t)mixer_vis_elems(probs[q].nant, probs[q].nch) * eq;
            if (a0 < b1 && b0 < a1) b->shared_cube[p] = 1;
        }
    }
    for (int p = 0; p < nprob && rc == MIXER_OK; ++p) {
        const mixer_xcorr_problem& q = probs[p];
        rc = mixer::xcorr_encode_maps(&maps[2 * p], q.planes, q.nant, q.nch, q.kt, q.kbeg + q.klen);
        const int nb = nblk_of(q.nant);
        if (q.nant % 128) b->ragged = true;
        b->tprobs[p] = mixer::XcorrProblem{q.nant, q.nch, nb * (nb + 1) / 2, (int32_t)q.kbeg, q.mode, 0,
                                           q.vis};
    }
    auto fail = [&](int r) {
        mixer_batch_destroy(b);
        return r;
    };
    if (rc != MIXER_OK) return fail(rc);
    cudaError_t e;
    if ((e = cudaGetDevice(&b->dev)) != cudaSuccess) return fail(mixer::cuda_status(e, "cudaGetDevice"));
    if ((e = cudaMalloc(&b->d_maps, maps.size() * sizeof(CUtensorMap))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_probs, nprob * sizeof(mixer::XcorrProblem))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_err, sizeof(int32_t))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_ctr, sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMemcpy(b->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(b->d_probs, b->tprobs.data(), nprob * sizeof(mixer::XcorrProblem),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemset(b->d_err, 0, sizeof(int32_t))) != cudaSuccess)
        return fail(mixer::cuda_status(e, "batch tables"));
    b->grid = mixer::xcorr_sm_count();
    rc = upload_plan(b);
    if (rc != MIXER_OK) return fail(rc);
    *out = b;
    return MIXER_OK;
}

extern "C" int mixer_batch_plan(mixer_batch* b, const int32_t* split_per_class, int32_t nclass,
                                int32_t order) {
    if (!b || (order != MIXER_ORDER_LPT && order != MIXER_ORDER_CHANNEL)) return MIXER_EINVAL;
    if (nclass < 0 || nclass > kMaxClass + 1 || (nclass > 0 && !split_per_class)) return MIXER_EINVAL;
    for (int c = 0; c < nclass; ++c)
        if (split_per_class[c] < 1 || split_per_class[c] > 4096) return MIXER_EINVAL;
    for (int c = 0; c < nclass; ++c) b->split[c] = split_per_class[c];
    b->order = order;
    return upload_plan(b);
}

extern "C" int mixer_batch_run(mixer_batch* b, void* stream) {
    if (!b) return MIXER_EINVAL;
    return mixer::xcorr_launch_table(b->d_maps, b->d_probs, b->d_work, b->nwork, b->grid, b->d_err,
                                     b->d_ctr, b->ragged,
                                     static_cast<cudaStream_t>(stream));
}

static int time_plan(mixer_batch* b, int reps, cudaStream_t st, float* ms) {
    int rc = mixer_batch_run(b, st);   // warm
    if (rc != MIXER_OK) return rc;
    cudaEvent_t e0, e1;
    MIXER_CK(cudaEventCreate(&e0));
    MIXER_CK(cudaEventCreate(&e1));
    MIXER_CK(cudaEventRecord(e0, st));
    for (int r = 0; r < reps && rc == MIXER_OK; ++r) rc = mixer_batch_run(b, st);
    MIXER_CK(cudaEventRecord(e1, st));
    MIXER_CK(cudaEventSynchronize(e1));
    float t = 0.f;
    MIXER_CK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / (float)reps;
    return rc;
}

// A candidate replaces the incumbent only when it is at least 2 % faster: the
// paired ratio of one launch varies by about 1 % from run to run.
constexpr float kGain = 0.98f;

// Paired comparison of a candidate plan against the incumbent: A B B A, so a
// slow drift of the GPU clock (the power cap settling in) cancels out of the
// ratio candidate / incumbent.
static int plan_ratio(mixer_batch* b, const int32_t* inc, int inc_order, const int32_t* cand,
                      int cand_order, int reps, cudaStream_t st, float* ratio, float* inc_ms) {
    float t[4];
    const int32_t* sp[4] = {inc, cand, cand, inc};
    const int ord[4] = {inc_order, cand_order, cand_order, inc_order};
    for (int i = 0; i < 4; ++i) {
        int rc = mixer_batch_plan(b, sp[i], kMaxClass + 1, ord[i]);
        if (rc == MIXER_OK) rc = time_plan(b, reps, st, &t[i]);
        if (rc != MIXER_OK) return rc;
    }
    *ratio = (t[1] + t[2]) / (t[0] + t[3]);
    if (inc_ms) *inc_ms = 0.5f * (t[0] + t[3]);
    return MIXER_OK;
}

extern "C" int mixer_batch_autotune(mixer_batch* b, int32_t reps, void* stream, float* best_ms) {
    if (!b || reps <= 0) return MIXER_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // classes present, heaviest first (tile-samples of work)
    std::vector<std::pair<double, int>> cls;
    for (int c = 1; c <= kMaxClass; ++c) {
        double work = 0.0;
        for (const auto& q : b->probs)
            if (std::min(nblk_of(q.nant), kMaxClass) == c)
                work += (double)q.nch * (c * (c + 1) / 2) * (double)q.klen;
        if (work > 0.0) cls.push_back({work, c});
    }
    std::sort(cls.rbegin(), cls.rend());
    // greedy K-split per size class, heaviest class first, with longest-first order
    int32_t inc[kMaxClass + 1];
    for (int c = 0; c <= kMaxClass; ++c) inc[c] = 1;
    for (const auto& wc : cls) {
        const int c = wc.second;
        for (int s : {2, 4, 8}) {
            int32_t cand[kMaxClass + 1];
            memcpy(cand, inc, sizeof(cand));
            cand[c] = s;
            float r;
            const int rc = plan_ratio(b, inc, MIXER_ORDER_LPT, cand, MIXER_ORDER_LPT, reps, st, &r, nullptr);
            if (rc != MIXER_OK) return rc;
            if (r < kGain) inc[c] = s;           // keep a split only for a clear gain
        }
    }
    // then the channel-major order with those splits
    int best_order = MIXER_ORDER_LPT;
    {
        float r;
        const int rc = plan_ratio(b, inc, MIXER_ORDER_LPT, inc, MIXER_ORDER_CHANNEL, reps, st, &r, nullptr);
        if (rc != MIXER_OK) return rc;
        if (r < kGain) best_order = MIXER_ORDER_CHANNEL;
    }
    // the result against the default plan (longest-first, no split), which it must
    // clearly beat
    float r;
    int rc;
    int32_t dflt[kMaxClass + 1];
    for (int c = 0; c <= kMaxClass; ++c) dflt[c] = 1;
    rc = plan_ratio(b, dflt, MIXER_ORDER_LPT, inc, best_order, reps, st, &r, nullptr);
    if (rc != MIXER_OK) return rc;
    if (r < kGain)
        rc = mixer_batch_plan(b, inc, kMaxClass + 1, best_order);
    else
        rc = mixer_batch_plan(b, dflt, kMaxClass + 1, MIXER_ORDER_LPT);
    if (rc == MIXER_OK && best_ms) rc = time_plan(b, reps, st, best_ms);
    return rc;
}

extern "C" int mixer_batch_capture_graph(mixer_batch* b, void* stream) {
    if (!b) return MIXER_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!st) return MIXER_EINVAL;   // the legacy default stream cannot be captured
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    MIXER_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = mixer_batch_run(b, st);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != MIXER_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return mixer::cuda_status(e, "cudaStreamEndCapture");
    b->graph = g;
    MIXER_CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    return MIXER_OK;
}

extern "C" int mixer_batch_replay(mixer_batch* b, void* stream) {
    if (!b || !b->exec) return MIXER_EINVAL;
    MIXER_CK(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)));
    return MIXER_OK;
}

extern "C" int mixer_batch_info(mixer_batch* b, int64_t* nwork, int32_t* order,
                                int32_t* split_per_class, int32_t* kernel_err) {
    if (!b) return MIXER_EINVAL;
    if (nwork) *nwork = b->nwork;
    if (order) *order = b->order;
    if (split_per_class) memcpy(split_per_class, b->split, sizeof(b->split));
    if (kernel_err) {
        MIXER_CK(cudaMemcpy(kernel_err, b->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost));
        if (*kernel_err) return MIXER_ETIMEOUT;
    }
    return MIXER_OK;
}
