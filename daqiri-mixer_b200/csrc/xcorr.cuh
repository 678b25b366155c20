// xcorr.cuh -- internal interface of the triangle cGEMM kernel for the batch
// planner (batch.cu): device table entries and launch helpers.
#pragma once
#include "common.cuh"

namespace mixer {

// One array of a batched launch (device table entry).  excl != 0 promises
// that no other item of the launch adds into the same cube entries (one item
// per tile and channel, and a cube no other array shares), so the int64
// epilogue may read-add-write instead of using atomics.
struct XcorrProblem {
    int32_t nant, nch, ntiles, kbeg;   // kbeg: first sample of the array's range
    int32_t mode, excl;
    void* vis;
};
// One work item: array `prob`, channel `chan`, lower-triangle tile `tile`,
// 128-sample chunks [kc0, kc0 + nkc) of the array's range.
struct XcorrWork {
    uint16_t prob, tile;
    uint32_t chan;
    uint32_t kc0, nkc;
};
static_assert(sizeof(XcorrWork) == 16, "work item is 16 bytes");

// Tensor map over planes [2][nch][nant][kt] whose sample dimension ends at kend.
int xcorr_encode_map(CUtensorMap* map, const int8_t* planes, int32_t nant, int32_t nch, int64_t kt,
                     int64_t kend);
// The two maps an array needs in a work table: maps[0] as above, maps[1] the
// ragged last 128-row block (both planes in one box).
int xcorr_encode_maps(CUtensorMap* maps, const int8_t* planes, int32_t nant, int32_t nch, int64_t kt,
                      int64_t kend);
// One persistent launch over a device work list (`grid` CTAs at most; d_tmaps
// holds two maps per array, from xcorr_encode_maps).  The CTAs take items in
// list order from *ctr (device memory of the caller's, zeroed on `st` before
// the launch); ragged: some array's N is not a multiple of 128.
int xcorr_launch_table(const CUtensorMap* d_tmaps, const XcorrProblem* d_probs,
                       const XcorrWork* d_work, int64_t nwork, int grid, int32_t* err,
                       unsigned long long* ctr, bool ragged, cudaStream_t st);
int xcorr_sm_count();

}  // namespace mixer
