// One radius-0 BM3D stage over any number of planes, each with its own size,
// sigma and buffers: match -> group filter (+ aggregation) -> finish. Planes
// of one shape (block, group, step, bm_range, Wiener or not) share one launch
// per kernel, up to kMaxBatchPlanes planes a launch. Used by the per-frame
// engine (the three planes of a frame) and by the batched form (every plane
// of every frame of a batch).
// Reference counterparts: process_planes_batched (src/cuda/bm3d/filter_bm3d.cpp:73-339),
// filter_center / first stage (src/cuda/common/group_driver.cpp:760-898).
#pragma once

#include "kernels.cuh"
#include "params.hpp"

#include <vector>

namespace nssb {

// Fixed-point accumulators of one target plane.
struct AccPlane {
    long long* num = nullptr;   // per pixel; zero between stages (finish clears it)
    long long* wsum = nullptr;  // per patch origin; cleared at the start of each stage
    int64_t pitch = 0;
};

// Scratch of one stage pass: match lists, group cubes.
struct StageScratch {
    int32_t* pos = nullptr;
    int32_t* slot = nullptr;
    float* dist = nullptr;
    int32_t* count = nullptr;
    size_t jobs_cap = 0, group_cap = 0;
    float* cube = nullptr;
    size_t cube_floats = 0;
};

// One plane of one stage, fully resolved.
struct StagePlane {
    const StageParams* sp;
    const float* src;  // filtered plane
    int64_t sstride;
    const float* ref;  // Wiener reference and match source, or null (hard threshold)
    int64_t rstride;
    float* dst;
    int64_t dstride;
    int w, h;
    AccPlane acc;
    const StageScratch* sc;
    const int32_t* shared_pos;    // CBM3D: groups matched on another plane of the same stage
    const int32_t* shared_count;
    const float* win = nullptr;   // opt-in aggregation window (block x block, device), or null
};

// Launch shapes of the specialised kernels (results do not depend on them).
struct LaunchTunes {
    MatchTune match;
    GroupTune group;
};

// Kernel bookkeeping of a stage run: launch counts, optional event timing,
// algorithmic matching work.
class StageClock {
public:
    enum Kind { kMatch = 0, kGroup = 1, kFinish = 2, kOther = 3 };  // kOther: clears and copies
    virtual ~StageClock() = default;
    virtual void begin(Kind kind) = 0;
    virtual void end(Kind kind) = 0;
    virtual void count_match(int w, int h, const StageParams& sp) = 0;
};

// Batch tables of the three kernels (large: kept off the stack).
struct StageTables {
    MatchBatch match;
    GroupBatch group;
    FinishBatch finish;
};

// Enqueues the stage on `stream`. Sigma-0 planes are copied. Planes whose
// shared_pos is set must come after the plane they share with.
void run_stage_planes(const StagePlane* planes, int n, cudaStream_t stream, const LaunchTunes& tunes,
                      StageClock& clock, StageTables& tables);

// Reference-candidate pairs of one matching pass over a w x h plane:
// every reference against every other position of its clamped window.
double match_pairs(int w, int h, const StageParams& sp);

}  // namespace nssb
