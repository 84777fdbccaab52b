// Resolved BM3D arguments and the creation-time checks of nss_cuda.BM3D.
//
// The checks, their order and their messages are part of the filter's
// interface (the reference pins them with 900 creation cases,
// tests/data/plugin_interface_v1.json). They follow, in order:
//   checked_create: numeric representability, memory_limit_mb   src/frontend/validate.hpp:36-52, validate.cpp:13-45
//   radius, parse_temporal_mode (default rolling)               src/cuda/bm3d/filter.cpp:21-24, temporal_args.cpp:10-27
//   parse_bm3d                                                   src/frontend/bm3d_args.cpp:115-145 (+ :17-112)
//   parse_rolling (adaptive cache)                               src/frontend/temporal_args.cpp:29-56
//   parse_backend_args                                           src/cuda/runtime/context.cpp:23-41
#pragma once

#include "nss_b200.h"

#include <cstdint>
#include <stdexcept>
#include <string>

namespace nssb {

constexpr int kMaxGroup = 64;
constexpr int kMaxBlock = 32;
constexpr int kMaxRange = 64;
constexpr int kMaxRadius = 16;
constexpr int kMaxStreams = 16;

// An argument error; what() is the exact message the filter reports.
struct ArgumentError : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};

// One processing stage of one plane. sigma is effective (0 = copy).
struct StageParams {
    float sigma = 0.f;
    int block = 8, group = 8, step = 8, bm_range = 9, ps_num = 2, ps_range = 4;
};

struct Bm3dConfig {
    nssb_video_info vi{};
    nssb_video_info out_vi{};
    int planes = 1;
    int plane_w[3]{}, plane_h[3]{};
    StageParams final_stage[3];  // the call's own stage (Wiener when ref/final)
    StageParams basic_stage[3];  // final=1: the basic estimate
    bool has_ref = false;        // an external ref clip (Wiener with it)
    bool two_stage = false;      // final=1
    bool chroma = false;         // CBM3D
    int radius = 0;
    bool rolling = false;        // temporal_mode resolves to rolling (radius > 0)
    int rolling_chunk = 1, rolling_cache_chunks = 1, rolling_cache_limit = 16;
    int64_t memory_limit_mb = 0; // 0 = none
    int device_id = 0;
    int num_streams = 1;
    // Opt-in Kaiser aggregation window (nssb_bm3d_set_window; not a filter
    // argument): 0 = the reference's flat per-group weights.
    float kaiser_beta = 0.f;
};

// Throws ArgumentError with the filter's message.
Bm3dConfig parse_bm3d_call(const nssb_video_info& clip, const nssb_video_info* ref, const nssb_arg* args, int nargs);

float effective_sigma(float user_sigma);

}  // namespace nssb
