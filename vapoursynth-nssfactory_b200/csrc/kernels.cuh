// Kernel launchers of the BM3D path (sm_100a). All device pointers; strides in
// elements; every launcher enqueues on `stream` and returns immediately.
#pragma once

#include "common.cuh"

#include <cstdint>

namespace nssb {

constexpr int kMaxSlots = 33;  // 2 * 16 + 1 temporal slots

// Spatial matching of the whole raster grid of one plane (see nss_b200.h).
void launch_match_spatial(const float* plane, int64_t stride, int width, int height, int block, int step,
                          int bm_range, int group, int32_t* pos, float* dist, int32_t* count, cudaStream_t stream);

// A batch of planes sharing one stage shape, processed by one launch per
// kernel (the planes of a frame, or of many frames in the batched form).
constexpr int kMaxBatchPlanes = 192;
struct MatchPlane {
    const float* src;  // match source plane
    int64_t stride;
    int32_t* pos;      // njobs x group
    float* dist;       // njobs x group, or null
    int32_t* count;    // njobs
    int W, H, nx, ny;
    int cta0;          // first CTA of this plane in the launch
    // 8x8 matcher only: int64 words to zero while matching (the plane's
    // origin weights, cleared for the group filter that follows), or null
    long long* clear = nullptr;
    int64_t clear_words = 0;
    // 8x8 matchers: the grid columns [rx_begin, rx_end) of references to
    // match (rx_end 0: up to the last)
    int rx_begin = 0, rx_end = 0;
};
struct MatchBatch {
    int n, step;
    int range;         // the search range (set by the 8x8 launcher; may be below the kernel's built range)
    int total_ctas;    // tiles of the launch (set by the launcher)
    int* queue;        // persistent form: next-tile counter, else null (set by the launcher)
    MatchPlane p[kMaxBatchPlanes];
};
// Launch shape of the 8x8 matcher; every choice gives the same lists.
struct TcCounters;
struct MatchTune {
    int parts = 2;           // warp pairs splitting the window columns: 1, 2 or 4
    int persistent = 0;      // 1: one resident wave taking tiles from a device counter
    int* queue = nullptr;    // that counter (one int of device memory)
    int form = 0;            // 0: FP32 SIMT matcher; 1: tensor-core distances + exact re-rank (same lists);
                             // 2: automatic, the form that measured faster for the shape
    TcCounters* tc = nullptr;  // counters of the tensor form (device memory)
};
// The specialised exact matcher for 8x8 blocks (match8.cu) over a batch of
// planes; false when the shape (bm_range, group, step) has no specialisation.
bool launch_match8_batch(MatchBatch& batch, int bm_range, int group, cudaStream_t stream,
                         const MatchTune* tune = nullptr);
bool launch_match8(const float* plane, int64_t stride, int width, int height, int step, int bm_range, int group,
                   int32_t* pos, float* dist, int32_t* count, cudaStream_t stream);
// The 8x8 direct matcher alone (every reference's 64 columns on its own lanes).
bool launch_match8_direct(MatchBatch& batch, int bm_range, int group, cudaStream_t stream, const MatchTune* tune);
// The column-reuse matcher for 8x8 blocks at steps 1-4 (match_col8.cu):
// whether it takes the shape, and the launch (false when it does not).
bool matchcol_takes(int step, int bm_range, int group);
bool launch_matchcol_batch(MatchBatch& batch, int bm_range, int group, cudaStream_t stream);

// Precision form of the 8x8 matcher (match_tc.cu): BF16 tensor-core distances,
// exact FP32 re-rank; the same lists as launch_match8_batch. Counters (device
// memory, accumulated across launches): survivors re-ranked, references,
// tiles with non-finite pixels, the largest |approx - exact| / margin seen,
// and barrier waits that gave up (0 unless the device misbehaves).
struct TcCounters {
    unsigned long long survivors, refs;
    unsigned int max_ratio_bits, flagged_tiles, timeouts, pad;
};
// Whether a stage of 8x8 blocks with this search range and block step takes
// the precision form: asked for (form 1), or automatically (form 2) where it
// measured faster on 1080p YUV420 frames. Beyond range 31 the FP32 matcher
// sweeps the window in bands of 63 x 63 candidates, its time growing with
// (2R + 1) x the number of row bands; the tensor form's grows with 2R + 1 and
// shares more candidate columns between references at smaller steps. At
// steps 1-7 the tensor form wins from range 32 (range 40: 1.15x at step 7,
// 1.18x at step 6, 1.58x at step 4); at step 8 only from range 63, where the
// FP32 matcher needs a third row band (1.46x at range 64; at ranges 40-56 it
// is 2-8 % faster itself). Lists are identical either way.
inline bool tensor_matcher_takes(int form, int bm_range, int step) {
    return form == 1 || (form == 2 && bm_range >= (step >= 8 ? 63 : 32));
}
// The precision form: bm_range 9 on match_tc.cu's kernel, 10-64 on match_tcw.cu's
// (references on the MMA's M side); false where neither covers the shape.
bool launch_match_tc_batch(MatchBatch& batch, int bm_range, int group, TcCounters* counters, cudaStream_t stream);
bool launch_match_tcw_batch(MatchBatch& batch, int bm_range, int group, TcCounters* counters, cudaStream_t stream);

struct GroupPlane {
    const float* src;
    const float* ref;  // Wiener reference, or null
    int64_t stride, ref_stride;
    long long* num;
    long long* wsum;
    int64_t acc_stride;
    const int32_t* pos;
    const int32_t* count;
    int job0, njobs;
    float sigma;
    int W, H;   // plane size
    int cta0;   // first CTA of this plane
    // opt-in aggregation window (block x block weights, device memory), or
    // null: each pixel then adds w * win to num (times the value) and to a
    // per-pixel den in wsum (finished with a 1 x 1 box)
    const float* win = nullptr;
};
struct GroupBatch {
    int n, total_jobs;
    GroupPlane p[kMaxBatchPlanes];
};
// Launch shape of the warp-per-group filter; every choice gives the same sums.
struct GroupTune {
    int warps = 4;          // groups (warps) per CTA: 2, 4 or 8
    int ctas_per_sm = 16;   // grid = min(groups / warps, SMs x this); warps loop over the rest
};
// Warp-per-group filter for 8x8 blocks and groups of 4/8/16 over a batch of
// planes (all Wiener or all hard threshold); false when the shape has none.
bool launch_group8_batch(const GroupBatch& batch, int group, bool wiener, cudaStream_t stream,
                         const GroupTune* tune = nullptr);

struct FinishPlane {
    long long* num;          // cleared by the kernel after use
    const long long* wsum;
    int64_t acc_stride;
    const float* src;
    int64_t sstride;
    float* dst;
    int64_t dstride;
    int W, H, tiles_x, cta0;
};
struct FinishBatch {
    int n, block, total_ctas;
    FinishPlane p[kMaxBatchPlanes];
};
void launch_finish_batch(const FinishBatch& batch, cudaStream_t stream);
int finish_tiles_x(int w);
int finish_tiles(int w, int h);

// Predictive temporal layers on top of a spatial result already in pos/dist/count
// (slot t0). Fills slot[] and extends each group across the valid slots.
struct TemporalPlanes {
    const float* plane[kMaxSlots];
    int64_t stride[kMaxSlots];
};
void launch_match_temporal(const TemporalPlanes& planes, int ntemp, int t0, int valid_begin, int valid_end,
                           int width, int height, int block, int step, int group, int ps_num, int ps_range,
                           int32_t* pos, int32_t* slot, float* dist, int32_t* count, cudaStream_t stream);
// The temporal layers of up to three planes of one centre in one launch (the
// streaming kernel: 8x8 blocks, ps_range 4, ps_num <= 2, groups 2/4/8/16);
// false when the shape is not covered (launch per plane instead).
struct TemporalBatchPlane {
    TemporalPlanes tp;
    int W, H, jobs, cta0;
    int32_t* pos;
    int32_t* slot;
    float* dist;
    int32_t* count;
};
struct TemporalBatch {
    int n, ntemp, t0, first, last, group, ps_num, ps_range, total_ctas;
    TemporalBatchPlane p[3];
};
bool launch_match_temporal_batch(TemporalBatch& batch, cudaStream_t stream);

// Group filtering + aggregation of one stage (hard threshold, or Wiener when
// ref planes are given). Sums go to fixed-point num (per pixel) and wsum (per
// patch origin) of the slot each patch came from.
struct GroupIO {
    const float* src[kMaxSlots];
    const float* ref[kMaxSlots];  // Wiener reference planes (nullptr: hard threshold)
    int64_t stride;               // element stride of src planes
    int64_t ref_stride;           // element stride of ref planes
    long long* num[kMaxSlots];
    long long* wsum[kMaxSlots];
    int64_t acc_stride;           // element stride of num/wsum
    const float* win = nullptr;   // opt-in aggregation window, as in GroupPlane
};
void launch_group_filter(const GroupIO& io, int width, int height, const int32_t* pos, const int32_t* slot,
                         const int32_t* count, int njobs, int block, int group, float sigma, bool wiener,
                         float* scratch, size_t scratch_floats, cudaStream_t stream);
// The specialised warp-per-group filter for 8x8 blocks and groups of 4/8/16
// (group8.cu); false when the shape has none.
bool launch_group8(const GroupIO& io, const int32_t* pos, const int32_t* slot, const int32_t* count, int njobs,
                   int group, float sigma, bool wiener, cudaStream_t stream);
// The same over up to three planes of one temporal centre in one launch.
struct GroupSlotPlane {
    GroupIO io;
    const int32_t* pos;
    const int32_t* slot;
    const int32_t* count;
    int njobs, job0;
    float sigma;
};
struct GroupSlotBatch {
    int n, total_jobs;
    GroupSlotPlane p[3];
};
bool launch_group8_slots_batch(const GroupSlotBatch& batch, int group, bool wiener, cudaStream_t stream);
// Device scratch (floats) the generic group kernel needs for this shape, 0 if none.
size_t group_filter_scratch_floats(int block, int group, bool wiener);
// The generic group kernel's DCT tables on the current device (once per device).
void ensure_group_tables();

// out = den > 1e-12 ? num / den : src, den the B x B box sum of the origin
// weights; num and wsum are read, not cleared.
void launch_finish(const long long* num, const long long* wsum, int64_t acc_stride, const float* src,
                   int64_t sstride, float* dst, int64_t dstride, int width, int height, int block,
                   cudaStream_t stream);

// The legacy fat slice of one target: num and den as float planes.
void launch_fat_slice(const long long* num, const long long* wsum, int64_t acc_stride, float* dst_num,
                      float* dst_den, int64_t dstride, int width, int height, int block, cudaStream_t stream);

}  // namespace nssb
