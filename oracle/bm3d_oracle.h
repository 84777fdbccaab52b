/*
 * CPU oracle for the BM3D hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference CPU plugin (nss.BM3D) semantics. It
 * is the parity checker for the CUDA library: only tests/, the smoke check of
 * __graft_entry__.py and the cpu_baseline / reference legs of bench.py load it.
 * The product path never calls into it and has no CPU fallback.
 *
 * What it restates (reference files, paths inside the reference project):
 *   - raster reference grid with clamped last row/column  src/host/batch_runner.hpp:17-53
 *   - Match ordering, StableTopK, collect_spatial_coords,
 *     collect_temporal (predictive search)                 src/cpu/bm/matcher.hpp:27-373
 *   - SSD of a block pair                                  src/cpu/bm/ssd.cpp:30-64
 *   - orthonormal DCT-II table                             src/cpu/bm/dct8.cpp:69-89
 *   - in-place orthonormal Haar along the group            src/cpu/bm/dct8.cpp:576-644
 *   - hard threshold / Wiener shrinkage and group weight   src/cpu/bm/dct8.cpp:926-1133
 *   - pack / unpack (aggregate_add) / aggregate_finish     src/cpu/bm/pack.cpp:23-87, agg.cpp:17-42
 *   - VAggregate target reduction (ascending centres)      src/cpu/bm/agg.cpp:151-200
 *   - per-plane orchestration, commit order, fat slices    src/host/filter_bm3d.cpp:73-339, 359-494
 *   - temporal slot mapping                                src/frontend/temporal.hpp:11-36
 *   - noise profile sigma_eff = sigma/255*0.75             include/nss/contracts.hpp:19-30
 *
 * Summation order of the SSD: per candidate, every block column takes one
 * FMA chain down the rows (c_j = fma(d, d, c_j), d = a - b), then the
 * columns are added pairwise (halves first, recursively). The reference's SIMD
 * trees are Highway-target dependent; this order is the one the CUDA
 * matcher also uses, so oracle and device distances are bit-identical and
 * groups agree exactly (om_ssd_lanes8 restates the reference's 8-lane AVX2
 * tree of SpatialMatch8, ssd.cpp:104-302, for reporting the near-tie rate
 * against that order).
 */
#ifndef NSS_B200_ORACLE_H
#define NSS_B200_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OM_MAX_GROUP 64
#define OM_MAX_RADIUS 16

typedef struct om_match {
    int32_t x, y, t;
    float dist;
    uint32_t ordinal;
} om_match;

typedef struct om_search {
    int block, step, group, bm_range, radius, ps_num, ps_range;
    int valid_t_begin, valid_t_end; /* valid slots [begin, end); end -1 = ntemp */
} om_search;

/* Per-plane, per-stage settings. sigma is the effective (profile-scaled) value. */
typedef struct om_stage {
    float sigma;
    int block, group, step, bm_range, ps_num, ps_range;
} om_stage;

/* ---- distances ---- */
float om_ssd(const float* a, ptrdiff_t sa, const float* b, ptrdiff_t sb, int block);
float om_ssd_lanes8(const float* a, ptrdiff_t sa, const float* b, ptrdiff_t sb);
int om_match_less(const om_match* a, const om_match* b);

/* ---- matching ---- */
/* collect_spatial_coords semantics: out[0] is the (clamped) reference, then
 * the group-1 best non-self candidates in match_less order. lanes8 != 0 uses
 * the reference's 8-lane tree for block 8. Returns the count. */
int om_spatial_match(const float* plane, ptrdiff_t stride, int width, int height, int bx, int by, int block,
                     int bm_range, int group, om_match* out, int lanes8);
/* predictive_match semantics (match.cpp:10-33): spatial match on slot t0,
 * then collect_temporal over the valid slots. */
int om_predictive_match(const float* const* planes, const ptrdiff_t* strides, int ntemp, int width, int height,
                        int bx, int by, int t0, const om_search* cfg, om_match* out);
/* Raster grid (batch_runner.hpp:17-31): count of positions per axis. */
int om_grid_count(int extent, int block, int step);
int om_grid_pos(int i, int extent, int block, int step);

/* ---- transforms ---- */
const float* om_dct_table(int n);
float om_haar_scale(int n, int j);
/* Bm3dFilterGroup: cube holds group*block*block floats, the first k patches
 * real, the rest zero. ref (Wiener) likewise, or NULL for hard threshold.
 * Filters in place; returns the group weight. */
float om_filter_group(float* cube, const float* ref, int group, int block, float sigma, int wiener);
/* The same in double precision with exact cosines: the FP64 recomputation. */
double om_filter_group_f64(double* cube, const double* ref, int group, int block, double sigma, int wiener);
/* One radius-0 stage with the group filter and sums in FP64 on the FP32
 * matcher's groups (matched on ref when wiener, else on src). */
int om_bm3d_plane_f64(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride, int width, int height,
                      const om_stage* st, int wiener, double* dst, ptrdiff_t dstride);
/* References whose groups differ between this build's SSD order and the
 * reference's 8-lane AVX2 order; *refs receives the reference count. */
long om_order_mismatch(const float* plane, ptrdiff_t stride, int width, int height, const om_stage* st, long* refs);

/* ---- plane passes ---- */
/* One stage of one plane at radius 0: match on ref (when wiener) or src,
 * filter, aggregate in raster commit order, finish into dst.
 * If matches != NULL it receives per reference `group` packed entries
 * (y << 16 | x, unused -1) and counts[] the group sizes. Returns 0 or -1. */
int om_bm3d_plane(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride, int width, int height,
                  const om_stage* st, int wiener, float* dst, ptrdiff_t dstride, int32_t* matches, int32_t* counts);

/* The same with the groups matched on another plane (CBM3D, filter_bm3d.cpp:
 * 451-486: every plane filtered with plane 0's groups); match NULL = as above. */
int om_bm3d_plane_matched(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride,
                          const float* match, ptrdiff_t mstride, int width, int height, const om_stage* st,
                          int wiener, float* dst, ptrdiff_t dstride, int32_t* matches, int32_t* counts);

/* om_bm3d_plane with an aggregation window: each patch pixel adds w * win
 * (block x block weights, row-major) to num (times the value) and den. This
 * is this build's opt-in Kaiser mode, not the reference's BM3D (whose weights
 * are flat per group): it checks the device's windowed mode, nothing else. */
int om_bm3d_plane_window(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride, int width,
                         int height, const om_stage* st, int wiener, const float* win, float* dst, ptrdiff_t dstride);

/* Radius > 0, one plane of a whole clip: each centre c matches predictively
 * over its 2r+1 slots (temporal.hpp:19-21), filters and adds to num/den
 * slices of its target frames; each frame is then reduced over its centres
 * in ascending order (VAggregate). src/ref/dst are arrays of nframes planes of
 * stride `stride`. ref NULL = hard threshold on src. Returns 0 or -1. */
int om_bm3d_plane_clip(const float* const* src, const float* const* ref, int nframes, int width, int height,
                       ptrdiff_t stride, const om_stage* st, int radius, int wiener, float* const* dst);

/* The legacy fat intermediate of centre n (filter_bm3d.cpp:306-320): 2r+1
 * slices of (num, den) planes, each height rows; dst is (2r+1)*2*height rows
 * of stride dstride. */
int om_bm3d_plane_fat(const float* const* src, const float* const* ref, int nframes, int n, int width, int height,
                      ptrdiff_t stride, const om_stage* st, int radius, int wiener, float* dst, ptrdiff_t dstride);

/* VAggregate of one frame from fat intermediates (agg.cpp:151-200). */
void om_vaggregate(const float* const* fats, int count, const float* src, int width, int height, ptrdiff_t fstride,
                   ptrdiff_t sstride, int radius, const int* slices, float* dst, ptrdiff_t dstride);

/* Frame-parallel driver for timing: nframes independent frames of one plane
 * size, radius 0, one stage or two (basic then Wiener with basic as ref),
 * on `threads` POSIX threads. */
int om_bm3d_frames_mt(const float* const* src, float* const* dst, float* const* basic_scratch, int nframes,
                      int width, int height, ptrdiff_t stride, const om_stage* basic, const om_stage* fin,
                      int two_stage, int threads);

float om_noise_effective(float user_sigma);

#ifdef __cplusplus
}
#endif
#endif
