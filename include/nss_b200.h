/*
 * nss_b200 -- C ABI of the B200 (sm_100a) BM3D library.
 *
 * The reference exposes this path only as a VapourSynth API4 filter,
 * core.nss_cuda.BM3D (registered in src/cuda/plugin.cpp:76-98 and
 * src/cuda/bm3d/filter.cpp:118-122, arguments from
 * src/frontend/bm3d_args.hpp:8-12 plus src/cuda/runtime/context.hpp:17).
 * This header is the boundary under a VapourSynth shim and under the ctypes
 * mirror: plain pointers, sizes and status codes, no exceptions, no C++ or
 * torch types. Each entry point names the reference interface it replaces.
 *
 * Threading: every handle may be used from several threads; calls on one
 * handle serialise internally. nssb_last_error() is per thread.
 */
#ifndef NSS_B200_H
#define NSS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define NSSB_OK 0
#define NSSB_ERR_ARGUMENT 1 /* creation error; the text is the filter's error message */
#define NSSB_ERR_CUDA 2     /* a CUDA call failed; context preserved where possible */
#define NSSB_ERR_RESOURCE 3 /* allocation or memory-limit failure */
#define NSSB_ERR_STATE 4    /* call not valid for this handle / these inputs */
#define NSSB_ERR_TIMEOUT 5  /* a bounded device-side wait gave up */

/* Last error text of the calling thread ("" when none). The creation errors
 * carry the reference's exact messages, e.g. "nss_cuda.BM3D: radius must be
 * in [0, 16]" (checked_create/mapSetError, src/frontend/validate.hpp:36-52). */
const char* nssb_last_error(void);

/* Library version string (the plugin's Version(), src/cuda/plugin.cpp:80). */
const char* nssb_version(void);

/* Device report (the plugin's Backend([device_id]), src/cuda/plugin.cpp:36-72):
 * writes a one-line JSON object into buf (NUL-terminated, truncated to cap). */
int nssb_backend_info(int device_id, char* buf, size_t cap);

/* ---- video description (VSVideoInfo / VSVideoFormat fields used by the path) ---- */
#define NSSB_GRAY 1
#define NSSB_RGB 2
#define NSSB_YUV 3
typedef struct nssb_video_info {
    int color_family;    /* NSSB_GRAY / NSSB_RGB / NSSB_YUV, 0 = variable */
    int sample_float;    /* 1 for float samples */
    int bits_per_sample; /* 32 for the accepted format */
    int subsampling_w, subsampling_h;
    int width, height, num_frames;
} nssb_video_info;

/* ---- creation arguments: the VSMap of the call, key by key, in map order ---- */
#define NSSB_ARG_INT 1
#define NSSB_ARG_FLOAT 2
#define NSSB_ARG_DATA 3
typedef struct nssb_arg {
    const char* key;
    int type;              /* NSSB_ARG_* */
    int count;             /* elements (1 for data) */
    const int64_t* ints;   /* NSSB_ARG_INT */
    const double* floats;  /* NSSB_ARG_FLOAT */
    const char* data;      /* NSSB_ARG_DATA, NUL-terminated */
} nssb_arg;

typedef struct nssb_bm3d nssb_bm3d;

/* Argument resolution without a device: every creation check of
 * nss_cuda.BM3D in the reference's order (checked_create ->
 * validate_numeric_args and memory_limit_mb, src/frontend/validate.hpp:36-52;
 * parse_temporal_mode, parse_bm3d, parse_rolling, parse_backend_args,
 * src/cuda/bm3d/filter.cpp:19-114, src/frontend/bm3d_args.cpp:115-145,
 * src/frontend/temporal_args.cpp:10-56, src/cuda/runtime/context.cpp:23-41).
 * ref may be NULL. On success writes the output video info (the legacy
 * temporal intermediate is (2r+1)*2 planes tall). */
int nssb_bm3d_check(const nssb_video_info* clip, const nssb_video_info* ref, const nssb_arg* args, int nargs,
                    nssb_video_info* out_vi);

/* Creation (the `create` of src/cuda/bm3d/filter.cpp:19-114): the checks
 * above, then device acquisition and device memory for the plan. */
int nssb_bm3d_create(const nssb_video_info* clip, const nssb_video_info* ref, const nssb_arg* args, int nargs,
                     nssb_bm3d** out);
void nssb_bm3d_free(nssb_bm3d* h);
int nssb_bm3d_output_info(const nssb_bm3d* h, nssb_video_info* out_vi);

/* Input frames that output frame n needs: [*first, *last] of clip (and of
 * ref when given) -- the arInitial requests of getFrame. */
int nssb_bm3d_frame_window(const nssb_bm3d* h, int n, int* first, int* last);

/* One frame's planes; strides in elements (float). */
typedef struct nssb_frame {
    const float* planes[3];
    int64_t strides[3];
} nssb_frame;
typedef struct nssb_frame_out {
    float* planes[3];
    int64_t strides[3];
} nssb_frame_out;
#define NSSB_MEM_HOST 0
#define NSSB_MEM_DEVICE 1

/* Output frame n (the getFrame of the group driver,
 * src/cuda/common/group_driver.cpp:1803 and :968-1107). clip_frames[i] (and
 * ref_frames[i], or NULL) are frames first+i, i < count, covering the
 * window above. memory says where all planes live. With NSSB_MEM_HOST the
 * copies to and from the device are part of the call. Several threads may
 * call it at once on one handle (VapourSynth's fmParallel): a radius-0 frame
 * takes one of the node's num_streams slots -- a stream and a set of frame
 * buffers, the reference's slot pool (src/cuda/runtime/stream_pool.hpp:62-140)
 * -- so the copies and kernels of frames on different slots overlap, and
 * waits while all slots are busy; temporal frames run one at a time. */
int nssb_bm3d_get_frame(nssb_bm3d* h, int n, const nssb_frame* clip_frames, const nssb_frame* ref_frames, int first,
                        int count, int memory, nssb_frame_out* out);

/* Frame properties the filter stamps on output frame n (stamp_contribution,
 * src/frontend/contribution.hpp:12-27; constants include/nss/contracts.hpp:6-17
 * of the reference): _NSSModel = 1 (BM3D), _NSSModelVersion = 3,
 * _NSSNoiseProfile = 1, and on the legacy temporal intermediate also
 * _NSSFatVersion = 2, _NSSFatRadius = r, _NSSFatCenter = n, _NSSFatLayout = 1
 * (num/den slices), which nss.VAggregate checks. A shim copies the source
 * frame's properties, then sets these (and deletes the _NSSFat* keys when
 * they are not listed). Writes up to cap entries and their number to *count. */
typedef struct nssb_prop {
    const char* key; /* static string */
    int64_t value;
} nssb_prop;
int nssb_bm3d_frame_props(const nssb_bm3d* h, int n, nssb_prop* out, int cap, int* count);

/* Kernel accounting of a handle, for measurement (no reference counterpart;
 * the reference measures through Nsight, tests/cuda/run_ncu.py). With
 * timing on, the engine brackets its matching, group and finish launches
 * with CUDA events on its own stream and adds their durations once a frame
 * completes. flops are the matcher's algorithmic count: 3 * B^2 per
 * reference-candidate pair (subtract, multiply, add). */
typedef struct nssb_kernel_stats {
    int64_t launches;        /* kernels launched by the handle */
    int64_t match_launches, group_launches, finish_launches;
    double match_ms, group_ms, finish_ms; /* summed event durations (timing on) */
    double match_flops;      /* algorithmic matcher flops of the counted launches */
    double match_pairs;      /* reference-candidate pairs evaluated */
    int64_t tc_survivors;    /* precision form: candidates re-ranked exactly */
    int64_t tc_refs;         /* precision form: references matched */
    double tc_max_error_ratio; /* precision form: largest |approximate - exact| / margin */
} nssb_kernel_stats;
int nssb_bm3d_stats(nssb_bm3d* h, int enable_timing, int reset, nssb_kernel_stats* out);

/* Matcher of a handle's 8x8 stages (spatial and the centre frame of
 * temporal): 0 = FP32, 1 = the tensor-core precision form of
 * nssb_match_spatial_tc, 2 = automatic (the default): the precision form
 * where it measured faster -- from bm_range 32 on at block steps 1-7, from
 * 63 on at step 8 -- and FP32 elsewhere. Outputs are
 * bit-identical whichever form runs. No reference counterpart (the
 * reference picks its CUDA matcher by shape, src/cuda/common/match.cu:1605-1611). */
#define NSSB_MATCHER_FP32 0
#define NSSB_MATCHER_TENSOR 1
#define NSSB_MATCHER_AUTO 2
int nssb_bm3d_set_matcher(nssb_bm3d* h, int form);

/* Opt-in Kaiser aggregation window. No counterpart in the reference's BM3D,
 * whose aggregation weights every pixel of a group's patches by one flat
 * per-group weight (src/cpu/bm/dct8.cpp:1126-1131,
 * src/cuda/bm3d/kernels.cu:292-301); the reference windows only its BM4D
 * (src/cuda/bm4d/kernels.cu:734). With beta > 0 each patch pixel (i, j) is
 * weighted by w * K(i) K(j), K(n) = I0(beta sqrt(1 - (2n/(B-1) - 1)^2)) / I0(beta),
 * in num and den alike; beta = 0 (the default) is the reference's aggregation
 * bit for bit. Radius-0 filters rendered by nssb_bm3d_get_frame only
 * (NSSB_ERR_STATE otherwise; the batched form rejects such nodes). Not
 * parity-checked against the reference, which has no such mode. */
int nssb_bm3d_set_window(nssb_bm3d* h, float beta);

/* ---- stage primitives on device memory (the kernels the filter runs) ----
 * Strides are in elements. stream is a cudaStream_t (NULL = default). */

/* Spatial block matching of every reference of the raster grid
 * (batch_runner.hpp:17-53; matcher contract src/cpu/bm/matcher.hpp:27-283,
 * the reference's device form src/cuda/common/match.cu:1685).
 * pos[j*group+q] = y << 16 | x of match q of reference j (raster order),
 * -1 past count[j]; dist (may be NULL) the matching SSDs. */
int nssb_match_spatial(const float* plane, int64_t stride, int width, int height, int block, int step,
                       int bm_range, int group, int32_t* pos, float* dist, int32_t* count, void* stream);

/* Precision form of nssb_match_spatial for 8x8 blocks, bm_range 9 (groups 2,
 * 4, 8, 16) and bm_range 10-64 (groups 2-32): candidate distances
 * |r|^2 + |c|^2 - 2 r.c with the dot
 * products on the tensor cores (tcgen05.mma, BF16 hi/lo split of every pixel,
 * FP32 accumulation in tensor memory), then every candidate within a proven
 * error margin of the K-th distance re-ranked with the exact FP32 distance,
 * so pos, dist and count equal nssb_match_spatial's bit for bit. stats (may
 * be NULL) receives the re-rank accounting of this call. Returns
 * NSSB_ERR_STATE for shapes it does not cover, NSSB_ERR_TIMEOUT if a bounded
 * device wait gave up. No reference counterpart in this form: the
 * reference's tensor matcher (src/cuda/common/match.cu, mma.sync, large
 * windows) orders ties differently (src/cuda/common/match.hpp:2-8). */
typedef struct nssb_tc_stats {
    int64_t survivors;      /* candidates re-ranked exactly */
    int64_t refs;           /* references matched */
    float max_error_ratio;  /* largest |approximate - exact| / margin among survivors (must stay < 1) */
    int flagged_tiles;      /* tiles with non-finite pixels (every candidate re-ranked) */
    int timeouts;           /* bounded device waits that gave up */
} nssb_tc_stats;
int nssb_match_spatial_tc(const float* plane, int64_t stride, int width, int height, int step, int bm_range,
                          int group, int32_t* pos, float* dist, int32_t* count, nssb_tc_stats* stats,
                          void* stream);

/* Predictive temporal matching (collect_temporal, matcher.hpp:319-373; device
 * form match.cu:1707-1757). planes/strides: host arrays of ntemp device
 * planes; reference slot t0; valid slots [valid_begin, valid_end). slot[j*group+q]
 * receives the frame slot of each match. */
int nssb_match_temporal(const float* const* planes, const int64_t* strides, int ntemp, int t0, int valid_begin,
                        int valid_end, int width, int height, int block, int step, int bm_range, int group,
                        int ps_num, int ps_range, int32_t* pos, int32_t* slot, float* dist, int32_t* count,
                        void* stream);

/* One full stage of one plane at radius 0 (process_planes_batched,
 * src/host/filter_bm3d.cpp:73-339; filter_center, group_driver.cpp:760-856):
 * match on ref (Wiener) or src (hard threshold, ref NULL), filter every group,
 * aggregate, finish into dst. sigma is the effective value. */
int nssb_bm3d_plane_stage(const float* src, const float* ref, float* dst, int64_t stride, int width, int height,
                          float sigma, int block, int group, int step, int bm_range, void* stream);

/* The stage above without allocating anything. No counterpart in the
 * reference: it is for callers that cannot allocate device memory while they
 * run -- hosts whose device memory is owned and budgeted by their own pool
 * (a frame pool sized at start-up), or latency-critical loops where
 * cudaMalloc/cudaFree would block or synchronise the device. Scratch comes
 * from one file-scope device array of about 37 MiB that every GPU loading the
 * library keeps until exit; planes up to 2 MiPx (stride x height <= 2097152),
 * 262144 references and 1048576 match entries (references x group) are
 * accepted, larger ones rejected with NSSB_ERR_STATE. Shapes whose group
 * cube needs global scratch (block 32 with groups of 32 or more, Wiener
 * block 16 with 64, ...) are rejected too. The first call on a device looks
 * up the array's device address (cudaGetSymbolAddress); make it before any
 * stream capture. Calls share the array: calls that overlap on the GPU race,
 * so serialise them; each call clears the sums it uses. */
int nssb_bm3d_plane_stage_noalloc(const float* src, const float* ref, float* dst, int64_t stride, int width,
                                  int height, float sigma, int block, int group, int step, int bm_range,
                                  void* stream);

/* ---- batched form ----
 * Many output frames of radius-0 filter instances -- different clips,
 * resolutions, formats, sigmas and stage arguments -- rendered in one pass:
 * each stage is one launch per kernel and block shape over every plane of
 * every frame, the two-stage pipeline is captured once per batch layout as
 * a CUDA graph and replayed, and the kernels' launch shapes are chosen by
 * timing the candidates on the first batch of each layout. The output of
 * every frame is bit-identical to nssb_bm3d_get_frame of the same node.
 * No single reference counterpart: the reference renders frame by frame
 * through VapourSynth's frame threads (src/cuda/bm3d/filter_bm3d.cpp:73-494,
 * the getFrame of src/cuda/common/group_driver.cpp:1803). */
typedef struct nssb_batch nssb_batch;
typedef struct nssb_batch_item {
    nssb_bm3d* node;        /* a radius-0 filter instance on the batch's device */
    const nssb_frame* clip; /* the output frame's input planes */
    const nssb_frame* ref;  /* its ref-clip frame when the node has one, else NULL */
    int memory;             /* NSSB_MEM_HOST / NSSB_MEM_DEVICE for clip, ref and out */
    nssb_frame_out* out;
} nssb_batch_item;
typedef struct nssb_batch_info {
    int match_parts, match_persistent;  /* matcher shape in use */
    int match_form;                     /* 0: FP32 matcher, 1: tensor-core precision form (same lists) */
    int group_warps, group_ctas_per_sm; /* group-filter shape in use */
    int graphs;                         /* 1: runs replay a captured graph */
    int64_t runs, frames;               /* batches and frames rendered */
    int64_t kernel_launches;            /* kernels per run of the current layout */
    int64_t graph_builds, tunings;
    int chunks;                         /* chunks of the last run */
    double last_run_ms;                 /* device time of the last run, copies included (CUDA events) */
    size_t arena_bytes;                 /* device memory of the kept layouts */
} nssb_batch_info;
/* args (ints): "autotune" (default 1), "graph" (default 1), "chunk_frames"
 * (frames per chunk; default 0: one chunk when every item is on the device,
 * else up to ten equal chunks on three streams so that host copies overlap
 * the kernels), and the shapes
 * used when autotune is 0: "match_form" (0 FP32, 1 tensor-core precision
 * form; default 0), "match_parts" (1, 2, 4; default 2),
 * "match_persistent" (0/1; default 0), "group_warps" (2, 4, 8; default 4),
 * "group_ctas_per_sm" (1..64; default 16). */
int nssb_batch_create(int device_id, const nssb_arg* args, int nargs, nssb_batch** out);
/* Renders items[0..n); returns when every output is written. Every node
 * must have radius 0 and live on the batch's device. Host planes should be
 * page-locked for the copies to overlap. */
int nssb_batch_run(nssb_batch* b, const nssb_batch_item* items, int n);
int nssb_batch_get_info(nssb_batch* b, nssb_batch_info* out);
void nssb_batch_free(nssb_batch* b);

/* ---- serving form ----
 * A request loop on one device. A request is a short clip with the
 * arguments of nss_cuda.BM3D (any radius in rolling mode, final, chroma,
 * sigma ...). Requests are admitted in arrival order while their device
 * footprint fits the memory budget; admitted radius-0 requests are rendered
 * together in continuously formed batches (requests arriving meanwhile join
 * the next batch), radius > 0 requests on pooled engines whose window frames
 * and rolling sums stay on the device, concurrently with the batches. Every
 * output equals what nssb_bm3d_get_frame gives for the same clip and
 * arguments, alone or in any mix. No reference counterpart: the reference
 * serves frames through VapourSynth's frame threads
 * (src/cuda/runtime/stream_pool.hpp:62-140). */
typedef struct nssb_server nssb_server;
typedef struct nssb_serve_request {
    nssb_video_info vi;     /* the clip: format, size, num_frames = frames of the request */
    const nssb_arg* args;   /* nss_cuda.BM3D arguments (device_id is the server's) */
    int nargs;
    const nssb_frame* clip; /* vi.num_frames frames */
    const nssb_frame* ref;  /* vi.num_frames ref-clip frames (same format), or NULL */
    int memory;             /* NSSB_MEM_HOST / NSSB_MEM_DEVICE for clip, ref and out */
    nssb_frame_out* out;    /* vi.num_frames output frames; written when the request completes */
} nssb_serve_request;
typedef struct nssb_serve_result {
    int status;              /* NSSB_OK or the request's error code */
    int frames;
    double queue_ms;         /* submission -> admission */
    double latency_ms;       /* submission -> every output written */
    int64_t footprint_bytes; /* device memory reserved at admission */
    char error[192];         /* error text when status != NSSB_OK */
} nssb_serve_result;
typedef struct nssb_server_stats {
    int64_t submitted, completed, failed, frames;
    int64_t ticks, tick_frames, temporal_frames; /* batched ticks and their frames; radius > 0 frames */
    int64_t queued, active, peak_active;
    int64_t budget_bytes, reserved_bytes, peak_reserved_bytes;
    int64_t engines_created, engines_reused;
} nssb_server_stats;
/* args (ints): "memory_budget_mb" (default 0: 80 % of the free device memory),
 * "max_tick_mpx" (pixels per batch, all planes, in millions; default 64),
 * "workers" (radius > 0 requests in flight; default 8). */
int nssb_server_create(int device_id, const nssb_arg* args, int nargs, nssb_server** out);
/* Checks the arguments (creation errors carry nss_cuda.BM3D's messages) and
 * queues the request. The request's frame arrays and planes must stay valid
 * until its result has been collected by nssb_server_wait. */
int nssb_server_submit(nssb_server* s, const nssb_serve_request* req, int64_t* ticket);
/* Waits for a request (timeout_ms < 0: no limit) and collects its result:
 * NSSB_OK when it completed (its own status is in out->status),
 * NSSB_ERR_TIMEOUT when the time ran out first (collect it later). */
int nssb_server_wait(nssb_server* s, int64_t ticket, int64_t timeout_ms, nssb_serve_result* out);
int nssb_server_get_stats(nssb_server* s, nssb_server_stats* out);
/* Finishes the admitted work, fails what is still queued, releases everything. */
void nssb_server_free(nssb_server* s);

#ifdef __cplusplus
}
#endif
#endif
