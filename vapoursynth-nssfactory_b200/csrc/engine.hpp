// Host engine of one BM3D filter instance: device buffers, the stage pipeline
// (match -> group filter -> finish) and the frame-level drivers (spatial,
// two-stage, CBM3D, rolling temporal and the legacy intermediate).
// Reference counterparts: the group driver src/cuda/common/group_driver.{hpp,cpp}
// (memory plan :571-600, filter_center :760-856, first stage :877-898, frame
// path :968-1107, rolling :1207-1800).
#pragma once

#include "kernels.cuh"
#include "params.hpp"
#include "stage.hpp"

#include <condition_variable>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

namespace nssb {

// A pitched device plane owned by the engine.
struct DevPlane {
    float* p = nullptr;
    int64_t pitch = 0;  // elements
    int w = 0, h = 0;
};

// One plane of one stage of a frame: where it reads, matches and writes.
struct StageItem {
    int plane;                 // engine plane (scratch and accumulators)
    const StageParams* sp;
    const float* src;          // filtered plane
    int64_t sstride;
    const float* ref;          // Wiener reference and match source, or null (hard threshold)
    int64_t rstride;
    float* dst;
    int64_t dstride;
    const int32_t* shared_pos = nullptr;  // CBM3D: groups matched on another plane
    const int32_t* shared_count = nullptr;
};

// Plane pointers of one stage invocation on the device.
struct StagePlanes {
    const float* src[kMaxSlots]{};    // filtered planes per slot
    int64_t src_stride = 0;
    const float* ref[kMaxSlots]{};    // Wiener reference per slot (also the match source), or null
    int64_t ref_stride = 0;
};

class Engine {
public:
    explicit Engine(const Bm3dConfig& cfg);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    const Bm3dConfig& config() const { return cfg_; }
    void frame_window(int n, int* first, int* last) const;
    void get_frame(int n, const nssb_frame* clip, const nssb_frame* ref, int first, int count, int memory,
                   nssb_frame_out* out);

    // Starts a new clip of num_frames frames on this engine's buffers (the
    // serving form reuses engines): cached window frames and rolling sums are
    // dropped.
    void reset_clip(int num_frames);
    // Device bytes an engine of this configuration allocates (temporal plan
    // and window caches included; host_frames: frames arrive in host memory).
    static size_t footprint(const Bm3dConfig& cfg, bool host_frames);

    // 8x8 matcher form: 0 FP32, 1 tensor-core precision form (same lists).
    void set_matcher(int form);
    int matcher() const { return tunes_.match.form; }

    // Kernel accounting (nssb_bm3d_stats).
    void stats(int enable_timing, int reset, nssb_kernel_stats* out);

    // One radius-0 stage of one plane on caller device memory (the C ABI's
    // nssb_bm3d_plane_stage).
    static void plane_stage(const float* src, const float* ref, float* dst, int64_t stride, int w, int h,
                            const StageParams& sp, cudaStream_t stream);

    // Slots the engine renders radius-0 frames on (num_streams).
    int slots() const { return (int)slots_.size(); }

    // Opt-in Kaiser aggregation window: every patch pixel is weighted by the
    // separable Kaiser window of the block (beta > 0) on top of the group's
    // flat weight; 0 restores the reference's flat weights. Radius 0 only.
    void set_window(float beta);

private:
    struct Plan;
    // The buffers and stream of one frame in flight -- the reference's slots
    // (SlotPool, src/cuda/runtime/stream_pool.hpp:62-140; num_streams,
    // src/cuda/runtime/context.hpp:17-23). A radius-0 frame leases a free
    // slot for the whole call, so frames requested from several host threads
    // (VapourSynth's frame threads) overlap: one frame's copies and another's
    // kernels run on different streams. Temporal frames carry rolling state
    // from frame to frame and run on slot 0 under the engine lock.
    struct Slot {
        cudaStream_t stream = nullptr;
        DevPlane in[3], refin[3], basic[3], out[3];
        AccPlane acc[3];
        StageScratch scratch[3];
        StageTables tables;
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;  // timing pool
        std::vector<std::pair<int, size_t>> pending;               // (kind, event pair index)
        bool busy = false;
    };
    void alloc();
    void alloc_slot(Slot& s);
    void release();
    Slot* lease(bool primary);
    void give_back(Slot* s);
    const float* device_input(Slot& s, int plane, const nssb_frame* frames, int first, int n, int memory,
                              bool is_ref, int64_t* stride);
    void spatial_frame(Slot& s, int n, const nssb_frame* clip, const nssb_frame* ref, int first, int memory);
    // Runs one stage over several planes: one launch per kernel and shape.
    void run_stage(Slot& s, StageItem* items, int n);
    void temporal_frame(int n, const nssb_frame* clip, const nssb_frame* ref, int first, int count, int memory,
                        nssb_frame_out* out);

    using Kind = StageClock::Kind;
    static constexpr Kind kMatch = StageClock::kMatch, kGroup = StageClock::kGroup, kFinish = StageClock::kFinish;
    void clock_begin(Slot& s, Kind kind);
    void clock_end(Slot& s, Kind kind);
    template <class F>
    void timed(Slot& s, Kind kind, F&& launch) {
        clock_begin(s, kind);
        launch();
        clock_end(s, kind);
    }
    void collect_timing(Slot& s);
    void count_match(int w, int h, const StageParams& sp);
    struct Clock : StageClock {
        Engine* e;
        Slot* s;
        Clock(Engine* en, Slot* sl) : e(en), s(sl) {}
        void begin(Kind k) override { e->clock_begin(*s, k); }
        void end(Kind k) override { e->clock_end(*s, k); }
        void count_match(int w, int h, const StageParams& sp) override { e->count_match(w, h, sp); }
    };

    Bm3dConfig cfg_;
    int device_ = 0;
    bool timing_ = false;
    nssb_kernel_stats stats_{};
    std::mutex stats_mu_;                        // stats_, timing_ and the tensor-core counters
    std::vector<std::unique_ptr<Slot>> slots_;   // slot 0 also serves temporal frames
    std::mutex slot_mu_;
    std::condition_variable slot_cv_;
    cudaStream_t stream_ = nullptr;              // slot 0's stream (the temporal drivers')
    std::mutex mu_;                              // temporal frames, matcher changes
    LaunchTunes tunes_;
    std::unique_ptr<Clock> clock_;               // slot 0's accounting (the temporal drivers')
    std::map<int, float*> windows_;              // block size -> its window (device), when windowed
    std::vector<void*> allocations_;
    struct PlanDeleter {
        void operator()(Plan* p) const;
    };
    std::unique_ptr<Plan, PlanDeleter> plan_;
};

// The one-plane stage without any allocation (noalloc.cu): scratch comes from
// a file-scope device array of fixed size; sizes beyond it are rejected.
void plane_stage_noalloc(const float* src, const float* ref, float* dst, int64_t stride, int w, int h,
                         const StageParams& sp, cudaStream_t stream);

// Device memory helpers: the library's stream-ordered pool (see dev_alloc).
void* dev_alloc(size_t bytes);
void dev_free(void* p);
// Returns to the device what the library's pool on device dev keeps from
// freed blocks (so cudaMemGetInfo counts it as free again).
void dev_pool_trim(int dev);

}  // namespace nssb
