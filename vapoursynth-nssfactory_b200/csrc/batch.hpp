// Batched form: many radius-0 frames -- of different filter instances,
// resolutions, formats and sigmas -- in one pass. Every plane of every frame
// gets its buffers in one device arena; each stage is one launch per kernel
// and shape over all of them (the matcher optionally persistent over a device
// tile counter), the whole two-stage pipeline is captured once as a CUDA
// graph per batch layout and replayed, and the kernels' launch shapes are
// picked by timing the candidates on the batch itself (the results do not
// depend on them).
// No single reference counterpart: the reference batches 32-job windows of
// one plane (src/cuda/bm3d/filter_bm3d.cpp:73-339, group_driver.cpp:760-856)
// and runs frames through VapourSynth's frame threads.
#pragma once

#include "nss_b200.h"
#include "stage.hpp"

#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace nssb {

// One output frame of a radius-0 filter instance.
struct BatchItem {
    const Bm3dConfig* cfg;   // the instance's resolved arguments
    const nssb_frame* clip;  // the frame's planes
    const nssb_frame* ref;   // the external ref frame, or null
    int memory;              // NSSB_MEM_HOST / NSSB_MEM_DEVICE
    nssb_frame_out* out;
};

// Stage clock that counts launches and, when asked, times them with events.
class EventClock : public StageClock {
public:
    EventClock(cudaStream_t s, bool timing) : stream_(s), timing_(timing) {}
    ~EventClock() override;
    void begin(Kind k) override;
    void end(Kind k) override;
    void count_match(int w, int h, const StageParams& sp) override;
    // After the stream is synchronised.
    void collect();
    double ms[4] = {0, 0, 0, 0};
    int64_t launches[4] = {0, 0, 0, 0};
    double match_flops = 0, match_pairs = 0;

private:
    cudaStream_t stream_;
    bool timing_;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events_;
    std::vector<int> kinds_;
    size_t used_ = 0;
};

// Device layout of one batch: the arena, the stage plane lists and the
// captured graph.
class BatchPlan {
public:
    explicit BatchPlan(int device);
    ~BatchPlan();
    BatchPlan(const BatchPlan&) = delete;
    BatchPlan& operator=(const BatchPlan&) = delete;

    // Lays the batch out; keeps the arena (and graph) when the layout is
    // unchanged. A new layout first waits for the plan's work on `s`.
    void layout(const BatchItem* items, int n, cudaStream_t s);
    void bind(const BatchItem* items, int n);
    static std::string signature_of(const BatchItem* items, int n);
    const std::string& signature() const { return sig_; }
    size_t arena_bytes() const { return arena_bytes_; }
    // Bytes the batch needs on the device (without laying it out).
    static size_t footprint(const BatchItem* items, int n);

    void upload(const BatchItem* items, int n, cudaStream_t s);
    // Both stages, directly (clock sees every launch) or as the captured graph.
    void compute(cudaStream_t s, const LaunchTunes& tunes, StageClock& clock);
    void compute_graph(cudaStream_t s, const LaunchTunes& tunes);
    void download(const BatchItem* items, int n, cudaStream_t s);
    int64_t launches_per_run() const { return launches_per_run_; }
    int64_t graph_builds() const { return graph_builds_; }

private:
    struct Plane;
    struct PreMatch;
    void release_graph();
    int device_;
    std::string sig_;
    char* arena_ = nullptr;
    size_t arena_bytes_ = 0, arena_cap_ = 0;
    std::vector<Plane> planes_;
    std::vector<StageScratch> scratch_;
    std::vector<StagePlane> stage_[2];
    std::vector<PreMatch> prematch_[2];
    std::unique_ptr<StageTables> tables_;
    int* queue_ = nullptr;
    cudaGraphExec_t graph_ = nullptr;
    LaunchTunes graph_tunes_{};
    int64_t launches_per_run_ = 0, graph_builds_ = 0;
};

struct BatchOptions {
    bool autotune = true;
    bool graphs = true;
    int chunk_frames = 0;  // 0: one chunk for device items, up to 6 equal chunks with host items
    bool plan_per_stream = false;  // one plan per stream, re-laid out as layouts change (serving)
    LaunchTunes fixed;     // the launch shapes used when autotune is off
};

// Runs batches in chunks on two streams, each chunk uploaded, computed (a
// graph replay) and downloaded on its stream, so that one chunk's host copies
// overlap the other's kernels. Plans (arena + graph) are kept per chunk
// layout and stream; the tuned shapes per layout.
class BatchEngine {
public:
    BatchEngine(int device, const BatchOptions& opt);
    ~BatchEngine();
    // Renders every item; returns when the outputs are written.
    void run(const BatchItem* items, int n);
    void info(nssb_batch_info* out);

private:
    static constexpr size_t kMaxPlans = 6;
    LaunchTunes tune(BatchPlan& plan, cudaStream_t s);
    BatchPlan& plan_for(const std::string& sig, int lane);
    std::vector<std::pair<int, int>> chunks(const BatchItem* items, int n) const;
    int device_;
    BatchOptions opt_;
    // chunks rotate over kLanes streams: a chunk's download and the upload
    // of the chunk after next on the same stream hide behind the kernels of
    // the chunks between them
    static constexpr int kLanes = 3;
    cudaStream_t streams_[kLanes] = {};
    cudaEvent_t t0_ = nullptr, t1_[kLanes] = {};
    std::vector<std::pair<std::string, std::unique_ptr<BatchPlan>>> plans_;  // least recently used first
    std::map<std::string, LaunchTunes> tuned_;
    std::mutex mu_;
    nssb_batch_info info_{};
};

// The launch-shape candidates the tuner times (index 0 is the default).
const std::vector<MatchTune>& match_candidates();
const std::vector<GroupTune>& group_candidates();

}  // namespace nssb
