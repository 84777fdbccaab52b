// Batched form (see batch.hpp).
#include "batch.hpp"
#include "engine.hpp"

#include <algorithm>
#include <cstring>
#include <sstream>

namespace nssb {

// ---- clock ----

EventClock::~EventClock() {
    for (auto& e : events_) {
        (void)cudaEventDestroy(e.first);
        (void)cudaEventDestroy(e.second);
    }
}

void EventClock::begin(Kind) {
    if (!timing_) return;
    if (used_ >= events_.size()) {
        cudaEvent_t a, b;
        NSSB_CUDA(cudaEventCreate(&a));
        NSSB_CUDA(cudaEventCreate(&b));
        events_.emplace_back(a, b);
    }
    NSSB_CUDA(cudaEventRecord(events_[used_].first, stream_));
}

void EventClock::end(Kind k) {
    ++launches[k];
    if (!timing_) return;
    NSSB_CUDA(cudaEventRecord(events_[used_].second, stream_));
    kinds_.push_back(k);
    ++used_;
}

void EventClock::count_match(int w, int h, const StageParams& sp) {
    const double pairs = nssb::match_pairs(w, h, sp);
    match_pairs += pairs;
    match_flops += pairs * 3.0 * sp.block * sp.block;
}

void EventClock::collect() {
    for (size_t i = 0; i < used_; ++i) {
        float t = 0.f;
        NSSB_CUDA(cudaEventElapsedTime(&t, events_[i].first, events_[i].second));
        ms[kinds_[i]] += t;
    }
    used_ = 0;
    kinds_.clear();
}

// ---- tuner candidates ----

const std::vector<MatchTune>& match_candidates() {
    static const std::vector<MatchTune> c = {
        {2, 0, nullptr, 0, nullptr}, {2, 1, nullptr, 0, nullptr}, {1, 0, nullptr, 0, nullptr},
        {4, 0, nullptr, 0, nullptr}, {4, 1, nullptr, 0, nullptr}, {2, 0, nullptr, 1, nullptr}};
    return c;
}

const std::vector<GroupTune>& group_candidates() {
    static const std::vector<GroupTune> c = {{4, 16}, {2, 32}, {8, 8}, {4, 8}, {8, 16}};
    return c;
}

// ---- plan ----

struct BatchPlan::Plane {
    int item, plane, w, h;
    int64_t pitch;
    size_t in, refin, basic, out, num, wsum, pos, count, cube;  // arena offsets (SIZE_MAX: none)
    size_t cube_floats;
};

struct BatchPlan::PreMatch {  // CBM3D with a plane-0 sigma of 0: plane 0 still matches
    const StageParams* sp;
    int plane;                // index into planes_
    bool on_ref;              // match on the stage's reference plane
    size_t src_off;
};

namespace {

constexpr size_t kNone = ~size_t(0);
constexpr size_t kAlign = 256;

int64_t pitch_of(int w) { return (int64_t)((w + 31) / 32) * 32; }
size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Stage A: the basic estimate (final=1) or the only hard-threshold stage.
// Stage B: the Wiener stage (final=1 on the basic estimate, or a ref clip).
bool has_stage_a(const Bm3dConfig& c) { return c.two_stage || !c.has_ref; }
bool has_stage_b(const Bm3dConfig& c) { return c.two_stage || c.has_ref; }

void append_signature(std::ostringstream& os, const Bm3dConfig& c) {
    os << c.planes << ':' << c.two_stage << c.has_ref << c.chroma;
    for (int p = 0; p < c.planes; ++p) {
        os << '|' << c.plane_w[p] << 'x' << c.plane_h[p];
        for (const StageParams* s : {&c.basic_stage[p], &c.final_stage[p]}) {
            uint32_t bits;
            std::memcpy(&bits, &s->sigma, 4);
            os << ',' << bits << '/' << s->block << '/' << s->group << '/' << s->step << '/' << s->bm_range;
        }
    }
    os << ';';
}

}  // namespace

BatchPlan::BatchPlan(int device) : device_(device), tables_(new StageTables) {}

BatchPlan::~BatchPlan() {
    release_graph();
    if (arena_) dev_free(arena_);
    if (queue_) dev_free(queue_);
}

void BatchPlan::release_graph() {
    if (graph_) (void)cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
}

size_t BatchPlan::footprint(const BatchItem* items, int n) {
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
        const Bm3dConfig& c = *items[i].cfg;
        for (int p = 0; p < c.planes; ++p) {
            const int w = c.plane_w[p], h = c.plane_h[p];
            const size_t px = (size_t)pitch_of(w) * h;
            size_t jobs = 0, group = 0, cube = 0;
            for (const StageParams* sp : {&c.final_stage[p], &c.basic_stage[p]}) {
                jobs = std::max(jobs, (size_t)grid_count(w, sp->block, sp->step) * grid_count(h, sp->block, sp->step));
                group = std::max(group, (size_t)sp->group);
                cube = std::max(cube, group_filter_scratch_floats(sp->block, sp->group, true));
            }
            total += align_up(px * 4) * (2 + c.has_ref + c.two_stage) + align_up(px * 8) * 2 +
                     align_up(jobs * group * 4) + align_up(jobs * 4) + (cube ? align_up(cube * 4) : 0);
        }
    }
    return total;
}

std::string BatchPlan::signature_of(const BatchItem* items, int n) {
    std::ostringstream os;
    for (int i = 0; i < n; ++i) append_signature(os, *items[i].cfg);
    return os.str();
}

void BatchPlan::layout(const BatchItem* items, int n, cudaStream_t stream) {
    std::string sig = signature_of(items, n);
    if (arena_ && sig == sig_) {
        // the same layout: the arena stays, the stage lists point at this run's items
        bind(items, n);
        return;
    }
    NSSB_CUDA(cudaSetDevice(device_));
    NSSB_CUDA(cudaStreamSynchronize(stream));  // the arena's previous layout is done with
    release_graph();
    sig_.clear();
    planes_.clear();
    scratch_.clear();
    for (int s = 0; s < 2; ++s) {
        stage_[s].clear();
        prematch_[s].clear();
    }
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += align_up(bytes);
        return o;
    };
    for (int i = 0; i < n; ++i) {
        const Bm3dConfig& c = *items[i].cfg;
        for (int p = 0; p < c.planes; ++p) {
            Plane pl{};
            pl.item = i;
            pl.plane = p;
            pl.w = c.plane_w[p];
            pl.h = c.plane_h[p];
            pl.pitch = pitch_of(pl.w);
            const size_t px = (size_t)pl.pitch * pl.h;
            pl.in = take(px * 4);
            pl.refin = c.has_ref ? take(px * 4) : kNone;
            pl.basic = c.two_stage ? take(px * 4) : kNone;
            pl.out = take(px * 4);
            pl.num = take(px * 8);
            pl.wsum = take(px * 8);
            size_t jobs = 0, group = 0, cube = 0;
            for (const StageParams* sp : {&c.final_stage[p], &c.basic_stage[p]}) {
                jobs = std::max(jobs, (size_t)grid_count(pl.w, sp->block, sp->step) *
                                          grid_count(pl.h, sp->block, sp->step));
                group = std::max(group, (size_t)sp->group);
                cube = std::max(cube, group_filter_scratch_floats(sp->block, sp->group, true));
            }
            pl.pos = take(jobs * group * 4);
            pl.count = take(jobs * 4);
            pl.cube = cube ? take(cube * 4) : kNone;
            pl.cube_floats = cube;
            planes_.push_back(pl);
            StageScratch sc{};
            sc.jobs_cap = jobs;
            sc.group_cap = group;
            sc.cube_floats = cube;
            scratch_.push_back(sc);
        }
    }
    if (off > arena_cap_) {
        if (arena_) dev_free(arena_);
        arena_ = nullptr;
        arena_cap_ = 0;
        arena_ = static_cast<char*>(dev_alloc(off));
        arena_cap_ = off;
    }
    if (!queue_) {
        // bytes 0..3: the persistent matcher's tile counter; 64..: the tensor form's counters
        queue_ = static_cast<int*>(dev_alloc(256));
        NSSB_CUDA(cudaMemsetAsync(queue_, 0, 256, stream));
    }
    arena_bytes_ = off;
    // num must start at zero; every finish leaves it zero again
    NSSB_CUDA(cudaMemsetAsync(arena_, 0, off, stream));
    auto F = [&](size_t o) { return o == kNone ? nullptr : reinterpret_cast<float*>(arena_ + o); };
    for (size_t k = 0; k < planes_.size(); ++k) {
        const Plane& pl = planes_[k];
        scratch_[k].pos = reinterpret_cast<int32_t*>(arena_ + pl.pos);
        scratch_[k].count = reinterpret_cast<int32_t*>(arena_ + pl.count);
        scratch_[k].cube = F(pl.cube);
    }
    bind(items, n);
    sig_ = std::move(sig);
}

// The stage lists of the laid-out arena for these items: each plane's stage
// parameters are the item's own (items of equal signatures have equal
// values, but an earlier run's items may be gone).
void BatchPlan::bind(const BatchItem* items, int n) {
    for (int s = 0; s < 2; ++s) {
        stage_[s].clear();
        prematch_[s].clear();
    }
    auto F = [&](size_t o) { return o == kNone ? nullptr : reinterpret_cast<float*>(arena_ + o); };
    size_t k = 0;
    for (int i = 0; i < n; ++i) {
        const Bm3dConfig& c = *items[i].cfg;
        const size_t k0 = k;
        for (int p = 0; p < c.planes; ++p, ++k) {
            const Plane& pl = planes_[k];
            const AccPlane acc{reinterpret_cast<long long*>(arena_ + pl.num),
                               reinterpret_cast<long long*>(arena_ + pl.wsum), pl.pitch};
            const int32_t* spos = (c.chroma && p > 0) ? scratch_[k0].pos : nullptr;
            const int32_t* scnt = (c.chroma && p > 0) ? scratch_[k0].count : nullptr;
            if (has_stage_a(c)) {
                const StageParams* sp = c.two_stage ? &c.basic_stage[p] : &c.final_stage[p];
                stage_[0].push_back(StagePlane{sp, F(pl.in), pl.pitch, nullptr, 0, F(c.two_stage ? pl.basic : pl.out),
                                               pl.pitch, pl.w, pl.h, acc, &scratch_[k], spos, scnt});
                if (c.chroma && p == 0 && sp->sigma == 0.f) prematch_[0].push_back(PreMatch{sp, (int)k, false, pl.in});
            }
            if (has_stage_b(c)) {
                const size_t ref = c.two_stage ? pl.basic : pl.refin;
                stage_[1].push_back(StagePlane{&c.final_stage[p], F(pl.in), pl.pitch, F(ref), pl.pitch, F(pl.out),
                                               pl.pitch, pl.w, pl.h, acc, &scratch_[k], spos, scnt});
                if (c.chroma && p == 0 && c.final_stage[p].sigma == 0.f)
                    prematch_[1].push_back(PreMatch{&c.final_stage[p], (int)k, true, ref});
            }
        }
    }
}

void BatchPlan::upload(const BatchItem* items, int n, cudaStream_t s) {
    for (const Plane& pl : planes_) {
        const BatchItem& it = items[pl.item];
        const cudaMemcpyKind kind = it.memory == NSSB_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        NSSB_CUDA(cudaMemcpy2DAsync(arena_ + pl.in, pl.pitch * 4, it.clip->planes[pl.plane],
                                    it.clip->strides[pl.plane] * 4, pl.w * 4, pl.h, kind, s));
        if (pl.refin != kNone)
            NSSB_CUDA(cudaMemcpy2DAsync(arena_ + pl.refin, pl.pitch * 4, it.ref->planes[pl.plane],
                                        it.ref->strides[pl.plane] * 4, pl.w * 4, pl.h, kind, s));
    }
    (void)n;
}

void BatchPlan::download(const BatchItem* items, int n, cudaStream_t s) {
    for (const Plane& pl : planes_) {
        const BatchItem& it = items[pl.item];
        const cudaMemcpyKind kind = it.memory == NSSB_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        NSSB_CUDA(cudaMemcpy2DAsync(it.out->planes[pl.plane], it.out->strides[pl.plane] * 4, arena_ + pl.out,
                                    pl.pitch * 4, pl.w * 4, pl.h, kind, s));
    }
    (void)n;
}

void BatchPlan::compute(cudaStream_t s, const LaunchTunes& tunes, StageClock& clock) {
    LaunchTunes t = tunes;
    t.match.queue = queue_;
    t.match.tc = reinterpret_cast<TcCounters*>(queue_ + 16);
    for (int st = 0; st < 2; ++st) {
        for (const PreMatch& pm : prematch_[st]) {
            const Plane& pl = planes_[pm.plane];
            const StageParams& sp = *pm.sp;
            clock.count_match(pl.w, pl.h, sp);
            clock.begin(StageClock::kMatch);
            launch_match_spatial(reinterpret_cast<const float*>(arena_ + pm.src_off), pl.pitch, pl.w, pl.h, sp.block,
                                 sp.step, sp.bm_range, sp.group, scratch_[pm.plane].pos, nullptr,
                                 scratch_[pm.plane].count, s);
            clock.end(StageClock::kMatch);
        }
        if (!stage_[st].empty()) run_stage_planes(stage_[st].data(), (int)stage_[st].size(), s, t, clock, *tables_);
    }
}

namespace {
bool same_tunes(const LaunchTunes& a, const LaunchTunes& b) {
    return a.match.parts == b.match.parts && a.match.persistent == b.match.persistent && a.match.form == b.match.form &&
           a.group.warps == b.group.warps && a.group.ctas_per_sm == b.group.ctas_per_sm;
}
}  // namespace

void BatchPlan::compute_graph(cudaStream_t s, const LaunchTunes& tunes) {
    if (graph_ && !same_tunes(tunes, graph_tunes_)) release_graph();
    if (!graph_) {
        EventClock counter(s, false);
        cudaGraph_t g = nullptr;
        NSSB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        try {
            compute(s, tunes, counter);
        } catch (...) {
            (void)cudaStreamEndCapture(s, &g);
            if (g) (void)cudaGraphDestroy(g);
            throw;
        }
        NSSB_CUDA(cudaStreamEndCapture(s, &g));
        size_t nodes = 0;
        int64_t kernels = 0;
        if (cudaGraphGetNodes(g, nullptr, &nodes) == cudaSuccess && nodes > 0) {
            std::vector<cudaGraphNode_t> list(nodes);
            if (cudaGraphGetNodes(g, list.data(), &nodes) == cudaSuccess)
                for (size_t i = 0; i < nodes; ++i) {
                    cudaGraphNodeType type;
                    if (cudaGraphNodeGetType(list[i], &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) ++kernels;
                }
        }
        const cudaError_t e = cudaGraphInstantiate(&graph_, g, 0);
        (void)cudaGraphDestroy(g);
        NSSB_CUDA(e);
        launches_per_run_ = kernels;
        graph_tunes_ = tunes;
        ++graph_builds_;
    }
    NSSB_CUDA(cudaGraphLaunch(graph_, s));
}

// ---- engine ----

BatchEngine::BatchEngine(int device, const BatchOptions& opt) : device_(device), opt_(opt) {
    NSSB_CUDA(cudaSetDevice(device_));
    for (auto& st : streams_) NSSB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    NSSB_CUDA(cudaEventCreate(&t0_));
    for (auto& e : t1_) NSSB_CUDA(cudaEventCreate(&e));
    info_.match_parts = opt_.fixed.match.parts;
    info_.match_persistent = opt_.fixed.match.persistent;
    info_.match_form = opt_.fixed.match.form;
    info_.group_warps = opt_.fixed.group.warps;
    info_.group_ctas_per_sm = opt_.fixed.group.ctas_per_sm;
    info_.graphs = opt_.graphs ? 1 : 0;
}

BatchEngine::~BatchEngine() {
    for (auto& st : streams_)
        if (st) (void)cudaStreamSynchronize(st);
    plans_.clear();
    (void)cudaEventDestroy(t0_);
    for (auto& e : t1_) (void)cudaEventDestroy(e);
    for (auto& st : streams_)
        if (st) (void)cudaStreamDestroy(st);
}

// Times every candidate shape on the batch itself, twice (the first pass
// also pays each variant's first launch), and keeps the fastest of each
// kernel; the candidates compute identical results.
LaunchTunes BatchEngine::tune(BatchPlan& plan, cudaStream_t s) {
    const auto& mc = match_candidates();
    const auto& gc = group_candidates();
    const size_t trials = std::max(mc.size(), gc.size());
    std::vector<double> mt(mc.size(), 1e30), gt(gc.size(), 1e30);
    for (int pass = 0; pass < 2; ++pass) {
        for (size_t i = 0; i < trials; ++i) {
            LaunchTunes t;
            t.match = mc[i % mc.size()];
            t.group = gc[i % gc.size()];
            EventClock clock(s, true);
            plan.compute(s, t, clock);
            NSSB_CUDA(cudaStreamSynchronize(s));
            clock.collect();
            if (clock.launches[StageClock::kMatch] > 0) mt[i % mc.size()] = std::min(mt[i % mc.size()], clock.ms[0]);
            if (clock.launches[StageClock::kGroup] > 0) gt[i % gc.size()] = std::min(gt[i % gc.size()], clock.ms[1]);
        }
    }
    LaunchTunes best;
    best.match = mc[std::min_element(mt.begin(), mt.end()) - mt.begin()];
    best.group = gc[std::min_element(gt.begin(), gt.end()) - gt.begin()];
    ++info_.tunings;
    return best;
}

BatchPlan& BatchEngine::plan_for(const std::string& sig, int lane) {
    const std::string key = sig + "#" + std::to_string(lane);
    for (size_t i = 0; i < plans_.size(); ++i) {
        if (plans_[i].first == key) {
            if (i + 1 != plans_.size()) std::rotate(plans_.begin() + i, plans_.begin() + i + 1, plans_.end());
            return *plans_.back().second;
        }
    }
    if (plans_.size() >= kMaxPlans) {
        // the evicted plan may still be in flight earlier in this run
        for (auto& st : streams_) NSSB_CUDA(cudaStreamSynchronize(st));
        plans_.erase(plans_.begin());
    }
    plans_.emplace_back(key, std::make_unique<BatchPlan>(device_));
    return *plans_.back().second;
}

constexpr int kMaxChunks = 10, kMinChunkFrames = 3;

// Chunks of the batch: one when every item is on the device (nothing to
// overlap), else up to ten equal chunks so that the host copies of one
// chunk overlap the kernels of its neighbours.
std::vector<std::pair<int, int>> BatchEngine::chunks(const BatchItem* items, int n) const {
    bool host = false;
    for (int i = 0; i < n; ++i) host |= items[i].memory == NSSB_MEM_HOST;
    int size = n;
    if (opt_.chunk_frames > 0) {
        size = opt_.chunk_frames;
    } else if (host && n >= 2) {
        // up to kMaxChunks equal chunks of at least kMinChunkFrames frames: the
        // first upload and the last download are the only copies not hidden
        int k = 0;
        const int most = std::max(1, std::min(kMaxChunks, n / kMinChunkFrames));
        for (int c = most; c >= 2 && !k; --c)
            if (n % c == 0) k = c;
        if (!k) k = std::min(most, n);
        size = (n + k - 1) / k;
    }
    std::vector<std::pair<int, int>> out;
    for (int a = 0; a < n; a += size) out.emplace_back(a, std::min(size, n - a));
    return out;
}

void BatchEngine::run(const BatchItem* items, int n) {
    std::lock_guard<std::mutex> lock(mu_);
    if (n <= 0) return;
    for (int i = 0; i < n; ++i) {
        const BatchItem& it = items[i];
        if (!it.cfg || !it.clip || !it.out) throw std::invalid_argument("nssb_batch_run: item without node, clip or out");
        if (it.cfg->radius != 0) throw std::invalid_argument("nssb_batch_run: the batched form takes radius-0 filters");
        if (it.cfg->kaiser_beta != 0.f)
            throw std::invalid_argument("nssb_batch_run: a node with the Kaiser window renders per frame only");
        if (it.cfg->device_id != device_)
            throw std::invalid_argument("nssb_batch_run: node lives on another device than the batch");
        if (it.cfg->has_ref && !it.ref) throw std::invalid_argument("nssb_batch_run: ref frame missing");
        if (it.memory != NSSB_MEM_HOST && it.memory != NSSB_MEM_DEVICE)
            throw std::invalid_argument("nssb_batch_run: memory must be NSSB_MEM_HOST or NSSB_MEM_DEVICE");
    }
    NSSB_CUDA(cudaSetDevice(device_));
    const auto parts = chunks(items, n);
    int64_t launches = 0;
    LaunchTunes last{};
    bool started = false;
    try {
        for (size_t k = 0; k < parts.size(); ++k) {
            const int lane = (int)(k % kLanes);
            cudaStream_t s = streams_[lane];
            const BatchItem* c = items + parts[k].first;
            const int m = parts[k].second;
            BatchPlan& plan = plan_for(opt_.plan_per_stream ? std::string() : BatchPlan::signature_of(c, m), lane);
            plan.layout(c, m, s);
            LaunchTunes t = opt_.fixed;
            const bool need_tune = opt_.autotune && tuned_.find(plan.signature()) == tuned_.end();
            if (opt_.autotune && !need_tune) t = tuned_[plan.signature()];
            if (need_tune) {
                plan.upload(c, m, s);
                t = tuned_[plan.signature()] = tune(plan, s);
            }
            if (!started) {
                NSSB_CUDA(cudaEventRecord(t0_, streams_[0]));
                for (int l = 1; l < kLanes; ++l) NSSB_CUDA(cudaStreamWaitEvent(streams_[l], t0_, 0));
                started = true;
            }
            if (!need_tune) plan.upload(c, m, s);
            if (opt_.graphs) {
                plan.compute_graph(s, t);
                launches += plan.launches_per_run();
            } else {
                EventClock clock(s, false);
                plan.compute(s, t, clock);
                launches += clock.launches[0] + clock.launches[1] + clock.launches[2] + clock.launches[3];
            }
            plan.download(c, m, s);
            last = t;
        }
        for (int l = 0; l < kLanes; ++l) NSSB_CUDA(cudaEventRecord(t1_[l], streams_[l]));
        for (auto& st : streams_) NSSB_CUDA(cudaStreamSynchronize(st));
    } catch (...) {
        for (auto& st : streams_) (void)cudaStreamSynchronize(st);
        plans_.clear();  // sums may be left mid-stage: lay out afresh
        throw;
    }
    float ms = 0.f;
    for (int l = 0; l < kLanes; ++l) {
        float m = 0.f;
        NSSB_CUDA(cudaEventElapsedTime(&m, t0_, t1_[l]));
        ms = std::max(ms, m);
    }
    info_.last_run_ms = ms;
    info_.kernel_launches = launches;
    info_.chunks = (int)parts.size();
    info_.match_parts = last.match.parts;
    info_.match_persistent = last.match.persistent;
    info_.match_form = last.match.form;
    info_.group_warps = last.group.warps;
    info_.group_ctas_per_sm = last.group.ctas_per_sm;
    info_.runs += 1;
    info_.frames += n;
    int64_t builds = 0;
    size_t bytes = 0;
    for (const auto& p : plans_) {
        builds += p.second->graph_builds();
        bytes += p.second->arena_bytes();
    }
    info_.graph_builds = std::max(info_.graph_builds, builds);
    info_.arena_bytes = bytes;
}

void BatchEngine::info(nssb_batch_info* out) {
    std::lock_guard<std::mutex> lock(mu_);
    if (out) *out = info_;
}

}  // namespace nssb
