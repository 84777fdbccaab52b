// Host engine (see engine.hpp). Radius-0 frames run the stages per plane on
// device-resident copies; the temporal drivers live in temporal_engine.cu.
#include "engine.hpp"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <cstring>
#include <vector>

namespace nssb {

namespace {

// The library's device memory: one stream-ordered pool per device that keeps
// what is freed (release threshold: unlimited), served on a private stream.
// Creating and destroying engines then neither blocks on cudaMalloc's device
// synchronisation nor stalls other streams the way cudaFree does.
struct DevicePool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
};

DevicePool& device_pool(int dev) {
    static std::mutex mu;
    static std::map<int, DevicePool> pools;
    std::lock_guard<std::mutex> lock(mu);
    DevicePool& d = pools[dev];
    if (!d.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        NSSB_CUDA(cudaMemPoolCreate(&d.pool, &props));
        uint64_t keep = ~0ull;
        NSSB_CUDA(cudaMemPoolSetAttribute(d.pool, cudaMemPoolAttrReleaseThreshold, &keep));
        NSSB_CUDA(cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking));
    }
    return d;
}

}  // namespace

// Memory from dev_alloc is ready for any stream when it returns. dev_free
// requires that no queued work still uses the block (callers synchronise
// their streams first).
void* dev_alloc(size_t bytes) {
    void* p = nullptr;
    if (bytes == 0) return nullptr;
    int dev = 0;
    NSSB_CUDA(cudaGetDevice(&dev));
    DevicePool& d = device_pool(dev);
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, d.pool, d.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d.stream);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        throw std::bad_alloc();
    }
    return p;
}

void dev_free(void* p) {
    if (!p) return;
    cudaPointerAttributes attr{};
    int dev = 0;
    if (cudaPointerGetAttributes(&attr, p) == cudaSuccess) dev = attr.device;
    (void)cudaGetLastError();
    (void)cudaFreeAsync(p, device_pool(dev).stream);
}

void dev_pool_trim(int dev) {
    DevicePool& d = device_pool(dev);
    NSSB_CUDA(cudaStreamSynchronize(d.stream));  // frees queued on the pool's stream have landed
    NSSB_CUDA(cudaMemPoolTrimTo(d.pool, 0));
}

namespace {

int64_t pitch_of(int w) { return (int64_t)((w + 31) / 32) * 32; }

}  // namespace

Engine::Engine(const Bm3dConfig& cfg) : cfg_(cfg) {
    device_ = cfg.device_id;
    NSSB_CUDA(cudaSetDevice(device_));
    // radius 0: num_streams slots; temporal: one (its rolling state is sequential)
    const int n = cfg_.radius > 0 ? 1 : std::max(1, cfg_.num_streams);
    for (int i = 0; i < n; ++i) slots_.emplace_back(new Slot());
    try {
        for (auto& s : slots_) NSSB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        stream_ = slots_[0]->stream;
        clock_.reset(new Clock(this, slots_[0].get()));
        alloc();
    } catch (...) {
        release();
        throw;
    }
}

void Engine::release() {
    for (auto& s : slots_) {
        if (!s->stream) continue;
        (void)cudaStreamSynchronize(s->stream);  // nothing queued may still use the buffers
        for (auto& e : s->events) {
            (void)cudaEventDestroy(e.first);
            (void)cudaEventDestroy(e.second);
        }
        s->events.clear();
    }
    for (void* p : allocations_) dev_free(p);
    allocations_.clear();
    for (auto& s : slots_) {
        if (s->stream) (void)cudaStreamDestroy(s->stream);
        s->stream = nullptr;
    }
    stream_ = nullptr;
}

Engine::Slot* Engine::lease(bool primary) {
    std::unique_lock<std::mutex> lock(slot_mu_);
    for (;;) {
        for (size_t i = 0; i < slots_.size(); ++i) {
            Slot* s = slots_[i].get();
            if (!s->busy && (!primary || i == 0)) {
                s->busy = true;
                return s;
            }
        }
        slot_cv_.wait(lock);
    }
}

void Engine::give_back(Slot* s) {
    {
        std::lock_guard<std::mutex> lock(slot_mu_);
        s->busy = false;
    }
    slot_cv_.notify_all();
}

void Engine::alloc() {
    for (auto& s : slots_) alloc_slot(*s);
    // the automatic matcher form (the default) may take the precision form: its counters
    auto* c = static_cast<TcCounters*>(dev_alloc(sizeof(TcCounters)));
    allocations_.push_back(c);
    NSSB_CUDA(cudaMemsetAsync(c, 0, sizeof(TcCounters), stream_));
    NSSB_CUDA(cudaStreamSynchronize(stream_));
    tunes_.match.tc = c;
    tunes_.match.form = 2;
}

void Engine::alloc_slot(Slot& s) {
    auto take = [&](size_t bytes) {
        void* p = dev_alloc(bytes);
        allocations_.push_back(p);
        return p;
    };
    for (int p = 0; p < cfg_.planes; ++p) {
        const int w = cfg_.plane_w[p], h = cfg_.plane_h[p];
        const int64_t pitch = pitch_of(w);
        for (DevPlane* d : {&s.in[p], &s.refin[p], &s.basic[p], &s.out[p]}) {
            d->p = static_cast<float*>(take((size_t)pitch * h * sizeof(float)));
            d->pitch = pitch;
            d->w = w;
            d->h = h;
        }
        // num stays zero between stages: every finish clears what it consumed
        s.acc[p].pitch = pitch;
        s.acc[p].num = static_cast<long long*>(take((size_t)pitch * h * sizeof(long long)));
        s.acc[p].wsum = static_cast<long long*>(take((size_t)pitch * h * sizeof(long long)));
        NSSB_CUDA(cudaMemsetAsync(s.acc[p].num, 0, (size_t)pitch * h * sizeof(long long), s.stream));
        size_t jobs = 0, group = 0, cube = 0;
        for (const StageParams* sp : {&cfg_.final_stage[p], &cfg_.basic_stage[p]}) {
            jobs = std::max(jobs, (size_t)grid_count(w, sp->block, sp->step) * grid_count(h, sp->block, sp->step));
            group = std::max(group, (size_t)sp->group);
            cube = std::max(cube, group_filter_scratch_floats(sp->block, sp->group, true));
        }
        StageScratch& sc = s.scratch[p];
        sc.jobs_cap = jobs;
        sc.group_cap = group;
        sc.pos = static_cast<int32_t*>(take(jobs * group * sizeof(int32_t)));
        sc.slot = static_cast<int32_t*>(take(jobs * group * sizeof(int32_t)));
        sc.dist = static_cast<float*>(take(jobs * group * sizeof(float)));
        sc.count = static_cast<int32_t*>(take(jobs * sizeof(int32_t)));
        sc.cube_floats = cube;
        if (cube) sc.cube = static_cast<float*>(take(cube * sizeof(float)));
    }
}

void Engine::frame_window(int n, int* first, int* last) const {
    // The arInitial requests of getFrame: a rolling stage needs the windows of
    // the centres n-r..n+r, final=1 those of the basic frames behind them.
    const int r = cfg_.radius;
    const int reach = r == 0 ? 0 : cfg_.rolling ? (cfg_.two_stage ? 4 * r : 2 * r) : (cfg_.two_stage ? 3 * r : r);
    *first = std::max(0, n - reach);
    *last = std::min(cfg_.vi.num_frames - 1, n + reach);
}

const float* Engine::device_input(Slot& s, int plane, const nssb_frame* frames, int first, int n, int memory,
                                  bool is_ref, int64_t* stride) {
    const nssb_frame& f = frames[n - first];
    if (memory == NSSB_MEM_DEVICE) {
        *stride = f.strides[plane];
        return f.planes[plane];
    }
    DevPlane& d = is_ref ? s.refin[plane] : s.in[plane];
    NSSB_CUDA(cudaMemcpy2DAsync(d.p, d.pitch * sizeof(float), f.planes[plane], f.strides[plane] * sizeof(float),
                                d.w * sizeof(float), d.h, cudaMemcpyHostToDevice, s.stream));
    *stride = d.pitch;
    return d.p;
}

void Engine::clock_begin(Slot& s, Kind) {
    bool timing;
    {
        std::lock_guard<std::mutex> lock(stats_mu_);
        timing = timing_;
    }
    if (!timing) return;
    const size_t i = s.pending.size();
    if (i >= s.events.size()) {
        cudaEvent_t a, b;
        NSSB_CUDA(cudaEventCreate(&a));
        NSSB_CUDA(cudaEventCreate(&b));
        s.events.emplace_back(a, b);
    }
    NSSB_CUDA(cudaEventRecord(s.events[i].first, s.stream));
    s.pending.emplace_back(-1, i);  // open until clock_end names its kind
}

void Engine::clock_end(Slot& s, Kind kind) {
    if (!s.pending.empty() && s.pending.back().first < 0) {
        NSSB_CUDA(cudaEventRecord(s.events[s.pending.back().second].second, s.stream));
        s.pending.back().first = (int)kind;
    }
    std::lock_guard<std::mutex> lock(stats_mu_);
    ++stats_.launches;
    if (kind == kMatch) ++stats_.match_launches;
    if (kind == kGroup) ++stats_.group_launches;
    if (kind == kFinish) ++stats_.finish_launches;
}

// After the slot's stream is synchronised: add the bracketed durations.
void Engine::collect_timing(Slot& s) {
    double ms_by_kind[3] = {0, 0, 0};
    for (const auto& p : s.pending) {
        if (p.first < 0 || p.first > 2) continue;
        float ms = 0.f;
        NSSB_CUDA(cudaEventElapsedTime(&ms, s.events[p.second].first, s.events[p.second].second));
        ms_by_kind[p.first] += ms;
    }
    s.pending.clear();
    std::lock_guard<std::mutex> lock(stats_mu_);
    stats_.match_ms += ms_by_kind[kMatch];
    stats_.group_ms += ms_by_kind[kGroup];
    stats_.finish_ms += ms_by_kind[kFinish];
}

// Algorithmic work of one matching launch: every reference against every
// other position of its clamped window, 3 * B^2 flops per pair.
void Engine::count_match(int w, int h, const StageParams& sp) {
    const double pairs = match_pairs(w, h, sp);
    std::lock_guard<std::mutex> lock(stats_mu_);
    stats_.match_pairs += pairs;
    stats_.match_flops += pairs * 3.0 * sp.block * sp.block;
}

void Engine::set_matcher(int form) {
    std::lock_guard<std::mutex> lock(mu_);
    // every slot idle: no frame may be reading the tunes
    std::vector<Slot*> held;
    for (size_t i = 0; i < slots_.size(); ++i) held.push_back(lease(false));
    if (form != 0 && !tunes_.match.tc) {
        auto* c = static_cast<TcCounters*>(dev_alloc(sizeof(TcCounters)));
        allocations_.push_back(c);
        NSSB_CUDA(cudaMemsetAsync(c, 0, sizeof(TcCounters), stream_));
        NSSB_CUDA(cudaStreamSynchronize(stream_));
        tunes_.match.tc = c;
    }
    tunes_.match.form = form;
    for (Slot* s : held) give_back(s);
}

void Engine::stats(int enable_timing, int reset, nssb_kernel_stats* out) {
    std::lock_guard<std::mutex> lock(stats_mu_);
    if (tunes_.match.tc) {
        // every slot's precision-form kernels add to the counters
        for (auto& s : slots_) NSSB_CUDA(cudaStreamSynchronize(s->stream));
        TcCounters c{};
        NSSB_CUDA(cudaMemcpyAsync(&c, tunes_.match.tc, sizeof c, cudaMemcpyDeviceToHost, stream_));
        NSSB_CUDA(cudaStreamSynchronize(stream_));
        stats_.tc_survivors = (int64_t)c.survivors;
        stats_.tc_refs = (int64_t)c.refs;
        float r;
        std::memcpy(&r, &c.max_ratio_bits, 4);
        stats_.tc_max_error_ratio = r;
        if (reset) NSSB_CUDA(cudaMemsetAsync(tunes_.match.tc, 0, sizeof(TcCounters), stream_));
    }
    if (out) *out = stats_;
    if (reset) stats_ = nssb_kernel_stats{};
    timing_ = enable_timing != 0;
}

namespace {

// Modified Bessel function of the first kind, order 0, by its power series
// sum_k ((x/2)^k / k!)^2 (terms added until they fall below 1e-17 of the sum).
double bessel_i0(double x) {
    double term = 1.0, sum = 1.0;
    int k = 1;
    while (term > 1e-17 * sum) {
        const double y = x / (2.0 * k);
        term *= y * y;
        sum += term;
        ++k;
    }
    return sum;
}

// The separable n x n Kaiser window: w(i) = I0(beta sqrt(1 - r_i^2)) / I0(beta),
// r_i = 2i/(n-1) - 1, and win(i, j) = w(i) w(j) rounded to float.
std::vector<float> kaiser_window(int n, double beta) {
    std::vector<double> w1(n, 1.0);
    if (n > 1) {
        for (int i = 0; i < n; ++i) {
            const double r = 2.0 * i / (n - 1) - 1.0;
            w1[i] = bessel_i0(beta * std::sqrt(std::max(0.0, 1.0 - r * r))) / bessel_i0(beta);
        }
    }
    std::vector<float> w((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) w[(size_t)i * n + j] = (float)(w1[i] * w1[j]);
    return w;
}

}  // namespace

void Engine::set_window(float beta) {
    if (!(beta >= 0.f) || !std::isfinite(beta))
        throw std::invalid_argument("nss_cuda.BM3D: the Kaiser window's beta must be finite and non-negative");
    if (beta > 0.f && cfg_.radius > 0)
        throw std::invalid_argument("nss_cuda.BM3D: the Kaiser window applies to radius-0 filters");
    std::lock_guard<std::mutex> lock(mu_);
    std::vector<Slot*> held;  // every slot idle: no frame may be reading the windows
    for (size_t i = 0; i < slots_.size(); ++i) held.push_back(lease(false));
    struct Back {
        Engine* e;
        std::vector<Slot*>& h;
        ~Back() {
            for (Slot* s : h) e->give_back(s);
        }
    } back{this, held};
    windows_.clear();  // the old tables stay allocated until the engine goes
    if (beta > 0.f) {
        for (int p = 0; p < cfg_.planes; ++p) {
            for (const StageParams* sp : {&cfg_.final_stage[p], &cfg_.basic_stage[p]}) {
                const int b = sp->block;
                if (windows_.count(b)) continue;
                const std::vector<float> w = kaiser_window(b, beta);
                auto* d = static_cast<float*>(dev_alloc(w.size() * sizeof(float)));
                allocations_.push_back(d);
                NSSB_CUDA(cudaMemcpy(d, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
                windows_[b] = d;
            }
        }
    }
    cfg_.kaiser_beta = beta;
}

// One stage over the planes of a frame (radius 0), one launch per kernel and shape.
void Engine::run_stage(Slot& s, StageItem* items, int n) {
    StagePlane planes[3];
    for (int i = 0; i < n; ++i) {
        const StageItem& it = items[i];
        planes[i] = StagePlane{it.sp, it.src, it.sstride, it.ref, it.rstride, it.dst, it.dstride,
                               cfg_.plane_w[it.plane], cfg_.plane_h[it.plane], s.acc[it.plane], &s.scratch[it.plane],
                               it.shared_pos, it.shared_count};
        if (!windows_.empty()) planes[i].win = windows_.at(it.sp->block);
    }
    Clock clock(this, &s);
    run_stage_planes(planes, n, s.stream, tunes_, clock, s.tables);
}

void Engine::spatial_frame(Slot& s, int n, const nssb_frame* clip, const nssb_frame* ref, int first, int memory) {
    const float* src[3]{};
    const float* rp[3]{};
    int64_t ss[3]{}, rs[3]{};
    for (int p = 0; p < cfg_.planes; ++p) {
        src[p] = device_input(s, p, clip, first, n, memory, false, &ss[p]);
        if (cfg_.has_ref) rp[p] = device_input(s, p, ref, first, n, memory, true, &rs[p]);
    }
    StageItem items[3];
    const int np = cfg_.planes;
    // CBM3D (filter_bm3d.cpp:451-486): plane 0's groups serve every plane; a
    // plane-0 sigma of 0 still matches (on plane 0) for the others.
    auto chroma_link = [&](const StageParams* sps, bool wiener) {
        if (!cfg_.chroma) return;
        if (sps[0].sigma == 0.f) {
            const StageParams& s0 = sps[0];
            const int w = cfg_.plane_w[0], h = cfg_.plane_h[0];
            StageScratch& sc = s.scratch[0];
            timed(s, kMatch, [&] {
                launch_match_spatial(wiener ? items[0].ref : items[0].src, wiener ? items[0].rstride : items[0].sstride,
                                     w, h, s0.block, s0.step, s0.bm_range, s0.group, sc.pos, sc.dist, sc.count,
                                     s.stream);
            });
        }
        for (int p = 1; p < np; ++p) {
            items[p].shared_pos = s.scratch[0].pos;
            items[p].shared_count = s.scratch[0].count;
        }
    };
    if (cfg_.two_stage) {
        for (int p = 0; p < np; ++p)
            items[p] = StageItem{p, &cfg_.basic_stage[p], src[p], ss[p], nullptr, 0, s.basic[p].p, s.basic[p].pitch};
        chroma_link(cfg_.basic_stage, false);
        run_stage(s, items, np);
        for (int p = 0; p < np; ++p)
            items[p] = StageItem{p, &cfg_.final_stage[p], src[p], ss[p], s.basic[p].p, s.basic[p].pitch, s.out[p].p,
                                 s.out[p].pitch};
        chroma_link(cfg_.final_stage, true);
        run_stage(s, items, np);
    } else {
        for (int p = 0; p < np; ++p)
            items[p] = StageItem{p, &cfg_.final_stage[p], src[p], ss[p], cfg_.has_ref ? rp[p] : nullptr, rs[p],
                                 s.out[p].p, s.out[p].pitch};
        chroma_link(cfg_.final_stage, cfg_.has_ref);
        run_stage(s, items, np);
    }
}

void Engine::get_frame(int n, const nssb_frame* clip, const nssb_frame* ref, int first, int count, int memory,
                       nssb_frame_out* out) {
    NSSB_CUDA(cudaSetDevice(device_));
    if (n < 0 || n >= cfg_.vi.num_frames) throw std::out_of_range("nss_cuda.BM3D: frame number out of range");
    int wf = 0, wl = 0;
    frame_window(n, &wf, &wl);
    if (first > wf || first + count - 1 < wl) throw std::out_of_range("nss_cuda.BM3D: input frames do not cover the window");
    if (cfg_.has_ref && !ref) throw std::invalid_argument("nss_cuda.BM3D: ref frames missing");
    if (cfg_.radius > 0) {
        std::lock_guard<std::mutex> lock(mu_);
        Slot* s = lease(true);
        struct Back {
            Engine* e;
            Slot* s;
            ~Back() { e->give_back(s); }
        } back{this, s};
        temporal_frame(n, clip, ref, first, count, memory, out);
        collect_timing(*s);
        return;
    }
    // radius 0: any free slot; frames on different slots overlap
    Slot* s = lease(false);
    struct Back {
        Engine* e;
        Slot* s;
        ~Back() {
            (void)cudaStreamSynchronize(s->stream);  // an error path leaves nothing queued on the slot
            e->give_back(s);
        }
    } back{this, s};
    spatial_frame(*s, n, clip, ref, first, memory);
    for (int p = 0; p < cfg_.planes; ++p) {
        const DevPlane& o = s->out[p];
        NSSB_CUDA(cudaMemcpy2DAsync(out->planes[p], out->strides[p] * sizeof(float), o.p, o.pitch * sizeof(float),
                                    o.w * sizeof(float), o.h,
                                    memory == NSSB_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                    s->stream));
    }
    NSSB_CUDA(cudaStreamSynchronize(s->stream));
    collect_timing(*s);
}

void Engine::plane_stage(const float* src, const float* ref, float* dst, int64_t stride, int w, int h,
                         const StageParams& sp, cudaStream_t stream) {
    if (sp.sigma == 0.f) {
        NSSB_CUDA(cudaMemcpy2DAsync(dst, stride * 4, src, stride * 4, w * 4, h, cudaMemcpyDeviceToDevice, stream));
        return;
    }
    const size_t jobs = (size_t)grid_count(w, sp.block, sp.step) * grid_count(h, sp.block, sp.step);
    const size_t cube = group_filter_scratch_floats(sp.block, sp.group, ref != nullptr);
    int32_t *pos = nullptr, *count = nullptr;
    float* dist = nullptr;
    long long *num = nullptr, *wsum = nullptr;
    float* cubes = nullptr;
    const size_t plane = (size_t)stride * h;
    NSSB_CUDA(cudaMallocAsync(&pos, jobs * sp.group * 4, stream));
    NSSB_CUDA(cudaMallocAsync(&dist, jobs * sp.group * 4, stream));
    NSSB_CUDA(cudaMallocAsync(&count, jobs * 4, stream));
    NSSB_CUDA(cudaMallocAsync(&num, plane * 8, stream));
    NSSB_CUDA(cudaMallocAsync(&wsum, plane * 8, stream));
    if (cube) NSSB_CUDA(cudaMallocAsync(&cubes, cube * 4, stream));
    launch_match_spatial(ref ? ref : src, stride, w, h, sp.block, sp.step, sp.bm_range, sp.group, pos, dist, count,
                         stream);
    NSSB_CUDA(cudaMemsetAsync(num, 0, plane * 8, stream));
    NSSB_CUDA(cudaMemsetAsync(wsum, 0, plane * 8, stream));
    GroupIO io{};
    io.src[0] = src;
    io.ref[0] = ref;
    io.stride = stride;
    io.ref_stride = stride;
    io.num[0] = num;
    io.wsum[0] = wsum;
    io.acc_stride = stride;
    launch_group_filter(io, w, h, pos, nullptr, count, (int)jobs, sp.block, sp.group, sp.sigma, ref != nullptr, cubes,
                        cube, stream);
    launch_finish(num, wsum, stride, src, stride, dst, stride, w, h, sp.block, stream);
    for (void* p : {(void*)pos, (void*)dist, (void*)count, (void*)num, (void*)wsum, (void*)cubes})
        if (p) NSSB_CUDA(cudaFreeAsync(p, stream));
}

}  // namespace nssb
