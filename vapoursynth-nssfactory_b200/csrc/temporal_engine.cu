// Temporal drivers of the engine (radius > 0).
//
// Output frame n sums the contributions of the centres c in [n-r, n+r]: each
// centre matches predictively over its 2r+1 slots (frames c-r..c+r clamped,
// temporal.hpp:19-21; valid slots filter_bm3d.cpp:95-97), filters its groups
// and adds every patch to the sums of the frame it came from. The reference
// reduces these per-centre slices in ascending centre order (VAggregate,
// agg.cpp:151-200); here the sums are fixed-point integers, so adding them
// straight into one accumulator per target frame gives the same value in any
// order.
//
// Rolling mode (the device default, finished frames): a ring of 2r+1 target
// accumulators per plane; centres run in ascending order and target m is
// complete once centre m+r has run, so frames rendered in order cost one
// centre each (the reference's rolling chunks with carry,
// group_driver.cpp:1207-1800). A request out of that order restarts the ring.
// Legacy mode: the fat intermediate of centre n, 2r+1 (num, den) slices
// (filter_bm3d.cpp:306-320). final=1 chains a rolling basic stage, whose
// finished frames are cached on the device, into the Wiener stage
// (bm3d_args.cpp:161-196: the basic stage is rolling when r > 0).
#include "engine.hpp"

#include <algorithm>
#include <functional>

namespace nssb {

namespace {

struct DevFrameSet {
    float* p[3]{};
    int64_t pitch[3]{};
    int index = -1;
};

__global__ void fill_ones_kernel(float* d, int64_t stride, int w, int h) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x < w && y < h) d[(int64_t)y * stride + x] = 1.f;
}

}  // namespace

// One temporal stage (hard threshold, or Wiener with per-frame references).
class TemporalStage {
public:
    // A new clip: nothing in the ring belongs to it.
    void invalidate() {
        for (int s = 0; s < kMaxSlots; ++s) target_[s] = -1;
        next_c_ = 0;
    }

    using Getter = std::function<void(int frame, const float* planes[3], int64_t strides[3])>;

    TemporalStage(const Bm3dConfig& cfg, const StageParams* sp, bool wiener, cudaStream_t stream,
                  const MatchTune* tune, StageClock* clock)
        : cfg_(cfg), sp_(sp), wiener_(wiener), r_(cfg.radius), slots_(2 * cfg.radius + 1), stream_(stream),
          tune_(tune), clock_(clock) {
        for (int p = 0; p < cfg_.planes; ++p) {
            const int w = cfg_.plane_w[p], h = cfg_.plane_h[p];
            pitch_[p] = (int64_t)((w + 31) / 32) * 32;
            for (int s = 0; s < slots_; ++s) {
                num_[p][s] = static_cast<long long*>(take((size_t)pitch_[p] * h * 8));
                wsum_[p][s] = static_cast<long long*>(take((size_t)pitch_[p] * h * 8));
            }
            const StageParams& st = sp_[p];
            const size_t jobs = (size_t)grid_count(w, st.block, st.step) * grid_count(h, st.block, st.step);
            pos_[p] = static_cast<int32_t*>(take(jobs * st.group * 4));
            slot_[p] = static_cast<int32_t*>(take(jobs * st.group * 4));
            dist_[p] = static_cast<float*>(take(jobs * st.group * 4));
            count_[p] = static_cast<int32_t*>(take(jobs * 4));
            cube_floats_[p] = group_filter_scratch_floats(st.block, st.group, wiener_);
            cube_[p] = cube_floats_[p] ? static_cast<float*>(take(cube_floats_[p] * 4)) : nullptr;
        }
        for (int s = 0; s < kMaxSlots; ++s) target_[s] = -1;
    }
    ~TemporalStage() {
        for (void* p : mem_) dev_free(p);
    }

    // Finished frame n into dst (device planes).
    void render(int n, const Getter& src, const Getter& ref, float* const dst[3], const int64_t dstride[3]) {
        const int N = cfg_.vi.num_frames;
        const int lo = std::max(0, n - r_), hi = std::min(N - 1, n + r_);
        const int sl = n % slots_;
        const bool ready = target_[sl] == n && first_[sl] == lo && last_[sl] == hi && !finished_[sl];
        if (!ready) {
            // carry on with the run in progress when target n is in it from its first centre
            const bool carry = target_[sl] == n && first_[sl] == lo && !finished_[sl] && next_c_ > lo &&
                               next_c_ <= hi + 1;
            if (!carry) restart(lo);
            while (next_c_ <= hi) process_centre(next_c_++, src, ref, false);
        }
        // finish: out = den > 1e-12 ? num / den : src (clears num)
        const float* sp[3];
        int64_t ss[3];
        src(n, sp, ss);
        FinishBatch& fb = fbatch_;
        fb.n = 0;
        fb.total_ctas = 0;
        fb.block = 0;
        for (int p = 0; p < cfg_.planes; ++p) {
            if (sp_[p].sigma == 0.f) {
                NSSB_CUDA(cudaMemcpy2DAsync(dst[p], dstride[p] * 4, sp[p], ss[p] * 4, cfg_.plane_w[p] * 4,
                                            cfg_.plane_h[p], cudaMemcpyDeviceToDevice, stream_));
                continue;
            }
            if (fb.n > 0 && sp_[p].block != fb.block) {
                clock_->begin(StageClock::kFinish);
                launch_finish_batch(fb, stream_);
                clock_->end(StageClock::kFinish);
                fb.n = 0;
                fb.total_ctas = 0;
            }
            fb.block = sp_[p].block;
            const int w = cfg_.plane_w[p], h = cfg_.plane_h[p];
            fb.p[fb.n++] = FinishPlane{num_[p][sl], wsum_[p][sl], pitch_[p], sp[p], ss[p], dst[p], dstride[p], w, h,
                                       finish_tiles_x(w), fb.total_ctas};
            fb.total_ctas += finish_tiles(w, h);
        }
        if (fb.n > 0) {
            clock_->begin(StageClock::kFinish);
            launch_finish_batch(fb, stream_);
            clock_->end(StageClock::kFinish);
        }
        finished_[sl] = true;
    }

    // Legacy fat intermediate of centre n: 2r+1 (num, den) slices per plane.
    void legacy(int n, const Getter& src, const Getter& ref, float* const dst[3], const int64_t dstride[3]) {
        for (int s = 0; s < slots_; ++s) {
            clear_slot(s);
            target_[s] = -1;
        }
        process_centre(n, src, ref, true);
        const float* sp[3];
        int64_t ss[3];
        src(n, sp, ss);
        for (int p = 0; p < cfg_.planes; ++p) {
            const int w = cfg_.plane_w[p], h = cfg_.plane_h[p];
            for (int t = 0; t < slots_; ++t) {
                float* dn = dst[p] + (int64_t)(2 * t) * h * dstride[p];
                float* dd = dst[p] + (int64_t)(2 * t + 1) * h * dstride[p];
                if (sp_[p].sigma == 0.f) {
                    // temporal_identity (temporal.hpp:24-35): slice r carries src with unit weight
                    if (t == r_) {
                        NSSB_CUDA(cudaMemcpy2DAsync(dn, dstride[p] * 4, sp[p], ss[p] * 4, w * 4, h,
                                                    cudaMemcpyDeviceToDevice, stream_));
                        fill_ones_kernel<<<dim3(ceil_div(w, 256), h), 256, 0, stream_>>>(dd, dstride[p], w, h);
                        NSSB_CUDA(cudaGetLastError());
                    } else {
                        NSSB_CUDA(cudaMemset2DAsync(dn, dstride[p] * 4, 0, w * 4, h, stream_));
                        NSSB_CUDA(cudaMemset2DAsync(dd, dstride[p] * 4, 0, w * 4, h, stream_));
                    }
                    continue;
                }
                launch_fat_slice(num_[p][t], wsum_[p][t], pitch_[p], dn, dd, dstride[p], w, h, sp_[p].block, stream_);
            }
        }
        // the slots hold one centre's slices now: a rolling request restarts
        for (int s = 0; s < slots_; ++s) target_[s] = -1;
    }

private:
    void* take(size_t bytes) {
        void* p = dev_alloc(bytes);
        mem_.push_back(p);
        return p;
    }

    void clear_slot(int s) {
        for (int p = 0; p < cfg_.planes; ++p) {
            const size_t bytes = (size_t)pitch_[p] * cfg_.plane_h[p] * 8;
            NSSB_CUDA(cudaMemsetAsync(num_[p][s], 0, bytes, stream_));
            NSSB_CUDA(cudaMemsetAsync(wsum_[p][s], 0, bytes, stream_));
        }
    }

    void enter_target(int m) {
        const int s = m % slots_;
        clear_slot(s);
        target_[s] = m;
        first_[s] = -1;
        last_[s] = -1;
        finished_[s] = false;
    }

    // A fresh run from centre c0: the targets it touches start from zero.
    void restart(int c0) {
        const int N = cfg_.vi.num_frames;
        for (int s = 0; s < slots_; ++s) target_[s] = -1;
        for (int m = std::max(0, c0 - r_); m <= std::min(N - 1, c0 + r_); ++m) enter_target(m);
        next_c_ = c0;
    }

    void process_centre(int c, const Getter& src, const Getter& ref, bool legacy) {
        const int N = cfg_.vi.num_frames;
        const int ntemp = slots_;
        const int vbegin = std::max(0, r_ - c), vend = r_ + std::min(r_ + 1, N - c);
        if (!legacy && c + r_ < N && target_[(c + r_) % slots_] != c + r_) enter_target(c + r_);
        const float* sp[kMaxSlots][3];
        const float* rp[kMaxSlots][3];
        int64_t ss[kMaxSlots][3], rs[kMaxSlots][3];
        for (int t = 0; t < ntemp; ++t) {
            const int f = c + std::clamp(t - r_, -c, N - 1 - c);
            src(f, sp[t], ss[t]);
            if (wiener_) ref(f, rp[t], rs[t]);
        }
        // the planes that match: every plane with a sigma, or plane 0 alone for
        // CBM3D (its groups serve every plane, filter_bm3d.cpp:451-486)
        int mpl[3], nm = 0;
        bool any = false;
        for (int p = 0; p < cfg_.planes; ++p) any |= sp_[p].sigma != 0.f;
        if (cfg_.chroma) {
            if (any) mpl[nm++] = 0;
        } else {
            for (int p = 0; p < cfg_.planes; ++p)
                if (sp_[p].sigma != 0.f) mpl[nm++] = p;
        }
        auto same_match = [&](const StageParams& a, const StageParams& b) {
            return a.block == b.block && a.step == b.step && a.bm_range == b.bm_range && a.group == b.group &&
                   a.ps_num == b.ps_num && a.ps_range == b.ps_range;
        };
        bool uniform = nm > 0;
        for (int q = 1; q < nm; ++q) uniform &= same_match(sp_[mpl[q]], sp_[mpl[0]]);
        TemporalPlanes tps[3]{};
        for (int q = 0; q < nm; ++q)
            for (int t = 0; t < ntemp; ++t) {
                tps[q].plane[t] = wiener_ ? rp[t][mpl[q]] : sp[t][mpl[q]];
                tps[q].stride[t] = wiener_ ? rs[t][mpl[q]] : ss[t][mpl[q]];
            }
        if (nm > 0) {
            clock_->begin(StageClock::kMatch);
            for (int q = 0; q < nm; ++q) clock_->count_match(cfg_.plane_w[mpl[q]], cfg_.plane_h[mpl[q]], sp_[mpl[q]]);
            // the centre frame: one batched launch over the planes when they share a shape
            bool done = false;
            const StageParams& m0 = sp_[mpl[0]];
            if (uniform && m0.block == 8) {
                mbatch_.n = nm;
                mbatch_.step = m0.step;
                for (int q = 0; q < nm; ++q) {
                    const int mp = mpl[q];
                    mbatch_.p[q] = MatchPlane{tps[q].plane[r_], tps[q].stride[r_], pos_[mp], dist_[mp], count_[mp],
                                              cfg_.plane_w[mp], cfg_.plane_h[mp], 0, 0, 0};
                }
                if (tune_ && tensor_matcher_takes(tune_->form, m0.bm_range, m0.step) && tune_->tc)
                    done = launch_match_tc_batch(mbatch_, m0.bm_range, m0.group, tune_->tc, stream_);
                if (!done) done = launch_match8_batch(mbatch_, m0.bm_range, m0.group, stream_);
            }
            if (!done)
                for (int q = 0; q < nm; ++q) {
                    const int mp = mpl[q];
                    const StageParams& ms = sp_[mp];
                    launch_match_spatial(tps[q].plane[r_], tps[q].stride[r_], cfg_.plane_w[mp], cfg_.plane_h[mp],
                                         ms.block, ms.step, ms.bm_range, ms.group, pos_[mp], dist_[mp], count_[mp],
                                         stream_);
                }
            // the temporal layers: one launch over the planes when the streaming kernel covers them
            done = false;
            if (uniform && m0.block == 8) {
                tbatch_.n = nm;
                tbatch_.ntemp = ntemp;
                tbatch_.t0 = r_;
                tbatch_.first = vbegin;
                tbatch_.last = vend;
                tbatch_.group = m0.group;
                tbatch_.ps_num = m0.ps_num;
                tbatch_.ps_range = m0.ps_range;
                for (int q = 0; q < nm; ++q) {
                    const int mp = mpl[q];
                    const int jobs = grid_count(cfg_.plane_w[mp], m0.block, m0.step) *
                                     grid_count(cfg_.plane_h[mp], m0.block, m0.step);
                    tbatch_.p[q] = TemporalBatchPlane{tps[q], cfg_.plane_w[mp], cfg_.plane_h[mp], jobs, 0,
                                                      pos_[mp], slot_[mp], dist_[mp], count_[mp]};
                }
                done = launch_match_temporal_batch(tbatch_, stream_);
            }
            if (!done)
                for (int q = 0; q < nm; ++q) {
                    const int mp = mpl[q];
                    const StageParams& ms = sp_[mp];
                    launch_match_temporal(tps[q], ntemp, r_, vbegin, vend, cfg_.plane_w[mp], cfg_.plane_h[mp],
                                          ms.block, ms.step, ms.group, ms.ps_num, ms.ps_range, pos_[mp], slot_[mp],
                                          dist_[mp], count_[mp], stream_);
                }
            clock_->end(StageClock::kMatch);
        }
        // group filtering into the target frames' sums
        gbatch_.n = 0;
        gbatch_.total_jobs = 0;
        bool batchable = true;
        int gshape = -1;
        for (int p = 0; p < cfg_.planes; ++p) {
            const StageParams& st = sp_[p];
            if (st.sigma == 0.f) continue;
            const int w = cfg_.plane_w[p], h = cfg_.plane_h[p];
            const int mp = cfg_.chroma ? 0 : p;
            GroupIO io{};
            const int64_t stride = ss[r_][p], rstride = wiener_ ? rs[r_][p] : 0;
            for (int t = 0; t < ntemp; ++t) {
                io.src[t] = sp[t][p];
                io.ref[t] = wiener_ ? rp[t][p] : nullptr;
                if (ss[t][p] != stride || (wiener_ && rs[t][p] != rstride))
                    throw std::invalid_argument("nss_cuda.BM3D: the frames of a temporal window must share strides");
                const int target = c + t - r_;
                const int s = legacy ? t : ((target >= 0 && target < N) ? target % slots_ : 0);
                io.num[t] = num_[p][s];
                io.wsum[t] = wsum_[p][s];
            }
            io.stride = stride;
            io.ref_stride = rstride;
            io.acc_stride = pitch_[p];
            const int jobs = grid_count(w, st.block, st.step) * grid_count(h, st.block, st.step);
            const bool fits = st.block == 8 && (st.group == 4 || st.group == 8 || st.group == 16 || st.group == 32) &&
                              (gshape < 0 || gshape == st.group);
            if (batchable && fits) {
                gshape = st.group;
                gbatch_.p[gbatch_.n++] = GroupSlotPlane{io, pos_[mp], slot_[mp], count_[mp], jobs,
                                                         gbatch_.total_jobs, st.sigma};
                gbatch_.total_jobs += jobs;
            } else {
                batchable = false;
                clock_->begin(StageClock::kGroup);
                launch_group_filter(io, w, h, pos_[mp], slot_[mp], count_[mp], jobs, st.block, st.group, st.sigma,
                                    wiener_, cube_[p], cube_floats_[p], stream_);
                clock_->end(StageClock::kGroup);
            }
        }
        if (gbatch_.n > 0) {
            clock_->begin(StageClock::kGroup);
            launch_group8_slots_batch(gbatch_, gshape, wiener_, stream_);
            clock_->end(StageClock::kGroup);
        }
        if (!legacy) {
            for (int m = std::max(0, c - r_); m <= std::min(N - 1, c + r_); ++m) {
                const int s = m % slots_;
                if (target_[s] != m) continue;
                if (first_[s] < 0) first_[s] = c;
                last_[s] = c;
            }
        }
    }

    const Bm3dConfig& cfg_;
    const StageParams* sp_;
    bool wiener_;
    int r_, slots_;
    cudaStream_t stream_;
    int64_t pitch_[3]{};
    long long* num_[3][kMaxSlots]{};
    long long* wsum_[3][kMaxSlots]{};
    int32_t *pos_[3]{}, *slot_[3]{}, *count_[3]{};
    float* dist_[3]{};
    float* cube_[3]{};
    size_t cube_floats_[3]{};
    int target_[kMaxSlots], first_[kMaxSlots]{}, last_[kMaxSlots]{};
    bool finished_[kMaxSlots]{};
    int next_c_ = 0;
    std::vector<void*> mem_;
    FinishBatch fbatch_;
    const MatchTune* tune_;  // the engine's matcher form (read at each centre)
    StageClock* clock_;      // the engine's launch accounting
    MatchBatch mbatch_;
    TemporalBatch tbatch_;
    GroupSlotBatch gbatch_;
};

// Device frames of the temporal window: host frames are uploaded once and kept
// while they stay inside the window (the reference's rolling chunk cache,
// gpuhost/chunk_cache.hpp).
class FrameCache {
public:
    FrameCache(const Bm3dConfig& cfg, int capacity, cudaStream_t stream) : cfg_(cfg), stream_(stream) {
        slots_.resize(capacity);
        for (auto& s : slots_) {
            for (int p = 0; p < cfg_.planes; ++p) {
                s.pitch[p] = (int64_t)((cfg_.plane_w[p] + 31) / 32) * 32;
                s.p[p] = static_cast<float*>(dev_alloc((size_t)s.pitch[p] * cfg_.plane_h[p] * 4));
            }
        }
    }
    ~FrameCache() {
        for (auto& s : slots_)
            for (int p = 0; p < cfg_.planes; ++p) dev_free(s.p[p]);
    }
    DevFrameSet* find(int idx) {
        for (auto& s : slots_)
            if (s.index == idx) return &s;
        return nullptr;
    }
    // a slot for idx: an empty one, else the frame farthest from `centre`
    DevFrameSet* claim(int idx, int centre) {
        DevFrameSet* best = nullptr;
        long far = -1;
        for (auto& s : slots_) {
            const long d = s.index < 0 ? (1L << 40) : std::abs((long)s.index - centre);
            if (d > far) {
                far = d;
                best = &s;
            }
        }
        best->index = idx;
        return best;
    }
    void invalidate() {
        for (auto& s : slots_) s.index = -1;
    }
    void upload(DevFrameSet* s, const nssb_frame& f) {
        for (int p = 0; p < cfg_.planes; ++p)
            NSSB_CUDA(cudaMemcpy2DAsync(s->p[p], s->pitch[p] * 4, f.planes[p], f.strides[p] * 4,
                                        cfg_.plane_w[p] * 4, cfg_.plane_h[p], cudaMemcpyHostToDevice, stream_));
    }

private:
    const Bm3dConfig& cfg_;
    cudaStream_t stream_;
    std::vector<DevFrameSet> slots_;
};

struct Engine::Plan {
    std::unique_ptr<TemporalStage> basic, final;
    std::unique_ptr<FrameCache> src_cache, ref_cache, basic_cache;
};

void Engine::PlanDeleter::operator()(Plan* p) const { delete p; }

void Engine::reset_clip(int num_frames) {
    std::lock_guard<std::mutex> lock(mu_);
    if (num_frames < 1) throw std::invalid_argument("nss_cuda.BM3D: a clip needs at least one frame");
    cfg_.vi.num_frames = num_frames;
    cfg_.out_vi.num_frames = num_frames;
    if (!plan_) return;
    for (TemporalStage* st : {plan_->basic.get(), plan_->final.get()})
        if (st) st->invalidate();
    for (FrameCache* c : {plan_->src_cache.get(), plan_->ref_cache.get(), plan_->basic_cache.get()})
        if (c) c->invalidate();
}

size_t Engine::footprint(const Bm3dConfig& cfg, bool host_frames) {
    auto px = [&](int p) { return (size_t)((cfg.plane_w[p] + 31) / 32 * 32) * cfg.plane_h[p]; };
    size_t total = 0, frame = 0, slot = 0;
    const int r = cfg.radius;
    for (int p = 0; p < cfg.planes; ++p) {
        frame += px(p) * 4;
        size_t jobs = 0, group = 0, cube = 0;
        for (const StageParams* sp : {&cfg.final_stage[p], &cfg.basic_stage[p]}) {
            jobs = std::max(jobs, (size_t)grid_count(cfg.plane_w[p], sp->block, sp->step) *
                                      grid_count(cfg.plane_h[p], sp->block, sp->step));
            group = std::max(group, (size_t)sp->group);
            cube = std::max(cube, group_filter_scratch_floats(sp->block, sp->group, true));
        }
        // per slot: in, refin, basic, out + num, wsum + pos, slot, dist, count, cube
        slot += px(p) * (4 * 4 + 2 * 8) + jobs * group * 12 + jobs * 4 + cube * 4;
        if (r > 0) {
            // per temporal stage: 2r+1 target sums + match lists
            const size_t stage = (2 * r + 1) * px(p) * 16 + jobs * group * 12 + jobs * 4 + cube * 4;
            total += stage * (cfg.two_stage ? 2 : 1);
        }
    }
    // radius 0 renders on num_streams slots, temporal frames on one
    total += slot * (size_t)(r > 0 ? 1 : std::max(1, cfg.num_streams));
    if (r > 0) {
        size_t frames = cfg.two_stage ? 2 * r + 2 : 0;
        if (host_frames) frames += 8 * r + 2 + (cfg.has_ref ? 4 * r + 2 : 0);
        total += frames * frame;
    }
    return total;
}

void Engine::temporal_frame(int n, const nssb_frame* clip, const nssb_frame* ref, int first, int count, int memory,
                            nssb_frame_out* out) {
    const int r = cfg_.radius;
    if (!plan_) {
        plan_.reset(new Plan());
        const bool wiener_final = cfg_.two_stage || cfg_.has_ref;
        plan_->final = std::make_unique<TemporalStage>(cfg_, cfg_.final_stage, wiener_final, stream_, &tunes_.match, clock_.get());
        if (cfg_.two_stage) {
            plan_->basic = std::make_unique<TemporalStage>(cfg_, cfg_.basic_stage, false, stream_, &tunes_.match, clock_.get());
            plan_->basic_cache = std::make_unique<FrameCache>(cfg_, 2 * r + 2, stream_);
        }
    }
    if (memory == NSSB_MEM_HOST && !plan_->src_cache) {
        plan_->src_cache = std::make_unique<FrameCache>(cfg_, 8 * r + 2, stream_);
        if (cfg_.has_ref) plan_->ref_cache = std::make_unique<FrameCache>(cfg_, 4 * r + 2, stream_);
    }
    auto window_frame = [&](const nssb_frame* frames, FrameCache* cache, int m, const float* planes[3],
                            int64_t strides[3]) {
        if (m < first || m >= first + count) throw std::out_of_range("nss_cuda.BM3D: a window frame is missing");
        const nssb_frame& f = frames[m - first];
        if (memory == NSSB_MEM_DEVICE) {
            for (int p = 0; p < cfg_.planes; ++p) {
                planes[p] = f.planes[p];
                strides[p] = f.strides[p];
            }
            return;
        }
        DevFrameSet* s = cache->find(m);
        if (!s) {
            s = cache->claim(m, n);
            cache->upload(s, f);
        }
        for (int p = 0; p < cfg_.planes; ++p) {
            planes[p] = s->p[p];
            strides[p] = s->pitch[p];
        }
    };
    TemporalStage::Getter src = [&](int m, const float* planes[3], int64_t strides[3]) {
        window_frame(clip, plan_->src_cache.get(), m, planes, strides);
    };
    TemporalStage::Getter refg = [&](int m, const float* planes[3], int64_t strides[3]) {
        window_frame(ref, plan_->ref_cache.get(), m, planes, strides);
    };
    TemporalStage::Getter basic_getter = [&](int m, const float* planes[3], int64_t strides[3]) {
        DevFrameSet* s = plan_->basic_cache->find(m);
        if (!s) {
            s = plan_->basic_cache->claim(m, m);
            float* dst[3] = {s->p[0], s->p[1], s->p[2]};
            plan_->basic->render(m, src, src, dst, s->pitch);
        }
        for (int p = 0; p < cfg_.planes; ++p) {
            planes[p] = s->p[p];
            strides[p] = s->pitch[p];
        }
    };
    const TemporalStage::Getter& final_ref = cfg_.two_stage ? basic_getter : refg;
    const bool host_out = memory == NSSB_MEM_HOST;
    float* dst[3]{};
    int64_t dstride[3]{};
    if (cfg_.rolling) {
        for (int p = 0; p < cfg_.planes; ++p) {
            dst[p] = host_out ? slots_[0]->out[p].p : out->planes[p];
            dstride[p] = host_out ? slots_[0]->out[p].pitch : out->strides[p];
        }
        plan_->final->render(n, src, final_ref, dst, dstride);
        if (host_out) {
            for (int p = 0; p < cfg_.planes; ++p)
                NSSB_CUDA(cudaMemcpy2DAsync(out->planes[p], out->strides[p] * 4, dst[p], dstride[p] * 4,
                                            cfg_.plane_w[p] * 4, cfg_.plane_h[p], cudaMemcpyDeviceToHost, stream_));
        }
        NSSB_CUDA(cudaStreamSynchronize(stream_));
        return;
    }
    // legacy: (2r+1) * 2 planes tall; staged on the device when the caller's planes are on the host
    std::vector<void*> tmp;
    for (int p = 0; p < cfg_.planes; ++p) {
        if (host_out) {
            dstride[p] = slots_[0]->out[p].pitch;
            dst[p] = static_cast<float*>(dev_alloc((size_t)dstride[p] * cfg_.plane_h[p] * (2 * r + 1) * 2 * 4));
            tmp.push_back(dst[p]);
        } else {
            dst[p] = out->planes[p];
            dstride[p] = out->strides[p];
        }
    }
    try {
        plan_->final->legacy(n, src, final_ref, dst, dstride);
        if (host_out) {
            for (int p = 0; p < cfg_.planes; ++p)
                NSSB_CUDA(cudaMemcpy2DAsync(out->planes[p], out->strides[p] * 4, dst[p], dstride[p] * 4,
                                            cfg_.plane_w[p] * 4, cfg_.plane_h[p] * (2 * r + 1) * 2,
                                            cudaMemcpyDeviceToHost, stream_));
        }
        NSSB_CUDA(cudaStreamSynchronize(stream_));
    } catch (...) {
        (void)cudaStreamSynchronize(stream_);
        for (void* p : tmp) dev_free(p);
        throw;
    }
    for (void* p : tmp) dev_free(p);
}

Engine::~Engine() {
    for (auto& s : slots_)
        if (s->stream) (void)cudaStreamSynchronize(s->stream);
    plan_.reset();
    release();
}

}  // namespace nssb
