// run_stage_planes (see stage.hpp).
#include "stage.hpp"

#include <algorithm>

namespace nssb {
namespace {

// wsum = 0 over every plane of a group batch: blockIdx.y is the plane, the
// x blocks stride over its rows, threads over 16-byte column pairs.
__global__ void clear_wsum_kernel(const __grid_constant__ GroupBatch gb) {
    const GroupPlane& P = gb.p[blockIdx.y];
    const int pairs = (P.W + 1) / 2;  // acc_stride is even (32-element pitch)
    for (int y = blockIdx.x; y < P.H; y += gridDim.x) {
        longlong2* row = reinterpret_cast<longlong2*>(P.wsum + (int64_t)y * P.acc_stride);
        for (int c = threadIdx.x; c < pairs; c += blockDim.x) row[c] = make_longlong2(0, 0);
    }
}

bool same_shape(const StagePlane& a, const StagePlane& b) {
    const StageParams &x = *a.sp, &y = *b.sp;
    return x.block == y.block && x.group == y.group && x.step == y.step && x.bm_range == y.bm_range &&
           (a.ref != nullptr) == (b.ref != nullptr) && a.win == b.win;
}

// One launch set over planes[set[0..ns)] (same shape, ns <= kMaxBatchPlanes).
void run_set(const StagePlane* planes, const int* set, int ns, cudaStream_t stream, const LaunchTunes& tunes,
             StageClock& clock, StageTables& t) {
    const StagePlane& first = planes[set[0]];
    const StageParams& sp = *first.sp;
    const bool wiener = first.ref != nullptr;
    // matching: the batched 8x8 kernel when the shape has it, else the generic one per plane
    MatchBatch& mb = t.match;
    mb.n = 0;
    mb.step = sp.step;
    // the 8x8 matcher zeroes the planes' origin weights while it runs when
    // every plane of the set is matched here (no plane borrowing another's
    // groups) and the weights allow 16-byte stores
    bool fuse_clear = true;
    for (int q = 0; q < ns; ++q) {
        const StagePlane& it = planes[set[q]];
        fuse_clear &= !it.shared_pos && (it.acc.pitch * it.h) % 2 == 0 &&
                      reinterpret_cast<uintptr_t>(it.acc.wsum) % 16 == 0;
    }
    for (int q = 0; q < ns; ++q) {
        const StagePlane& it = planes[set[q]];
        if (it.shared_pos) continue;
        MatchPlane m{wiener ? it.ref : it.src, wiener ? it.rstride : it.sstride, it.sc->pos, nullptr,
                     it.sc->count, it.w, it.h, 0, 0, 0};
        if (fuse_clear) {
            m.clear = it.acc.wsum;
            m.clear_words = it.acc.pitch * it.h;
        }
        mb.p[mb.n++] = m;
        clock.count_match(it.w, it.h, sp);
    }
    bool cleared = false;
    if (mb.n > 0) {
        bool ok = false;
        if (sp.block == 8) {
            clock.begin(StageClock::kMatch);
            if (tensor_matcher_takes(tunes.match.form, sp.bm_range, sp.step) && tunes.match.tc)
                ok = launch_match_tc_batch(mb, sp.bm_range, sp.group, tunes.match.tc, stream);
            if (!ok) cleared = ok = launch_match8_batch(mb, sp.bm_range, sp.group, stream, &tunes.match);
            clock.end(StageClock::kMatch);
        }
        if (!ok) {
            for (int q = 0; q < mb.n; ++q) {
                const MatchPlane& m = mb.p[q];
                clock.begin(StageClock::kMatch);
                launch_match_spatial(m.src, m.stride, m.W, m.H, sp.block, sp.step, sp.bm_range, sp.group, m.pos,
                                     nullptr, m.count, stream);
                clock.end(StageClock::kMatch);
            }
        }
    }
    // group filtering into cleared origin weights
    GroupBatch& gb = t.group;
    gb.n = 0;
    gb.total_jobs = 0;
    for (int q = 0; q < ns; ++q) {
        const StagePlane& it = planes[set[q]];
        const int jobs = grid_count(it.w, sp.block, sp.step) * grid_count(it.h, sp.block, sp.step);
        gb.p[gb.n++] = GroupPlane{it.src, it.ref, it.sstride, it.rstride, it.acc.num, it.acc.wsum, it.acc.pitch,
                                  it.shared_pos ? it.shared_pos : it.sc->pos,
                                  it.shared_count ? it.shared_count : it.sc->count, gb.total_jobs, jobs,
                                  it.sp->sigma, it.w, it.h, 0, it.win};
        gb.total_jobs += jobs;
    }
    if (!(cleared && fuse_clear)) {
        clock.begin(StageClock::kOther);
        // about four CTAs per SM over all planes of the set (rows grid-strided)
        clear_wsum_kernel<<<dim3(std::max(8, std::min(512, ceil_div(592, gb.n))), gb.n), 256, 0, stream>>>(gb);
        NSSB_CUDA(cudaGetLastError());
        clock.end(StageClock::kOther);
    }
    bool gok = false;
    if (sp.block == 8) {
        clock.begin(StageClock::kGroup);
        gok = launch_group8_batch(gb, sp.group, wiener, stream, &tunes.group);
        clock.end(StageClock::kGroup);
    }
    if (!gok) {
        for (int q = 0; q < gb.n; ++q) {
            const GroupPlane& g = gb.p[q];
            const StagePlane& it = planes[set[q]];
            GroupIO io{};
            io.src[0] = g.src;
            io.ref[0] = g.ref;
            io.stride = g.stride;
            io.ref_stride = g.ref_stride;
            io.num[0] = g.num;
            io.wsum[0] = g.wsum;
            io.acc_stride = g.acc_stride;
            io.win = g.win;
            clock.begin(StageClock::kGroup);
            launch_group_filter(io, it.w, it.h, g.pos, nullptr, g.count, g.njobs, sp.block, sp.group, g.sigma,
                                wiener, it.sc->cube, it.sc->cube_floats, stream);
            clock.end(StageClock::kGroup);
        }
    }
    // finish (clears num)
    FinishBatch& fb = t.finish;
    fb.n = 0;
    fb.block = first.win ? 1 : sp.block;  // windowed: wsum already holds each pixel's den
    fb.total_ctas = 0;
    for (int q = 0; q < ns; ++q) {
        const StagePlane& it = planes[set[q]];
        fb.p[fb.n++] = FinishPlane{it.acc.num, it.acc.wsum, it.acc.pitch, it.src, it.sstride, it.dst, it.dstride,
                                   it.w, it.h, finish_tiles_x(it.w), fb.total_ctas};
        fb.total_ctas += finish_tiles(it.w, it.h);
    }
    clock.begin(StageClock::kFinish);
    launch_finish_batch(fb, stream);
    clock.end(StageClock::kFinish);
}

}  // namespace

double match_pairs(int w, int h, const StageParams& sp) {
    auto axis = [&](int extent) {
        const int n = grid_count(extent, sp.block, sp.step);
        double sum = 0;
        for (int i = 0; i < n; ++i) {
            const int c = grid_pos(i, extent, sp.block, sp.step);
            sum += std::min(c + sp.bm_range, extent - sp.block) - std::max(c - sp.bm_range, 0) + 1;
        }
        return std::make_pair(sum, (double)n);
    };
    const auto ax = axis(w), ay = axis(h);
    return ax.first * ay.first - ax.second * ay.second;
}

void run_stage_planes(const StagePlane* planes, int n, cudaStream_t stream, const LaunchTunes& tunes,
                      StageClock& clock, StageTables& tables) {
    std::vector<int> live;
    live.reserve(n);
    for (int i = 0; i < n; ++i) {
        const StagePlane& it = planes[i];
        if (it.sp->sigma == 0.f) {
            NSSB_CUDA(cudaMemcpy2DAsync(it.dst, it.dstride * sizeof(float), it.src, it.sstride * sizeof(float),
                                        it.w * sizeof(float), it.h, cudaMemcpyDeviceToDevice, stream));
        } else {
            live.push_back(i);
        }
    }
    std::vector<char> done(live.size(), 0);
    std::vector<int> set;
    for (size_t a = 0; a < live.size(); ++a) {
        if (done[a]) continue;
        set.clear();
        for (size_t b = a; b < live.size(); ++b) {
            if (!done[b] && same_shape(planes[live[b]], planes[live[a]])) {
                set.push_back(live[b]);
                done[b] = 1;
            }
        }
        for (size_t s0 = 0; s0 < set.size(); s0 += kMaxBatchPlanes) {
            const int ns = (int)std::min(set.size() - s0, (size_t)kMaxBatchPlanes);
            run_set(planes, set.data() + s0, ns, stream, tunes, clock, tables);
        }
    }
}

}  // namespace nssb
