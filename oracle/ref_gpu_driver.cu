// Test and benchmark infrastructure, never part of the product: drives the
// reference's OWN CUDA BM3D kernels, compiled unchanged from the reference
// tree for sm_100a (make -C oracle refgpu -> _ref/libref_bm3d_gpu.so), the
// way its per-frame driver does for one plane of one radius-0 stage
// (filter_center, src/cuda/common/group_driver.cpp:760-856, with the
// filter launch of src/cuda/bm3d/filter.cpp:86-111):
//
//   fixed_clear -> spatial matching (column / square / tensor / window / lane
//   kernels, chosen by the reference's own predicates) -> bm3d_filter_groups
//   -> fixed_finish (or the ordered aggregator + aggregate_finish for the
//   shapes the reference does not fuse).
//
// The tests load it to pin this build's outputs and match lists to reference
// code on the GPU, and bench.py times it beside this build's kernels on the
// same device-resident frames. Planes are dense (pitch = width floats), as in
// the reference's slots. C linkage, status codes and a last-error string.
#include "cuda/bm3d/kernels.hpp"
#include "cuda/common/aggregate.hpp"
#include "cuda/common/match.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <functional>
#include <stdexcept>
#include <memory>
#include <string>

namespace {

thread_local std::string g_error;

struct Ctx {
    int max_w = 0, max_h = 0;
    nss_cuda::DeviceBuffer matches, counts, fixed_num, fixed_den, rows, values, patches, ref_cube, fnum, fden, ptrs,
        tensor, frames;
    std::unique_ptr<nss_cuda::OrderedAggregator> agg;
    size_t cap_entries = 0;
};

// The one-frame plane table [src, ref] of the group kernels, written on the
// stream from kernel arguments (so calls queued back to back cannot see each
// other's pointers, as they could through a reused host staging buffer).
__global__ void set_table_kernel(const float** table, const float* src, const float* ref) {
    table[0] = src;
    table[1] = ref;
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Grows a buffer to at least `bytes` (outside any timed region: callers warm up first).
void ensure(nss_cuda::DeviceBuffer& b, size_t bytes) {
    if (b.bytes() < bytes) b = nss_cuda::DeviceBuffer(bytes);
}

nss_cuda::MatchGeometry geometry_of(int w, int h, int block, int range, int group) {
    nss_cuda::MatchGeometry g{w, h, w, block, range, group};
    return g;
}

// The reference's matcher choice for a radius-0 plane (filter_center).
void match_plane(Ctx& c, const float* plane, const nss_cuda::MatchGeometry& g, const nss_cuda::RasterGrid& grid,
                 cudaStream_t stream) {
    using namespace nss_cuda;
    auto* out = c.matches.as<DeviceMatch>();
    auto* counts = c.counts.as<int>();
    const int n = grid.count();
    bool tensor_ok = false;
    if (spatial_match_tensor(g, grid)) {
        const size_t bytes = spatial_match_scratch_bytes(g.width, g.height);
        ensure(c.tensor, bytes);
        tensor_ok = !spatial_match_window_over_tensor(g, grid);
    }
    const bool column = spatial_match_column_takes(g, grid);
    const bool square = spatial_match_square_takes(g, grid) && !(tensor_ok && g.lo() >= kSquareTensorRadius);
    const bool tensor = !column && !square && tensor_ok;
    if (tensor) spatial_match_prepare(plane, g, c.tensor.get(), stream);
    if (column) {
        if (!spatial_match_column(plane, g, grid, 0, n, out, counts, stream))
            spatial_match(plane, g, grid, 0, n, out, counts, stream);
    } else if (!square || !spatial_match_square(plane, g, grid, 0, n, out, counts, stream)) {
        spatial_match(plane, g, grid, 0, n, out, counts, stream, tensor ? c.tensor.get() : nullptr);
    }
}

void reserve(Ctx& c, int w, int h, int block, int step, int group, bool wiener) {
    using namespace nss_cuda;
    const RasterGrid grid = make_raster_grid(w, h, block, step);
    const size_t refs = (size_t)grid.count();
    const size_t entries = refs * (size_t)group;
    ensure(c.matches, entries * sizeof(DeviceMatch));
    ensure(c.counts, refs * sizeof(int));
    const size_t px = (size_t)w * h;
    ensure(c.fixed_num, px * sizeof(unsigned long long));
    ensure(c.fixed_den, px * sizeof(unsigned long long));
    ensure(c.rows, px * sizeof(unsigned long long));
    const size_t cube = refs * bm3d_scratch_floats(block, group, wiener);
    if (cube) ensure(c.ref_cube, cube * sizeof(float));
    if (!bm3d_fuses(block, group, wiener)) {
        ensure(c.values, entries * block * block * sizeof(float));
        ensure(c.patches, entries * sizeof(AggregatePatch));
        ensure(c.fnum, px * sizeof(float));
        ensure(c.fden, px * sizeof(float));
        if (!c.agg || c.cap_entries < entries || c.max_w < w || c.max_h < h) {
            c.max_w = std::max(c.max_w, w);
            c.max_h = std::max(c.max_h, h);
            c.cap_entries = std::max(c.cap_entries, entries);
            c.agg = std::make_unique<OrderedAggregator>(c.max_w, c.max_h, 1, c.cap_entries, nullptr, true);
        }
    }
}

int guarded(const std::function<void()>& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

}  // namespace

extern "C" {

const char* refgpu_last_error(void) { return g_error.c_str(); }

int refgpu_create(void** out) {
    return guarded([&] {
        auto* c = new Ctx();
        c->ptrs = nss_cuda::DeviceBuffer(2 * sizeof(float*));
        *out = c;
    });
}

void refgpu_destroy(void* ctx) {
    auto* c = static_cast<Ctx*>(ctx);
    delete c;
}

// Matching only: ref_count = grid count records of `group` DeviceMatch
// {x, y, t, dist} (16 bytes each) into matches, and the counts.
int refgpu_match(void* ctx, const float* plane, int w, int h, int block, int step, int range, int group,
                 void* matches, int* counts, void* stream_) {
    return guarded([&] {
        using namespace nss_cuda;
        Ctx& c = *static_cast<Ctx*>(ctx);
        auto stream = static_cast<cudaStream_t>(stream_);
        reserve(c, w, h, block, step, group, false);
        const RasterGrid grid = make_raster_grid(w, h, block, step);
        const MatchGeometry g = geometry_of(w, h, block, range, group);
        match_plane(c, plane, g, grid, stream);
        const size_t n = (size_t)grid.count();
        check(cudaMemcpyAsync(matches, c.matches.get(), n * group * sizeof(DeviceMatch), cudaMemcpyDeviceToDevice,
                              stream),
              "copy matches");
        check(cudaMemcpyAsync(counts, c.counts.get(), n * sizeof(int), cudaMemcpyDeviceToDevice, stream),
              "copy counts");
    });
}

// One radius-0 stage of one plane: ref == nullptr is the hard-threshold
// (basic) stage, otherwise the Wiener stage matching on and shrinking
// against ref. sigma is the effective sigma (sigma / 255 * 0.75).
int refgpu_stage(void* ctx, const float* src, const float* ref, float* dst, int w, int h, int block, int step,
                 int range, int group, float sigma, void* stream_) {
    return guarded([&] {
        using namespace nss_cuda;
        Ctx& c = *static_cast<Ctx*>(ctx);
        auto stream = static_cast<cudaStream_t>(stream_);
        const bool wiener = ref != nullptr;
        reserve(c, w, h, block, step, group, wiener);
        const RasterGrid grid = make_raster_grid(w, h, block, step);
        const MatchGeometry g = geometry_of(w, h, block, range, group);
        const size_t px = (size_t)w * h;
        // the plane table the group kernels index by match t (one frame)
        set_table_kernel<<<1, 1, 0, stream>>>(c.ptrs.as<const float*>(), src, ref);
        check(cudaGetLastError(), "set_table_kernel");
        const auto* table = c.ptrs.as<const float*>();
        const bool fused = bm3d_fuses(block, group, wiener);
        FixedTarget fixed{c.fixed_num.as<unsigned long long>(), c.fixed_den.as<unsigned long long>(), w, px};
        fixed.channel_step = px;
        if (fused) fixed_clear(fixed, px, stream);
        match_plane(c, wiener ? ref : src, g, grid, stream);
        Bm3dGroupArgs a{};
        a.src = table;
        a.ref = wiener ? table + 1 : nullptr;
        a.pitch = w;
        a.matches = c.matches.as<DeviceMatch>();
        a.plane_offset = 0;
        a.counts = c.counts.as<int>();
        a.batch = grid.count();
        a.block = block;
        a.group = group;
        a.sigma = sigma;
        a.values = fused ? nullptr : c.values.as<float>();
        a.ref_cube = c.ref_cube.as<float>();
        a.patches = fused ? nullptr : c.patches.as<AggregatePatch>();
        if (fused) a.fused = fixed;
        bm3d_filter_groups(a, stream);
        if (fused) {
            fixed_finish(fixed, block, src, w, h, c.rows.as<unsigned long long>(), dst, stream);
        } else {
            const AggregateTarget target{c.fnum.as<float>(), c.fden.as<float>(), w, h, w, 1, px};
            c.agg->run(c.values.as<float>(), c.patches.as<AggregatePatch>(), grid.count() * group, block, target,
                       stream, false);
            aggregate_finish(c.fnum.as<float>(), c.fden.as<float>(), src, w, h, w, dst, stream);
        }
    });
}

// Temporal (predictive) matching of every reference of the centre slot t0
// over ntemp frames (host array of device plane pointers, dense, pitch =
// width), valid slots [valid_begin, valid_end): the reference's choice of
// filter_center for radius > 0 (group_driver.cpp:800-810): its square
// matcher's centre frame where that takes the shape, else the window
// matcher's, else the lane kernels throughout.
int refgpu_match_temporal(void* ctx, const float* const* planes, int ntemp, int t0, int valid_begin, int valid_end,
                          int w, int h, int block, int step, int range, int group, int ps_num, int ps_range,
                          void* matches, int* counts, void* stream_) {
    return guarded([&] {
        using namespace nss_cuda;
        Ctx& c = *static_cast<Ctx*>(ctx);
        auto stream = static_cast<cudaStream_t>(stream_);
        if (ntemp < 1 || ntemp > 33) throw std::invalid_argument("refgpu_match_temporal: 1 to 33 frames");
        reserve(c, w, h, block, step, group, false);
        ensure(c.frames, 33 * sizeof(float*));
        check(cudaMemcpyAsync(c.frames.get(), planes, ntemp * sizeof(float*), cudaMemcpyHostToDevice, stream),
              "frame table");
        check(cudaStreamSynchronize(stream), "frame table");  // pageable source: the copy is done before it changes
        const RasterGrid grid = make_raster_grid(w, h, block, step);
        const MatchGeometry g = geometry_of(w, h, block, range, group);
        TemporalWindow win{};
        win.frames = c.frames.as<const float*>();
        win.ntemp = ntemp;
        win.t0 = t0;
        win.radius = t0;
        win.valid_begin = valid_begin;
        win.valid_end = valid_end;
        win.ps_num = ps_num;
        win.ps_range = ps_range;
        const int n = grid.count();
        auto* out = c.matches.as<DeviceMatch>();
        auto* cnt = c.counts.as<int>();
        if (!predictive_match_square(g, win, grid, 0, n, out, cnt, stream) &&
            !predictive_match_window(g, win, grid, 0, n, out, cnt, stream))
            predictive_match(g, win, grid, 0, n, out, cnt, stream);
        check(cudaMemcpyAsync(matches, out, (size_t)n * group * sizeof(DeviceMatch), cudaMemcpyDeviceToDevice,
                              stream),
              "copy matches");
        check(cudaMemcpyAsync(counts, cnt, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, stream),
              "copy counts");
    });
}

// Which of the reference's matchers filter_center would take for this
// plane: 1 column, 2 square, 3 tensor, 0 the window / lane / generic kernels.
int refgpu_matcher_kind(int w, int h, int block, int step, int range, int group) {
    using namespace nss_cuda;
    const RasterGrid grid = make_raster_grid(w, h, block, step);
    const MatchGeometry g = geometry_of(w, h, block, range, group);
    const bool tensor_ok = spatial_match_tensor(g, grid) && !spatial_match_window_over_tensor(g, grid);
    if (spatial_match_column_takes(g, grid)) return 1;
    if (spatial_match_square_takes(g, grid) && !(tensor_ok && g.lo() >= kSquareTensorRadius)) return 2;
    return tensor_ok ? 3 : 0;
}

}  // extern "C"
