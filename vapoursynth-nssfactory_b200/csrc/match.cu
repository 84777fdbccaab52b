// Exact FP32 spatial block matching (sm_100a).
//
// Semantics (reference src/cpu/bm/matcher.hpp:27-283, batch_runner.hpp:17-53):
// for every reference of the raster grid (last row/column clamped to W-B/H-B)
// the group is the reference itself, then the group-1 smallest SSDs of the
// other positions of the clamped (2R+1)^2 window, ordered by distance, then y,
// then x; non-finite distances after every finite one. The SSD order: one
// FMA chain per block column down the rows, then the columns added pairwise
// (column_tree) -- the order of the CPU oracle, so device and oracle
// distances are bit-identical.
//
// Layout: one thread per reference; a CTA covers TX x TY references and stages
// the union of their windows in shared memory once. Keys are 64-bit
// (dist_bits << 32 | y << 16 | x): their unsigned order is the match order.
#include "kernels.cuh"

#include <algorithm>

namespace nssb {
namespace {

__device__ __forceinline__ uint64_t match_key(float d, int x, int y) {
    uint32_t b = __float_as_uint(d);
    if ((b & 0x7f800000u) == 0x7f800000u) b = 0x7f800000u;  // every non-finite ties, then y, x
    return (uint64_t(b) << 32) | (uint64_t(uint32_t(y)) << 16) | uint64_t(uint32_t(x));
}

// K smallest keys, ascending, in registers (K known at compile time).
template <int K>
struct RegTopK {
    uint64_t k[K > 0 ? K : 1];
    __device__ void init() {
#pragma unroll
        for (int q = 0; q < K; ++q) k[q] = ~0ull;
    }
    __device__ __forceinline__ void add(uint64_t v) {
        if constexpr (K > 0) {
            if (!(v < k[K - 1])) return;
#pragma unroll
            for (int q = 0; q < K; ++q) {
                const uint64_t a = k[q];
                const bool s = v < a;
                k[q] = s ? v : a;
                v = s ? a : v;
            }
        }
    }
    __device__ uint64_t get(int q) const {
        uint64_t r = ~0ull;
#pragma unroll
        for (int i = 0; i < K; ++i)
            if (i == q) r = k[i];
        return r;
    }
};

// Runtime capacity up to 63 (groups of 32 and 64): a local-memory list.
struct LocalTopK {
    uint64_t k[63];
    int cap, n;
    __device__ void init(int c) {
        cap = c;
        n = 0;
    }
    __device__ void add(uint64_t v) {
        if (cap <= 0) return;
        if (n == cap) {
            if (!(v < k[n - 1])) return;
            --n;
        }
        int p = n;
        while (p > 0 && v < k[p - 1]) {
            k[p] = k[p - 1];
            --p;
        }
        k[p] = v;
        ++n;
    }
    __device__ uint64_t get(int q) const { return q < n ? k[q] : ~0ull; }
};

struct TileGeom {
    int tx, ty;         // references per CTA in x / y
    int pitch, rows;    // shared tile extent (floats)
};

template <int B, class TopK>
__device__ void match_one(const float* __restrict__ tile, int tp, int x0, int y0, int cx, int cy, int left,
                          int right, int top, int bottom, TopK& topk) {
    constexpr bool kRegs = B <= 8;
    float ref[kRegs ? B * B : 1];
    if constexpr (kRegs) {
#pragma unroll
        for (int i = 0; i < B; ++i)
#pragma unroll
            for (int j = 0; j < B; ++j) ref[i * B + j] = tile[(cy - y0 + i) * tp + (cx - x0 + j)];
    }
    const float* rb = tile + (cy - y0) * tp + (cx - x0);
    for (int y = top; y <= bottom; ++y) {
        const float* rowbase = tile + (y - y0) * tp - x0;
        for (int x = left; x <= right; ++x) {
            if (x == cx && y == cy) continue;
            const float* cb = rowbase + x;
            float c[B];
#pragma unroll
            for (int j = 0; j < B; ++j) c[j] = 0.f;
            if constexpr (kRegs) {
#pragma unroll
                for (int i = 0; i < B; ++i)
#pragma unroll
                    for (int j = 0; j < B; ++j) {
                        const float d = __fsub_rn(ref[i * B + j], cb[i * tp + j]);
                        c[j] = __fmaf_rn(d, d, c[j]);
                    }
            } else {
                for (int i = 0; i < B; ++i)
#pragma unroll
                    for (int j = 0; j < B; ++j) {
                        const float d = __fsub_rn(rb[i * tp + j], cb[i * tp + j]);
                        c[j] = __fmaf_rn(d, d, c[j]);
                    }
            }
            topk.add(match_key(column_tree<B>(c), x, y));
        }
    }
}

template <int B, int K>
__global__ void __launch_bounds__(128) spatial_match_kernel(const float* __restrict__ plane, int64_t stride,
                                                            int W, int H, int step, int R, int G, int nx, int ny,
                                                            TileGeom tg, int32_t* __restrict__ pos,
                                                            float* __restrict__ dist, int32_t* __restrict__ count) {
    extern __shared__ float tile[];
    const int rx0 = blockIdx.x * tg.tx, ry0 = blockIdx.y * tg.ty;
    const int rx1 = min(rx0 + tg.tx, nx) - 1, ry1 = min(ry0 + tg.ty, ny) - 1;
    const int x0 = max(0, grid_pos(rx0, W, B, step) - R);
    const int x1 = min(W - 1, grid_pos(rx1, W, B, step) + R + B - 1);
    const int y0 = max(0, grid_pos(ry0, H, B, step) - R);
    const int y1 = min(H - 1, grid_pos(ry1, H, B, step) + R + B - 1);
    const int tw = x1 - x0 + 1, th = y1 - y0 + 1;
    const int tp = tg.pitch;
    for (int i = threadIdx.x; i < tw * th; i += blockDim.x) {
        const int yy = i / tw, xx = i - yy * tw;
        tile[yy * tp + xx] = __ldg(plane + (int64_t)(y0 + yy) * stride + x0 + xx);
    }
    __syncthreads();
    const int rx = rx0 + int(threadIdx.x) % tg.tx, ry = ry0 + int(threadIdx.x) / tg.tx;
    if (rx >= nx || ry >= ny || int(threadIdx.x) >= tg.tx * tg.ty) return;
    const int cx = grid_pos(rx, W, B, step), cy = grid_pos(ry, H, B, step);
    const int left = max(cx - R, 0), right = min(cx + R, W - B);
    const int top = max(cy - R, 0), bottom = min(cy + R, H - B);
    const int64_t job = (int64_t)ry * nx + rx;
    int32_t* op = pos + job * G;
    float* od = dist ? dist + job * G : nullptr;
    op[0] = pack_pos(cx, cy);
    if (od) od[0] = 0.f;
    int n = 0;
    if constexpr (K >= 0) {
        RegTopK<K> topk;
        topk.init();
        if (K > 0) match_one<B>(tile, tp, x0, y0, cx, cy, left, right, top, bottom, topk);
        for (int q = 0; q < G - 1; ++q) {
            const uint64_t key = topk.get(q);
            const bool valid = key != ~0ull;
            n += valid;
            op[1 + q] = valid ? int32_t(uint32_t(key)) : -1;
            if (od) od[1 + q] = valid ? __uint_as_float(uint32_t(key >> 32)) : 0.f;
        }
    } else {
        LocalTopK topk;
        topk.init(G - 1);
        match_one<B>(tile, tp, x0, y0, cx, cy, left, right, top, bottom, topk);
        for (int q = 0; q < G - 1; ++q) {
            const uint64_t key = topk.get(q);
            const bool valid = q < topk.n;
            n += valid;
            op[1 + q] = valid ? int32_t(uint32_t(key)) : -1;
            if (od) od[1 + q] = valid ? __uint_as_float(uint32_t(key >> 32)) : 0.f;
        }
    }
    count[job] = 1 + n;
}

TileGeom choose_tile(int block, int step, int R, int nx, int ny) {
    // Largest tile (up to 32 x 4 references) whose window union fits in 96 KB.
    TileGeom g{};
    int tx = std::min(32, nx), ty = std::min(4, ny);
    for (;;) {
        const int w = (tx - 1) * step + 2 * R + block, h = (ty - 1) * step + 2 * R + block;
        if ((size_t)w * h * sizeof(float) <= 96 * 1024 || (tx == 1 && ty == 1)) {
            g.tx = tx;
            g.ty = ty;
            g.pitch = w;
            g.rows = h;
            return g;
        }
        if (ty > 1)
            ty = (ty + 1) / 2;
        else
            tx = (tx + 1) / 2;
    }
}

template <int B, int K>
void launch_bk(const float* plane, int64_t stride, int W, int H, int step, int R, int G, int32_t* pos, float* dist,
               int32_t* count, cudaStream_t stream) {
    const int nx = grid_count(W, B, step), ny = grid_count(H, B, step);
    if (nx == 0 || ny == 0) return;
    const TileGeom tg = choose_tile(B, step, R, nx, ny);
    const size_t smem = (size_t)tg.pitch * tg.rows * sizeof(float);
    auto kern = spatial_match_kernel<B, K>;
    NSSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 grid(ceil_div(nx, tg.tx), ceil_div(ny, tg.ty));
    kern<<<grid, 128, smem, stream>>>(plane, stride, W, H, step, R, G, nx, ny, tg, pos, dist, count);
    NSSB_CUDA(cudaGetLastError());
}

template <int B>
void launch_b(const float* plane, int64_t stride, int W, int H, int step, int R, int G, int32_t* pos, float* dist,
              int32_t* count, cudaStream_t stream) {
    switch (G) {
        case 1: return launch_bk<B, 0>(plane, stride, W, H, step, R, G, pos, dist, count, stream);
        case 2: return launch_bk<B, 1>(plane, stride, W, H, step, R, G, pos, dist, count, stream);
        case 4: return launch_bk<B, 3>(plane, stride, W, H, step, R, G, pos, dist, count, stream);
        case 8: return launch_bk<B, 7>(plane, stride, W, H, step, R, G, pos, dist, count, stream);
        case 16: return launch_bk<B, 15>(plane, stride, W, H, step, R, G, pos, dist, count, stream);
        default: return launch_bk<B, -1>(plane, stride, W, H, step, R, G, pos, dist, count, stream);
    }
}

}  // namespace

void launch_match_spatial(const float* plane, int64_t stride, int width, int height, int block, int step,
                          int bm_range, int group, int32_t* pos, float* dist, int32_t* count, cudaStream_t stream) {
    if (block == 8 && launch_match8(plane, stride, width, height, step, bm_range, group, pos, dist, count, stream))
        return;
    switch (block) {
        case 1: return launch_b<1>(plane, stride, width, height, step, bm_range, group, pos, dist, count, stream);
        case 2: return launch_b<2>(plane, stride, width, height, step, bm_range, group, pos, dist, count, stream);
        case 4: return launch_b<4>(plane, stride, width, height, step, bm_range, group, pos, dist, count, stream);
        case 8: return launch_b<8>(plane, stride, width, height, step, bm_range, group, pos, dist, count, stream);
        case 12: return launch_b<12>(plane, stride, width, height, step, bm_range, group, pos, dist, count, stream);
        case 16: return launch_b<16>(plane, stride, width, height, step, bm_range, group, pos, dist, count, stream);
        case 32: return launch_b<32>(plane, stride, width, height, step, bm_range, group, pos, dist, count, stream);
        default: throw std::invalid_argument("nss_cuda: unsupported block size");
    }
}

}  // namespace nssb
