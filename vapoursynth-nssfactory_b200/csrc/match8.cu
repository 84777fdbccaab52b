// Exact FP32 block matching for 8x8 blocks (sm_100a): the default BM3D shape.
//
// Same contract as match.cu (the reference's matcher.hpp:27-283 ordering,
// row-major FMA chain per candidate, keys dist << 32 | y << 16 | x); only the
// schedule differs:
//   - a CTA is 32 consecutive references of one grid row (one per lane) of
//     one plane of a batch; its P warps split the 2R+1 window columns, each
//     lane holding its reference block in 64 registers;
//   - the CTA stages the 2R+8 rows of its windows once in shared memory with a
//     skewed layout (column c at c + c/32), so 32 lanes whose references sit
//     8 columns apart read 32 different banks;
//   - a lane walks its columns one by one: the column's 2R+8 image rows stream
//     through and each row is applied to the 8 candidates that overlap it.
//     Candidate k lives in accumulator k & 7; with the row loop unrolled the
//     slots are register names, so a row costs 8 shared loads and 64
//     subtract/FMA pairs. A finished candidate enters the lane's register
//     top-k; the P partial lists of a reference merge in shared memory.
#include "kernels.cuh"

#include <algorithm>

namespace nssb {
namespace {

__device__ __forceinline__ int skew(int col) { return col + (col >> 5); }

__device__ __forceinline__ uint64_t key_of(float d, int x, int y) {
    uint32_t b = __float_as_uint(d);
    if ((b & 0x7f800000u) == 0x7f800000u) b = 0x7f800000u;
    return (uint64_t(b) << 32) | (uint64_t(uint32_t(y)) << 16) | uint64_t(uint32_t(x));
}

template <int K>
struct TopK {
    uint64_t k[K];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int q = 0; q < K; ++q) k[q] = ~0ull;
    }
    __device__ __forceinline__ void add(uint64_t v) {
        if (!(v < k[K - 1])) return;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const uint64_t a = k[q];
            const bool s = v < a;
            k[q] = s ? v : a;
            v = s ? a : v;
        }
    }
};

constexpr int kLanes = 32;

template <int R>
__host__ __device__ constexpr int tile_rows() { return 2 * R + 8; }

int tile_pitch(int step, int R) {
    const int tw = (kLanes - 1) * step + 2 * R + 8;
    return ((tw - 1 + ((tw - 1) >> 5)) / 32 + 1) * 32;
}

template <int R, int K, int P>
__global__ void __launch_bounds__(kLanes* P, (K <= 7 ? 4 : 3))
    match8_kernel(const __grid_constant__ MatchBatch mb, int pitch) {
    constexpr int B = 8;
    constexpr int NC = 2 * R + 1;            // candidates per window column
    constexpr int TR = tile_rows<R>();
    constexpr int CPW = (NC + P - 1) / P;    // window columns per warp
    extern __shared__ float tile[];
    // this CTA's plane
    int pl = 0;
    {
        int lo = 0, hi = mb.n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (mb.p[mid].cta0 <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
        }
        pl = lo;
    }
    const MatchPlane& P_ = mb.p[pl];
    const int W = P_.W, H = P_.H, step = mb.step, nx = P_.nx;
    const int local = blockIdx.x - P_.cta0;
    const int chunks = (nx + kLanes - 1) / kLanes;
    const int ry = local / chunks, rx0 = (local - ry * chunks) * kLanes;
    const int rx1 = min(rx0 + kLanes, nx) - 1;
    const int cy = grid_pos(ry, H, B, step);
    const int X0 = grid_pos(rx0, W, B, step) - R, Y0 = cy - R;
    const int TW = grid_pos(rx1, W, B, step) + R + B - X0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < TR; r += P) {
        const int gy = Y0 + r;
        const bool yok = gy >= 0 && gy < H;
        const float* src = P_.src + (int64_t)(yok ? gy : 0) * P_.stride;
        float* dst = tile + r * pitch;
        for (int c = lane; c < TW; c += kLanes) {
            const int gx = X0 + c;
            dst[skew(c)] = (yok && gx >= 0 && gx < W) ? __ldg(src + gx) : 0.f;
        }
    }
    __syncthreads();

    const int rx = rx0 + lane;
    const bool active = rx < nx;
    const int cx = grid_pos(min(rx, nx - 1), W, B, step);
    const int left = max(cx - R, 0), right = min(cx + R, W - B);
    const int kmin = max(cy - R, 0) - (cy - R), kmax = min(cy + R, H - B) - (cy - R);
    const int tc0 = cx - R - X0;

    float ref[B * B];
#pragma unroll
    for (int i = 0; i < B; ++i)
#pragma unroll
        for (int j = 0; j < B; ++j) ref[i * B + j] = tile[(R + i) * pitch + skew(tc0 + R + j)];

    TopK<K> topk;
    topk.init();
    const int d0 = warp * CPW, d1 = min(NC, d0 + CPW);
    for (int dxi = d0; dxi < d1; ++dxi) {
        const int x = cx - R + dxi;
        const bool xok = x >= left && x <= right;
        int col[B];
#pragma unroll
        for (int j = 0; j < B; ++j) col[j] = skew(tc0 + dxi + j);
        float acc[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = 0.f;
#pragma unroll
        for (int s = 0; s < NC + B - 1; ++s) {
            const float* rp = tile + s * pitch;
            float p[B];
#pragma unroll
            for (int j = 0; j < B; ++j) p[j] = rp[col[j]];
#pragma unroll
            for (int i = 0; i < B; ++i) {
                const int k = s - i;
                if (k >= 0 && k < NC) {
#pragma unroll
                    for (int j = 0; j < B; ++j) {
                        const float d = __fsub_rn(ref[i * B + j], p[j]);
                        acc[k & 7] = __fmaf_rn(d, d, acc[k & 7]);
                    }
                }
            }
            const int kd = s - (B - 1);
            if (kd >= 0 && kd < NC) {
                const float dd = acc[kd & 7];
                acc[kd & 7] = 0.f;
                if (xok && kd >= kmin && kd <= kmax && !(dxi == R && kd == R))
                    topk.add(key_of(dd, x, cy - R + kd));
            }
        }
    }
    // merge the P partial lists of each reference (exact: keys are a total order)
    if constexpr (P > 1) {
        __syncthreads();
        uint64_t* keys = reinterpret_cast<uint64_t*>(tile);  // [P][K][32]
        if (warp > 0) {
#pragma unroll
            for (int q = 0; q < K; ++q) keys[(warp * K + q) * kLanes + lane] = topk.k[q];
        }
        __syncthreads();
        if (warp > 0) return;
        for (int w = 1; w < P; ++w)
#pragma unroll
            for (int q = 0; q < K; ++q) topk.add(keys[(w * K + q) * kLanes + lane]);
    }
    if (!active) return;
    const int64_t job = (int64_t)ry * nx + rx;
    constexpr int G = K + 1;
    int32_t* op = P_.pos + job * G;
    op[0] = pack_pos(cx, cy);
    int n = 0;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const bool valid = topk.k[q] != ~0ull;
        n += valid;
        op[1 + q] = valid ? int32_t(uint32_t(topk.k[q])) : -1;
    }
    if (P_.dist) {
        float* od = P_.dist + job * G;
        od[0] = 0.f;
#pragma unroll
        for (int q = 0; q < K; ++q)
            od[1 + q] = topk.k[q] != ~0ull ? __uint_as_float(uint32_t(topk.k[q] >> 32)) : 0.f;
    }
    P_.count[job] = 1 + n;
}

constexpr int kParts = 4;

template <int R, int K>
void launch_rk(MatchBatch& mb, cudaStream_t stream) {
    int ctas = 0;
    for (int i = 0; i < mb.n; ++i) {
        MatchPlane& p = mb.p[i];
        p.nx = grid_count(p.W, 8, mb.step);
        p.ny = grid_count(p.H, 8, mb.step);
        p.cta0 = ctas;
        ctas += ceil_div(p.nx, kLanes) * p.ny;
    }
    if (ctas == 0) return;
    const int pitch = tile_pitch(mb.step, R);
    const size_t smem = std::max((size_t)pitch * tile_rows<R>() * sizeof(float),
                                 (size_t)kParts * K * kLanes * sizeof(uint64_t));
    auto kern = match8_kernel<R, K, kParts>;
    NSSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<ctas, kLanes * kParts, smem, stream>>>(mb, pitch);
    NSSB_CUDA(cudaGetLastError());
}

template <int R>
bool launch_r(MatchBatch& mb, int group, cudaStream_t stream) {
    switch (group) {
        case 2: launch_rk<R, 1>(mb, stream); return true;
        case 4: launch_rk<R, 3>(mb, stream); return true;
        case 8: launch_rk<R, 7>(mb, stream); return true;
        case 16: launch_rk<R, 15>(mb, stream); return true;
        default: return false;
    }
}

}  // namespace

bool launch_match8_batch(MatchBatch& mb, int bm_range, int group, cudaStream_t stream) {
    if (mb.step < 1 || mb.step > 8 || mb.n < 1 || mb.n > kMaxBatchPlanes) return false;
    for (int i = 0; i < mb.n; ++i)
        if (mb.p[i].W < 8 || mb.p[i].H < 8) return false;
    switch (bm_range) {
        case 9: return launch_r<9>(mb, group, stream);
        default: return false;
    }
}

bool launch_match8(const float* plane, int64_t stride, int width, int height, int step, int bm_range, int group,
                   int32_t* pos, float* dist, int32_t* count, cudaStream_t stream) {
    static thread_local MatchBatch mb;
    mb.n = 1;
    mb.step = step;
    mb.p[0] = MatchPlane{plane, stride, pos, dist, count, width, height, 0, 0, 0};
    return launch_match8_batch(mb, bm_range, group, stream);
}

}  // namespace nssb
