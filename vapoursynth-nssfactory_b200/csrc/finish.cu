// Finish of a stage (sm_100a): den is recovered exactly from the per-origin
// weights by a B x B box sum in int64, then out = den > 1e-12 ? num / den : src
// (reference aggregate_finish, src/cpu/bm/agg.cpp:17-42; the device form keeps
// den at the patch origin too, src/cuda/common/aggregate.cu:300-323).
#include "kernels.cuh"

namespace nssb {
namespace {

constexpr int kTX = 32, kTY = 8, kMaxB = 32;

// Box-summed den of the tile's pixels into den_tile[kTY][kTX] (int64).
__device__ void box_den(const long long* __restrict__ wsum, int64_t as, int W, int H, int B, int x0, int y0,
                        long long (*wt)[kTX + kMaxB - 1], long long (*hs)[kTX], long long (*den)[kTX]) {
    const int rows = kTY + B - 1, cols = kTX + B - 1;
    for (int i = threadIdx.x; i < rows * cols; i += blockDim.x) {
        const int r = i / cols, c = i - r * cols;
        const int yy = y0 - B + 1 + r, xx = x0 - B + 1 + c;
        wt[r][c] = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? wsum[(int64_t)yy * as + xx] : 0ll;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < rows * kTX; i += blockDim.x) {
        const int r = i / kTX, c = i - r * kTX;
        long long s = 0;
        for (int q = 0; q < B; ++q) s += wt[r][c + q];
        hs[r][c] = s;
    }
    __syncthreads();
    {
        const int r = threadIdx.x / kTX, c = threadIdx.x % kTX;
        long long s = 0;
        for (int q = 0; q < B; ++q) s += hs[r + q][c];
        den[r][c] = s;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kTX* kTY) finish_kernel(const long long* __restrict__ num,
                                                          const long long* __restrict__ wsum, int64_t as,
                                                          const float* __restrict__ src, int64_t ss,
                                                          float* __restrict__ dst, int64_t ds, int W, int H, int B) {
    __shared__ long long wt[kTY + kMaxB - 1][kTX + kMaxB - 1];
    __shared__ long long hs[kTY + kMaxB - 1][kTX];
    __shared__ long long den[kTY][kTX];
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    box_den(wsum, as, W, H, B, x0, y0, wt, hs, den);
    const int r = threadIdx.x / kTX, c = threadIdx.x % kTX;
    const int x = x0 + c, y = y0 + r;
    if (x >= W || y >= H) return;
    const long long d = den[r][c];
    const double dd = (double)d * kFixedInv;
    float out;
    if ((float)dd > 1e-12f) {
        out = (float)((double)num[(int64_t)y * as + x] / (double)d);
    } else {
        out = src[(int64_t)y * ss + x];
    }
    dst[(int64_t)y * ds + x] = out;
}

__global__ void __launch_bounds__(kTX* kTY) fat_kernel(const long long* __restrict__ num,
                                                       const long long* __restrict__ wsum, int64_t as,
                                                       float* __restrict__ dnum, float* __restrict__ dden,
                                                       int64_t ds, int W, int H, int B) {
    __shared__ long long wt[kTY + kMaxB - 1][kTX + kMaxB - 1];
    __shared__ long long hs[kTY + kMaxB - 1][kTX];
    __shared__ long long den[kTY][kTX];
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    box_den(wsum, as, W, H, B, x0, y0, wt, hs, den);
    const int r = threadIdx.x / kTX, c = threadIdx.x % kTX;
    const int x = x0 + c, y = y0 + r;
    if (x >= W || y >= H) return;
    dnum[(int64_t)y * ds + x] = (float)((double)num[(int64_t)y * as + x] * kFixedInv);
    dden[(int64_t)y * ds + x] = (float)((double)den[r][c] * kFixedInv);
}

// Batched finish over a plane table. A CTA finishes a 64 x 32 tile, 8
// pixels per thread (one column, 8 rows): the origin weights of the tile and
// its (B-1)-pixel halo, num and src are all requested before the first
// barrier; den comes from sliding B-wide row sums, then B-tall column sums,
// exact in int64. num is cleared as it is consumed (each pixel's num is read
// by exactly one thread), so the next stage finds it zero.
constexpr int kFX = 64, kFY = 32, kFT = 256;

// BT > 0: the block size known at compile time (8, the default), so the
// halo tile's loads are a fixed, fully unrolled set issued before any of them
// is stored; BT = 0: any block size.
template <int BT>
__global__ void __launch_bounds__(kFT) finish_batch_kernel(const __grid_constant__ FinishBatch fb) {
    extern __shared__ long long fsm[];  // wt[(kFY + B - 1)][(kFX + B - 1)], then hs[(kFY + B - 1)][kFX]
    int pl = 0;
    {
        int lo = 0, hi = fb.n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (fb.p[mid].cta0 <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
        }
        pl = lo;
    }
    const FinishPlane& P = fb.p[pl];
    const int B = BT > 0 ? BT : fb.block;
    const int local = blockIdx.x - P.cta0;
    const int ty = local / P.tiles_x, tx = local - ty * P.tiles_x;
    const int x0 = tx * kFX, y0 = ty * kFY;
    const int c = threadIdx.x & (kFX - 1), q = threadIdx.x / kFX;  // column, 8-row quarter
    const int x = x0 + c;
    // this thread's num and src, requested first
    long long nv[8];
    float sv[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int y = y0 + q * 8 + r;
        const bool ok = x < P.W && y < P.H;
        nv[r] = ok ? P.num[(int64_t)y * P.acc_stride + x] : 0;
        sv[r] = ok ? P.src[(int64_t)y * P.sstride + x] : 0.f;
    }
    const int rows = kFY + B - 1, cols = kFX + B - 1;
    long long* wtp = fsm;
    long long* hsp = fsm + rows * cols;
#define wt(r, cc) wtp[(r) * cols + (cc)]
#define hs(r, cc) hsp[(r) * kFX + (cc)]
    if constexpr (BT > 0) {
        constexpr int kRows = kFY + BT - 1, kCols = kFX + BT - 1, kN = (kRows * kCols + kFT - 1) / kFT;
        long long v[kN];
#pragma unroll
        for (int t = 0; t < kN; ++t) {
            const int i = threadIdx.x + t * kFT;
            const int r = i / kCols, cc = i - r * kCols;
            const int yy = y0 - BT + 1 + r, xx = x0 - BT + 1 + cc;
            v[t] = (i < kRows * kCols && yy >= 0 && yy < P.H && xx >= 0 && xx < P.W)
                       ? P.wsum[(int64_t)yy * P.acc_stride + xx]
                       : 0ll;
        }
#pragma unroll
        for (int t = 0; t < kN; ++t) {
            const int i = threadIdx.x + t * kFT;
            if (i < kRows * kCols) wtp[i] = v[t];
        }
    } else {
        for (int i = threadIdx.x; i < rows * cols; i += kFT) {
            const int r = i / cols, cc = i - r * cols;
            const int yy = y0 - B + 1 + r, xx = x0 - B + 1 + cc;
            wt(r, cc) = (yy >= 0 && yy < P.H && xx >= 0 && xx < P.W) ? P.wsum[(int64_t)yy * P.acc_stride + xx] : 0ll;
        }
    }
    __syncthreads();
    // row sums: 8 consecutive columns of one row per task, sliding
    for (int t = threadIdx.x; t < rows * (kFX / 8); t += kFT) {
        const int r = t / (kFX / 8), c0 = (t - r * (kFX / 8)) * 8;
        long long sum = 0;
        for (int k = 0; k < B; ++k) sum += wt(r, c0 + k);
        hs(r, c0) = sum;
#pragma unroll
        for (int j = 1; j < 8; ++j) {
            sum += wt(r, c0 + j + B - 1) - wt(r, c0 + j - 1);
            hs(r, c0 + j) = sum;
        }
    }
    __syncthreads();
    // column sums down this thread's 8 rows, then the finish
    long long den = 0;
    for (int k = 0; k < B; ++k) den += hs(q * 8 + k, c);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        if (r > 0) den += hs(q * 8 + r + B - 1, c) - hs(q * 8 + r - 1, c);
        const int y = y0 + q * 8 + r;
        if (x < P.W && y < P.H) {
            P.num[(int64_t)y * P.acc_stride + x] = 0;
            const float dd = (float)((double)den * kFixedInv);
            P.dst[(int64_t)y * P.dstride + x] = dd > 1e-12f ? (float)((double)nv[r] / (double)den) : sv[r];
        }
    }
#undef wt
#undef hs
}

}  // namespace

void launch_finish_batch(const FinishBatch& fb, cudaStream_t stream) {
    if (fb.total_ctas <= 0) return;
    const size_t smem = (size_t)(kFY + fb.block - 1) * (kFX + fb.block - 1 + kFX) * sizeof(long long);
    auto kern = fb.block == 8 ? finish_batch_kernel<8> : finish_batch_kernel<0>;
    NSSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<fb.total_ctas, kFT, smem, stream>>>(fb);
    NSSB_CUDA(cudaGetLastError());
}

int finish_tiles_x(int w) { return ceil_div(w, kFX); }
int finish_tiles(int w, int h) { return ceil_div(w, kFX) * ceil_div(h, kFY); }

void launch_finish(const long long* num, const long long* wsum, int64_t acc_stride, const float* src,
                   int64_t sstride, float* dst, int64_t dstride, int width, int height, int block,
                   cudaStream_t stream) {
    const dim3 grid(ceil_div(width, kTX), ceil_div(height, kTY));
    finish_kernel<<<grid, kTX * kTY, 0, stream>>>(num, wsum, acc_stride, src, sstride, dst, dstride, width, height,
                                                  block);
    NSSB_CUDA(cudaGetLastError());
}

void launch_fat_slice(const long long* num, const long long* wsum, int64_t acc_stride, float* dst_num,
                      float* dst_den, int64_t dstride, int width, int height, int block, cudaStream_t stream) {
    const dim3 grid(ceil_div(width, kTX), ceil_div(height, kTY));
    fat_kernel<<<grid, kTX * kTY, 0, stream>>>(num, wsum, acc_stride, dst_num, dst_den, dstride, width, height,
                                               block);
    NSSB_CUDA(cudaGetLastError());
}

}  // namespace nssb
