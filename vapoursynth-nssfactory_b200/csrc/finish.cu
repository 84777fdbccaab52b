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
    // den > 1e-12 in real units is d >= 1 in units of 2^-32
    dst[(int64_t)y * ds + x] = d > 0 ? fixed_quotient(num[(int64_t)y * as + x], d) : src[(int64_t)y * ss + x];
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
    dnum[(int64_t)y * ds + x] = __ll2float_rn(num[(int64_t)y * as + x]) * kFixedInv;
    dden[(int64_t)y * ds + x] = __ll2float_rn(den[r][c]) * kFixedInv;
}

// Batched finish over a plane table. A CTA finishes a 64 x 32 tile:
//   - first every thread requests the num and src of its 8 output pixels (8
//     consecutive pixels of one row), so they arrive while den is formed;
//   - vertical B-tall sums of the origin weights: a thread per (8-row
//     quarter, column) of the tile and of its B-1 halo columns on the left
//     reads 8 + B - 1 weights down its column and slides the sum, exact in
//     int64, into a shared table vs[32 rows][64 + B - 1 columns];
//   - horizontal B-wide sums: each thread slides along its 8 pixels.
// vs column cc is stored at cc + cc / 8 in a row of kVsPitch(B) words with
// the pitch = 8 (mod 16), so the 16 lanes of a half-warp (2 rows x 8
// segments) read 16 different bank pairs. num is cleared as it is consumed
// (each pixel's num is read by exactly one thread), so the next stage finds
// it zero.
constexpr int kFX = 64, kFY = 32, kFT = 256;

__host__ __device__ constexpr int vs_col(int cc) { return cc + (cc >> 3); }
__host__ __device__ constexpr int vs_pitch(int B) { return (vs_col(kFX + B - 2) + 1 + 7) / 16 * 16 + 8; }

template <int BT>
__global__ void __launch_bounds__(kFT) finish_batch_kernel(const __grid_constant__ FinishBatch fb) {
    extern __shared__ long long vs[];
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
    const int pitch = vs_pitch(B);
    const int local = blockIdx.x - P.cta0;
    const int ty = local / P.tiles_x, tx = local - ty * P.tiles_x;
    const int x0 = tx * kFX, y0 = ty * kFY;
    // output mapping: row r of the tile, pixels 8 * seg .. 8 * seg + 7
    const int r = threadIdx.x >> 3, seg = threadIdx.x & 7;
    const int y = y0 + r, xs = x0 + 8 * seg;
    // a full segment of 16-byte aligned rows moves as vectors
    const bool vec = y < P.H && xs + 8 <= P.W &&
                     ((reinterpret_cast<uintptr_t>(P.num) | reinterpret_cast<uintptr_t>(P.src) |
                       reinterpret_cast<uintptr_t>(P.dst)) & 15) == 0 &&
                     ((P.acc_stride | P.sstride | P.dstride) & 3) == 0;
    // vertical sums: quarter q, tile column c (vs column c + B - 1) and, for
    // c < B - 1, halo column c (vs column c)
    {
        const int c = threadIdx.x & (kFX - 1), q = threadIdx.x / kFX;
        const int ytop = y0 + 8 * q - (B - 1);
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1 && c >= B - 1) break;
            const int cc = pass == 0 ? c + B - 1 : c;
            const int xx = x0 - (B - 1) + cc;
            const bool xok = xx >= 0 && xx < P.W;
            const long long* col = P.wsum + xx;
            long long* out = vs + (8 * q) * pitch + vs_col(cc);
            if constexpr (BT > 0) {
                long long w[8 + BT - 1];
#pragma unroll
                for (int i = 0; i < 8 + BT - 1; ++i) {
                    const int yy = ytop + i;
                    w[i] = (xok && yy >= 0 && yy < P.H) ? __ldg(col + (int64_t)yy * P.acc_stride) : 0ll;
                }
                long long sum = 0;
#pragma unroll
                for (int k = 0; k < BT; ++k) sum += w[k];
                out[0] = sum;
#pragma unroll
                for (int rr = 1; rr < 8; ++rr) {
                    sum += w[rr + BT - 1] - w[rr - 1];
                    out[rr * pitch] = sum;
                }
            } else {
                const auto at = [&](int i) {
                    const int yy = ytop + i;
                    return (xok && yy >= 0 && yy < P.H) ? __ldg(col + (int64_t)yy * P.acc_stride) : 0ll;
                };
                long long sum = 0;
                for (int k = 0; k < B; ++k) sum += at(k);
                out[0] = sum;
                for (int rr = 1; rr < 8; ++rr) {
                    sum += at(rr + B - 1) - at(rr - 1);
                    out[rr * pitch] = sum;
                }
            }
        }
    }
    __syncthreads();
    long long* const np = P.num + (int64_t)y * P.acc_stride + xs;
    float* const dp = P.dst + (int64_t)y * P.dstride + xs;
    long long nv[8];
    float sv[8];
    if (vec) {
        const float* sp = P.src + (int64_t)y * P.sstride + xs;
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            const longlong2 t = reinterpret_cast<const longlong2*>(np)[h];
            nv[2 * h] = t.x;
            nv[2 * h + 1] = t.y;
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(sp) + h);
            sv[4 * h] = t.x;
            sv[4 * h + 1] = t.y;
            sv[4 * h + 2] = t.z;
            sv[4 * h + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const bool ok = xs + j < P.W && y < P.H;
            nv[j] = ok ? np[j] : 0;
            sv[j] = ok ? __ldg(P.src + (int64_t)y * P.sstride + xs + j) : 0.f;
        }
    }
    // horizontal sums along this thread's 8 pixels, then the finish
    const long long* row = vs + r * pitch;
    long long den = 0;
    for (int k = 0; k < B; ++k) den += row[vs_col(8 * seg + k)];
    float out[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (j > 0) den += row[vs_col(8 * seg + j + B - 1)] - row[vs_col(8 * seg + j - 1)];
        // den > 1e-12 in real units is den >= 1 in units of 2^-32 (the
        // smallest positive den, 2^-32 = 2.3e-10, already passes)
        out[j] = den > 0 ? fixed_quotient(nv[j], den) : sv[j];
    }
    if (vec) {
#pragma unroll
        for (int h = 0; h < 4; ++h) reinterpret_cast<longlong2*>(np)[h] = make_longlong2(0, 0);
#pragma unroll
        for (int h = 0; h < 2; ++h)
            reinterpret_cast<float4*>(dp)[h] = make_float4(out[4 * h], out[4 * h + 1], out[4 * h + 2], out[4 * h + 3]);
    } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (xs + j < P.W && y < P.H) {
                np[j] = 0;
                dp[j] = out[j];
            }
        }
    }
}

}  // namespace

void launch_finish_batch(const FinishBatch& fb, cudaStream_t stream) {
    if (fb.total_ctas <= 0) return;
    const size_t smem = (size_t)kFY * vs_pitch(fb.block) * sizeof(long long);
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
