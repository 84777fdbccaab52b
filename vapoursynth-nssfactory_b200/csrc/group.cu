// Collaborative filtering of the groups and aggregation (sm_100a), every
// block x group shape.
//
// Semantics (reference Bm3dFilterGroup, src/cpu/bm/dct8.cpp:926-1133; the
// device form src/cuda/bm3d/kernels.cu:247-327): the k patches of a group,
// zero-padded to `group`, take the orthonormal 2-D DCT-II (rows, then
// columns), then the orthonormal Haar transform along the group in its
// in-place layout (dct8.cpp:576-644). Hard threshold keeps the coefficients
// with |c| >= 2.7 sigma and always the DC of the DC; the weight is 1/kept.
// Wiener takes w = r^2 / (r^2 + sigma^2) from the reference cube (w = 1 at the
// DC of the DC), the weight is 1 / max(sum w^2, 1e-12). The inverse transforms
// run in the same order; every real patch then adds w * value to num of its
// pixels and w to the weight of its origin (den is the box sum of those,
// taken by the finish kernel).
//
// One CTA per group (grid-stride), the cube in shared memory, or in a global
// scratch slice per CTA when the shape does not fit (blocks 16/32 with big
// groups). Line transforms run one thread per line from the DCT matrix, with
// the same FMA order as the CPU oracle's matrix form.
#include "kernels.cuh"

#include <cmath>
#include <mutex>

namespace nssb {

// DCT-II tables of the block sizes 1, 2, 4, 8, 12, 16, 32, row k = frequency.
__device__ float g_dct_tables[1 + 4 + 16 + 64 + 144 + 256 + 1024];

namespace {

__host__ __device__ constexpr int dct_offset(int n) {
    return n == 1 ? 0 : n == 2 ? 1 : n == 4 ? 5 : n == 8 ? 21 : n == 12 ? 85 : n == 16 ? 229 : 485;
}

std::once_flag g_tables_once[64];

}  // namespace

// Uploads the DCT tables to the current device once (a synchronous copy: the
// first call on a device must not be made under stream capture). An upload
// that throws leaves the flag unset, so the next call tries again.
void ensure_group_tables() {
    int dev = 0;
    NSSB_CUDA(cudaGetDevice(&dev));
    std::call_once(g_tables_once[dev & 63], [] {
        static float host[1509];
        const double pi = 3.14159265358979323846264338327950288;
        for (int n : {1, 2, 4, 8, 12, 16, 32}) {
            const double s0 = std::sqrt(1.0 / n), s1 = std::sqrt(2.0 / n);
            for (int k = 0; k < n; ++k)
                for (int i = 0; i < n; ++i)
                    host[dct_offset(n) + k * n + i] = (float)((k == 0 ? s0 : s1) * std::cos(pi * (i + 0.5) * k / n));
        }
        NSSB_CUDA(cudaMemcpyToSymbol(g_dct_tables, host, sizeof host));
    });
}

namespace {

__device__ __forceinline__ float haar_scale(int n, int j) {
    int e = 0;
    if (j == 0) {
        while ((1 << e) < n) ++e;
    } else {
        while (((j >> e) & 1) == 0) ++e;
        ++e;
    }
    float f = 1.f;
    for (int i = 0; i < e / 2; ++i) f *= 0.5f;
    return e % 2 ? f * 0.70710678118654752f : f;
}

// count lines of B samples, sample i of line v at base[v*ls + i*ss]
template <int B>
__device__ void dct_line(float* p, int ss, const float* T, bool inverse) {
    float x[B];
#pragma unroll
    for (int i = 0; i < B; ++i) x[i] = p[i * ss];
#pragma unroll
    for (int o = 0; o < B; ++o) {
        float acc = 0.f;
#pragma unroll
        for (int q = 0; q < B; ++q) acc = __fmaf_rn(inverse ? T[q * B + o] : T[o * B + q], x[q], acc);
        p[o * ss] = acc;
    }
}

__device__ void haar_line(float* p, int n, int ss, bool inverse) {
    if (n <= 1) return;
    if (inverse) {
        for (int j = 0; j < n; ++j) p[j * ss] = __fmul_rn(p[j * ss], haar_scale(n, j));
        for (int h = n / 2; h >= 1; h >>= 1)
            for (int i = 0; i < n; i += 2 * h) {
                const float a = p[i * ss], b = p[(i + h) * ss];
                p[i * ss] = __fadd_rn(a, b);
                p[(i + h) * ss] = __fsub_rn(a, b);
            }
    } else {
        for (int h = 1; h < n; h <<= 1)
            for (int i = 0; i < n; i += 2 * h) {
                const float a = p[i * ss], b = p[(i + h) * ss];
                p[i * ss] = __fadd_rn(a, b);
                p[(i + h) * ss] = __fsub_rn(a, b);
            }
        for (int j = 0; j < n; ++j) p[j * ss] = __fmul_rn(p[j * ss], haar_scale(n, j));
    }
}

// rows of every patch, then columns (forward and inverse alike)
template <int B>
__device__ void dct2(float* cube, int G, const float* T, bool inverse, int cubes, int cube_stride) {
    constexpr int A = B * B;
    if constexpr (B == 1) return;
    for (int l = threadIdx.x; l < G * B * cubes; l += blockDim.x) {
        const int c = l / (G * B), r = l - c * (G * B);
        dct_line<B>(cube + c * cube_stride + r * B, 1, T, inverse);
    }
    __syncthreads();
    for (int l = threadIdx.x; l < G * B * cubes; l += blockDim.x) {
        const int c = l / (G * B), r = l - c * (G * B);
        const int g = r / B, j = r - g * B;
        dct_line<B>(cube + c * cube_stride + g * A + j, B, T, inverse);
    }
    __syncthreads();
}

template <int B>
__global__ void __launch_bounds__(128) group_kernel(GroupIO io, int W, int H, const int32_t* __restrict__ pos,
                                                    const int32_t* __restrict__ slot,
                                                    const int32_t* __restrict__ count, int njobs, int G, float sigma,
                                                    int wiener, float* scratch, int in_smem) {
    constexpr int A = B * B;
    extern __shared__ float sm[];
    float* T = sm;                         // A
    float* redf = sm + A;                  // 4 warps
    int* redi = reinterpret_cast<int*>(redf + 4);
    float* smcube = redf + 8;
    const float* tab = g_dct_tables + dct_offset(B);
    for (int i = threadIdx.x; i < A; i += blockDim.x) T[i] = tab[i];
    const int ncubes = wiener ? 2 : 1;
    const int cs = G * A;
    float* cube = in_smem ? smcube : scratch + (size_t)blockIdx.x * cs * ncubes;
    float* rcube = cube + cs;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    __syncthreads();
    for (int job = blockIdx.x; job < njobs; job += gridDim.x) {
        const int k = count[job];
        if (k <= 0) continue;
        const int32_t* jp = pos + (size_t)job * G;
        const int32_t* js = slot ? slot + (size_t)job * G : nullptr;
        for (int idx = tid; idx < cs; idx += blockDim.x) {
            const int g = idx / A, e = idx - g * A, i = e / B, j = e - i * B;
            float v = 0.f, r = 0.f;
            if (g < k) {
                const int32_t p = jp[g];
                const int s = js ? js[g] : 0;
                const int64_t row = pos_y(p) + i, col = pos_x(p) + j;
                v = __ldg(io.src[s] + row * io.stride + col);
                if (wiener) r = __ldg(io.ref[s] + row * io.ref_stride + col);
            }
            cube[idx] = v;
            if (wiener) rcube[idx] = r;
        }
        __syncthreads();
        dct2<B>(cube, G, T, false, ncubes, cs);
        for (int l = tid; l < A * ncubes; l += blockDim.x) haar_line(cube + (l / A) * cs + (l % A), G, A, false);
        __syncthreads();
        // shrinkage
        int kept = 0;
        float w2 = 0.f;
        if (wiener) {
            const float sig2 = __fmul_rn(sigma, sigma);
            for (int i = tid; i < cs; i += blockDim.x) {
                float w = 1.f;
                if (i != 0) {
                    const float rr = rcube[i];
                    const float r2 = __fmul_rn(rr, rr);
                    const float den = __fadd_rn(r2, sig2);
                    w = den > 0.f ? __fdiv_rn(r2, den) : 0.f;
                }
                cube[i] = __fmul_rn(cube[i], w);
                w2 = __fmaf_rn(w, w, w2);
            }
        } else {
            const float thr = __fmul_rn(2.7f, sigma);
            for (int i = tid; i < cs; i += blockDim.x) {
                const float c = cube[i];
                if (i != 0 && fabsf(c) < thr) {
                    cube[i] = 0.f;
                } else {
                    ++kept;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            w2 = __fadd_rn(w2, __shfl_down_sync(0xffffffffu, w2, o));
            kept += __shfl_down_sync(0xffffffffu, kept, o);
        }
        if (lane == 0) {
            redf[warp] = w2;
            redi[warp] = kept;
        }
        __syncthreads();
        float weight;
        if (wiener) {
            float s = 0.f;
            for (int q = 0; q < int(blockDim.x >> 5); ++q) s = __fadd_rn(s, redf[q]);
            weight = __fdiv_rn(1.f, fmaxf(s, 1e-12f));
        } else {
            int s = 0;
            for (int q = 0; q < int(blockDim.x >> 5); ++q) s += redi[q];
            weight = __fdiv_rn(1.f, (float)(s > 1 ? s : 1));
        }
        for (int l = tid; l < A; l += blockDim.x) haar_line(cube + l, G, A, true);
        __syncthreads();
        dct2<B>(cube, G, T, true, 1, cs);
        // aggregation
        for (int idx = tid; idx < k * A; idx += blockDim.x) {
            const int g = idx / A, e = idx - g * A, i = e / B, j = e - i * B;
            const int32_t p = jp[g];
            const int s = js ? js[g] : 0;
            const int64_t off = (int64_t)(pos_y(p) + i) * io.acc_stride + pos_x(p) + j;
            // opt-in window: the pixel's own weight, its den per pixel
            const float ww = io.win ? __fmul_rn(weight, __ldg(io.win + e)) : weight;
            atomicAdd(reinterpret_cast<unsigned long long*>(io.num[s] + off),
                      static_cast<unsigned long long>(to_fixed(__fmul_rn(ww, cube[idx]))));
            if (io.win)
                atomicAdd(reinterpret_cast<unsigned long long*>(io.wsum[s] + off),
                          static_cast<unsigned long long>(to_fixed(ww)));
        }
        for (int g = tid; g < k && !io.win; g += blockDim.x) {
            const int32_t p = jp[g];
            const int s = js ? js[g] : 0;
            const int64_t off = (int64_t)pos_y(p) * io.acc_stride + pos_x(p);
            atomicAdd(reinterpret_cast<unsigned long long*>(io.wsum[s] + off),
                      static_cast<unsigned long long>(to_fixed(weight)));
        }
        __syncthreads();
    }
}

size_t cube_floats(int block, int group, bool wiener) { return (size_t)group * block * block * (wiener ? 2 : 1); }
constexpr size_t kSmemCubeLimit = 160 * 1024;

template <int B>
void launch_group_b(const GroupIO& io, int W, int H, const int32_t* pos, const int32_t* slot, const int32_t* count,
                    int njobs, int G, float sigma, bool wiener, float* scratch, size_t scratch_floats,
                    cudaStream_t stream) {
    const size_t cf = cube_floats(B, G, wiener);
    const size_t head = (size_t)B * B + 8;
    const bool in_smem = cf * sizeof(float) <= kSmemCubeLimit;
    const size_t smem = (head + (in_smem ? cf : 0)) * sizeof(float);
    int grid = njobs;
    if (!in_smem) {
        const size_t slices = scratch_floats / cf;
        if (slices == 0) throw std::invalid_argument("nss_cuda: group scratch too small");
        grid = (int)std::min<size_t>(slices, (size_t)njobs);
    }
    auto kern = group_kernel<B>;
    NSSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<grid, 128, smem, stream>>>(io, W, H, pos, slot, count, njobs, G, sigma, wiener ? 1 : 0, scratch,
                                      in_smem ? 1 : 0);
    NSSB_CUDA(cudaGetLastError());
}

}  // namespace

size_t group_filter_scratch_floats(int block, int group, bool wiener) {
    const size_t cf = cube_floats(block, group, wiener);
    if (cf * sizeof(float) <= kSmemCubeLimit) return 0;
    return cf * 296;  // two slices per SM of a 148-SM part
}

void launch_group_filter(const GroupIO& io, int width, int height, const int32_t* pos, const int32_t* slot,
                         const int32_t* count, int njobs, int block, int group, float sigma, bool wiener,
                         float* scratch, size_t scratch_floats, cudaStream_t stream) {
    if (njobs <= 0) return;
    if (block == 8 && launch_group8(io, pos, slot, count, njobs, group, sigma, wiener, stream)) return;
    ensure_group_tables();
    switch (block) {
        case 1: return launch_group_b<1>(io, width, height, pos, slot, count, njobs, group, sigma, wiener, scratch, scratch_floats, stream);
        case 2: return launch_group_b<2>(io, width, height, pos, slot, count, njobs, group, sigma, wiener, scratch, scratch_floats, stream);
        case 4: return launch_group_b<4>(io, width, height, pos, slot, count, njobs, group, sigma, wiener, scratch, scratch_floats, stream);
        case 8: return launch_group_b<8>(io, width, height, pos, slot, count, njobs, group, sigma, wiener, scratch, scratch_floats, stream);
        case 12: return launch_group_b<12>(io, width, height, pos, slot, count, njobs, group, sigma, wiener, scratch, scratch_floats, stream);
        case 16: return launch_group_b<16>(io, width, height, pos, slot, count, njobs, group, sigma, wiener, scratch, scratch_floats, stream);
        case 32: return launch_group_b<32>(io, width, height, pos, slot, count, njobs, group, sigma, wiener, scratch, scratch_floats, stream);
        default: throw std::invalid_argument("nss_cuda: unsupported block size");
    }
}

}  // namespace nssb
