// Collaborative filtering for 8x8 blocks and groups of 4, 8, 16 or 32 (sm_100a):
// the default BM3D shapes. Same semantics as group.cu (the reference's
// Bm3dFilterGroup, src/cpu/bm/dct8.cpp:926-1133); the schedule is one warp
// per group, the cube in registers and a padded per-warp shared buffer:
//   - 32/G lanes per patch, each holding 8G/32 rows, then as many columns,
//     then two Haar tubes (coefficient positions l and l+32 across the group);
//     with 32 patches (the "heavy" final stage) a lane holds a whole patch;
//   - the per-patch stride is 64 + 32/G floats and a coefficient's column is
//     XORed with its row's owner lane, so the row, column and tube phases of
//     the 32 lanes each touch 32 different banks;
//   - the inverse runs rows first, then columns (the oracle's order); for
//     groups of up to 8 the columns stay in registers and each lane adds its
//     own patch's pixels to the sums from there;
//   - the 8-point DCT-II is evaluated through its even/odd symmetry: with
//     a_n = x_n + x_{7-n}, b_n = x_n - x_{7-n}, the even outputs are a 4-point
//     DCT of a (split again the same way) and the odd outputs a 4x4 cosine
//     product with b, 36 operations instead of 64 multiply-adds; the inverse
//     is the transpose of the same factorisation.
#include "kernels.cuh"

#include <cmath>

namespace nssb {
namespace {

// cos(pi * m / 16) for m = 1..7
constexpr float kC1 = 0.98078528040323044913f, kC2 = 0.92387953251128675613f, kC3 = 0.83146961230254523708f;
constexpr float kC5 = 0.55557023301960222474f, kC6 = 0.38268343236508977173f, kC7 = 0.19509032201612826785f;
constexpr float kS8 = 0.35355339059327376220f;  // 1/sqrt(8)

__device__ __forceinline__ void fdct8(float* x) {
    const float a0 = x[0] + x[7], a1 = x[1] + x[6], a2 = x[2] + x[5], a3 = x[3] + x[4];
    const float b0 = x[0] - x[7], b1 = x[1] - x[6], b2 = x[2] - x[5], b3 = x[3] - x[4];
    const float e0 = a0 + a3, e1 = a1 + a2, o0 = a0 - a3, o1 = a1 - a2;
    x[0] = (e0 + e1) * kS8;
    x[4] = (e0 - e1) * kS8;
    x[2] = fmaf(0.5f * kC2, o0, 0.5f * kC6 * o1);
    x[6] = fmaf(0.5f * kC6, o0, -0.5f * kC2 * o1);
    // odd: X_k = 1/2 sum_n cos(pi (2n+1) k / 16) b_n
    x[1] = 0.5f * fmaf(kC1, b0, fmaf(kC3, b1, fmaf(kC5, b2, kC7 * b3)));
    x[3] = 0.5f * fmaf(kC3, b0, fmaf(-kC7, b1, fmaf(-kC1, b2, -kC5 * b3)));
    x[5] = 0.5f * fmaf(kC5, b0, fmaf(-kC1, b1, fmaf(kC7, b2, kC3 * b3)));
    x[7] = 0.5f * fmaf(kC7, b0, fmaf(-kC5, b1, fmaf(kC3, b2, -kC1 * b3)));
}

__device__ __forceinline__ void idct8(float* x) {
    const float e0 = (x[0] + x[4]) * kS8, e1 = (x[0] - x[4]) * kS8;
    const float o0 = fmaf(0.5f * kC2, x[2], 0.5f * kC6 * x[6]);
    const float o1 = fmaf(0.5f * kC6, x[2], -0.5f * kC2 * x[6]);
    const float a0 = e0 + o0, a3 = e0 - o0, a1 = e1 + o1, a2 = e1 - o1;
    const float X1 = 0.5f * x[1], X3 = 0.5f * x[3], X5 = 0.5f * x[5], X7 = 0.5f * x[7];
    const float b0 = fmaf(kC1, X1, fmaf(kC3, X3, fmaf(kC5, X5, kC7 * X7)));
    const float b1 = fmaf(kC3, X1, fmaf(-kC7, X3, fmaf(-kC1, X5, -kC5 * X7)));
    const float b2 = fmaf(kC5, X1, fmaf(-kC1, X3, fmaf(kC7, X5, kC3 * X7)));
    const float b3 = fmaf(kC7, X1, fmaf(-kC5, X3, fmaf(kC3, X5, -kC1 * X7)));
    x[0] = a0 + b0;
    x[7] = a0 - b0;
    x[1] = a1 + b1;
    x[6] = a1 - b1;
    x[2] = a2 + b2;
    x[5] = a2 - b2;
    x[3] = a3 + b3;
    x[4] = a3 - b3;
}

template <int G>
__device__ __forceinline__ float haar_scale_c(int j) {
    int e = 0;
    if (j == 0) {
        while ((1 << e) < G) ++e;
    } else {
        while (((j >> e) & 1) == 0) ++e;
        ++e;
    }
    float f = 1.f;
    for (int i = 0; i < e / 2; ++i) f *= 0.5f;
    return e % 2 ? f * 0.70710678118654752f : f;
}

// in-place orthonormal Haar of G samples (dct8.cpp:601-642 layout)
template <int G>
__device__ __forceinline__ void haar_fwd(float* t) {
#pragma unroll
    for (int h = 1; h < G; h <<= 1)
#pragma unroll
        for (int i = 0; i < G; i += 2 * h) {
            const float a = t[i], b = t[i + h];
            t[i] = a + b;
            t[i + h] = a - b;
        }
#pragma unroll
    for (int j = 0; j < G; ++j) t[j] *= haar_scale_c<G>(j);
}

template <int G>
__device__ __forceinline__ void haar_inv(float* t) {
#pragma unroll
    for (int j = 0; j < G; ++j) t[j] *= haar_scale_c<G>(j);
#pragma unroll
    for (int h = G / 2; h >= 1; h >>= 1)
#pragma unroll
        for (int i = 0; i < G; i += 2 * h) {
            const float a = t[i], b = t[i + h];
            t[i] = a + b;
            t[i + h] = a - b;
        }
}

constexpr int kWarps = 4;

// Warps per CTA: the requested count, or fewer where the per-warp cubes (the
// reference cube too for Wiener) would exceed 48 KB of static shared memory
// (groups of 32: 8.3 KB per cube).
template <int G, bool WIENER>
__host__ __device__ constexpr int warps_fit(int want) {
    const int bytes = G * (64 + 32 / G) * 4 * (WIENER ? 2 : 1);
    int w = want;
    while (w > 1 && w * bytes > 48 * 1024) w /= 2;
    return w;
}

template <int G>
struct Shape {
    static constexpr int LP = 32 / G;      // lanes per patch
    static constexpr int RPL = 8 / LP;     // rows (and columns) per lane
    static constexpr int S = 64 + LP;      // patch stride in the shared cube
    // word of coefficient (row, col) within a patch: the column is XORed
    // with the row's owner lane (row / RPL < LP), so row, column and tube
    // accesses of the 32 lanes each touch 32 different banks
    __device__ static __forceinline__ int at(int row, int col) { return row * 8 + (col ^ (row / RPL)); }
};

// rows -> (DCT on rows) -> cube, cube -> columns -> (DCT) -> cube
template <int G, bool INV>
__device__ __forceinline__ void col_pass(float* cube, int g, int q) {
    using Sh = Shape<G>;
#pragma unroll
    for (int t = 0; t < Sh::RPL; ++t) {
        const int c = q + Sh::LP * t;
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = cube[g * Sh::S + Sh::at(i, c)];
        if (INV)
            idct8(v);
        else
            fdct8(v);
#pragma unroll
        for (int i = 0; i < 8; ++i) cube[g * Sh::S + Sh::at(i, c)] = v[i];
    }
}

// Eight consecutive floats of a row starting at any column: from 16-byte
// aligned rows (vec) as the two or three aligned 16-byte chunks covering
// them (a chunk holding a valid float never leaves its allocation), else
// one float at a time.
__device__ __forceinline__ void load_row8(const float* rowp, int px, bool vec, float (&v)[8]) {
    if (vec) {
        const int o = px & 3;
        const float4* a = reinterpret_cast<const float4*>(rowp + (px - o));
        const float4 c0 = __ldg(a), c1 = __ldg(a + 1);
        const float4 c2 = o != 0 ? __ldg(a + 2) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float w[12] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w, c2.x, c2.y, c2.z, c2.w};
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = o == 0 ? w[j] : o == 1 ? w[j + 1] : o == 2 ? w[j + 2] : w[j + 3];
    } else {
        const float* sp = rowp + px;
#pragma unroll
        for (int j = 0; j < 8; ++j) v[j] = __ldg(sp + j);
    }
}

__device__ __forceinline__ bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// One group on one warp. Acc(s) gives the (num, wsum, stride) of slot s,
// Src(s, row, x) / Ref(s, row, x) the source rows. win: the opt-in 8x8
// aggregation window or null; with it each pixel adds its own weight
// w * win to num (times the value) and to its den in wsum.
template <int G, bool WIENER, class SrcRow, class RefRow, class AddNum, class AddWeight>
__device__ __forceinline__ void filter_group(float* cube, float* rcube, int lane, int k, int32_t p, int s,
                                             float sigma, bool vec, SrcRow src_row, RefRow ref_row,
                                             AddNum add_num, AddWeight add_weight, const float* win) {
    using Sh = Shape<G>;
    const int g = lane / Sh::LP, q = lane % Sh::LP;
    const int px = pos_x(p), py = pos_y(p);
    // gather and row transforms
#pragma unroll
    for (int r = 0; r < Sh::RPL; ++r) {
        const int row = q * Sh::RPL + r;
        float v[8], w[8];
        if (g < k) {
            load_row8(src_row(s, py + row), px, vec, v);
            if (WIENER) load_row8(ref_row(s, py + row), px, vec, w);
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = w[j] = 0.f;
        }
        fdct8(v);
#pragma unroll
        for (int j = 0; j < 8; ++j) cube[g * Sh::S + Sh::at(row, j)] = v[j];
        if (WIENER) {
            fdct8(w);
#pragma unroll
            for (int j = 0; j < 8; ++j) rcube[g * Sh::S + Sh::at(row, j)] = w[j];
        }
    }
    __syncwarp();
    col_pass<G, false>(cube, g, q);
    if (WIENER) col_pass<G, false>(rcube, g, q);
    __syncwarp();
    // Haar tubes, shrinkage, inverse Haar: positions lane and lane + 32
    int kept = 0;
    float w2 = 0.f;
#pragma unroll (G >= 16 ? 1 : 2)  // large groups: one copy of the tube code (instruction cache)
    for (int h = 0; h < 2; ++h) {
        const int f = lane + 32 * h, fa = Sh::at(f >> 3, f & 7);
        float t[G];
#pragma unroll
        for (int gg = 0; gg < G; ++gg) t[gg] = cube[gg * Sh::S + fa];
        haar_fwd<G>(t);
        if (WIENER) {
            float r[G];
#pragma unroll
            for (int gg = 0; gg < G; ++gg) r[gg] = rcube[gg * Sh::S + fa];
            haar_fwd<G>(r);
            const float sig2 = sigma * sigma;
#pragma unroll
            for (int gg = 0; gg < G; ++gg) {
                float wt = 1.f;
                if (!(gg == 0 && f == 0)) {
                    const float r2 = r[gg] * r[gg];
                    const float den = r2 + sig2;
                    wt = den > 0.f ? __fdiv_rn(r2, den) : 0.f;
                }
                t[gg] *= wt;
                w2 = fmaf(wt, wt, w2);
            }
        } else {
            const float thr = 2.7f * sigma;
#pragma unroll
            for (int gg = 0; gg < G; ++gg) {
                if (!(gg == 0 && f == 0) && fabsf(t[gg]) < thr) {
                    t[gg] = 0.f;
                } else {
                    ++kept;
                }
            }
        }
        haar_inv<G>(t);
#pragma unroll
        for (int gg = 0; gg < G; ++gg) cube[gg * Sh::S + fa] = t[gg];
    }
    float weight;
    if (WIENER) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w2 += __shfl_xor_sync(0xffffffffu, w2, o);
        weight = __fdiv_rn(1.f, fmaxf(w2, 1e-12f));
    } else {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) kept += __shfl_xor_sync(0xffffffffu, kept, o);
        weight = __fdiv_rn(1.f, (float)(kept > 1 ? kept : 1));
    }
    // w * v rounds once in FP32; the 2^32 scale is exact, so it goes on the
    // weight first: (w 2^32) v == (w v) 2^32 bit for bit (barring overflow)
    const float wscaled = weight * kFixedScale;
    __syncwarp();
    if constexpr (G <= 8) {
        // inverse rows in the cube, then inverse columns kept in registers and
        // added from there: lane (g, q) holds columns q + LP t of its own
        // patch, so the LP lanes of a patch add LP adjacent pixels of a row
#pragma unroll
        for (int r = 0; r < Sh::RPL; ++r) {
            const int row = q * Sh::RPL + r;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = cube[g * Sh::S + Sh::at(row, j)];
            idct8(v);
#pragma unroll
            for (int j = 0; j < 8; ++j) cube[g * Sh::S + Sh::at(row, j)] = v[j];
        }
        __syncwarp();
        if (g < k) {
            if (q == 0 && !win) add_weight(s, px, py, __float2ll_rn(wscaled));
#pragma unroll
            for (int t = 0; t < Sh::RPL; ++t) {
                const int c = q + Sh::LP * t;
                float v[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] = cube[g * Sh::S + Sh::at(i, c)];
                idct8(v);
                if (win) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const float ww = __fmul_rn(weight, __ldg(win + i * 8 + c));
                        add_num(s, px + c, py + i, to_fixed(__fmul_rn(ww, v[i])));
                        add_weight(s, px + c, py + i, to_fixed(ww));
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        add_num(s, px + c, py + i, __float2ll_rn(__fmul_rn(wscaled, v[i])));
                }
            }
        }
    } else {
        // groups of 16 (two lanes per patch): inverse columns, inverse rows,
        // then 8 consecutive lanes on 8 consecutive pixels of a row, a warp
        // instruction covering 4 rows of one patch (k is the same on every
        // lane, so the loop ends for the whole warp at once)
        col_pass<G, true>(cube, g, q);
        __syncwarp();
#pragma unroll
        for (int r = 0; r < Sh::RPL; ++r) {
            const int row = q * Sh::RPL + r;
            float v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = cube[g * Sh::S + Sh::at(row, j)];
            idct8(v);
#pragma unroll
            for (int j = 0; j < 8; ++j) cube[g * Sh::S + Sh::at(row, j)] = v[j];
        }
        if (g < k && q == 0 && !win) add_weight(s, px, py, __float2ll_rn(wscaled));
        __syncwarp();
#pragma unroll (G >= 16 ? 1 : G)
        for (int gg = 0; gg < G; ++gg) {
            if (gg >= k) break;
            const int32_t pp = __shfl_sync(0xffffffffu, p, gg * Sh::LP);
            const int ss = __shfl_sync(0xffffffffu, s, gg * Sh::LP);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i = 4 * h + (lane >> 3), j = lane & 7;
                const float v = cube[gg * Sh::S + Sh::at(i, j)];
                if (win) {
                    const float ww = __fmul_rn(weight, __ldg(win + i * 8 + j));
                    add_num(ss, pos_x(pp) + j, pos_y(pp) + i, to_fixed(__fmul_rn(ww, v)));
                    add_weight(ss, pos_x(pp) + j, pos_y(pp) + i, to_fixed(ww));
                } else {
                    add_num(ss, pos_x(pp) + j, pos_y(pp) + i, __float2ll_rn(__fmul_rn(wscaled, v)));
                }
            }
        }
    }
    __syncwarp();
}

// Temporal / single-plane form: slots of GroupIO.
template <int G, bool WIENER, int NW = warps_fit<G, WIENER>(kWarps)>
__global__ void __launch_bounds__(32 * NW) group8_kernel(GroupIO io, const int32_t* __restrict__ pos,
                                                         const int32_t* __restrict__ slot,
                                                         const int32_t* __restrict__ count, int njobs,
                                                         float sigma) {
    using Sh = Shape<G>;
    constexpr int CUBE = G * Sh::S;
    __shared__ float smem[NW][WIENER ? 2 * CUBE : CUBE];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / Sh::LP;
    const int stride_w = gridDim.x * NW;
    bool vec = io.stride % 4 == 0 && io.ref_stride % 4 == 0;
    for (int q = 0; q < kMaxSlots; ++q) vec = vec && aligned16(io.src[q]) && aligned16(io.ref[q]);
    for (int job = blockIdx.x * NW + warp; job < njobs; job += stride_w) {
        const int k = count[job];
        if (k <= 0) continue;
        const int32_t p = g < k ? pos[(size_t)job * G + g] : 0;
        const int s = (slot && g < k) ? slot[(size_t)job * G + g] : 0;
        filter_group<G, WIENER>(
            smem[warp], smem[warp] + CUBE, lane, k, p, s, sigma, vec,
            [&](int sl, int row) { return io.src[sl] + (int64_t)row * io.stride; },
            [&](int sl, int row) { return io.ref[sl] + (int64_t)row * io.ref_stride; },
            [&](int sl, int x, int y, long long v) {
                atomicAdd(reinterpret_cast<unsigned long long*>(io.num[sl] + (int64_t)y * io.acc_stride + x),
                          (unsigned long long)v);
            },
            [&](int sl, int x, int y, long long v) {
                atomicAdd(reinterpret_cast<unsigned long long*>(io.wsum[sl] + (int64_t)y * io.acc_stride + x),
                          (unsigned long long)v);
            },
            io.win);
    }
}

// Temporal centre, batched over its planes: each plane with its own slots;
// the next job's count, positions and slots are read ahead as in the
// batched form below.
template <int G, bool WIENER, int NW = warps_fit<G, WIENER>(kWarps)>
__global__ void __launch_bounds__(32 * NW) group8_slots_batch_kernel(const __grid_constant__ GroupSlotBatch gb) {
    using Sh = Shape<G>;
    constexpr int CUBE = G * Sh::S;
    __shared__ float smem[NW][WIENER ? 2 * CUBE : CUBE];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / Sh::LP;
    const int stride_w = gridDim.x * NW;
    // planes whose every slot row is 16-byte aligned
    int vec_mask = 0;
    for (int q = 0; q < gb.n; ++q) {
        const GroupIO& io = gb.p[q].io;
        bool vec = io.stride % 4 == 0 && io.ref_stride % 4 == 0;
        for (int t = 0; t < kMaxSlots; ++t) vec = vec && aligned16(io.src[t]) && aligned16(io.ref[t]);
        vec_mask |= int(vec) << q;
    }
    int pl = 0;
    const auto fetch = [&](int jb, int& k, int32_t& p, int& s, int& plane) {
        while (pl + 1 < gb.n && gb.p[pl + 1].job0 <= jb) ++pl;
        const GroupSlotPlane& P_ = gb.p[pl];
        const int lj = jb - P_.job0;
        k = P_.count[lj];
        p = g < k ? P_.pos[(size_t)lj * G + g] : 0;
        s = (P_.slot && g < k) ? P_.slot[(size_t)lj * G + g] : 0;
        plane = pl;
    };
    int job = blockIdx.x * NW + warp;
    int k = 0, s = 0, plane = 0;
    int32_t p = 0;
    if (job < gb.total_jobs) fetch(job, k, p, s, plane);
    for (; job < gb.total_jobs; job += stride_w) {
        int kn = 0, sn = 0, plane_n = plane;
        int32_t pn = 0;
        if (job + stride_w < gb.total_jobs) fetch(job + stride_w, kn, pn, sn, plane_n);
        if (k > 0) {
            const GroupSlotPlane& P_ = gb.p[plane];
            const GroupIO& io = P_.io;
            filter_group<G, WIENER>(
                smem[warp], smem[warp] + CUBE, lane, k, p, s, P_.sigma, (vec_mask >> plane) & 1,
                [&](int sl, int row) { return io.src[sl] + (int64_t)row * io.stride; },
                [&](int sl, int row) { return io.ref[sl] + (int64_t)row * io.ref_stride; },
                [&](int sl, int x, int y, long long v) {
                    atomicAdd(reinterpret_cast<unsigned long long*>(io.num[sl] + (int64_t)y * io.acc_stride + x),
                              (unsigned long long)v);
                },
                [&](int sl, int x, int y, long long v) {
                    atomicAdd(reinterpret_cast<unsigned long long*>(io.wsum[sl] + (int64_t)y * io.acc_stride + x),
                              (unsigned long long)v);
                },
                io.win);
        }
        k = kn;
        s = sn;
        p = pn;
        plane = plane_n;
    }
}

// Batched form: every job of every plane of the batch, a warp per group. A
// warp reads its next job's count and positions before it filters the
// current one, so that dependent pair of loads overlaps the transforms.
template <int G, bool WIENER, int NW>
__global__ void __launch_bounds__(32 * NW) group8_batch_kernel(const __grid_constant__ GroupBatch gb) {
    using Sh = Shape<G>;
    constexpr int CUBE = G * Sh::S;
    __shared__ float smem[NW][WIENER ? 2 * CUBE : CUBE];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane / Sh::LP;
    const int stride_w = gridDim.x * NW;
    int pl = 0;
    const auto fetch = [&](int jb, int& k, int32_t& p, int& plane) {
        while (pl + 1 < gb.n && gb.p[pl + 1].job0 <= jb) ++pl;
        const GroupPlane& P_ = gb.p[pl];
        const int lj = jb - P_.job0;
        k = P_.count[lj];
        p = g < k ? P_.pos[(size_t)lj * G + g] : 0;
        plane = pl;
    };
    int job = blockIdx.x * NW + warp;
    int k = 0, plane = 0;
    int32_t p = 0;
    if (job < gb.total_jobs) fetch(job, k, p, plane);
    for (; job < gb.total_jobs; job += stride_w) {
        int kn = 0, plane_n = plane;
        int32_t pn = 0;
        if (job + stride_w < gb.total_jobs) fetch(job + stride_w, kn, pn, plane_n);
        if (k > 0) {
            const GroupPlane& P_ = gb.p[plane];
            const bool vec = P_.stride % 4 == 0 && P_.ref_stride % 4 == 0 && aligned16(P_.src) && aligned16(P_.ref);
            filter_group<G, WIENER>(
                smem[warp], smem[warp] + CUBE, lane, k, p, 0, P_.sigma, vec,
                [&](int, int row) { return P_.src + (int64_t)row * P_.stride; },
                [&](int, int row) { return P_.ref + (int64_t)row * P_.ref_stride; },
                [&](int, int x, int y, long long v) {
                    atomicAdd(reinterpret_cast<unsigned long long*>(P_.num + (int64_t)y * P_.acc_stride + x),
                              (unsigned long long)v);
                },
                [&](int, int x, int y, long long v) {
                    atomicAdd(reinterpret_cast<unsigned long long*>(P_.wsum + (int64_t)y * P_.acc_stride + x),
                              (unsigned long long)v);
                },
                P_.win);
        }
        k = kn;
        p = pn;
        plane = plane_n;
    }
}

template <int G, bool W>
void launch_gw(const GroupIO& io, const int32_t* pos, const int32_t* slot, const int32_t* count, int njobs,
               float sigma, cudaStream_t stream) {
    constexpr int NW = warps_fit<G, W>(kWarps);
    const int blocks = std::min(ceil_div(njobs, NW), 148 * 16);
    group8_kernel<G, W><<<blocks, 32 * NW, 0, stream>>>(io, pos, slot, count, njobs, sigma);
    NSSB_CUDA(cudaGetLastError());
}

template <int G, bool W, int NW>
void launch_batch_gwn(const GroupBatch& gb, int ctas_per_sm, cudaStream_t stream) {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        NSSB_CUDA(cudaGetDevice(&dev));
        NSSB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    const int blocks = std::min(ceil_div(gb.total_jobs, NW), sms * std::max(1, ctas_per_sm));
    group8_batch_kernel<G, W, NW><<<blocks, 32 * NW, 0, stream>>>(gb);
    NSSB_CUDA(cudaGetLastError());
}

template <int G, bool W>
void launch_batch_gw(const GroupBatch& gb, const GroupTune& t, cudaStream_t stream) {
    // the requested warps per CTA, fewer where the cubes would not fit
    switch (t.warps) {
        case 2: launch_batch_gwn<G, W, warps_fit<G, W>(2)>(gb, t.ctas_per_sm, stream); break;
        case 8: launch_batch_gwn<G, W, warps_fit<G, W>(8)>(gb, t.ctas_per_sm, stream); break;
        default: launch_batch_gwn<G, W, warps_fit<G, W>(4)>(gb, t.ctas_per_sm, stream); break;
    }
}

}  // namespace

bool launch_group8(const GroupIO& io, const int32_t* pos, const int32_t* slot, const int32_t* count, int njobs,
                   int group, float sigma, bool wiener, cudaStream_t stream) {
    if (njobs <= 0) return true;
    switch (group) {
        case 4:
            wiener ? launch_gw<4, true>(io, pos, slot, count, njobs, sigma, stream)
                   : launch_gw<4, false>(io, pos, slot, count, njobs, sigma, stream);
            return true;
        case 8:
            wiener ? launch_gw<8, true>(io, pos, slot, count, njobs, sigma, stream)
                   : launch_gw<8, false>(io, pos, slot, count, njobs, sigma, stream);
            return true;
        case 16:
            wiener ? launch_gw<16, true>(io, pos, slot, count, njobs, sigma, stream)
                   : launch_gw<16, false>(io, pos, slot, count, njobs, sigma, stream);
            return true;
        case 32:
            wiener ? launch_gw<32, true>(io, pos, slot, count, njobs, sigma, stream)
                   : launch_gw<32, false>(io, pos, slot, count, njobs, sigma, stream);
            return true;
        default:
            return false;
    }
}

bool launch_group8_slots_batch(const GroupSlotBatch& gb, int group, bool wiener, cudaStream_t stream) {
    if (gb.total_jobs <= 0) return true;
    auto go = [&](auto kern) {
        cudaFuncAttributes fa{};
        NSSB_CUDA(cudaFuncGetAttributes(&fa, kern));
        const int nw = fa.maxThreadsPerBlock >= 32 * kWarps ? kWarps : fa.maxThreadsPerBlock / 32;
        const int blocks = std::min(ceil_div(gb.total_jobs, nw), 148 * 16);
        kern<<<blocks, 32 * nw, 0, stream>>>(gb);
        NSSB_CUDA(cudaGetLastError());
    };
    switch (group) {
        case 4: wiener ? go(group8_slots_batch_kernel<4, true>) : go(group8_slots_batch_kernel<4, false>); return true;
        case 8: wiener ? go(group8_slots_batch_kernel<8, true>) : go(group8_slots_batch_kernel<8, false>); return true;
        case 16:
            wiener ? go(group8_slots_batch_kernel<16, true>) : go(group8_slots_batch_kernel<16, false>);
            return true;
        case 32:
            wiener ? go(group8_slots_batch_kernel<32, true>) : go(group8_slots_batch_kernel<32, false>);
            return true;
        default: return false;
    }
}

bool launch_group8_batch(const GroupBatch& gb, int group, bool wiener, cudaStream_t stream, const GroupTune* tune) {
    if (gb.total_jobs <= 0) return true;
    const GroupTune t = tune ? *tune : GroupTune{};
    switch (group) {
        case 4: wiener ? launch_batch_gw<4, true>(gb, t, stream) : launch_batch_gw<4, false>(gb, t, stream); return true;
        case 8: wiener ? launch_batch_gw<8, true>(gb, t, stream) : launch_batch_gw<8, false>(gb, t, stream); return true;
        case 16:
            wiener ? launch_batch_gw<16, true>(gb, t, stream) : launch_batch_gw<16, false>(gb, t, stream);
            return true;
        case 32:
            wiener ? launch_batch_gw<32, true>(gb, t, stream) : launch_batch_gw<32, false>(gb, t, stream);
            return true;
        default: return false;
    }
}

}  // namespace nssb
