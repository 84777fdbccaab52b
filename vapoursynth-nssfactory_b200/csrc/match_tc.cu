// Precision form of the 8x8 matcher: distances scored on the sm_100a tensor
// cores, groups re-ranked exactly (the result equals match8.cu's, bit for bit).
//
// d(r, c) = |r|^2 + |c|^2 - 2 r.c. The dot products come from tcgen05.mma
// (kind::f16, BF16 inputs, FP32 accumulation in tensor memory) with every
// pixel split as hi = bf16(v), lo = bf16(v - hi): r.c ~ rh.ch + rh.cl + rl.ch,
// three MMAs into one accumulator. With u = 2^-8, the split leaves
// |r.c - that| <= ~3.1 u^2 S plus FP32 accumulation, S = sum |r_i c_i| <=
// sqrt(|r|^2 |c|^2), i.e. |d~ - d| <= 1.42e-4 S + (norm and final roundings);
// the kernel takes E = 2.9e-4 sqrt(|r|^2 max|c|^2) + 1e-5 (|r|^2 + max|c|^2)
// + 2e-6 |U| (twice the derived bound) as the per-reference error margin. With U >= the K-th smallest approximate
// distance, every exact top-K candidate c has d~(c) <= U + 2E; those
// "survivors" get the exact FP32 distance in this build's order (per-column
// FMA chains, then the column tree) and the exact keys pick the group. A tile
// with any non-finite pixel treats every candidate as a survivor.
//
// Tile: 14 references of one grid row (x span 104 + 2R + 1 <= 128) of one
// plane of a batch; one CTA of 256 threads.
//   A (M = 128 candidates x K = 64 pixels) is MN-major and never materialised
//     per candidate row: image row Y is stored once as a "shift block"
//     S_Y[g][j][m'] = v(Y, X0 + 8g + j + m') (16 groups x 8 shifts x 8, bf16),
//     so the K-slice (pixel rows i, i+1) of candidate row y is the pair of
//     blocks S_{y+i}, S_{y+i+1}: descriptor start at S_{y+i}, core-matrix
//     stride (SBO) 128 B along M, block stride (LBO) along K. Each image row
//     is converted once and serves the 8 candidate rows overlapping it.
//   B (N = 16 references x K = 64) is K-major: 8 references x 8 pixels per
//     128-byte core matrix, pixel rows 128 B apart (LBO), the two reference
//     groups 1 KB apart (SBO).
//   D: 128 lanes x 16 FP32 columns, two buffers in 32 allocated columns, so
//     the MMAs of candidate row c+1 run while row c is read back.
// Reference counterpart: the reference's large-window tensor matcher
// (src/cuda/common/match.cu, mma.sync path; docs/api/cuda/bm3d.md:20-59) --
// this one is tcgen05/TMEM-based and exact.
#include "kernels.cuh"
#include "tcgen05.cuh"

#include <algorithm>

namespace nssb {
namespace {

using namespace tc;

constexpr int kTcRefs = 14;
constexpr int kTcThreads = 256;
constexpr int kBlockBytes = 2048;  // one image row's shift block (bf16)

template <int R>
struct Tc {
    static constexpr int NC = 2 * R + 1;  // candidates per window axis
    static constexpr int RB = NC + 7;     // image rows of a tile
    static constexpr int NW = NC * NC;    // window entries per reference
    // dynamic shared memory layout (bytes)
    static constexpr int A_HI = 0;
    static constexpr int A_LO = A_HI + RB * kBlockBytes;
    static constexpr int B_HI = A_LO + RB * kBlockBytes;
    static constexpr int B_LO = B_HI + 2048;
    static constexpr int DIST = B_LO + 2048;                  // float [kTcRefs][NW]
    static constexpr int NCS = DIST + kTcRefs * NW * 4;       // float [NC][128] candidate norms
    static constexpr int RS = NCS + NC * 128 * 4;             // float [RB][128] row sums of squares
    static constexpr int SURV = RS + RB * 128 * 4;            // uint16 [8 warps][NW] survivor indices
    static constexpr int TP = 136;                            // FP32 tile pitch (>= 128 + 7)
    static constexpr int TILE = SURV + 8 * NW * 2;            // float [RB][TP] the tile's pixels, exact
    static constexpr int BYTES = TILE + RB * TP * 4;
};

// kind::f16: F32 accumulate, BF16 A (MN-major) and B (K-major), M = 128, N = 16.
constexpr uint32_t kIdesc = tc::idesc_bf16(128, 16, true, false);

__device__ __forceinline__ uint64_t tc_key(float d, int x, int y) {
    uint32_t b = __float_as_uint(d);
    if ((b & 0x7f800000u) == 0x7f800000u) b = 0x7f800000u;
    return (uint64_t(b) << 32) | (uint64_t(uint32_t(y)) << 16) | uint64_t(uint32_t(x));
}

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u < v ? u : v;
    }
    return v;
}

__device__ __forceinline__ float warp_max_ratio(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_min_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Exact SSD in this build's order (per-column FMA chains, column tree).
__device__ __forceinline__ float ssd8_exact(const float* a, int sa, const float* b, int sb) {
    float c[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) c[j] = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float d = __fsub_rn(a[i * sa + j], b[i * sb + j]);
            c[j] = __fmaf_rn(d, d, c[j]);
        }
    return column_tree<8>(c);
}

template <int KK>
struct TcTop {
    uint64_t k[KK];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int q = 0; q < KK; ++q) k[q] = ~0ull;
    }
    __device__ __forceinline__ void add(uint64_t v) {
        if (!(v < k[KK - 1])) return;
#pragma unroll
        for (int q = 0; q < KK; ++q) {
            const uint64_t a = k[q];
            const bool sw = v < a;
            k[q] = sw ? v : a;
            v = sw ? a : v;
        }
    }
    __device__ __forceinline__ void pop() {
#pragma unroll
        for (int q = 0; q + 1 < KK; ++q) k[q] = k[q + 1];
        k[KK - 1] = ~0ull;
    }
};

// The 12 MMAs of candidate row c into D buffer `col` (3 split terms x 4 K-steps).
template <int R>
__device__ __forceinline__ void issue_row(uint32_t smem0, uint32_t tmem, int c, uint64_t* bar) {
    using T = Tc<R>;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const uint32_t arow = (uint32_t)(c + 2 * s) * kBlockBytes;
        const uint64_t ah = umma_desc(smem0 + T::A_HI + arow, kBlockBytes, 128);
        const uint64_t al = umma_desc(smem0 + T::A_LO + arow, kBlockBytes, 128);
        const uint64_t bh = umma_desc(smem0 + T::B_HI + s * 256, 128, 1024);
        const uint64_t bl = umma_desc(smem0 + T::B_LO + s * 256, 128, 1024);
        mma_bf16(tmem, ah, bh, kIdesc, s > 0);
        mma_bf16(tmem, ah, bl, kIdesc, true);
        mma_bf16(tmem, al, bh, kIdesc, true);
    }
    mma_commit(bar);
}

template <int R, int K>
__global__ void __launch_bounds__(kTcThreads, 1) match_tc_kernel(const __grid_constant__ MatchBatch mb,
                                                                 TcCounters* __restrict__ ctr) {
    using T = Tc<R>;
    constexpr int NC = T::NC, NW = T::NW;
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t tmem_base;
    __shared__ float nr_s[16];
    __shared__ int cx_s[16];
    __shared__ unsigned int ncmax_bits;
    __shared__ int nonfinite;
    float* dist = reinterpret_cast<float*>(sm + T::DIST);
    float* ncs = reinterpret_cast<float*>(sm + T::NCS);
    float* rs = reinterpret_cast<float*>(sm + T::RS);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t smem0 = smem_u32(sm);

    // ---- the tile ----
    int pl = 0;
    {
        int lo = 0, hi = mb.n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (mb.p[mid].cta0 <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
        }
        pl = lo;
    }
    const MatchPlane& P = mb.p[pl];
    const int W = P.W, H = P.H, step = mb.step, nx = P.nx;
    const int local = blockIdx.x - P.cta0;
    const int chunks = (nx + kTcRefs - 1) / kTcRefs;
    const int ry = local / chunks, rx0 = (local - ry * chunks) * kTcRefs;
    const int nref = min(kTcRefs, nx - rx0);
    const int cy = grid_pos(ry, H, 8, step);
    const int X0 = max(0, grid_pos(rx0, W, 8, step) - R);
    const int ylo = max(0, cy - R), yhi = min(H - 8, cy + R);
    const int ncr = yhi - ylo + 1;  // candidate rows
    const int nrows = ncr + 7;      // image rows
    const float* src = P.src;
    const int64_t ss = P.stride;

    // ---- setup: tensor memory (32 columns = two 16-column D buffers), barriers ----
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(&tmem_base))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int b = 0; b < 2; ++b)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[b])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        nonfinite = 0;
        ncmax_bits = 0;
    }
    if (tid < 16) {
        cx_s[tid] = tid < nref ? grid_pos(rx0 + tid, W, 8, step) : 0;
        nr_s[tid] = 0.f;
    }
    for (int i = tid; i < kTcRefs * NW; i += kTcThreads) dist[i] = __int_as_float(0x7f800000);

    // ---- A: shift blocks (hi, lo) of the image rows; row sums of squares ----
    bool bad = false;
    {
        const int m = tid & 127, g = m >> 3, j = m & 7;
        const int x = X0 + m;
        for (int rr = tid >> 7; rr < nrows; rr += 2) {
            const float* rowp = src + (int64_t)(ylo + rr) * ss;
            float v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = (x + q < W) ? __ldg(rowp + x + q) : 0.f;
            float sq = 0.f;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                sq = __fmaf_rn(v[q], v[q], sq);
                bad |= !isfinite(v[q]);
            }
            rs[rr * 128 + m] = sq;
            float* trow = reinterpret_cast<float*>(sm + T::TILE) + rr * T::TP;
            trow[m] = v[0];
            if (m >= 121) {  // the last 7 columns of the tile's row
#pragma unroll
                for (int q = 1; q < 8; ++q)
                    if (m + q >= 128) trow[m + q] = v[q];
            }
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) split2(v[2 * q], v[2 * q + 1], hi[q], lo[q]);
            const int off = rr * kBlockBytes + g * 128 + j * 16;
            *reinterpret_cast<uint4*>(sm + T::A_HI + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<uint4*>(sm + T::A_LO + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        }
    }
    // ---- B: the references (hi, lo), their norms ----
    if (tid < 128) {
        const int n = tid >> 3, i = tid & 7;
        float v[8];
        const bool live = n < nref;
        const float* rowp = src + (int64_t)(cy + i) * ss + (live ? grid_pos(rx0 + n, W, 8, step) : 0);
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = live ? __ldg(rowp + q) : 0.f;
        float sq = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) sq = __fmaf_rn(v[q], v[q], sq);
        sq += __shfl_xor_sync(0xffffffffu, sq, 1);
        sq += __shfl_xor_sync(0xffffffffu, sq, 2);
        sq += __shfl_xor_sync(0xffffffffu, sq, 4);
        if (i == 0) nr_s[n] = sq;
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) split2(v[2 * q], v[2 * q + 1], hi[q], lo[q]);
        const int off = (n >> 3) * 1024 + i * 128 + (n & 7) * 16;
        *reinterpret_cast<uint4*>(sm + T::B_HI + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(sm + T::B_LO + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
    if (bad) nonfinite = 1;
    // operands written by the generic proxy become visible to the tensor core's async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    if (tid == 0) issue_row<R>(smem0, tmem, 0, &bars[0]);
    // candidate norms |c|^2 per (candidate row, column) while the first MMAs run
    {
        float mx = 0.f;
        for (int e = tid; e < ncr * 128; e += kTcThreads) {
            const int c = e >> 7, m = e & 127;
            float s = 0.f;
#pragma unroll
            for (int i = 0; i < 8; ++i) s += rs[(c + i) * 128 + m];
            ncs[e] = s;
            if (X0 + m <= W - 8) mx = fmaxf(mx, s);
        }
        mx = warp_max_ratio(mx);
        if (lane == 0) atomicMax(&ncmax_bits, __float_as_uint(mx));
    }
    __syncthreads();

    // ---- main loop: MMAs of row c+1 overlap the read-back of row c ----
    bool timed_out = false;
    const int quarter = warp & 3, colhalf = warp >> 2;
    const int m = quarter * 32 + lane;  // this thread's candidate (TMEM lane)
    const int x = X0 + m;
    int c = 0;
    for (; c < ncr; ++c) {
        if (tid == 0 && c + 1 < ncr) issue_row<R>(smem0, tmem + 16 * ((c + 1) & 1), c + 1, &bars[(c + 1) & 1]);
        const bool ok = mbar_wait(&bars[c & 1], (c >> 1) & 1);
        if (__syncthreads_or(!ok)) {
            timed_out = true;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        float d[8];
        tmem_ld8(tmem + ((uint32_t)(quarter * 32) << 16) + 16 * (c & 1) + 8 * colhalf, d);
        const int y = ylo + c, dy = y - (cy - R);
        const float nc = ncs[c * 128 + m];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int n = colhalf * 8 + q;
            if (n < nref) {
                const int cxn = cx_s[n];
                if (x >= max(0, cxn - R) && x <= min(W - 8, cxn + R) && !(x == cxn && y == cy))
                    dist[n * NW + dy * NC + (x - (cxn - R))] = __fmaf_rn(-2.f, d[q], nc + nr_s[n]);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (timed_out) {
        // let the MMAs in flight finish (bounded) before the columns are released
        if (tid == 0) {
            (void)mbar_wait(&bars[c & 1], (c >> 1) & 1);
            if (c + 1 < ncr) (void)mbar_wait(&bars[(c + 1) & 1], ((c + 1) >> 1) & 1);
            atomicAdd(&ctr->timeouts, 1u);
        }
        __syncthreads();
    }
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
    }
    if (timed_out) return;

    // ---- selection and exact re-rank, one warp per reference ----
    const float ncmax = __uint_as_float(ncmax_bits);
    const bool flagged = nonfinite != 0;
    if (flagged && tid == 0) atomicAdd(&ctr->flagged_tiles, 1u);
    uint16_t* surv = reinterpret_cast<uint16_t*>(sm + T::SURV) + warp * NW;
    const float kInf = __int_as_float(0x7f800000);
    for (int n = warp; n < nref; n += kTcThreads / 32) {
        const float* dn = dist + n * NW;
        const int cxn = cx_s[n];
        const int xl = max(0, cxn - R), xh = min(W - 8, cxn + R);
        // U: the K-th smallest of the 64 values made of each lane's two smallest
        float a = kInf, b = kInf;
        for (int q = lane; q < NW; q += 32) {
            const float v = dn[q];
            if (v < a) {
                b = a;
                a = v;
            } else if (v < b) {
                b = v;
            }
        }
        float U = kInf;
        int need = K;
        for (int round = 0; round < 2 * K && need > 0; ++round) {
            const float mv = warp_min_f(a);
            if (!(mv < kInf)) break;
            const unsigned hit = __ballot_sync(0xffffffffu, a == mv);
            need -= __popc(hit);
            if (a == mv) {
                a = b;
                b = kInf;
            }
            if (need <= 0) U = mv;
        }
        const float nr = nr_s[n];
        const float E = 2.9e-4f * sqrtf(nr * ncmax) + 1e-5f * (nr + ncmax) + (U < kInf ? 2e-6f * fabsf(U) : 0.f);
        const float theta = U + 2.f * E;
        // survivors, compacted in window order
        int S = 0;
        for (int q0 = 0; q0 < NW; q0 += 32) {
            const int q = q0 + lane;
            bool keep = false;
            if (q < NW) {
                const int dy = q / NC, dx = q - dy * NC;
                const int xx = cxn - R + dx, yy = cy - R + dy;
                const bool valid = xx >= xl && xx <= xh && yy >= ylo && yy <= yhi && !(dx == R && dy == R);
                keep = valid && (flagged || dn[q] <= theta);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (keep) surv[S + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)q;
            S += __popc(bal);
        }
        __syncwarp();
        // exact distances of the survivors, exact keys
        const float* tile = reinterpret_cast<const float*>(sm + T::TILE);
        const float* refp = tile + (cy - ylo) * T::TP + (cxn - X0);
        TcTop<K> top;
        top.init();
        float worst_ratio = 0.f;
        for (int i = lane; i < S; i += 32) {
            const int q = surv[i];
            const int dy = q / NC, dx = q - dy * NC;
            const int xx = cxn - R + dx, yy = cy - R + dy;
            const float de = ssd8_exact(refp, T::TP, tile + (yy - ylo) * T::TP + (xx - X0), T::TP);
            top.add(tc_key(de, xx, yy));
            if (!flagged) worst_ratio = fmaxf(worst_ratio, fabsf(dn[q] - de) / E);
        }
        uint64_t best[K];
        int nb = 0;
#pragma unroll
        for (int r = 0; r < K; ++r) {
            const uint64_t mk = warp_min_u64(top.k[0]);
            best[r] = mk;
            if (mk != ~0ull) {
                ++nb;
                if (top.k[0] == mk) top.pop();
            }
        }
        const float wr = warp_max_ratio(worst_ratio);
        if (lane == 0) {
            const int64_t job = (int64_t)ry * nx + rx0 + n;
            constexpr int G = K + 1;
            int32_t* op = P.pos + job * G;
            op[0] = pack_pos(cxn, cy);
#pragma unroll
            for (int r = 0; r < K; ++r) op[1 + r] = best[r] != ~0ull ? int32_t(uint32_t(best[r])) : -1;
            if (P.dist) {
                float* od = P.dist + job * G;
                od[0] = 0.f;
#pragma unroll
                for (int r = 0; r < K; ++r) od[1 + r] = best[r] != ~0ull ? __uint_as_float(uint32_t(best[r] >> 32)) : 0.f;
            }
            P.count[job] = 1 + nb;
            atomicAdd(&ctr->survivors, (unsigned long long)S);
            atomicAdd(&ctr->refs, 1ull);
            atomicMax(&ctr->max_ratio_bits, __float_as_uint(wr));
        }
        __syncwarp();
    }
}

template <int R, int K>
void launch_tc(MatchBatch& mb, TcCounters* ctr, cudaStream_t stream) {
    int ctas = 0;
    for (int i = 0; i < mb.n; ++i) {
        MatchPlane& p = mb.p[i];
        p.nx = grid_count(p.W, 8, mb.step);
        p.ny = grid_count(p.H, 8, mb.step);
        p.cta0 = ctas;
        ctas += ceil_div(p.nx, kTcRefs) * p.ny;
    }
    mb.total_ctas = ctas;
    mb.queue = nullptr;
    if (ctas == 0) return;
    static_assert(8 * (kTcRefs - 1) + 2 * R + 1 <= 128, "a tile's candidates must fit one M = 128 MMA");
    auto kern = match_tc_kernel<R, K>;
    NSSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Tc<R>::BYTES));
    kern<<<ctas, kTcThreads, Tc<R>::BYTES, stream>>>(mb, ctr);
    NSSB_CUDA(cudaGetLastError());
}

}  // namespace

bool launch_match_tc_batch(MatchBatch& mb, int bm_range, int group, TcCounters* counters, cudaStream_t stream) {
    if (!counters || mb.step < 1 || mb.step > 8 || mb.n < 1 || mb.n > kMaxBatchPlanes) return false;
    if (bm_range != 9) return launch_match_tcw_batch(mb, bm_range, group, counters, stream);
    for (int i = 0; i < mb.n; ++i)
        if (mb.p[i].W < 8 || mb.p[i].H < 8 || mb.p[i].W > 65535 || mb.p[i].H > 65535) return false;
    switch (group) {
        case 2: launch_tc<9, 1>(mb, counters, stream); return true;
        case 4: launch_tc<9, 3>(mb, counters, stream); return true;
        case 8: launch_tc<9, 7>(mb, counters, stream); return true;
        case 16: launch_tc<9, 15>(mb, counters, stream); return true;
        default: return false;
    }
}

}  // namespace nssb
