// Precision form of the 8x8 matcher for large windows (bm_range 10-64):
// distances scored on the sm_100a tensor cores with the references on the
// MMA's M side, groups re-ranked exactly (lists equal match8.cu's and the
// oracle's, bit for bit).
//
// d(r, c) = |r - c|^2 = |r'|^2 + |c'|^2 - 2 r'.c' with r' = r - mu, c' = c - mu
// for one shift mu per tile (the midrange of its pixels: the margin below
// then scales with the local contrast, not the brightness). The dot products
// come from tcgen05.mma (kind::f16, BF16 in, FP32 accumulated in tensor
// memory) with every shifted pixel split hi = bf16(v), lo = bf16(v - hi):
// r'.c' ~ rh.ch + rh.cl + rl.ch. The margin is match_tc.cu's, with the norm
// bound max|c'|^2 <= 64 max|v - mu|^2 and a term for the shift's roundings:
// |d~ - d| <= E = 2.9e-4 sqrt(|r'|^2 max|c'|^2) + 1.1e-5 (|r'|^2 + max|c'|^2).
//
// Tile: 128 references (NX x NY of a plane's grid, NX * NY = 128), one CTA of
// 256 threads. The MMA is D[128 references][N candidates] per candidate row
// y: N consecutive candidate columns X0 .. X0+N-1 cover every window of the
// tile along x, the candidate rows ylo..yhi every window along y.
//   A (M = 128 references x K = 64 pixels) is K-major: 8 references x 8
//     pixels per 128-byte core matrix, pixel rows 128 B apart (LBO), groups of
//     8 references 1 KB apart (SBO); written once per tile.
//   B (K = 64 x N candidates) is MN-major and never materialised per
//     candidate: image row Y is stored once as a block S_Y[g][j][m'] =
//     v(Y, X0 + 8g + j + m') (N/8 groups x 8 shifts x 8, BF16), so the
//     K-slice (pixel rows i, i+1) of candidate row y is the pair of blocks
//     S_{y+i}, S_{y+i+1}: descriptor start at S_{y+i}, LBO = the block
//     stride, SBO = 128 B. The blocks live in a ring of 10 image rows (plus a
//     copy of slot 0 after the last slot, so a pair never wraps).
//   D: lane t of tensor memory is reference t, column n candidate n; two
//     buffers of N columns, so the MMAs of candidate row c+1 run while row c
//     is read back. Warp w reads lanes 32 (w & 3) .. +31 and the column half
//     w >> 2: each thread owns one reference's half of the candidates.
// Two passes over the candidate rows (the MMAs run twice):
//   1. each thread takes the smallest d~ of every 16-column chunk of every row
//      in its window; U = the K-th smallest of those over both halves. They
//      are K distinct candidates, so d_K <= U + E and every exact top-K
//      candidate c has d~(c) <= d(c) + E <= U + 2E;
//   2. a candidate with d~ <= U + 2E (every candidate of a tile with a
//      non-finite pixel) is buffered by its thread; when a lane's buffer fills
//      (and at the end) the warp re-ranks all its lanes' buffers together --
//      lane i takes the warp's i-th survivor, whatever its reference: the
//      exact FP32 distance in this build's order (per-column FMA chains, then
//      the column tree) -- and each lane enters its survivors' exact keys into
//      its list. A full list's K-th distance also bounds d_K, so the threshold
//      drops to (the smaller of both halves' K-th distances) + E.
// The halves' lists then merge: the exact keys pick the FP32 matcher's group.
#include "kernels.cuh"
#include "tcgen05.cuh"

#include <algorithm>

namespace nssb {
namespace {

using namespace tc;

constexpr int kWThreads = 256;
constexpr int kWRefs = 128;  // references per tile = the MMA's M
constexpr int kRing = 10;    // image-row slots of the candidate operand (+ one copy of slot 0)
constexpr int kCap = 16;     // survivors a thread buffers before their exact re-rank

struct TcwGeom {
    int nx_refs, ny_refs;  // tile arrangement, nx_refs * ny_refs = 128
    int N;                 // candidate columns per MMA row (a multiple of 32, <= 256)
    int R;                 // search range
};

// dynamic shared memory layout (bytes)
struct TcwLayout {
    int blk;               // one image row's operand block: N x 8 BF16
    int a_hi, a_lo, b_hi, b_lo, rs, ncb, spos, se, wl, bytes;
};

__host__ __device__ inline TcwLayout tcw_layout(int N, int K) {
    TcwLayout L;
    L.blk = N * 16;
    L.a_hi = 0;
    L.a_lo = kWRefs * 128;
    L.b_hi = 2 * kWRefs * 128;
    L.b_lo = L.b_hi + (kRing + 1) * L.blk;
    const int ring_end = L.b_lo + (kRing + 1) * L.blk;
    const int scratch_end = L.b_hi + kWRefs * K * 8;  // list merges reuse the ring
    L.rs = ring_end > scratch_end ? ring_end : scratch_end;
    L.ncb = L.rs + kRing * N * 8;
    L.spos = L.ncb + 4 * N * 4;                 // uint16 [kCap][256] buffered survivors (row << 8 | column)
    L.se = L.spos + kCap * kWThreads * 2;        // float [kCap][256] their d~ - |r'|^2, then d
    L.wl = L.se + kCap * kWThreads * 4;          // uint16 [8 warps][32 * kCap] a warp's survivors in order
    L.bytes = L.wl + kWThreads * kCap * 2;
    return L;
}

__device__ __forceinline__ uint64_t key_of(float d, int x, int y) {
    uint32_t b = __float_as_uint(d);
    if ((b & 0x7f800000u) == 0x7f800000u) b = 0x7f800000u;
    return (uint64_t(b) << 32) | (uint64_t(uint32_t(y)) << 16) | uint64_t(uint32_t(x));
}

// Exact SSD of two 8x8 blocks of the plane in this build's order.
__device__ __forceinline__ float ssd8_plane(const float* a, const float* b, int64_t s) {
    float c[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) c[j] = 0.f;
#pragma unroll 2
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float d = __fsub_rn(__ldg(a + i * s + j), __ldg(b + i * s + j));
            c[j] = __fmaf_rn(d, d, c[j]);
        }
    return column_tree<8>(c);
}

// Sorted insert of v into k[0..S) when it beats the last entry (all
// comparisons first, then every slot takes its own entry, the one before it,
// or v).
template <int S, typename T>
__device__ __forceinline__ void sorted_insert(T* k, T v) {
    if (!(v < k[S - 1])) return;
    bool c[S];
#pragma unroll
    for (int q = 0; q < S; ++q) c[q] = v < k[q];
#pragma unroll
    for (int q = S - 1; q > 0; --q) k[q] = c[q] ? (c[q - 1] ? k[q - 1] : v) : k[q];
    k[0] = c[0] ? v : k[0];
}

// The columns [lo, hi] of a 16-column chunk starting at col0, as bits.
__device__ __forceinline__ uint32_t chunk_bits(int lo, int hi, int col0) {
    const int a = max(lo - col0, 0), b = min(hi - col0, 15);
    return a > b ? 0u : ((2u << b) - 1u) & ~((1u << a) - 1u);
}

template <int K>
__global__ void __launch_bounds__(kWThreads, (K <= 15 ? 2 : 1))
    match_tcw_kernel(const __grid_constant__ MatchBatch mb, const TcwGeom geo, TcCounters* __restrict__ ctr) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bars[2];
    __shared__ uint32_t tmem_base;
    __shared__ float nr_s[kWRefs];
    __shared__ float dk_s[2][kWRefs];  // each half's K-th exact distance so far
    __shared__ float wmin_s[kWThreads / 32], wmax_s[kWThreads / 32];
    __shared__ int nonfinite;
    const int N = geo.N, R = geo.R, NXr = geo.nx_refs, NYr = geo.ny_refs;
    const TcwLayout L = tcw_layout(N, K);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int quarter = warp & 3, half = warp >> 2;
    const uint32_t smem0 = smem_u32(sm);
    float* rs = reinterpret_cast<float*>(sm + L.rs);
    float* ncb = reinterpret_cast<float*>(sm + L.ncb);
    const float kInf = __int_as_float(0x7f800000);

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
    const int W = P.W, H = P.H, step = mb.step, nx = P.nx, ny = P.ny;
    const int local = blockIdx.x - P.cta0;
    const int tiles_x = (nx + NXr - 1) / NXr;
    const int ty = local / tiles_x, rx0 = (local - ty * tiles_x) * NXr, ry0 = ty * NYr;
    const int x_first = grid_pos(rx0, W, 8, step);
    const int y_first = grid_pos(ry0, H, 8, step), y_last = grid_pos(min(ry0 + NYr, ny) - 1, H, 8, step);
    const int X0 = max(0, x_first - R);
    const int ylo = max(0, y_first - R), yhi = min(H - 8, y_last + R);
    const int ncr = yhi - ylo + 1;  // candidate rows
    const int nrows = ncr + 7;      // image rows
    const int xend = min(W, X0 + N + 7);  // image columns [X0, xend) of the tile
    const float* src = P.src;
    const int64_t ss = P.stride;

    // this thread's reference (tensor-memory lane t) and column half
    const int t = quarter * 32 + lane;
    const int rx = rx0 + t % NXr, ry = ry0 + t / NXr;
    const bool active = rx < nx && ry < ny;
    const int cx = grid_pos(min(rx, nx - 1), W, 8, step), cy = grid_pos(min(ry, ny - 1), H, 8, step);
    const int xl = max(0, cx - R) - X0, xh = min(W - 8, cx + R) - X0;  // the window's tile columns
    const int yl = max(0, cy - R), yh = min(H - 8, cy + R);
    const int self_col = cx - X0;
    const int half_cols = N / 2, chunks = N / 32;

    // ---- setup: tensor memory (two N-column D buffers), barriers ----
    const uint32_t tcols = N <= 128 ? 256u : 512u;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(tcols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int b = 0; b < 2; ++b)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[b])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        nonfinite = 0;
    }
    if (tid < kWRefs) dk_s[0][tid] = dk_s[1][tid] = kInf;

    // ---- the tile's pixel range: the shift mu (midrange) and a bound on
    // every shifted candidate norm; non-finite pixels flag the tile ----
    // (distances are shift-invariant: the MMAs see v - mu, so the error
    // margin scales with the local contrast, not the brightness)
    {
        float lo = kInf, hi = -kInf;
        bool bad = false;
#pragma unroll 1
        for (int r = warp; r < nrows; r += kWThreads / 32) {
            const float* rowp = src + (int64_t)(ylo + r) * ss;
            for (int x = X0 + lane; x < xend; x += 32) {
                const float v = __ldg(rowp + x);
                bad |= !isfinite(v);
                lo = fminf(lo, v);
                hi = fmaxf(hi, v);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            wmin_s[warp] = lo;
            wmax_s[warp] = hi;
        }
        if (bad) nonfinite = 1;
    }
    __syncthreads();
    const bool flagged = nonfinite != 0;
    float mu, amax;
    {
        float lo = wmin_s[0], hi = wmax_s[0];
        for (int w = 1; w < kWThreads / 32; ++w) {
            lo = fminf(lo, wmin_s[w]);
            hi = fmaxf(hi, wmax_s[w]);
        }
        mu = flagged ? 0.f : 0.5f * lo + 0.5f * hi;
        // every shifted pixel |v - mu| <= amax (its rounding included)
        amax = flagged ? 0.f : fmaxf(fabsf(__fsub_rn(hi, mu)), fabsf(__fsub_rn(lo, mu))) * (1.f + 1e-6f);
    }
    const float ncmax = 64.f * amax * amax * (1.f + 1e-6f);  // >= every shifted candidate norm

    // ---- A: the 128 references (hi, lo) and their norms ----
#pragma unroll 1
    for (int e = tid; e < kWRefs * 8; e += kWThreads) {
        const int n = e >> 3, i = e & 7;
        const int rxn = rx0 + n % NXr, ryn = ry0 + n / NXr;
        const bool live = rxn < nx && ryn < ny;
        float v[8];
        if (live) {
            const float* rp = src + (int64_t)(grid_pos(ryn, H, 8, step) + i) * ss + grid_pos(rxn, W, 8, step);
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = __fsub_rn(__ldg(rp + q), mu);
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = 0.f;
        }
        float sq = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) sq = __fmaf_rn(v[q], v[q], sq);
        // the 8 rows of reference n sit in 8 consecutive lanes
        sq += __shfl_xor_sync(0xffffffffu, sq, 1);
        sq += __shfl_xor_sync(0xffffffffu, sq, 2);
        sq += __shfl_xor_sync(0xffffffffu, sq, 4);
        if (i == 0) nr_s[n] = sq;
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) split2(v[2 * q], v[2 * q + 1], hi[q], lo[q]);
        const int off = (n >> 3) * 1024 + i * 128 + (n & 7) * 16;
        *reinterpret_cast<uint4*>(sm + L.a_hi + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(sm + L.a_lo + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }

    // image row r of the tile (Y = ylo + r) into ring slot r % kRing: candidate
    // column n's 8 shifted pixels as column n of the block, hi and lo, and
    // their sum of squares (the row's share of candidate n's norm); two
    // threads per column, four pixels each
    auto convert = [&](int r) {
        if (r >= nrows) return;
        const int slot = r % kRing;
        const float* rowp = src + (int64_t)(ylo + r) * ss;
        for (int e = tid; e < 2 * N; e += kWThreads) {
            const int n = e >> 1, h = e & 1;
            float v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int x = X0 + n + 4 * h + q;
                v[q] = x < W ? __fsub_rn(__ldg(rowp + x), mu) : 0.f;
            }
            float sq = 0.f;
#pragma unroll
            for (int q = 0; q < 4; ++q) sq = __fmaf_rn(v[q], v[q], sq);
            rs[(slot * N + n) * 2 + h] = sq;
            uint32_t hi[2], lo[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) split2(v[2 * q], v[2 * q + 1], hi[q], lo[q]);
            const int off = (n >> 3) * 128 + (n & 7) * 16 + 8 * h;
            const uint2 h2 = make_uint2(hi[0], hi[1]), l2 = make_uint2(lo[0], lo[1]);
            *reinterpret_cast<uint2*>(sm + L.b_hi + slot * L.blk + off) = h2;
            *reinterpret_cast<uint2*>(sm + L.b_lo + slot * L.blk + off) = l2;
            if (slot == 0) {
                *reinterpret_cast<uint2*>(sm + L.b_hi + kRing * L.blk + off) = h2;
                *reinterpret_cast<uint2*>(sm + L.b_lo + kRing * L.blk + off) = l2;
            }
        }
    };
    // candidate row c's norms |c - mu|^2 per column (rows c .. c+7 converted)
    auto norms = [&](int c) {
        if (c >= ncr) return;
        for (int n = tid; n < N; n += kWThreads) {
            float s = 0.f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float2 p = *reinterpret_cast<const float2*>(rs + (((c + i) % kRing) * N + n) * 2);
                s += p.x + p.y;
            }
            ncb[(c & 3) * N + n] = s;
        }
    };

    const uint32_t idesc = idesc_bf16(128, N, false, true);
    // the 12 MMAs of candidate row c (3 split terms x 4 K-steps) into D buffer u & 1
    auto issue = [&](int c, int u) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem_base + (uint32_t)((u & 1) * N);
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const uint32_t brow = (uint32_t)((c + 2 * s) % kRing) * L.blk;
            const uint64_t bh = umma_desc(smem0 + L.b_hi + brow, L.blk, 128);
            const uint64_t bl = umma_desc(smem0 + L.b_lo + brow, L.blk, 128);
            const uint64_t ah = umma_desc(smem0 + L.a_hi + s * 256, 128, 1024);
            const uint64_t al = umma_desc(smem0 + L.a_lo + s * 256, 128, 1024);
            mma_bf16(d, ah, bh, idesc, s > 0);
            mma_bf16(d, ah, bl, idesc, true);
            mma_bf16(d, al, bh, idesc, true);
        }
        mma_commit(&bars[u & 1]);
    };

    // One pass over the candidate rows: the MMAs of row c+1 run while row c is
    // read back; chunk(y, col0, m, e) sees each 16-column chunk of this
    // thread's half (all lanes of a warp together) with m = the chunk's window
    // columns (self excluded) and e[j] = d~ - |r'|^2. c0: rows issued before
    // this pass (D buffer and barrier phase). False when a device wait gave up.
    int c0 = 0, cfail = -1;
    auto sweep = [&](auto&& chunk) -> bool {
        for (int r = 0; r <= 8; ++r) convert(r);
        __syncthreads();
        norms(0);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) issue(0, c0);
#pragma unroll 1
        for (int c = 0; c < ncr; ++c) {
            convert(c + 9);
            norms(c + 1);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (tid == 0 && c + 1 < ncr) issue(c + 1, c0 + c + 1);
            const int u = c0 + c;
            const bool done = mbar_wait(&bars[u & 1], (u >> 1) & 1);
            if (__syncthreads_or(!done)) {
                cfail = c;
                return false;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int y = ylo + c;
            const bool row_ok = active && y >= yl && y <= yh;
            const float* ncrow = ncb + (c & 3) * N;
            const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)((u & 1) * N);
#pragma unroll 1
            for (int k = 0; k < chunks; ++k) {
                const int col0 = half * half_cols + 16 * k;
                float D[16];
                __syncwarp();
                tmem_ld16(taddr + (uint32_t)col0, D);
                uint32_t m = row_ok ? chunk_bits(xl, xh, col0) : 0u;
                if (y == cy && self_col >= col0 && self_col < col0 + 16) m &= ~(1u << (self_col - col0));
                float e[16];
                if (m) {
                    const float2 m2 = make_float2(-2.f, -2.f);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float4 f = *reinterpret_cast<const float4*>(ncrow + col0 + 4 * q);
                        const float2 a = __ffma2_rn(make_float2(D[4 * q], D[4 * q + 1]), m2, make_float2(f.x, f.y));
                        const float2 b = __ffma2_rn(make_float2(D[4 * q + 2], D[4 * q + 3]), m2, make_float2(f.z, f.w));
                        e[4 * q] = a.x;
                        e[4 * q + 1] = a.y;
                        e[4 * q + 2] = b.x;
                        e[4 * q + 3] = b.y;
                    }
                }
                chunk(y, col0, m, e);
            }
        }
        c0 += ncr;
        // every MMA of the pass has completed: the ring is free
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        return true;
    };

    __syncthreads();  // the references' norms
    const float nrv = nr_s[t];
    // the margin: |d~ - d| <= E for every candidate of this reference
    const float E = 2.9e-4f * sqrtf(nrv * ncmax) + 1.1e-5f * (nrv + ncmax);
    float th_e = kInf;  // pass 2's threshold on d~ - |r'|^2
    bool ok;
    {
        // ---- pass 1: U = the K-th smallest 16-column chunk minimum of the
        // window over both halves (K distinct candidates: U >= the K-th
        // smallest d~, so every top-K candidate has d~ <= U + 2E) ----
        float top[K];
#pragma unroll
        for (int q = 0; q < K; ++q) top[q] = kInf;
        ok = sweep([&](int, int, uint32_t m, const float* e) {
            if (m == 0u) return;
            float mn = kInf;
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if ((m >> j) & 1u) mn = fminf(mn, e[j]);
            sorted_insert<K>(top, mn);
        });
        if (ok) {
            float* lists = reinterpret_cast<float*>(sm + L.b_hi);  // [2][128][K], over the free ring
#pragma unroll
            for (int q = 0; q < K; ++q) lists[(half * kWRefs + t) * K + q] = top[q];
            __syncthreads();
            const float* other = lists + ((1 - half) * kWRefs + t) * K;
            for (int q = 0; q < K; ++q) {
                const float v = other[q];
                if (!(v < top[K - 1])) break;
                sorted_insert<K>(top, v);
            }
            const float U = top[K - 1] + nrv;
            if (U < kInf) th_e = U + 2.f * E + 2e-6f * fabsf(U) - nrv;
            __syncthreads();  // the lists are read before pass 2 reuses the ring
        }
    }

    // ---- pass 2: survivors (d~ <= threshold) into per-thread buffers; when a
    // lane's buffer fills (and at the end) the warp re-ranks all its lanes'
    // buffers together: lane i takes the i-th survivor of the warp, whatever
    // its reference, for the exact distance; then each lane enters its own
    // survivors' exact keys into its list ----
    uint64_t ex[K];  // the K smallest exact keys of this half
#pragma unroll
    for (int q = 0; q < K; ++q) ex[q] = ~0ull;
    unsigned long long survivors = 0;
    float worst_ratio = 0.f;
    uint16_t* spos = reinterpret_cast<uint16_t*>(sm + L.spos);
    float* se = reinterpret_cast<float*>(sm + L.se);
    uint16_t* wlist = reinterpret_cast<uint16_t*>(sm + L.wl) + warp * 32 * kCap;
    int nbuf = 0;
    auto flush = [&]() {
        int incl = nbuf;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for (int q = 0; q < nbuf; ++q) wlist[incl - nbuf + q] = uint16_t((lane << 8) | q);
        __syncwarp();
        for (int g = lane; g < total; g += 32) {
            const int ent = wlist[g], ol = ent >> 8, q = ent & 255;
            const int otid = warp * 32 + ol, ot = quarter * 32 + ol;
            const int orx = min(rx0 + ot % NXr, nx - 1), ory = min(ry0 + ot / NXr, ny - 1);
            const int ocx = grid_pos(orx, W, 8, step), ocy = grid_pos(ory, H, 8, step);
            const int pk = spos[q * kWThreads + otid];
            const int x = X0 + (pk & 255), y = ylo + (pk >> 8);
            const float d = ssd8_plane(src + (int64_t)ocy * ss + ocx, src + (int64_t)y * ss + x, ss);
            if (!flagged) {
                const float onr = nr_s[ot];
                const float oE = 2.9e-4f * sqrtf(onr * ncmax) + 1.1e-5f * (onr + ncmax);
                if (oE > 0.f) worst_ratio = fmaxf(worst_ratio, fabsf(se[q * kWThreads + otid] + onr - d) / oE);
            }
            se[q * kWThreads + otid] = d;
        }
        __syncwarp();
        for (int q = 0; q < nbuf; ++q) {
            const int pk = spos[q * kWThreads + tid];
            sorted_insert<K>(ex, key_of(se[q * kWThreads + tid], X0 + (pk & 255), ylo + (pk >> 8)));
        }
        survivors += nbuf;
        nbuf = 0;
        // a full list bounds d_K by its K-th distance (the smaller of both
        // halves' is also a bound): every top-K candidate has d~ <= d_K + E
        if (!flagged) {
            float dk = ex[K - 1] == ~0ull ? kInf : __uint_as_float(uint32_t(ex[K - 1] >> 32));
            volatile float* dks = dk_s[0];
            if (dk < kInf) dks[half * kWRefs + t] = dk;
            dk = fminf(dk, dks[(1 - half) * kWRefs + t]);
            if (dk < kInf) th_e = fminf(th_e, dk + E + 2e-6f * dk - nrv);
        }
        __syncwarp();
    };
    if (ok) {
        ok = sweep([&](int y, int col0, uint32_t m, const float* e) {
            uint32_t pm = 0;
            if (m) {
                // most chunks hold no survivor: their smallest d~ decides
                float mn = kInf;
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if ((m >> j) & 1u) mn = fminf(mn, e[j]);
                if (flagged || mn <= th_e) {
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (((m >> j) & 1u) && (flagged || e[j] <= th_e)) pm |= 1u << j;
                }
            }
            if (__any_sync(0xffffffffu, nbuf + __popc(pm) > kCap)) flush();
            if (pm) {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if ((pm >> j) & 1u) {
                        spos[nbuf * kWThreads + tid] = uint16_t(((y - ylo) << 8) | (col0 + j));
                        se[nbuf * kWThreads + tid] = e[j];
                        ++nbuf;
                    }
            }
        });
        if (ok) flush();
    }
    if (!ok) {
        // let the MMAs in flight finish (bounded) before the columns are released
        if (tid == 0) {
            const int u = c0 + cfail;
            (void)mbar_wait(&bars[u & 1], (u >> 1) & 1);
            if (cfail + 1 < ncr) (void)mbar_wait(&bars[(u + 1) & 1], ((u + 1) >> 1) & 1);
            atomicAdd(&ctr->timeouts, 1u);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(tcols)
                     : "memory");
    }
    if (!ok) return;

    // ---- merge the halves' exact lists; half 0 writes the group ----
    uint64_t* keys = reinterpret_cast<uint64_t*>(sm + L.b_hi);  // [128][K], over the ring (every MMA is done)
    if (half == 1) {
#pragma unroll
        for (int q = 0; q < K; ++q) keys[t * K + q] = ex[q];
    }
    __syncthreads();
    // statistics: survivors of both halves, references, the largest error / margin
    {
        unsigned long long sv = survivors;
        float wr = worst_ratio;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sv += __shfl_xor_sync(0xffffffffu, sv, o);
            wr = fmaxf(wr, __shfl_xor_sync(0xffffffffu, wr, o));
        }
        const unsigned refs = __popc(__ballot_sync(0xffffffffu, active && half == 0));
        if (lane == 0) {
            if (sv) atomicAdd(&ctr->survivors, sv);
            if (refs) atomicAdd(&ctr->refs, (unsigned long long)refs);
            atomicMax(&ctr->max_ratio_bits, __float_as_uint(wr));
            if (warp == 0 && flagged) atomicAdd(&ctr->flagged_tiles, 1u);
        }
    }
    if (half == 1 || !active) return;
    for (int q = 0; q < K; ++q) {
        const uint64_t v = keys[t * K + q];
        if (!(v < ex[K - 1])) break;
        sorted_insert<K>(ex, v);
    }
    const int64_t job = (int64_t)ry * nx + rx;
    constexpr int G = K + 1;
    int32_t* op = P.pos + job * G;
    op[0] = pack_pos(cx, cy);
    int nb = 0;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        op[1 + q] = ex[q] != ~0ull ? int32_t(uint32_t(ex[q])) : -1;
        nb += ex[q] != ~0ull;
    }
    if (P.dist) {
        float* od = P.dist + job * G;
        od[0] = 0.f;
#pragma unroll
        for (int q = 0; q < K; ++q) od[1 + q] = ex[q] != ~0ull ? __uint_as_float(uint32_t(ex[q] >> 32)) : 0.f;
    }
    P.count[job] = 1 + nb;
}

template <int K>
void launch_tcw(MatchBatch& mb, const TcwGeom& geo, TcCounters* ctr, cudaStream_t stream) {
    int ctas = 0;
    for (int i = 0; i < mb.n; ++i) {
        MatchPlane& p = mb.p[i];
        p.nx = grid_count(p.W, 8, mb.step);
        p.ny = grid_count(p.H, 8, mb.step);
        p.cta0 = ctas;
        ctas += ceil_div(p.nx, geo.nx_refs) * ceil_div(p.ny, geo.ny_refs);
    }
    mb.total_ctas = ctas;
    mb.queue = nullptr;
    if (ctas == 0) return;
    const TcwLayout L = tcw_layout(geo.N, K);
    // tiles with more than 128 candidate columns take all 512 tensor-memory
    // columns: one CTA per SM (the shared memory asked for sees to it)
    const int bytes = geo.N > 128 ? std::max(L.bytes, 120 * 1024) : L.bytes;
    auto kern = match_tcw_kernel<K>;
    NSSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    kern<<<ctas, kWThreads, bytes, stream>>>(mb, geo, ctr);
    NSSB_CUDA(cudaGetLastError());
}

}  // namespace

bool launch_match_tcw_batch(MatchBatch& mb, int bm_range, int group, TcCounters* counters, cudaStream_t stream) {
    if (!counters || mb.step < 1 || mb.step > 8 || mb.n < 1 || mb.n > kMaxBatchPlanes) return false;
    if (bm_range < 10 || bm_range > 64) return false;
    for (int i = 0; i < mb.n; ++i)
        if (mb.p[i].W < 8 || mb.p[i].H < 8 || mb.p[i].W > 65535 || mb.p[i].H > 65535) return false;
    // the arrangement of the 128 references with the least MMA work (candidate
    // columns x candidate rows)
    TcwGeom geo{0, 0, 0, bm_range};
    long best = -1;
    for (int nxr = 32; nxr >= 4; nxr >>= 1) {
        const int nyr = kWRefs / nxr;
        const int n = ((nxr - 1) * mb.step + 2 * bm_range + 1 + 31) / 32 * 32;
        if (n > 256 || (nyr - 1) * mb.step + 2 * bm_range + 1 > 256) continue;  // columns, rows < 256
        const long cost = (long)n * ((nyr - 1) * mb.step + 2 * bm_range + 1);
        if (best < 0 || cost < best) {
            best = cost;
            geo.nx_refs = nxr;
            geo.ny_refs = nyr;
            geo.N = n;
        }
    }
    if (best < 0) return false;
    switch (group) {
        case 2: launch_tcw<1>(mb, geo, counters, stream); return true;
        case 4: launch_tcw<3>(mb, geo, counters, stream); return true;
        case 8: launch_tcw<7>(mb, geo, counters, stream); return true;
        case 16: launch_tcw<15>(mb, geo, counters, stream); return true;
        case 32: launch_tcw<31>(mb, geo, counters, stream); return true;
        default: return false;
    }
}

}  // namespace nssb
