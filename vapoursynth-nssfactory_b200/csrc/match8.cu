// Exact FP32 block matching for 8x8 blocks (sm_100a): the default BM3D shape
// (bm_range 9), and every range from 4 to 64 (kernels built for 4-9, 12,
// 15, 16, 19, 25 and 31; a range between two runs on the larger one, a range
// beyond 31 on the 31 kernel in bands of 63 x 63 candidates), groups of 2,
// 4, 8, 16 and 32.
//
// Same contract as match.cu (the reference's matcher.hpp:27-283 ordering,
// keys dist << 32 | y << 16 | x, and this build's SSD order: one FMA chain per
// block column down the rows, then ((c0+c1)+(c2+c3))+((c4+c5)+(c6+c7)));
// only the schedule differs:
//   - a CTA is 32 consecutive references of one grid row of one plane of a
//     batch. Two lanes serve each reference, one per column half, each with
//     its 8x4 half block in 32 registers; a warp is 16 references x 2 halves
//     and the CTA's P warp pairs split the 2R+1 window columns;
//   - the CTA stages the 2R+8 rows of its windows once in shared memory by
//     asynchronous copies (all issued, then one wait), the column c of a row
//     stored at c ^ ((c >> 5) & 3): the 32 lanes read 32 columns 4 apart,
//     which this swizzle sends to 32 different banks;
//   - a lane walks its window columns one by one: the column's 2R+8 image rows
//     stream through and every row is applied to the 8 candidates that
//     overlap it. Candidate k lives in accumulator k & 7; with the row loop
//     unrolled the slots are register names. The packed FP32 FMA of sm_100
//     (__ffma2_rn) carries two block columns per instruction, so a row costs 4
//     shared loads and 32 packed operations per lane. A finished candidate's
//     two half sums meet through one shuffle; the sum enters the reference's
//     register top-k, kept identically by both lanes (split over the two
//     lanes for groups of 32); the P partial lists merge in shared memory.
#include "kernels.cuh"

#include <algorithm>
#include <type_traits>

namespace nssb {
namespace {

__device__ __forceinline__ int swz(int col) { return col ^ ((col >> 5) & 3); }

__device__ __forceinline__ uint64_t key_of(float d, int x, int y) {
    uint32_t b = __float_as_uint(d);
    if ((b & 0x7f800000u) == 0x7f800000u) b = 0x7f800000u;
    return (uint64_t(b) << 32) | (uint64_t(uint32_t(y)) << 16) | uint64_t(uint32_t(x));
}

// Inserts v into the sorted list k[0..S) if it beats the last entry; returns
// what leaves the list (the old last entry, or v itself). All S comparisons
// first (independent), then every slot takes its own entry, the one before
// it, or v: no chain through the list.
template <int S>
__device__ __forceinline__ uint64_t sorted_insert(uint64_t* k, uint64_t v) {
    const uint64_t last = k[S - 1];
    if (!(v < last)) return v;
    bool c[S];
#pragma unroll
    for (int q = 0; q < S; ++q) c[q] = v < k[q];
#pragma unroll
    for (int q = S - 1; q > 0; --q) k[q] = c[q] ? (c[q - 1] ? k[q - 1] : v) : k[q];
    k[0] = c[0] ? v : k[0];
    return last;
}

// The K best keys of a reference, kept identically by both lanes of it.
template <int K>
struct TopK {
    static constexpr int kHeld = K;  // list entries in each lane
    uint64_t k[K];
    __device__ __forceinline__ void init(int) {
#pragma unroll
        for (int q = 0; q < K; ++q) k[q] = ~0ull;
    }
    __device__ __forceinline__ void add(uint64_t v) { (void)sorted_insert<K>(k, v); }
    __device__ __forceinline__ uint64_t worst() const { return k[K - 1]; }
    // entry q of the list, and whether this lane holds it
    __device__ __forceinline__ bool holds(int q, int half) const { return half == 0; }
    __device__ __forceinline__ uint64_t at(int q) const { return k[q]; }
};

// Groups of 32: the 31-entry list split over the two lanes of a reference
// (half 0 the 16 smallest keys, half 1 the next 15), so a lane holds no more
// registers than the 15-entry list. Every key of half 0's list is below every
// key of half 1's, so a new key v enters as follows, both lanes running the
// same instructions: half 0 inserts v (a no-op unless v beats its last key);
// half 1 inserts max(v, half 0's last key) -- v itself, or the key half 0
// lets go, which lands at half 1's front. Half 1's 16th slot is scratch.
// Both lanes then take the overall worst (half 1's 15th key), so they agree
// on every pass mask and run the same insertions (the pair's shuffles use
// the pair's own lane mask).
template <int K>
struct SplitTopK {
    static constexpr int LO = (K + 1) / 2, HI = K - LO, kHeld = LO;
    static_assert(HI <= LO, "half 1's list fits in half 0's length");
    uint64_t k[LO];
    uint64_t worst_;
    int half, lo_lane, hi_lane;
    unsigned pair;
    __device__ __forceinline__ void init(int lane) {
#pragma unroll
        for (int q = 0; q < LO; ++q) k[q] = ~0ull;
        worst_ = ~0ull;
        half = lane >> 4;
        lo_lane = lane & 15;
        hi_lane = lo_lane | 16;
        pair = (1u << lo_lane) | (1u << hi_lane);
    }
    __device__ __forceinline__ void add(uint64_t v) {
        if (!(v < worst_)) return;  // the same decision in both lanes
        const uint64_t lo_last = __shfl_sync(pair, k[LO - 1], lo_lane);
        (void)sorted_insert<LO>(k, half == 0 || v > lo_last ? v : lo_last);
        worst_ = __shfl_sync(pair, k[HI - 1], hi_lane);
    }
    __device__ __forceinline__ uint64_t worst() const { return worst_; }
    __device__ __forceinline__ bool holds(int q, int h) const { return h == (q < LO ? 0 : 1); }
    __device__ __forceinline__ uint64_t at(int q) const { return k[q < LO ? q : q - LO]; }
};

constexpr int kLanes = 32;   // references per CTA
// tile row pitch: the 31 * 8 + 2R + 8 columns of 32 references at step <= 8,
// rounded up to a multiple of 4 (the swizzle only permutes a column within
// its aligned group of 4; 276 floats at range 9)
template <int R>
__host__ __device__ constexpr int tile_pitch() { return (31 * 8 + 2 * R + 8 + 3) / 4 * 4; }

template <int R>
__host__ __device__ constexpr int tile_rows() { return 2 * R + 8; }

// one bit per candidate row of a window column: 32 bits up to range 15,
// 64 up to range 31
template <int R>
using RowMask = typename std::conditional<(2 * R + 1 <= 32), uint32_t, uint64_t>::type;

__device__ __forceinline__ int first_bit(uint32_t m) { return __ffs(m) - 1; }
__device__ __forceinline__ int first_bit(uint64_t m) { return __ffsll((long long)m) - 1; }

// Resident CTAs per SM the launch bounds ask for: 16 warps of 127 registers.
template <int K, int P>
__host__ __device__ constexpr int match8_min_blocks() { return (K <= 7 ? 16 : 12) / (2 * P) > 0 ? (K <= 7 ? 16 : 12) / (2 * P) : 1; }

// One tile: 32 consecutive references of one grid row of one plane. BANDED:
// the window's range exceeds R and is swept in bands (see below).
template <int R, int K, int P, bool BANDED>
__device__ __forceinline__ void match8_tile(const MatchBatch& mb, int tile_id, float* tile) {
    constexpr int B = 8, HB = 4;
    constexpr int NC = 2 * R + 1;            // candidates per window column
    constexpr int TR = tile_rows<R>();
    constexpr int kPitch = tile_pitch<R>();
    using Mask = RowMask<R>;
    int pl = 0;
    {
        int lo = 0, hi = mb.n - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (mb.p[mid].cta0 <= tile_id) lo = mid; else hi = mid - 1;
        }
        pl = lo;
    }
    const MatchPlane& P_ = mb.p[pl];
    const int W = P_.W, H = P_.H, step = mb.step, nx = P_.nx;
    const int rxe = P_.rx_end > 0 ? P_.rx_end : nx;  // grid columns [rx_begin, rxe)
    const int local = tile_id - P_.cta0;
    const int chunks = (rxe - P_.rx_begin + kLanes - 1) / kLanes;
    const int ry = local / chunks, rx0 = P_.rx_begin + (local - ry * chunks) * kLanes;
    const int rx1 = min(rx0 + kLanes, rxe) - 1;
    const int cy = grid_pos(ry, H, B, step);
    const int xr0 = grid_pos(rx0, W, B, step);
    const int TW = grid_pos(rx1, W, B, step) - xr0 + NC + B - 1;  // tile columns
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rg = warp & 1, part = warp >> 1, half = lane >> 4;
    const int l = rg * 16 + (lane & 15);
    const int rx = rx0 + l;
    const bool active = rx < rxe;
    const int cx = grid_pos(min(rx, rxe - 1), W, B, step);
    // The window's own range Rr: up to R, a kernel built for range R serves
    // it in one pass (rows and columns beyond Rr masked or skipped); beyond R
    // (ranges 32-64 on the R = 31 kernel) the window is swept in bands of
    // NC x NC candidates, the tile reloaded per band and the lists carried
    // in registers from band to band.
    const int Rr = mb.range;
    constexpr bool banded = BANDED;
    const int nb = banded ? (2 * Rr + NC) / NC : 1;  // bands per axis: ceil((2 Rr + 1) / NC)
    const int left = max(cx - Rr, 0), right = min(cx + Rr, W - B);
    const int tc0 = cx - xr0 + HB * half;  // tile column of this half's first block column at band column 0

    float2 ref[B][2];
    using List = typename std::conditional<(K > 15), SplitTopK<K>, TopK<K>>::type;
    List topk;
    topk.init(lane);
    // finished distances of the current column, one slot per candidate row:
    // an emit stores its sum and marks a bit when it may enter the list; the
    // insertions run after the column, once per marked candidate
    // one slot per reference and candidate row of the part's current column:
    // a reference's two lanes hold the same sum (their halves meet in one
    // commutative add), so both store it to the same slot and each reads
    // back its own store
    float* stash = tile + TR * kPitch + part * (NC * kLanes) + l;  // [P][NC][32 references]
    const float2 neg1 = make_float2(-1.f, -1.f);
    for (int band = 0; band < nb * nb; ++band) {
    // candidate (band column d, band row k) is (cx + ox + d, cy + oy + k)
    const int ox = banded ? -Rr + (band % nb) * NC : -R, oy = banded ? -Rr + (band / nb) * NC : -R;
    const int X0 = xr0 + ox, Y0 = cy + oy;
    if (band > 0) __syncthreads();  // every warp is done with the previous band's tile
    for (int r = warp; r < TR; r += 2 * P) {
        const int gy = Y0 + r;
        const bool yok = gy >= 0 && gy < H;
        const float* src = P_.src + (int64_t)(yok ? gy : 0) * P_.stride;
        float* dst = tile + r * kPitch;
        for (int c = lane; c < TW; c += 32) {
            const int gx = X0 + c;
            const bool ok = yok && gx >= 0 && gx < W;
            cp_async4(dst + swz(c), ok ? src + gx : src, ok ? 4 : 0);
        }
    }
    // this tile's share of the plane's words to clear, stored while the
    // window rows are in flight (an even count per tile: 16-byte stores)
    if (band == 0 && P_.clear) {
        const int tiles = chunks * P_.ny;
        const int64_t per = ((P_.clear_words + tiles - 1) / tiles + 1) & ~int64_t(1);
        const int64_t a = (int64_t)local * per, b = min(P_.clear_words, a + per);
        for (int64_t i = a + 2 * threadIdx.x; i + 1 < b; i += 2 * (int64_t)blockDim.x)
            *reinterpret_cast<longlong2*>(P_.clear + i) = make_longlong2(0, 0);
    }
    cp_async_wait_all();
    __syncthreads();
    if (band == 0) {
        // this half's 8x4 reference block as column pairs (c, c+1) of each
        // row: from the tile (rows R.. hold the block), or from the plane when banded
#pragma unroll
        for (int i = 0; i < B; ++i)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                if (banded) {
                    const float* rp = P_.src + (int64_t)(cy + i) * P_.stride + cx + HB * half + 2 * h;
                    ref[i][h] = make_float2(__ldg(rp), __ldg(rp + 1));
                } else {
                    ref[i][h] = make_float2(tile[(R + i) * kPitch + swz(tc0 + R + 2 * h)],
                                            tile[(R + i) * kPitch + swz(tc0 + R + 2 * h + 1)]);
                }
            }
    }
    // the band's candidate rows inside the reference's clamped window
    const int klo = max(max(cy - Rr, 0) - (cy + oy), 0), khi = min(min(cy + Rr, H - B) - (cy + oy), NC - 1);
    const Mask rows_ok = klo > khi ? Mask(0) : ((Mask(1) << (khi + 1)) - 1) & ~((Mask(1) << klo) - 1);
    // this part's columns: unbanded, walked outwards from the window centre
    // so the closest candidates (usually the best) fill the list first
    const int ncols = banded ? min(NC, Rr - ox + 1) : 2 * Rr + 1;
    const int cpw = (ncols + P - 1) / P;
    const int d0 = (banded ? 0 : R - Rr) + part * cpw, d1 = min((banded ? 0 : R - Rr) + ncols, d0 + cpw);
    const bool down = !banded && d1 - 1 <= R;
    // one part: the centre column, then outwards on alternate sides (R - 1,
    // R + 1, R - 2, ...), so the list's threshold tightens from both sides
    const bool alt = P == 1 && !banded;
    for (int m = 0; m < d1 - d0; ++m) {
        const int dxi = alt ? R + ((m & 1) ? -((m + 1) >> 1) : (m >> 1)) : down ? d1 - 1 - m : d0 + m;
        const int x = cx + ox + dxi;
        const bool xok = x >= left && x <= right;
        Mask pass = 0;
        // a candidate may enter unless it is farther than the current worst
        // (NaN never compares greater: non-finite sums always take the exact path)
        const float worst = __uint_as_float(uint32_t(topk.worst() >> 32));
        int col[HB];
#pragma unroll
        for (int j = 0; j < HB; ++j) col[j] = swz(tc0 + dxi + j);
        // per-column chains, two columns per packed FMA: acc[k & 7][h] holds
        // columns (2h, 2h+1) of this half for candidate k
        float2 acc[8][2];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q][0] = acc[q][1] = make_float2(0.f, 0.f);
        // window row s updates the candidates k = s - i it overlaps (block
        // row i, accumulator k & 7); once its last row is in (s = k + 7)
        // candidate k is emitted. SM8 = s & 7 and the range of i are
        // compile-time, so the accumulators stay register names.
        auto row = [&](int s, auto sm8_, auto ilo_, auto ihi_, auto emit_) {
            constexpr int SM8 = decltype(sm8_)::value, ILO = decltype(ilo_)::value, IHI = decltype(ihi_)::value;
            const float2 p01 = make_float2(tile[s * kPitch + col[0]], tile[s * kPitch + col[1]]);
            const float2 p23 = make_float2(tile[s * kPitch + col[2]], tile[s * kPitch + col[3]]);
#pragma unroll
            for (int i = ILO; i <= IHI; ++i) {
                const int ks = (SM8 - i) & 7;
                // r - p exactly as fma(p, -1, r), then the square added
                const float2 d01 = __ffma2_rn(p01, neg1, ref[i][0]);
                const float2 d23 = __ffma2_rn(p23, neg1, ref[i][1]);
                acc[ks][0] = __ffma2_rn(d01, d01, acc[ks][0]);
                acc[ks][1] = __ffma2_rn(d23, d23, acc[ks][1]);
            }
            if constexpr (decltype(emit_)::value) {
                constexpr int ks = (SM8 + 1) & 7;  // (s - 7) & 7
                const int kd = s - (B - 1);
                const float2 a = acc[ks][0], b = acc[ks][1];
                acc[ks][0] = acc[ks][1] = make_float2(0.f, 0.f);
                const float half_sum = __fadd_rn(__fadd_rn(a.x, a.y), __fadd_rn(b.x, b.y));
                const float dd = __fadd_rn(half_sum, __shfl_xor_sync(0xffffffffu, half_sum, 16));
                stash[kd * kLanes] = dd;
                pass |= Mask(dd > worst ? 0 : 1) << kd;
            }
        };
        // rows 0-6 (no candidate finished yet), then the rest: fully unrolled
        // for small windows; for ranges from 25 on, the middle rows in a
        // rolled loop of 8-row blocks so a column's code stays in the
        // instruction cache, then the last rows
        constexpr int NBLK = R >= 25 ? (NC - (B - 1)) / 8 : 0;
        static_for<0, B - 1>([&](auto S_) {
            constexpr int s = decltype(S_)::value;
            row(s, ic<s & 7>(), ic<0>(), ic<(s < NC - 1 ? s : NC - 1)>(), ic<0>());
        });
#pragma unroll 1
        for (int ob = 0; ob < NBLK; ++ob) {
            static_for<0, 8>([&](auto U_) {
                constexpr int u = decltype(U_)::value;
                row(B - 1 + 8 * ob + u, ic<(B - 1 + u) & 7>(), ic<0>(), ic<B - 1>(), ic<1>());
            });
        }
        static_for<B - 1 + 8 * NBLK, NC + B - 1>([&](auto S_) {
            constexpr int s = decltype(S_)::value;
            row(s, ic<s & 7>(), ic<(s - NC + 1 > 0 ? s - NC + 1 : 0)>(), ic<(s < B - 1 ? s : B - 1)>(),
                ic<(s >= B - 1)>());
        });
        pass &= xok ? rows_ok : Mask(0);
        if (dxi == -ox && -oy >= 0 && -oy < NC) pass &= ~(Mask(1) << -oy);  // the reference itself
        while (pass) {
            const int kd = first_bit(pass);
            pass &= pass - 1;
            topk.add(key_of(stash[kd * kLanes], x, cy + oy + kd));
        }
    }
    }  // bands
    // merge the P partial lists of each reference (exact: keys are a total order)
    if constexpr (P > 1) {
        __syncthreads();
        uint64_t* keys = reinterpret_cast<uint64_t*>(tile);  // [P][K][32 references]
        if (part > 0) {
#pragma unroll
            for (int q = 0; q < K; ++q)
                if (topk.holds(q, half)) keys[(part * K + q) * kLanes + l] = topk.at(q);
        }
        __syncthreads();
        if (part > 0) return;
        for (int w = 1; w < P; ++w)
#pragma unroll
            for (int q = 0; q < K; ++q) topk.add(keys[(w * K + q) * kLanes + l]);
    }
    // each lane writes the entries it holds; the pair adds up the count
    int n = 0;
#pragma unroll
    for (int q = 0; q < K; ++q) n += (topk.holds(q, half) && topk.at(q) != ~0ull) ? 1 : 0;
    n += __shfl_xor_sync(0xffffffffu, n, 16);
    if (!active) return;
    const int64_t job = (int64_t)ry * nx + rx;
    constexpr int G = K + 1;
    int32_t* op = P_.pos + job * G;
    float* od = P_.dist ? P_.dist + job * G : nullptr;
    if (half == 0) {
        op[0] = pack_pos(cx, cy);
        if (od) od[0] = 0.f;
        P_.count[job] = 1 + n;
    }
#pragma unroll
    for (int q = 0; q < K; ++q) {
        if (!topk.holds(q, half)) continue;
        const uint64_t e = topk.at(q);
        const bool valid = e != ~0ull;
        op[1 + q] = valid ? int32_t(uint32_t(e)) : -1;
        if (od) od[1 + q] = valid ? __uint_as_float(uint32_t(e >> 32)) : 0.f;
    }
}

// Grid form: CTA b takes tile b. Persistent form (mb.queue set): a CTA takes
// tile blockIdx.x, then keeps taking the next untaken tile from the device
// counter until none is left; the counter is zero at launch.
template <int R, int K, int P, bool BANDED>
__global__ void __launch_bounds__(64 * P, match8_min_blocks<K, P>())
    match8_kernel(const __grid_constant__ MatchBatch mb) {
    extern __shared__ float tile[];
    __shared__ int next_tile;
    int t = blockIdx.x;
    while (t < mb.total_ctas) {
        match8_tile<R, K, P, BANDED>(mb, t, tile);
        if (mb.queue == nullptr) break;
        __syncthreads();  // the tile buffer is free again
        if (threadIdx.x == 0) next_tile = atomicAdd(mb.queue, 1) + (int)gridDim.x;
        __syncthreads();
        t = next_tile;
    }
}

template <int R, int K, int P, bool BANDED = false>
void launch_rkp(MatchBatch& mb, const MatchTune& tune, cudaStream_t stream) {
    int ctas = 0;
    for (int i = 0; i < mb.n; ++i) {
        MatchPlane& p = mb.p[i];
        p.nx = grid_count(p.W, 8, mb.step);
        p.ny = grid_count(p.H, 8, mb.step);
        p.cta0 = ctas;
        ctas += ceil_div((p.rx_end > 0 ? p.rx_end : p.nx) - p.rx_begin, kLanes) * p.ny;
    }
    mb.total_ctas = ctas;
    mb.queue = nullptr;
    if (ctas == 0) return;
    static_assert(2 * R + 1 <= 64, "a column's candidates must fit the row mask");
    const size_t smem = std::max((size_t)(tile_pitch<R>() * tile_rows<R>() + (2 * R + 1) * kLanes * P) * sizeof(float),
                                 (size_t)P * K * kLanes * sizeof(uint64_t));
    auto kern = match8_kernel<R, K, P, BANDED>;
    NSSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int grid = ctas;
    if (tune.persistent && tune.queue) {
        int dev = 0, sms = 0, per_sm = 0;
        NSSB_CUDA(cudaGetDevice(&dev));
        NSSB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        NSSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 64 * P, smem));
        const int resident = sms * std::max(per_sm, 1);
        if (resident < ctas) {
            grid = resident;
            mb.queue = tune.queue;
            NSSB_CUDA(cudaMemsetAsync(tune.queue, 0, sizeof(int), stream));
        }
    }
    kern<<<grid, 64 * P, smem, stream>>>(mb);
    NSSB_CUDA(cudaGetLastError());
}

template <int R, int K>
void launch_rk(MatchBatch& mb, const MatchTune& tune, cudaStream_t stream) {
    if (mb.range > R) {  // ranges 32-64 on the 31 kernel, in bands
        if constexpr (R == 31) launch_rkp<R, K, 2, true>(mb, tune, stream);
        return;
    }
    if constexpr (R == 9) {  // the default range: every column split the tuner may pick
        switch (tune.parts) {
            case 1: launch_rkp<R, K, 1>(mb, tune, stream); break;
            case 4: launch_rkp<R, K, 4>(mb, tune, stream); break;
            default: launch_rkp<R, K, 2>(mb, tune, stream); break;
        }
    } else {
        launch_rkp<R, K, 2>(mb, tune, stream);
    }
}

template <int R>
bool launch_r(MatchBatch& mb, int group, const MatchTune& tune, cudaStream_t stream) {
    switch (group) {
        case 2: launch_rk<R, 1>(mb, tune, stream); return true;
        case 4: launch_rk<R, 3>(mb, tune, stream); return true;
        case 8: launch_rk<R, 7>(mb, tune, stream); return true;
        case 16: launch_rk<R, 15>(mb, tune, stream); return true;
        case 32: launch_rk<R, 31>(mb, tune, stream); return true;
        default: return false;
    }
}

}  // namespace

bool launch_match8_batch(MatchBatch& mb, int bm_range, int group, cudaStream_t stream, const MatchTune* tune) {
    // dense steps: the column-reuse matcher where it takes the shape
    if (matchcol_takes(mb.step, bm_range, group) && launch_matchcol_batch(mb, bm_range, group, stream)) return true;
    return launch_match8_direct(mb, bm_range, group, stream, tune);
}

bool launch_match8_direct(MatchBatch& mb, int bm_range, int group, cudaStream_t stream, const MatchTune* tune) {
    if (mb.step < 1 || mb.step > 8 || mb.n < 1 || mb.n > kMaxBatchPlanes) return false;
    for (int i = 0; i < mb.n; ++i)
        if (mb.p[i].W < 8 || mb.p[i].H < 8) return false;
    const MatchTune t = tune ? *tune : MatchTune{};
    // ranges 4-31 (a column's 2R + 1 candidates take one bit each of a 32- or
    // 64-bit pass mask): the kernel built for the range, or for the next
    // larger range that has one
    mb.range = bm_range;
    if (bm_range < 4) return false;
    if (bm_range <= 9) {
        switch (bm_range) {
            case 4: return launch_r<4>(mb, group, t, stream);
            case 5: return launch_r<5>(mb, group, t, stream);
            case 6: return launch_r<6>(mb, group, t, stream);
            case 7: return launch_r<7>(mb, group, t, stream);
            case 8: return launch_r<8>(mb, group, t, stream);
            default: return launch_r<9>(mb, group, t, stream);
        }
    }
    if (bm_range <= 12) return launch_r<12>(mb, group, t, stream);
    if (bm_range <= 15) return launch_r<15>(mb, group, t, stream);
    if (bm_range <= 16) return launch_r<16>(mb, group, t, stream);
    if (bm_range <= 19) return launch_r<19>(mb, group, t, stream);
    if (bm_range <= 25) return launch_r<25>(mb, group, t, stream);
    if (bm_range <= 64) return launch_r<31>(mb, group, t, stream);  // beyond 31: in bands
    return false;
}

bool launch_match8(const float* plane, int64_t stride, int width, int height, int step, int bm_range, int group,
                   int32_t* pos, float* dist, int32_t* count, cudaStream_t stream) {
    static thread_local MatchBatch mb;
    mb.n = 1;
    mb.step = step;
    mb.p[0] = MatchPlane{plane, stride, pos, dist, count, width, height, 0, 0, 0};
    return launch_match8_batch(mb, bm_range, group, stream, nullptr);
}

}  // namespace nssb
