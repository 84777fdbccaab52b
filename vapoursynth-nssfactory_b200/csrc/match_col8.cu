// Exact FP32 block matching for 8x8 blocks at steps 1-4 by column reuse
// (sm_100a): the dense-step shapes, the reference's "heavy" preset among
// them (block_step 3, bm_range 19, groups of 16 and 32).
//
// Below a step of 8, horizontally adjacent references share block columns.
// For a displacement (dx, dy) the column sum
//     S(c) = sum_i (I[y+i][c] - I[y+dy+i][c+dx])^2   (one FMA chain down the rows)
// of image column c is the same number for every reference whose block
// covers c, and a reference's distance is the canonical tree of its eight
// column sums, ((S0+S1)+(S2+S3))+((S4+S5)+(S6+S7)) -- the SSD order of every
// other matcher here, so the distances, keys and lists are bit-identical to
// theirs. (The reference's CUDA column matcher shares column sums the same
// way at steps 1-3, src/cuda/common/match_column.cu:97-100,360-366; the
// schedule below is this build's own.)
//   - a CTA is one grid row's run of 32 - h references (h = ceil(8/S) - 1
//     helper lanes) and P warps. Lane l of every warp owns the S image
//     columns l*S .. l*S+S-1 of the run, reference l's first S columns; the
//     P warps split the window columns dx;
//   - the run's window rows are staged once in shared memory (asynchronous
//     copies); a lane streams its columns' 2R+8 window rows and applies each
//     row to the 8 candidate rows that overlap it (accumulator dy & 7), two
//     columns per packed FMA where it can;
//   - a finished candidate's distance is assembled in the canonical order
//     from the next h lanes' column sums by shuffles, so each column sum is
//     formed once for the ceil(8/S) references that use it;
//   - one register top-k per reference (its lane); the P partial lists merge
//     in shared memory. While they run, each part publishes its list's last
//     key after every window column and filters its candidates against the
//     smallest of the parts' last keys: a candidate farther than some part's
//     K-th is beaten by K others and cannot make the merged list, so the
//     parts together insert about as often as one list would.
// The last grid column is clamped to W-8 when the step does not divide
// W-8; that reference's columns are off the lanes' grid, so the 8x8 direct
// matcher (match8.cu) takes that one grid column.
#include "kernels.cuh"

#include <algorithm>
#include <type_traits>

namespace nssb {
namespace {

__device__ __forceinline__ uint64_t col_key(float d, int x, int y) {
    uint32_t b = __float_as_uint(d);
    if ((b & 0x7f800000u) == 0x7f800000u) b = 0x7f800000u;
    return (uint64_t(b) << 32) | (uint64_t(uint32_t(y)) << 16) | uint64_t(uint32_t(x));
}

template <int K>
struct LaneTopK {
    uint64_t k[K];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int q = 0; q < K; ++q) k[q] = ~0ull;
    }
    // all K comparisons first, then every slot takes its own entry, the one
    // before it, or v
    __device__ __forceinline__ void add(uint64_t v) {
        if (!(v < k[K - 1])) return;
        bool c[K];
#pragma unroll
        for (int q = 0; q < K; ++q) c[q] = v < k[q];
#pragma unroll
        for (int q = K - 1; q > 0; --q) k[q] = c[q] ? (c[q - 1] ? k[q - 1] : v) : k[q];
        k[0] = c[0] ? v : k[0];
    }
};

template <int S>
__host__ __device__ constexpr int helpers() { return (8 + S - 1) / S - 1; }
template <int S>
__host__ __device__ constexpr int refs_per_cta() { return 32 - helpers<S>(); }
// tile column of run column c: even steps add one word per 32 columns, so
// the lanes' S-strided reads fall on distinct banks
template <int S>
__host__ __device__ constexpr int tcol(int c) { return S % 2 == 0 ? c + (c >> 5) : c; }
template <int S, int R>
__host__ __device__ constexpr int col_pitch() { return (tcol<S>(32 * S + 2 * R) + 1 + 3) / 4 * 4; }
template <int R>
__host__ __device__ constexpr int col_rows() { return 2 * R + 8; }

template <int R>
using ColMask = typename std::conditional<(2 * R + 1 <= 32), uint32_t, uint64_t>::type;
__device__ __forceinline__ int lowest_bit(uint32_t m) { return __ffs(m) - 1; }
__device__ __forceinline__ int lowest_bit(uint64_t m) { return __ffsll((long long)m) - 1; }

// The candidate's distance from this lane's S column sums and the next
// lanes' (all 32 lanes take part in the shuffles).
template <int S>
__device__ __forceinline__ float assemble(const float* c) {
    if constexpr (S == 1) {
        const float t1 = __fadd_rn(c[0], __shfl_down_sync(0xffffffffu, c[0], 1));
        const float t2 = __fadd_rn(t1, __shfl_down_sync(0xffffffffu, t1, 2));
        return __fadd_rn(t2, __shfl_down_sync(0xffffffffu, t2, 4));
    } else if constexpr (S == 2) {
        const float a = __fadd_rn(c[0], c[1]);
        const float t = __fadd_rn(a, __shfl_down_sync(0xffffffffu, a, 1));
        return __fadd_rn(t, __shfl_down_sync(0xffffffffu, t, 2));
    } else if constexpr (S == 3) {
        // columns 0-2 here, 3-5 on the next lane, 6-7 on the one after
        const float a = __fadd_rn(c[0], c[1]);  // (c0 + c1), and the next-but-one lane's (c6 + c7)
        const float b = __fadd_rn(c[1], c[2]);  // the next lane's (c4 + c5)
        const float x = __shfl_down_sync(0xffffffffu, c[0], 1);
        const float y = __shfl_down_sync(0xffffffffu, b, 1);
        const float z = __shfl_down_sync(0xffffffffu, a, 2);
        return __fadd_rn(__fadd_rn(a, __fadd_rn(c[2], x)), __fadd_rn(y, z));
    } else {
        const float t = __fadd_rn(__fadd_rn(c[0], c[1]), __fadd_rn(c[2], c[3]));
        return __fadd_rn(t, __shfl_down_sync(0xffffffffu, t, 1));
    }
}

// Resident CTAs per SM the launch bounds ask for: 16 warps (128 registers)
// up to groups of 16, 12 warps for groups of 32.
template <int K, int P>
__host__ __device__ constexpr int matchcol_min_blocks() { return (K <= 15 ? 16 : 12) / P; }

template <int S, int R, int K, int P>
__global__ void __launch_bounds__(32 * P, matchcol_min_blocks<K, P>()) matchcol_kernel(const __grid_constant__ MatchBatch mb) {
    constexpr int B = 8, NC = 2 * R + 1, TR = col_rows<R>(), kPitch = col_pitch<S, R>();
    constexpr int NREF = refs_per_cta<S>();
    constexpr int S2 = S / 2;  // packed column pairs
    using Mask = ColMask<R>;
    extern __shared__ float tile[];
    const int tile_id = blockIdx.x;
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
    const int W = P_.W, H = P_.H, nx = P_.nx;
    const int nreg = P_.rx_end;  // references on the lanes' grid: [0, nreg)
    const int local = tile_id - P_.cta0;
    const int chunks = (nreg + NREF - 1) / NREF;
    const int ry = local / chunks, rx0 = (local - ry * chunks) * NREF;
    const int cy = grid_pos(ry, H, B, S);
    const int xb = rx0 * S;  // the run's first column
    const int X0 = xb - R, Y0 = cy - R;
    constexpr int TW = 32 * S + 2 * R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < TR; r += P) {
        const int gy = Y0 + r;
        const bool yok = gy >= 0 && gy < H;
        const float* src = P_.src + (int64_t)(yok ? gy : 0) * P_.stride;
        float* dst = tile + r * kPitch;
        for (int c = lane; c < TW; c += 32) {
            const int gx = X0 + c;
            const bool ok = yok && gx >= 0 && gx < W;
            cp_async4(dst + tcol<S>(c), ok ? src + gx : src, ok ? 4 : 0);
        }
    }
    // this tile's share of the plane's words to clear (as the 8x8 matcher does)
    if (P_.clear) {
        const int tiles = chunks * P_.ny;
        const int64_t per = ((P_.clear_words + tiles - 1) / tiles + 1) & ~int64_t(1);
        const int64_t a = (int64_t)local * per, b = min(P_.clear_words, a + per);
        for (int64_t i = a + 2 * threadIdx.x; i + 1 < b; i += 2 * (int64_t)blockDim.x)
            *reinterpret_cast<longlong2*>(P_.clear + i) = make_longlong2(0, 0);
    }
    // each part's current last key per reference, for the shared filter
    volatile uint64_t* part_last = reinterpret_cast<volatile uint64_t*>(tile + TR * kPitch + NC * 32 * P);
    part_last[warp * 32 + lane] = ~0ull;
    cp_async_wait_all();
    __syncthreads();

    const int part = warp;
    const int rx = rx0 + lane;
    const bool is_ref = lane < NREF && rx < nreg;
    const int cx = xb + lane * S;  // this lane's first column (its reference's x)
    const int Rr = mb.range;
    const int left = max(cx - Rr, 0), right = min(cx + Rr, W - B);
    const int kmin = max(cy - Rr, 0) - (cy - R), kmax = min(cy + Rr, H - B) - (cy - R);
    const int c0 = lane * S;  // run column of the lane's first column at dx = -R, plus R below
    // this lane's S columns of the reference block (rows cy .. cy+7)
    float2 rp[B][S2 > 0 ? S2 : 1];
    float rs[B];
#pragma unroll
    for (int i = 0; i < B; ++i) {
#pragma unroll
        for (int h = 0; h < S2; ++h)
            rp[i][h] = make_float2(tile[(R + i) * kPitch + tcol<S>(c0 + R + 2 * h)],
                                   tile[(R + i) * kPitch + tcol<S>(c0 + R + 2 * h + 1)]);
        rs[i] = (S & 1) ? tile[(R + i) * kPitch + tcol<S>(c0 + R + S - 1)] : 0.f;
    }
    LaneTopK<K> topk;
    topk.init();
    float* stash = tile + TR * kPitch + threadIdx.x;  // [NC][32 P]
    const Mask rows_ok = ((Mask(1) << (kmax + 1)) - 1) & ~((Mask(1) << kmin) - 1);
    const float2 neg1 = make_float2(-1.f, -1.f);
    const int cpw = (2 * Rr + P) / P;
    const int d0 = (R - Rr) + part * cpw, d1 = min(R + Rr + 1, d0 + cpw);
    const bool down = d1 - 1 <= R;
    for (int m = 0; m < d1 - d0; ++m) {
        const int dxi = down ? d1 - 1 - m : d0 + m;
        const int x = cx - R + dxi;
        const bool xok = is_ref && x >= left && x <= right;
        Mask pass = 0;
        // the tightest last key of the P parts (a stale one is only looser)
        uint64_t last = topk.k[K - 1];
#pragma unroll
        for (int q = 0; q < P; ++q)
            if (q != part) last = min(last, (uint64_t)part_last[q * 32 + lane]);
        const float worst = __uint_as_float(uint32_t(last >> 32));
        int col[S];
#pragma unroll
        for (int j = 0; j < S; ++j) col[j] = tcol<S>(c0 + dxi + j);
        float2 a2[8][S2 > 0 ? S2 : 1];
        float a1[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
#pragma unroll
            for (int h = 0; h < S2; ++h) a2[q][h] = make_float2(0.f, 0.f);
            a1[q] = 0.f;
        }
        // window row s updates the candidates k = s - i it overlaps (block
        // row i, accumulator k & 7); once its last row is in (s = k + 7)
        // candidate k is emitted. SM8 = s & 7 and the range of i are
        // compile-time, so the accumulators stay register names.
        auto row = [&](int s, auto sm8_, auto ilo_, auto ihi_, auto emit_) {
            constexpr int SM8 = decltype(sm8_)::value, ILO = decltype(ilo_)::value, IHI = decltype(ihi_)::value;
            float2 p2[S2 > 0 ? S2 : 1];
#pragma unroll
            for (int h = 0; h < S2; ++h)
                p2[h] = make_float2(tile[s * kPitch + col[2 * h]], tile[s * kPitch + col[2 * h + 1]]);
            const float p1 = (S & 1) ? tile[s * kPitch + col[S - 1]] : 0.f;
#pragma unroll
            for (int i = ILO; i <= IHI; ++i) {
                const int ks = (SM8 - i) & 7;
#pragma unroll
                for (int h = 0; h < S2; ++h) {
                    const float2 d = __ffma2_rn(p2[h], neg1, rp[i][h]);
                    a2[ks][h] = __ffma2_rn(d, d, a2[ks][h]);
                }
                if (S & 1) {
                    const float d = __fmaf_rn(p1, -1.f, rs[i]);
                    a1[ks] = __fmaf_rn(d, d, a1[ks]);
                }
            }
            if constexpr (decltype(emit_)::value) {
                constexpr int ks = (SM8 + 1) & 7;  // (s - 7) & 7
                const int kd = s - (B - 1);
                float c[S];
#pragma unroll
                for (int h = 0; h < S2; ++h) {
                    c[2 * h] = a2[ks][h].x;
                    c[2 * h + 1] = a2[ks][h].y;
                    a2[ks][h] = make_float2(0.f, 0.f);
                }
                if (S & 1) {
                    c[S - 1] = a1[ks];
                    a1[ks] = 0.f;
                }
                const float dd = assemble<S>(c);
                stash[kd * (32 * P)] = dd;
                pass |= Mask(dd > worst ? 0 : 1) << kd;
            }
        };
        // rows 0-6: the first candidates, none finished yet
        static_for<0, B - 1>([&](auto S_) {
            constexpr int s = decltype(S_)::value;
            row(s, ic<s & 7>(), ic<0>(), ic<s>(), ic<false>());
        });
        // rows 7 .. NC-1 in blocks of 8: every row updates 8 candidates and finishes one
        constexpr int NBLK = (NC - (B - 1)) / 8;
#pragma unroll 1
        for (int ob = 0; ob < NBLK; ++ob) {
            static_for<0, 8>([&](auto U_) {
                constexpr int u = decltype(U_)::value;
                row(B - 1 + 8 * ob + u, ic<(B - 1 + u) & 7>(), ic<0>(), ic<B - 1>(), ic<true>());
            });
        }
        // the remaining rows up to NC + 6: the last candidates finish
        static_for<B - 1 + 8 * NBLK, NC + B - 1>([&](auto S_) {
            constexpr int s = decltype(S_)::value;
            row(s, ic<s & 7>(), ic<(s - NC + 1 > 0 ? s - NC + 1 : 0)>(), ic<(s < B - 1 ? s : B - 1)>(),
                ic<(s >= B - 1)>());
        });
        pass &= xok ? rows_ok : Mask(0);
        if (dxi == R) pass &= ~(Mask(1) << R);
        while (pass) {
            const int kd = lowest_bit(pass);
            pass &= pass - 1;
            topk.add(col_key(stash[kd * (32 * P)], x, cy - R + kd));
        }
        part_last[part * 32 + lane] = topk.k[K - 1];
    }
    if constexpr (P > 1) {
        __syncthreads();
        uint64_t* keys = reinterpret_cast<uint64_t*>(tile);  // [P][K][32 lanes]
        if (part > 0) {
#pragma unroll
            for (int q = 0; q < K; ++q) keys[(part * K + q) * 32 + lane] = topk.k[q];
        }
        __syncthreads();
        if (part > 0) return;
        for (int w = 1; w < P; ++w)
#pragma unroll
            for (int q = 0; q < K; ++q) topk.add(keys[(w * K + q) * 32 + lane]);
    }
    if (!is_ref) return;
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

template <int S, int R, int K>
void launch_srk(MatchBatch& mb, cudaStream_t stream) {
    int ctas = 0;
    for (int i = 0; i < mb.n; ++i) {
        MatchPlane& p = mb.p[i];
        p.cta0 = ctas;
        ctas += ceil_div(p.rx_end, refs_per_cta<S>()) * p.ny;
    }
    mb.total_ctas = ctas;
    mb.queue = nullptr;
    if (ctas == 0) return;
    static_assert(2 * R + 1 <= 64, "a column's candidates must fit the row mask");
    const size_t smem =
        std::max((size_t)(col_pitch<S, R>() * col_rows<R>() + (2 * R + 1) * 32 * kParts) * sizeof(float) +
                     (size_t)kParts * 32 * sizeof(uint64_t),
                 (size_t)kParts * K * 32 * sizeof(uint64_t));
    auto kern = matchcol_kernel<S, R, K, kParts>;
    NSSB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<ctas, 32 * kParts, smem, stream>>>(mb);
    NSSB_CUDA(cudaGetLastError());
}

template <int S, int R>
bool launch_sr(MatchBatch& mb, int group, cudaStream_t stream) {
    switch (group) {
        case 4: launch_srk<S, R, 3>(mb, stream); return true;
        case 8: launch_srk<S, R, 7>(mb, stream); return true;
        case 16: launch_srk<S, R, 15>(mb, stream); return true;
        case 32:
            if constexpr (S <= 3) {
                launch_srk<S, R, 31>(mb, stream);
                return true;
            }
            return false;
        default: return false;
    }
}

template <int S>
bool launch_s(MatchBatch& mb, int bm_range, int group, cudaStream_t stream) {
    if (bm_range <= 9) return launch_sr<S, 9>(mb, group, stream);
    if (bm_range <= 16) return launch_sr<S, 16>(mb, group, stream);
    if (bm_range <= 19) return launch_sr<S, 19>(mb, group, stream);
    if (bm_range <= 25) return launch_sr<S, 25>(mb, group, stream);
    if (bm_range <= 31) return launch_sr<S, 31>(mb, group, stream);
    return false;
}

}  // namespace

bool matchcol_takes(int step, int bm_range, int group) {
    if (step < 1 || step > 4 || bm_range < 9 || bm_range > 31) return false;
    return group == 4 || group == 8 || group == 16 || (group == 32 && step <= 3);
}

bool launch_matchcol_batch(MatchBatch& mb, int bm_range, int group, cudaStream_t stream) {
    if (!matchcol_takes(mb.step, bm_range, group) || mb.n < 1 || mb.n > kMaxBatchPlanes) return false;
    for (int i = 0; i < mb.n; ++i)
        if (mb.p[i].W < 8 || mb.p[i].H < 8) return false;
    mb.range = bm_range;
    // references on the lanes' grid, and the planes whose last grid column is clamped
    static thread_local MatchBatch tail;
    tail.n = 0;
    tail.step = mb.step;
    for (int i = 0; i < mb.n; ++i) {
        MatchPlane& p = mb.p[i];
        p.nx = grid_count(p.W, 8, mb.step);
        p.ny = grid_count(p.H, 8, mb.step);
        const bool clamped = grid_pos(p.nx - 1, p.W, 8, mb.step) != (p.nx - 1) * mb.step;
        p.rx_begin = 0;
        p.rx_end = clamped ? p.nx - 1 : p.nx;
        if (clamped) {
            MatchPlane t = p;
            t.rx_begin = p.nx - 1;
            t.rx_end = p.nx;
            t.clear = nullptr;  // the column kernel clears the whole plane
            t.clear_words = 0;
            tail.p[tail.n++] = t;
        }
    }
    bool ok = false;
    switch (mb.step) {
        case 1: ok = launch_s<1>(mb, bm_range, group, stream); break;
        case 2: ok = launch_s<2>(mb, bm_range, group, stream); break;
        case 3: ok = launch_s<3>(mb, bm_range, group, stream); break;
        default: ok = launch_s<4>(mb, bm_range, group, stream); break;
    }
    if (!ok) return false;
    if (tail.n > 0 && !launch_match8_direct(tail, bm_range, group, stream, nullptr))
        throw CudaError("nss_cuda: the 8x8 matcher declined the clamped grid column");
    return true;
}

}  // namespace nssb
