// Predictive temporal matching (sm_100a).
//
// Semantics (reference collect_temporal, src/cpu/bm/matcher.hpp:319-373, and
// predictive_match, src/cpu/bm/match.cpp:10-33): the spatial group of the
// reference on slot t0 seeds the search; in each direction the slots
// t0 +- 1, +- 2, ... (inside the valid range) are searched over the raster
// union of the ps_range windows around the ps_num best matches of the previous
// slot; each slot's ps_num best join the global group. Order: distance, then
// the reference first, then slot, y, x.
//
// One thread per reference, after the spatial kernel has written the slot-t0
// group into pos/dist/count. Pixels come through the read-only cache: the
// windows follow the motion of each group, so there is no shared tile.
#include "kernels.cuh"

namespace nssb {
namespace {

struct TKey {
    uint32_t d;    // canonical distance bits
    uint64_t tyx;  // slot << 32 | y << 16 | x  (x, y < 65536)
};

__device__ __forceinline__ uint64_t tyx_key(int t, int y, int x) {
    return (uint64_t(uint32_t(t)) << 32) | (uint64_t(uint32_t(y)) << 16) | uint64_t(uint32_t(x));
}
__device__ __forceinline__ int tyx_x(uint64_t k) { return int(k & 0xffffu); }
__device__ __forceinline__ int tyx_y(uint64_t k) { return int((k >> 16) & 0xffffu); }
__device__ __forceinline__ int tyx_t(uint64_t k) { return int(k >> 32); }

__device__ __forceinline__ bool tkey_less(const TKey& a, const TKey& b) {
    return a.d != b.d ? a.d < b.d : a.tyx < b.tyx;
}

__device__ __forceinline__ uint32_t canon(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x7f800000u) == 0x7f800000u ? 0x7f800000u : b;
}

struct TList {
    TKey k[64];
    int cap, n;
    __device__ void init(int c) {
        cap = c;
        n = 0;
    }
    __device__ void add(TKey v) {
        if (cap <= 0) return;
        if (n == cap) {
            if (!tkey_less(v, k[n - 1])) return;
            --n;
        }
        int p = n;
        while (p > 0 && tkey_less(v, k[p - 1])) {
            k[p] = k[p - 1];
            --p;
        }
        k[p] = v;
        ++n;
    }
};

// SSD in this build's order: per-column FMA chains down the rows, column_tree.
template <int B>
__device__ float ssd_global(const float* __restrict__ a, int64_t sa, const float* __restrict__ b, int64_t sb) {
    float c[B];
#pragma unroll
    for (int j = 0; j < B; ++j) c[j] = 0.f;
#pragma unroll
    for (int i = 0; i < B; ++i)
#pragma unroll
        for (int j = 0; j < B; ++j) {
            const float d = __fsub_rn(__ldg(a + i * sa + j), __ldg(b + i * sb + j));
            c[j] = __fmaf_rn(d, d, c[j]);
        }
    return column_tree<B>(c);
}

__device__ float ssd_global_rt(const float* __restrict__ a, int64_t sa, const float* __restrict__ b, int64_t sb,
                               int B) {
    switch (B) {
        case 1: return ssd_global<1>(a, sa, b, sb);
        case 2: return ssd_global<2>(a, sa, b, sb);
        case 4: return ssd_global<4>(a, sa, b, sb);
        case 8: return ssd_global<8>(a, sa, b, sb);
        case 12: return ssd_global<12>(a, sa, b, sb);
        case 16: return ssd_global<16>(a, sa, b, sb);
        default: return ssd_global<32>(a, sa, b, sb);
    }
}

template <int B>
__global__ void __launch_bounds__(64) temporal_kernel(TemporalPlanes tp, int ntemp, int t0, int first, int last,
                                                     int W, int H, int Bdyn, int step, int G, int ps_num,
                                                     int ps_range, int nx, int ny, int32_t* __restrict__ pos,
                                                     int32_t* __restrict__ slot, float* __restrict__ dist,
                                                     int32_t* __restrict__ count) {
    const int blk = B > 0 ? B : Bdyn;
    const int job = blockIdx.x * blockDim.x + threadIdx.x;
    if (job >= nx * ny) return;
    int32_t* op = pos + (int64_t)job * G;
    int32_t* os = slot + (int64_t)job * G;
    float* od = dist + (int64_t)job * G;
    const int n = count[job];
    const int cx = pos_x(op[0]), cy = pos_y(op[0]);
    const float* refp = tp.plane[t0] + (int64_t)cy * tp.stride[t0] + cx;
    const int64_t rs = tp.stride[t0];
    for (int q = 0; q < G; ++q) os[q] = q < n ? t0 : -1;
    if (n <= 0 || ntemp == 1 || G == 1 || first >= last) return;

    // seeds: the first min(n, ps_num) of the spatial group (self included)
    TKey seeds[64];
    const int nseed = min(n, ps_num);
    for (int i = 0; i < nseed; ++i) {
        seeds[i].d = canon(od[i]);
        seeds[i].tyx = tyx_key(t0, pos_y(op[i]), pos_x(op[i]));
    }
    TList global;
    global.init(G - 1);
    for (int i = 1; i < n; ++i) {
        TKey k;
        k.d = canon(od[i]);
        k.tyx = tyx_key(t0, pos_y(op[i]), pos_x(op[i]));
        global.add(k);
    }
    const int maxx = W - blk, maxy = H - blk;
    for (int si = 0; si < 2; ++si) {
        const int sign = si == 0 ? -1 : 1;
        TKey centers[64];
        int nc = nseed;
        for (int i = 0; i < nc; ++i) centers[i] = seeds[i];
        for (int dt = 1; dt < 64; ++dt) {
            const int t = t0 + sign * dt;
            if (t < first || t >= last || dt > (ntemp - 1) / 2) break;
            TList local;
            local.init(min(ps_num, G));
            int ymin = H, ymax = -1;
            for (int i = 0; i < nc; ++i) {
                const int cyy = tyx_y(centers[i].tyx);
                ymin = min(ymin, max(0, cyy - ps_range));
                ymax = max(ymax, min(maxy, cyy + ps_range));
            }
            const float* pl = tp.plane[t];
            const int64_t ps = tp.stride[t];
            for (int y = ymin; y <= ymax; ++y) {
                // the x intervals of the windows that cover row y, in ascending order
                int ia[64], ib[64], ni = 0;
                for (int i = 0; i < nc; ++i) {
                    const int cyy = tyx_y(centers[i].tyx), cxx = tyx_x(centers[i].tyx);
                    if (abs(y - cyy) <= ps_range) {
                        const int a = max(0, cxx - ps_range), b = min(maxx, cxx + ps_range);
                        int p = ni++;
                        while (p > 0 && (ia[p - 1] > a || (ia[p - 1] == a && ib[p - 1] > b))) {
                            ia[p] = ia[p - 1];
                            ib[p] = ib[p - 1];
                            --p;
                        }
                        ia[p] = a;
                        ib[p] = b;
                    }
                }
                int done = -1;
                for (int i = 0; i < ni; ++i) {
                    for (int x = max(done + 1, ia[i]); x <= ib[i]; ++x) {
                        const float* cb = pl + (int64_t)y * ps + x;
                        float d;
                        if constexpr (B > 0) {
                            d = ssd_global<B>(refp, rs, cb, ps);
                        } else {
                            d = ssd_global_rt(refp, rs, cb, ps, blk);
                        }
                        TKey k;
                        k.d = canon(d);
                        k.tyx = tyx_key(t, y, x);
                        local.add(k);
                    }
                    done = max(done, ib[i]);
                }
            }
            nc = local.n;
            for (int i = 0; i < nc; ++i) {
                global.add(local.k[i]);
                centers[i] = local.k[i];
            }
            if (nc == 0) break;
        }
    }
    // write back: self first, then the global list
    for (int q = 0; q < G - 1; ++q) {
        const bool valid = q < global.n;
        const TKey k = global.k[q];
        op[1 + q] = valid ? pack_pos(tyx_x(k.tyx), tyx_y(k.tyx)) : -1;
        os[1 + q] = valid ? tyx_t(k.tyx) : -1;
        od[1 + q] = valid ? __uint_as_float(k.d) : 0.f;
    }
    os[0] = t0;
    count[job] = 1 + global.n;
}

// ---- fast path: 8x8 blocks, ps_num <= 8, ps_range <= 12 ----
//
// A warp per reference searches the chain towards earlier slots, then the one
// towards later slots (4 references per CTA). In a layer the warp's
// lanes take the (window, column) pairs of the union of the ps_num windows;
// a lane streams the column's image rows from the read-only cache and applies
// each row to the (up to 8) candidates that overlap it -- candidate k in
// accumulator slot k & 7 -- in two passes over the block's column halves, so
// each distance is formed in this build's order: per-column chains down the
// rows, ((c0+c1)+(c2+c3)) + ((c4+c5)+(c6+c7)). A candidate already in an
// earlier window of the layer is skipped (the raster union's dedup). Each lane
// keeps its PS best keys; the layer's ps_num best are drawn by warp minima
// (keys are unique, so the result is the set's top, whatever the visit
// order). The layer bests of both chains then merge with the spatial group.
constexpr int kTRefs = 4;

__device__ __forceinline__ uint64_t tk64(uint32_t d, uint32_t tyx) { return (uint64_t(d) << 32) | tyx; }

template <int PS>
struct LaneTop {
    uint64_t k[PS];
    __device__ __forceinline__ void init() {
#pragma unroll
        for (int q = 0; q < PS; ++q) k[q] = ~0ull;
    }
    // all comparisons first, then each slot takes its own entry, the one
    // before it, or v (no dependency chain through the list)
    __device__ __forceinline__ void add(uint64_t v) {
        if (!(v < k[PS - 1])) return;
        bool c[PS];
#pragma unroll
        for (int q = 0; q < PS; ++q) c[q] = v < k[q];
#pragma unroll
        for (int q = PS - 1; q > 0; --q) k[q] = c[q] ? (c[q - 1] ? k[q - 1] : v) : k[q];
        k[0] = c[0] ? v : k[0];
    }
    __device__ __forceinline__ void pop() {
#pragma unroll
        for (int q = 0; q + 1 < PS; ++q) k[q] = k[q + 1];
        k[PS - 1] = ~0ull;
    }
};

__device__ __forceinline__ uint64_t warp_min64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const uint64_t u = __shfl_xor_sync(0xffffffffu, v, o);
        v = u < v ? u : v;
    }
    return v;
}

// One (window, column) task of a layer: the column's candidates (nk of them,
// rows ya.. of window i) against the reference, in two passes over the
// block's column halves; each finished, not-duplicated candidate enters the
// lane's top list. NK > 0: nk == NK known at compile time (a full window),
// every loop unrolled and the first-half sums kept in registers.
template <int NK, int PS>
__device__ __forceinline__ void temporal_column(const float* __restrict__ refp, int64_t rs,
                                                const float* __restrict__ colp, int64_t ps, int nk, int x, int ya,
                                                int i, const int (*cen)[2], int ps_range, int maxx, int maxy,
                                                uint32_t tbits, LaneTop<PS>& top, float* h0s) {
    constexpr int B = 8;
    constexpr int NKS = NK > 0 ? NK : 32;
    float h0r[NK > 0 ? NK : 1];
    const float2 neg1 = make_float2(-1.f, -1.f);
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        float2 rf[B][2];
#pragma unroll
        for (int ii = 0; ii < B; ++ii) {
            rf[ii][0] = make_float2(__ldg(refp + ii * rs + 4 * half), __ldg(refp + ii * rs + 4 * half + 1));
            rf[ii][1] = make_float2(__ldg(refp + ii * rs + 4 * half + 2), __ldg(refp + ii * rs + 4 * half + 3));
        }
        float2 acc[8][2];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q][0] = acc[q][1] = make_float2(0.f, 0.f);
        auto emit = [&](int kd, float hs) {
            if (half == 0) {
                if constexpr (NK > 0) {
#pragma unroll
                    for (int q = 0; q < NKS; ++q)
                        if (q == kd) h0r[q] = hs;
                } else {
                    h0s[kd] = hs;
                }
                return;
            }
            float first_half;
            if constexpr (NK > 0) {
                first_half = 0.f;
#pragma unroll
                for (int q = 0; q < NKS; ++q)
                    if (q == kd) first_half = h0r[q];
            } else {
                first_half = h0s[kd];
            }
            const int y = ya + kd;
            bool dup = false;
            for (int j = 0; j < i; ++j) {
                const int jx = cen[j][0], jy = cen[j][1];
                dup |= x >= max(0, jx - ps_range) && x <= min(maxx, jx + ps_range) && y >= max(0, jy - ps_range) &&
                       y <= min(maxy, jy + ps_range);
            }
            if (!dup) top.add(tk64(canon(__fadd_rn(first_half, hs)), tbits | (uint32_t(y) << 13) | uint32_t(x)));
        };
        auto row = [&](int s, int slot_base) {
            // image row ya + s: its 4 columns of this half, applied to the candidates k = s - ii
            const float* rowp = colp + (int64_t)s * ps + 4 * half;
            const float2 p01 = make_float2(__ldg(rowp), __ldg(rowp + 1));
            const float2 p23 = make_float2(__ldg(rowp + 2), __ldg(rowp + 3));
#pragma unroll
            for (int ii = 0; ii < B; ++ii) {
                const int k = s - ii;
                if (k >= 0 && k < (NK > 0 ? NK : nk)) {
                    const int sl = (slot_base - ii) & 7;
                    const float2 d01 = __ffma2_rn(p01, neg1, rf[ii][0]);
                    const float2 d23 = __ffma2_rn(p23, neg1, rf[ii][1]);
                    acc[sl][0] = __ffma2_rn(d01, d01, acc[sl][0]);
                    acc[sl][1] = __ffma2_rn(d23, d23, acc[sl][1]);
                }
            }
            const int kd = s - (B - 1);
            if (kd >= 0 && kd < (NK > 0 ? NK : nk)) {
                const int sl = (slot_base + 1) & 7;
                const float2 a = acc[sl][0], b = acc[sl][1];
                acc[sl][0] = acc[sl][1] = make_float2(0.f, 0.f);
                emit(kd, __fadd_rn(__fadd_rn(a.x, a.y), __fadd_rn(b.x, b.y)));
            }
        };
        if constexpr (NK > 0) {
#pragma unroll
            for (int s = 0; s < NK + B - 1; ++s) row(s, s);
        } else {
            for (int s0 = 0; s0 < nk + B - 1; s0 += 8) {
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (s0 + u < nk + B - 1) row(s0 + u, u);
            }
        }
    }
}

// A warp per reference: the chain towards earlier slots, then the one
// towards later slots, then the merge -- no block-level synchronisation.
template <int PS, int PR>
__global__ void __launch_bounds__(32 * kTRefs, 4)
    temporal8_kernel(TemporalPlanes tp, int ntemp, int t0, int first, int last, int W, int H, int G, int ps_num,
                     int ps_range, int jobs, int32_t* __restrict__ pos, int32_t* __restrict__ slot,
                     float* __restrict__ dist, int32_t* __restrict__ count) {
    constexpr int B = 8;
    __shared__ int cen[kTRefs][8][2];               // the layer's window centres (x, y)
    __shared__ uint64_t tops[kTRefs][2 * 16 * 8];   // every layer's bests, both directions
    __shared__ float h0s[32 * kTRefs][27];          // first-half sums (windows clamped by the image)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int job = blockIdx.x * kTRefs + w;
    if (job >= jobs) return;  // a whole warp
    const int n = count[job];
    int32_t* op = pos + (int64_t)job * G;
    int32_t* os = slot + (int64_t)job * G;
    for (int q = lane; q < G; q += 32) os[q] = q < n ? t0 : -1;
    if (n <= 0 || ntemp == 1 || G == 1 || first >= last) return;
    const int cx = pos_x(op[0]), cy = pos_y(op[0]);
    const float* refp = tp.plane[t0] + (int64_t)cy * tp.stride[t0] + cx;
    const int64_t rs = tp.stride[t0];
    const int nseed = min(n, ps_num);
    const int maxx = W - B, maxy = H - B, span = 2 * ps_range + 1;
    int ntop = 0;
    for (int dir = 0; dir < 2; ++dir) {
        __syncwarp();
        if (lane < nseed) {
            cen[w][lane][0] = pos_x(op[lane]);
            cen[w][lane][1] = pos_y(op[lane]);
        }
        __syncwarp();
        int nc = nseed;
        const int sign = dir == 0 ? -1 : 1;
        for (int dt = 1; dt <= (ntemp - 1) / 2; ++dt) {
            const int t = t0 + sign * dt;
            if (t < first || t >= last || nc == 0) break;
            const float* pl = tp.plane[t];
            const int64_t ps = tp.stride[t];
            LaneTop<PS> top;
            top.init();
            for (int task = lane; task < nc * span; task += 32) {
                const int i = task / span, col = task - i * span;
                const int wcx = cen[w][i][0], wcy = cen[w][i][1];
                const int x = max(0, wcx - ps_range) + col;
                if (x > min(maxx, wcx + ps_range)) continue;
                const int ya = max(0, wcy - ps_range), yb = min(maxy, wcy + ps_range);
                const int nk = yb - ya + 1;
                const float* colp = pl + (int64_t)ya * ps + x;
                const uint32_t tbits = uint32_t(t) << 26;
                if (PR > 0 && nk == 2 * PR + 1)
                    temporal_column<2 * PR + 1, PS>(refp, rs, colp, ps, nk, x, ya, i, cen[w], ps_range, maxx, maxy,
                                                    tbits, top, h0s[threadIdx.x]);
                else
                    temporal_column<0, PS>(refp, rs, colp, ps, nk, x, ya, i, cen[w], ps_range, maxx, maxy, tbits,
                                           top, h0s[threadIdx.x]);
            }
            // the layer's ps_num best over the warp
            int got = 0;
            for (int q = 0; q < ps_num; ++q) {
                const uint64_t m = warp_min64(top.k[0]);
                if (m == ~0ull) break;
                if (top.k[0] == m) top.pop();
                if (lane == 0) tops[w][ntop + q] = m;
                ++got;
            }
            __syncwarp();
            if (lane < got) {
                const uint64_t m = tops[w][ntop + lane];
                cen[w][lane][0] = int(m & 0x1fff);
                cen[w][lane][1] = int((m >> 13) & 0x1fff);
            }
            ntop += got;
            nc = got;
            __syncwarp();
        }
    }
    if (lane != 0) return;
    // the global group: the spatial matches (self excluded) and both chains' layer bests
    float* od = dist + (int64_t)job * G;
    uint64_t best[64] = {};
    int nb = 0;
    auto push = [&](uint64_t v) {
        if (nb > 0 && nb == G - 1 && !(v < best[nb - 1])) return;
        int p = nb < G - 1 ? nb++ : nb - 1;
        while (p > 0 && v < best[p - 1]) {
            best[p] = best[p - 1];
            --p;
        }
        best[p] = v;
    };
    for (int i = 1; i < n; ++i)
        push(tk64(canon(od[i]), (uint32_t(t0) << 26) | (uint32_t(pos_y(op[i])) << 13) | uint32_t(pos_x(op[i]))));
    for (int i = 0; i < ntop; ++i) push(tops[w][i]);
    for (int q = 0; q < G - 1; ++q) {
        const bool valid = q < nb;
        const uint64_t k = valid ? best[q] : 0;
        const uint32_t tyx = uint32_t(k);
        op[1 + q] = valid ? pack_pos(tyx & 0x1fff, (tyx >> 13) & 0x1fff) : -1;
        os[1 + q] = valid ? int32_t(tyx >> 26) : -1;
        od[1 + q] = valid ? __uint_as_float(uint32_t(k >> 32)) : 0.f;
    }
    os[0] = t0;
    count[job] = 1 + nb;
}

// ---- streaming form: 8x8 blocks, ps_range PR, ps_num PS (1 or 2) ----
//
// The spatial matcher's schedule applied to the temporal layers: two lanes
// per reference (block columns 0-3 and 4-7, each half of the reference in
// registers for the whole search), 16 references per warp, so every lane
// works on its own reference's windows. A lane walks each window of the layer
// column by column; the column's image rows stream through and each row is
// applied to the candidates overlapping it (slot k & 7); a finished
// candidate's halves meet through one shuffle. Every loop has a trip count
// shared by the warp (windows clipped by the image predicate their missing
// rows and columns off), so the shuffles stay converged. Both lanes of a
// reference keep identical lists: the layer's PS best, and the group itself
// (spatial matches, then every layer's best, inserted as they are found --
// the same set, hence the same top, as the reference's merge).
constexpr int kSRefs = 32;  // references per CTA (2 warps)

template <int K, int PS, int PR>
__global__ void __launch_bounds__(2 * kSRefs, 8) temporal8s_kernel(const __grid_constant__ TemporalBatch tb) {
    constexpr int B = 8, G = K + 1, SPAN = 2 * PR + 1, ROWS = SPAN + B - 1;
    int pl = 0;
    while (pl + 1 < tb.n && tb.p[pl + 1].cta0 <= (int)blockIdx.x) ++pl;
    const TemporalBatchPlane& P = tb.p[pl];
    const TemporalPlanes& tp = P.tp;
    const int ntemp = tb.ntemp, t0 = tb.t0, first = tb.first, last = tb.last, ps_num = tb.ps_num;
    const int W = P.W, H = P.H, jobs = P.jobs;
    int32_t* __restrict__ pos = P.pos;
    int32_t* __restrict__ slot = P.slot;
    float* __restrict__ dist = P.dist;
    int32_t* __restrict__ count = P.count;
    const int lane = threadIdx.x & 31, half = lane >> 4;
    const int job = (blockIdx.x - P.cta0) * kSRefs + (threadIdx.x >> 5) * 16 + (lane & 15);
    const bool live = job < jobs;
    const int n = live ? count[job] : 0;
    int32_t* op = pos + (int64_t)(live ? job : 0) * G;
    int32_t* os = slot + (int64_t)(live ? job : 0) * G;
    float* od = dist + (int64_t)(live ? job : 0) * G;
    if (live && half == 0)
        for (int q = 0; q < G; ++q) os[q] = q < n ? t0 : -1;
    const bool search = live && n > 0 && ntemp > 1 && first < last;
    // a warp with no searching reference leaves (uniform: no shuffle is pending)
    if (!__any_sync(0xffffffffu, search)) return;
    const int cx = search ? pos_x(op[0]) : 0, cy = search ? pos_y(op[0]) : 0;
    const int64_t rs = tp.stride[t0];
    float2 rf[B][2];
    {
        const float* refp = tp.plane[t0] + (int64_t)cy * rs + cx + 4 * half;
#pragma unroll
        for (int i = 0; i < B; ++i) {
            rf[i][0] = make_float2(__ldg(refp + i * rs), __ldg(refp + i * rs + 1));
            rf[i][1] = make_float2(__ldg(refp + i * rs + 2), __ldg(refp + i * rs + 3));
        }
    }
    // the group so far: the spatial matches without the reference itself
    LaneTop<K> group;
    group.init();
    for (int i = 1; i < (search ? n : 0); ++i)
        group.add(tk64(canon(od[i]), (uint32_t(t0) << 26) | (uint32_t(pos_y(op[i])) << 13) | uint32_t(pos_x(op[i]))));
    // window centres per direction: the first ps_num of the spatial group
    int cxs[2][PS], cys[2][PS], nc[2];
    const int nseed = search ? min(n, ps_num) : 0;
#pragma unroll
    for (int q = 0; q < PS; ++q) {
        const int32_t p = q < nseed ? op[q] : 0;
        cxs[0][q] = cxs[1][q] = pos_x(p);
        cys[0][q] = cys[1][q] = pos_y(p);
    }
    nc[0] = nc[1] = nseed;
    const int maxx = W - B, maxy = H - B;
    const float2 neg1 = make_float2(-1.f, -1.f);
    for (int dt = 1; dt <= (ntemp - 1) / 2; ++dt) {
#pragma unroll
        for (int dir = 0; dir < 2; ++dir) {
            const int t = t0 + (dir == 0 ? -dt : dt);
            if (t < first || t >= last) continue;  // the same for the whole warp
            const float* pl = tp.plane[t];
            const int64_t ps = tp.stride[t];
            LaneTop<PS> layer;
            layer.init();
#pragma unroll
            for (int i = 0; i < PS; ++i) {
                const bool win = i < nc[dir];
                const int xa = max(0, cxs[dir][i] - PR), xb = min(maxx, cxs[dir][i] + PR);
                const int ya = max(0, cys[dir][i] - PR), yb = min(maxy, cys[dir][i] + PR);
                const int nk = win ? yb - ya + 1 : 0;
                for (int col = 0; col < SPAN; ++col) {
                    const int x = xa + col;
                    const bool colok = win && x <= xb;
                    const float* colp = pl + (int64_t)(colok ? ya : 0) * ps + (colok ? x : 0) + 4 * half;
                    float2 acc[8][2];
#pragma unroll
                    for (int q = 0; q < 8; ++q) acc[q][0] = acc[q][1] = make_float2(0.f, 0.f);
                    // rows are read LA rows ahead of their use
                    constexpr int LA = 2;
                    float2 q01[LA], q23[LA];
#pragma unroll
                    for (int a = 0; a < LA; ++a) {
                        q01[a] = q23[a] = make_float2(0.f, 0.f);
                        if (colok && a < nk + B - 1) {
                            const float* rowp = colp + (int64_t)a * ps;
                            q01[a] = make_float2(__ldg(rowp), __ldg(rowp + 1));
                            q23[a] = make_float2(__ldg(rowp + 2), __ldg(rowp + 3));
                        }
                    }
#pragma unroll
                    for (int srow = 0; srow < ROWS; ++srow) {
                        const float2 p01 = q01[srow % LA], p23 = q23[srow % LA];
                        if (srow + LA < ROWS) {
                            q01[srow % LA] = q23[srow % LA] = make_float2(0.f, 0.f);
                            if (colok && srow + LA < nk + B - 1) {
                                const float* rowp = colp + (int64_t)(srow + LA) * ps;
                                q01[srow % LA] = make_float2(__ldg(rowp), __ldg(rowp + 1));
                                q23[srow % LA] = make_float2(__ldg(rowp + 2), __ldg(rowp + 3));
                            }
                        }
#pragma unroll
                        for (int ii = 0; ii < B; ++ii) {
                            const int k = srow - ii;
                            if (k >= 0 && k < SPAN) {
                                const float2 d01 = __ffma2_rn(p01, neg1, rf[ii][0]);
                                const float2 d23 = __ffma2_rn(p23, neg1, rf[ii][1]);
                                acc[k & 7][0] = __ffma2_rn(d01, d01, acc[k & 7][0]);
                                acc[k & 7][1] = __ffma2_rn(d23, d23, acc[k & 7][1]);
                            }
                        }
                        const int kd = srow - (B - 1);
                        if (kd >= 0 && kd < SPAN) {
                            const float2 a = acc[kd & 7][0], b = acc[kd & 7][1];
                            acc[kd & 7][0] = acc[kd & 7][1] = make_float2(0.f, 0.f);
                            const float hs = __fadd_rn(__fadd_rn(a.x, a.y), __fadd_rn(b.x, b.y));
                            const float dd = __fadd_rn(hs, __shfl_xor_sync(0xffffffffu, hs, 16));
                            if (colok && kd < nk) {
                                const int y = ya + kd;
                                bool dup = false;
#pragma unroll
                                for (int j = 0; j < PS; ++j)
                                    if (j < i)
                                        dup |= x >= max(0, cxs[dir][j] - PR) && x <= min(maxx, cxs[dir][j] + PR) &&
                                               y >= max(0, cys[dir][j] - PR) && y <= min(maxy, cys[dir][j] + PR);
                                if (!dup)
                                    layer.add(tk64(canon(dd), (uint32_t(t) << 26) | (uint32_t(y) << 13) | uint32_t(x)));
                            }
                        }
                    }
                }
            }
            // the layer's best: into the group, and the next layer's centres
            int got = 0;
#pragma unroll
            for (int q = 0; q < PS; ++q) {
                const uint64_t k = layer.k[q];
                if (q < ps_num && k != ~0ull) {
                    group.add(k);
                    cxs[dir][q] = int(k & 0x1fff);
                    cys[dir][q] = int((k >> 13) & 0x1fff);
                    ++got;
                }
            }
            nc[dir] = got;
        }
    }
    if (!search || half != 0) return;
    int nb = 0;
#pragma unroll
    for (int q = 0; q < K; ++q) {
        const bool valid = group.k[q] != ~0ull;
        nb += valid;
        const uint32_t tyx = uint32_t(group.k[q]);
        op[1 + q] = valid ? pack_pos(tyx & 0x1fff, (tyx >> 13) & 0x1fff) : -1;
        os[1 + q] = valid ? int32_t(tyx >> 26) : -1;
        od[1 + q] = valid ? __uint_as_float(uint32_t(group.k[q] >> 32)) : 0.f;
    }
    os[0] = t0;
    count[job] = 1 + nb;
}

}  // namespace

bool launch_match_temporal_batch(TemporalBatch& tb, cudaStream_t stream) {
    const int g = tb.group;
    if (tb.n < 1 || tb.n > 3 || tb.ps_range != 4 || tb.ps_num < 1 || tb.ps_num > 2 || tb.ntemp > 33 ||
        !(g == 2 || g == 4 || g == 8 || g == 16))
        return false;
    int ctas = 0;
    for (int i = 0; i < tb.n; ++i) {
        TemporalBatchPlane& p = tb.p[i];
        if (p.W >= 8192 || p.H >= 8192 || p.W < 8 || p.H < 8) return false;
        p.cta0 = ctas;
        ctas += ceil_div(p.jobs, kSRefs);
    }
    tb.total_ctas = ctas;
    if (ctas == 0) return true;
    const int first = tb.first < 0 ? 0 : tb.first;
    const int last = tb.last < 0 ? tb.ntemp : (tb.last < tb.ntemp ? tb.last : tb.ntemp);
    tb.first = first;
    tb.last = last;
    auto gos = [&](auto kern) { kern<<<ctas, 2 * kSRefs, 0, stream>>>(tb); };
    switch (g * 4 + tb.ps_num) {
        case 9: gos(temporal8s_kernel<1, 1, 4>); break;
        case 10: gos(temporal8s_kernel<1, 2, 4>); break;
        case 17: gos(temporal8s_kernel<3, 1, 4>); break;
        case 18: gos(temporal8s_kernel<3, 2, 4>); break;
        case 33: gos(temporal8s_kernel<7, 1, 4>); break;
        case 34: gos(temporal8s_kernel<7, 2, 4>); break;
        case 65: gos(temporal8s_kernel<15, 1, 4>); break;
        default: gos(temporal8s_kernel<15, 2, 4>); break;
    }
    NSSB_CUDA(cudaGetLastError());
    return true;
}

void launch_match_temporal(const TemporalPlanes& planes, int ntemp, int t0, int valid_begin, int valid_end,
                           int width, int height, int block, int step, int group, int ps_num, int ps_range,
                           int32_t* pos, int32_t* slot, float* dist, int32_t* count, cudaStream_t stream) {
    const int nx = grid_count(width, block, step), ny = grid_count(height, block, step);
    const int jobs = nx * ny;
    if (jobs == 0) return;
    const int first = valid_begin < 0 ? 0 : valid_begin;
    const int last = valid_end < 0 ? ntemp : (valid_end < ntemp ? valid_end : ntemp);
    const int layers = (ntemp - 1) / 2;
    // the fast path packs slot, y and x into 6 + 13 + 13 bits; larger planes take the generic kernel
    if (block == 8 && ps_num <= 8 && ps_range <= 12 && group <= 64 && 2 * layers * ps_num <= 2 * 16 * 8 &&
        ntemp <= 33 && width < 8192 && height < 8192) {
        const dim3 g8(ceil_div(jobs, kTRefs));
        auto go = [&](auto kern) {
            kern<<<g8, 32 * kTRefs, 0, stream>>>(planes, ntemp, t0, first, last, width, height, group, ps_num,
                                                 ps_range, jobs, pos, slot, dist, count);
        };
        const bool r4 = ps_range == 4;
        if (r4 && ps_num <= 2 && (group == 2 || group == 4 || group == 8 || group == 16)) {
            static thread_local TemporalBatch tb;
            tb.n = 1;
            tb.ntemp = ntemp;
            tb.t0 = t0;
            tb.first = first;
            tb.last = last;
            tb.group = group;
            tb.ps_num = ps_num;
            tb.ps_range = ps_range;
            tb.p[0] = TemporalBatchPlane{planes, width, height, jobs, 0, pos, slot, dist, count};
            if (launch_match_temporal_batch(tb, stream)) return;
        }
        if (ps_num <= 2) r4 ? go(temporal8_kernel<2, 4>) : go(temporal8_kernel<2, 0>);
        else if (ps_num <= 4) r4 ? go(temporal8_kernel<4, 4>) : go(temporal8_kernel<4, 0>);
        else r4 ? go(temporal8_kernel<8, 4>) : go(temporal8_kernel<8, 0>);
        NSSB_CUDA(cudaGetLastError());
        return;
    }
    const dim3 grid(ceil_div(jobs, 64));
    switch (block) {
        case 4:
            temporal_kernel<4><<<grid, 64, 0, stream>>>(planes, ntemp, t0, first, last, width, height, block, step,
                                                        group, ps_num, ps_range, nx, ny, pos, slot, dist, count);
            break;
        case 8:
            temporal_kernel<8><<<grid, 64, 0, stream>>>(planes, ntemp, t0, first, last, width, height, block, step,
                                                        group, ps_num, ps_range, nx, ny, pos, slot, dist, count);
            break;
        default:
            temporal_kernel<0><<<grid, 64, 0, stream>>>(planes, ntemp, t0, first, last, width, height, block, step,
                                                        group, ps_num, ps_range, nx, ny, pos, slot, dist, count);
            break;
    }
    NSSB_CUDA(cudaGetLastError());
}

}  // namespace nssb
