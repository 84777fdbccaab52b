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
    uint32_t tyx;  // slot << 26 | y << 13 | x  (x, y < 8192)
};

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
        seeds[i].tyx = (uint32_t(t0) << 26) | (uint32_t(pos_y(op[i])) << 13) | uint32_t(pos_x(op[i]));
    }
    TList global;
    global.init(G - 1);
    for (int i = 1; i < n; ++i) {
        TKey k;
        k.d = canon(od[i]);
        k.tyx = (uint32_t(t0) << 26) | (uint32_t(pos_y(op[i])) << 13) | uint32_t(pos_x(op[i]));
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
                const int cyy = (centers[i].tyx >> 13) & 0x1fff;
                ymin = min(ymin, max(0, cyy - ps_range));
                ymax = max(ymax, min(maxy, cyy + ps_range));
            }
            const float* pl = tp.plane[t];
            const int64_t ps = tp.stride[t];
            for (int y = ymin; y <= ymax; ++y) {
                // the x intervals of the windows that cover row y, in ascending order
                int ia[64], ib[64], ni = 0;
                for (int i = 0; i < nc; ++i) {
                    const int cyy = (centers[i].tyx >> 13) & 0x1fff, cxx = centers[i].tyx & 0x1fff;
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
                        k.tyx = (uint32_t(t) << 26) | (uint32_t(y) << 13) | uint32_t(x);
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
        op[1 + q] = valid ? pack_pos(k.tyx & 0x1fff, (k.tyx >> 13) & 0x1fff) : -1;
        os[1 + q] = valid ? int32_t(k.tyx >> 26) : -1;
        od[1 + q] = valid ? __uint_as_float(k.d) : 0.f;
    }
    os[0] = t0;
    count[job] = 1 + global.n;
}

}  // namespace

void launch_match_temporal(const TemporalPlanes& planes, int ntemp, int t0, int valid_begin, int valid_end,
                           int width, int height, int block, int step, int group, int ps_num, int ps_range,
                           int32_t* pos, int32_t* slot, float* dist, int32_t* count, cudaStream_t stream) {
    if (width >= 8192 || height >= 8192) throw std::invalid_argument("nss_cuda: temporal planes must be < 8192 wide");
    const int nx = grid_count(width, block, step), ny = grid_count(height, block, step);
    const int jobs = nx * ny;
    if (jobs == 0) return;
    const int first = valid_begin < 0 ? 0 : valid_begin;
    const int last = valid_end < 0 ? ntemp : (valid_end < ntemp ? valid_end : ntemp);
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
