/*
 * CPU oracle for the BM3D hot path -- TEST INFRASTRUCTURE ONLY (see
 * bm3d_oracle.h for what it restates and who may load it).
 *
 * Built with -ffp-contract=off: every fused multiply-add here is an explicit
 * fmaf(), every other operation rounds on its own, so results do not depend
 * on the compiler's contraction or vectorisation choices.
 */
#include "bm3d_oracle.h"

#include <math.h>
#if defined(__AVX2__) && defined(__FMA__)
#include <immintrin.h>
#endif
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }
static int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static int finite_bits(float v) {
    uint32_t u;
    memcpy(&u, &v, sizeof u);
    return (u & 0x7f800000u) != 0x7f800000u;
}

float om_noise_effective(float user_sigma) {
    /* contracts.hpp:27-29: (sigma * (1/255)) * 0.75, in float */
    return (user_sigma * (1.f / 255.f)) * 0.75f;
}

/* ---------------------------------------------------------------- distances */

/* Pairwise sum of n per-column partials: the halves' sums, added. */
static float column_tree(const float* c, int n) {
    if (n == 1) return c[0];
    const int h = n / 2;
    return column_tree(c, h) + column_tree(c + h, n - h);
}

/* The SSD order of this build: every block column j takes one FMA chain down
 * the rows (c_j = fma(d, d, c_j), d = a - b, rows in order), then the
 * columns are summed pairwise (column_tree: halves first, recursively). */
float om_ssd(const float* a, ptrdiff_t sa, const float* b, ptrdiff_t sb, int block) {
    float c[32];
    for (int j = 0; j < block; ++j) c[j] = 0.f;
    for (int i = 0; i < block; ++i) {
        for (int j = 0; j < block; ++j) {
            const float d = a[i * sa + j] - b[i * sb + j];
            c[j] = fmaf(d, d, c[j]);
        }
    }
    return column_tree(c, block);
}

/* The 8-lane tree of SpatialMatch8 (ssd.cpp:207-237): lane j accumulates rows
 * {k, k+4} in four accumulators, (a0 + a2) + (a1 + a3), then HSum8
 * (ssd_leaf-inl.hpp:8-11): low half + high half, then the 4-lane reduction,
 * taken here as (w0 + w2) + (w1 + w3). */
float om_ssd_lanes8(const float* a, ptrdiff_t sa, const float* b, ptrdiff_t sb) {
    float v[8];
    for (int j = 0; j < 8; ++j) {
        float acc[4];
        for (int k = 0; k < 4; ++k) {
            const float d0 = a[k * sa + j] - b[k * sb + j];
            const float d1 = a[(k + 4) * sa + j] - b[(k + 4) * sb + j];
            acc[k] = fmaf(d1, d1, fmaf(d0, d0, 0.f));
        }
        v[j] = (acc[0] + acc[2]) + (acc[1] + acc[3]);
    }
    float w[4];
    for (int k = 0; k < 4; ++k) w[k] = v[k] + v[k + 4];
    return (w[0] + w[2]) + (w[1] + w[3]);
}

/* ------------------------------------------------------------- match order */

/* match_tie_less / match_less (matcher.hpp:27-57) */
static int tie_less(const om_match* a, const om_match* b) {
    const int as = a->ordinal == 0, bs = b->ordinal == 0;
    if (as != bs) return as;
    if (a->t != b->t) return a->t < b->t;
    if (a->y != b->y) return a->y < b->y;
    if (a->x != b->x) return a->x < b->x;
    return a->ordinal < b->ordinal;
}

static inline int match_less(const om_match* a, const om_match* b) {
    const int af = finite_bits(a->dist), bf = finite_bits(b->dist);
    if (af != bf) return af;
    if (af && a->dist != b->dist) return a->dist < b->dist;
    return tie_less(a, b);
}

int om_match_less(const om_match* a, const om_match* b) { return match_less(a, b); }

/* A top-k set under match_less, kept sorted: the same final set and order as
 * StableTopK (matcher.hpp:59-109) because match_less is a total order on
 * distinct (t, y, x, ordinal). */
typedef struct topk {
    om_match* s;
    int cap, size;
} topk;

static void topk_add(topk* k, om_match m) {
    if (k->cap <= 0) return;
    if (k->size == k->cap) {
        if (!match_less(&m, &k->s[k->size - 1])) return;
        --k->size;
    }
    int pos = k->size;
    while (pos > 0 && match_less(&m, &k->s[pos - 1])) {
        k->s[pos] = k->s[pos - 1];
        --pos;
    }
    k->s[pos] = m;
    ++k->size;
}

/* adopt(n) of StableTopK followed by later adds: sort what is adopted. */
static void topk_adopt(topk* k, int n) {
    k->size = n < 0 ? 0 : (n > k->cap ? k->cap : n);
    for (int i = 1; i < k->size; ++i) {
        om_match m = k->s[i];
        int pos = i;
        while (pos > 0 && match_less(&m, &k->s[pos - 1])) {
            k->s[pos] = k->s[pos - 1];
            --pos;
        }
        k->s[pos] = m;
    }
}

/* ---------------------------------------------------------------- matching */

int om_grid_count(int extent, int block, int step) {
    if (extent < block || step < 1) return 0;
    return (extent - block + step - 1) / step + 1;
}

int om_grid_pos(int i, int extent, int block, int step) { return imin(i * step, extent - block); }

/* SSDs of n consecutive candidates of one row of a zero-padded window copy
 * (buf holds the window rows, each readable for n + 24 + block columns), 24
 * candidates per pass: each keeps its own row-major FMA chain, the lanes are
 * independent, so the compiler's vector form gives om_ssd's bits. */
#if defined(__AVX2__) && defined(__FMA__)
static __m256 column_tree8(const __m256* c, int n) {
    if (n == 1) return c[0];
    const int h = n / 2;
    return _mm256_add_ps(column_tree8(c, h), column_tree8(c + h, n - h));
}
#endif

#if defined(__AVX2__) && defined(__FMA__)
/* block 8: the same per-column chains and tree with the accumulators in registers */
static void ssd_span8(const float* refblk, const float* buf, ptrdiff_t bstride, int n, int nrows, float* out,
                      int ostride) {
    for (int q = 0; q < nrows; ++q) {
        for (int c0 = 0; c0 < n; c0 += 8) {
            __m256 a0 = _mm256_setzero_ps(), a1 = a0, a2 = a0, a3 = a0, a4 = a0, a5 = a0, a6 = a0, a7 = a0;
            for (int i = 0; i < 8; ++i) {
                const float* row = buf + (ptrdiff_t)(i + q) * bstride + c0;
                const float* r = refblk + i * 8;
#define NSSB_COL(k, acc)                                                                            \
    {                                                                                               \
        const __m256 d = _mm256_sub_ps(_mm256_set1_ps(r[k]), _mm256_loadu_ps(row + k));            \
        acc = _mm256_fmadd_ps(d, d, acc);                                                           \
    }
                NSSB_COL(0, a0) NSSB_COL(1, a1) NSSB_COL(2, a2) NSSB_COL(3, a3)
                NSSB_COL(4, a4) NSSB_COL(5, a5) NSSB_COL(6, a6) NSSB_COL(7, a7)
#undef NSSB_COL
            }
            const __m256 t = _mm256_add_ps(_mm256_add_ps(_mm256_add_ps(a0, a1), _mm256_add_ps(a2, a3)),
                                           _mm256_add_ps(_mm256_add_ps(a4, a5), _mm256_add_ps(a6, a7)));
            float tree[8];
            _mm256_storeu_ps(tree, t);
            const int mm = n - c0 < 8 ? n - c0 : 8;
            for (int l = 0; l < mm; ++l) out[q * ostride + c0 + l] = tree[l];
        }
    }
}
#endif

static void ssd_span(const float* refblk, int block, const float* buf, ptrdiff_t bstride, int n, int nrows,
                     float* out, int ostride) {
    /* nrows (<= 2) candidate rows x n candidates (8 per vector lane group);
     * candidate row q starts at buffer row q. Per-column chains and the
     * column tree as in om_ssd. */
#if defined(__AVX2__) && defined(__FMA__)
    if (block == 8) {
        ssd_span8(refblk, buf, bstride, n, nrows, out, ostride);
        return;
    }
#endif
    for (int q = 0; q < nrows; ++q) {
        for (int c0 = 0; c0 < n; c0 += 8) {
            float col[32][8];
#if defined(__AVX2__) && defined(__FMA__)
            /* vfmadd is the exactly rounded fma: the same bits as fmaf */
            __m256 acc[32];
            for (int j = 0; j < block; ++j) acc[j] = _mm256_setzero_ps();
            for (int i = 0; i < block; ++i) {
                const float* row = buf + (ptrdiff_t)(i + q) * bstride + c0;
                for (int j = 0; j < block; ++j) {
                    const __m256 d = _mm256_sub_ps(_mm256_set1_ps(refblk[i * block + j]), _mm256_loadu_ps(row + j));
                    acc[j] = _mm256_fmadd_ps(d, d, acc[j]);
                }
            }
            float tree[8];
            _mm256_storeu_ps(tree, column_tree8(acc, block));
            const int mm = n - c0 < 8 ? n - c0 : 8;
            for (int l = 0; l < mm; ++l) out[q * ostride + c0 + l] = tree[l];
            continue;
            (void)col;
#else
            for (int j = 0; j < block; ++j)
                for (int l = 0; l < 8; ++l) col[j][l] = 0.f;
            for (int i = 0; i < block; ++i) {
                const float* row = buf + (ptrdiff_t)(i + q) * bstride + c0;
                for (int j = 0; j < block; ++j) {
                    const float r = refblk[i * block + j];
                    for (int l = 0; l < 8; ++l) {
                        const float d = r - row[j + l];
                        col[j][l] = fmaf(d, d, col[j][l]);
                    }
                }
            }
#endif
            const int m = n - c0 < 8 ? n - c0 : 8;
            for (int l = 0; l < m; ++l) {
                float c[32];
                for (int j = 0; j < block; ++j) c[j] = col[j][l];
                out[q * ostride + c0 + l] = column_tree(c, block);
            }
        }
    }
}

int om_spatial_match(const float* plane, ptrdiff_t stride, int width, int height, int bx, int by, int block,
                     int bm_range, int group, om_match* out, int lanes8) {
    if (!plane || !out || width < 1 || height < 1 || block < 1 || width < block || height < block || group < 1)
        return 0;
    const int wanted = imin(group, OM_MAX_GROUP);
    const int max_x = width - block, max_y = height - block;
    const int cx = iclamp(bx, 0, max_x), cy = iclamp(by, 0, max_y);
    const int range = imax(bm_range, 0);
    const int top = imax(cy - range, 0), bottom = imin(cy + range, max_y);
    const int left = imax(cx - range, 0), right = imin(cx + range, max_x);
    out[0] = (om_match){cx, cy, 0, 0.f, 0};
    if (wanted == 1) return 1;
    topk k = {out + 1, wanted - 1, 0};
    float refblk[32 * 32];
    for (int i = 0; i < block; ++i)
        memcpy(refblk + i * block, plane + (ptrdiff_t)(cy + i) * stride + cx, (size_t)block * sizeof(float));
    const int span = right - left + 1;
    const int rows = bottom - top + block;
    /* the window rows, zero-padded right and below so every 4-row, 24-wide pass reads in bounds */
    const ptrdiff_t bstride = span + block + 24 + 8;
    static __thread float tbuf[(2 * 64 + 32 + 4) * (2 * 64 + 1 + 32 + 24 + 8)];
    float* buf = tbuf;
    for (int r = 0; r < rows + 4; ++r) {
        float* dst = buf + (ptrdiff_t)r * bstride;
        const int valid = r < rows ? span + block - 1 : 0;
        if (valid) memcpy(dst, plane + (ptrdiff_t)(top + r) * stride + left, (size_t)valid * sizeof(float));
        memset(dst + valid, 0, (size_t)(bstride - valid) * sizeof(float));
    }
    float dist[2][2 * 64 + 1 + 24];
    for (int y = top; y <= bottom; ++y) {
        const int q = (y - top) & 1;
        if (q == 0 && !(lanes8 && block == 8))
            ssd_span(refblk, block, buf + (ptrdiff_t)(y - top) * bstride, bstride, span, imin(2, bottom - y + 1),
                     dist[0], 2 * 64 + 1 + 24);
        if (lanes8 && block == 8) {
            for (int c = 0; c < span; ++c)
                dist[q][c] = om_ssd_lanes8(refblk, 8, plane + (ptrdiff_t)y * stride + left + c, stride);
        }
        for (int x = left; x <= right; ++x) {
            if (x == cx && y == cy) continue;
            const float d = dist[q][x - left];
            /* a finite distance above a full set's worst cannot enter it */
            if (k.size == k.cap && finite_bits(d) && finite_bits(k.s[k.cap - 1].dist) && d > k.s[k.cap - 1].dist)
                continue;
            const uint32_t ordinal = (uint32_t)((y - top) * span + (x - left) + 1);
            topk_add(&k, (om_match){x, y, 0, d, ordinal});
        }
    }
    return 1 + k.size;
}

/* assign_temporal_order (matcher.hpp:296-314) */
static void temporal_order(om_match* m, int count, int t, int t0, uint32_t* next) {
    const uint32_t kFrameStride = 1u << 20;
    for (int i = 0; i < count; ++i) {
        const uint32_t local = m[i].ordinal;
        m[i].t = t;
        if (t == t0 && local == 0) {
            m[i].ordinal = 0;
        } else {
            m[i].ordinal = (uint32_t)(imax(t, 0) + 1) * kFrameStride + local;
        }
        if (m[i].ordinal + 1u > *next) *next = m[i].ordinal + 1u;
    }
}

typedef struct interval {
    int a, b;
} interval;

static int interval_cmp(const void* p, const void* q) {
    const interval* x = (const interval*)p;
    const interval* y = (const interval*)q;
    if (x->a != y->a) return x->a < y->a ? -1 : 1;
    if (x->b != y->b) return x->b < y->b ? -1 : 1;
    return 0;
}

int om_predictive_match(const float* const* planes, const ptrdiff_t* strides, int ntemp, int width, int height,
                        int bx, int by, int t0, const om_search* cfg, om_match* out) {
    /* argument checks of predictive_match (match.cpp:12-24) */
    if (!planes || !strides || !out || ntemp < 1 || t0 < 0 || t0 >= ntemp || width < cfg->block ||
        height < cfg->block || cfg->block < 1 || cfg->group < 1 || cfg->group > OM_MAX_GROUP || cfg->step < 1 ||
        cfg->bm_range < 0 || cfg->ps_num < 1 || cfg->ps_range < 0 || cfg->radius < 0 ||
        cfg->radius > OM_MAX_RADIUS || !planes[t0] || strides[t0] < width)
        return 0;
    if (cfg->valid_t_begin < 0 || cfg->valid_t_begin > t0 ||
        (cfg->valid_t_end != -1 && (cfg->valid_t_end <= t0 || cfg->valid_t_end > ntemp)))
        return 0;
    for (int t = 0; t < ntemp; ++t)
        if (!planes[t] || strides[t] < width) return 0;
    const int block = cfg->block;
    int n = om_spatial_match(planes[t0], strides[t0], width, height, bx, by, block, cfg->bm_range, cfg->group, out,
                             0);
    const int cx = iclamp(bx, 0, width - block), cy = iclamp(by, 0, height - block);
    const float* reference = planes[t0] + (ptrdiff_t)cy * strides[t0] + cx;

    /* collect_temporal (matcher.hpp:319-373) */
    uint32_t ordinal = 0;
    temporal_order(out, n, t0, t0, &ordinal);
    if (n <= 0 || cfg->radius == 0 || ntemp == 1 || cfg->group == 1) return n;
    om_match seeds[OM_MAX_GROUP];
    const int seed_count = imin(imin(n, cfg->ps_num), OM_MAX_GROUP);
    memcpy(seeds, out, (size_t)seed_count * sizeof(om_match));
    topk global = {out + 1, cfg->group - 1, 0};
    topk_adopt(&global, n - 1);
    const int first = imax(0, cfg->valid_t_begin);
    const int last = cfg->valid_t_end < 0 ? ntemp : imin(ntemp, cfg->valid_t_end);
    for (int si = 0; si < 2; ++si) {
        const int sign = si == 0 ? -1 : 1;
        om_match centers[OM_MAX_GROUP];
        memcpy(centers, seeds, (size_t)seed_count * sizeof(om_match));
        int nc = seed_count;
        for (int dt = 1; dt <= cfg->radius; ++dt) {
            const int t = t0 + sign * dt;
            if (t < first || t >= last) break;
            om_match local[OM_MAX_GROUP];
            topk top = {local, imin(cfg->ps_num, cfg->group), 0};
            int ymin = height, ymax = -1;
            for (int i = 0; i < nc; ++i) {
                ymin = imin(ymin, imax(0, centers[i].y - cfg->ps_range));
                ymax = imax(ymax, imin(height - block, centers[i].y + cfg->ps_range));
            }
            uint32_t visit = 1;
            for (int y = ymin; y <= ymax; ++y) {
                interval iv[OM_MAX_GROUP];
                int ni = 0;
                for (int i = 0; i < nc; ++i) {
                    if (abs(y - centers[i].y) <= cfg->ps_range) {
                        iv[ni].a = imax(0, centers[i].x - cfg->ps_range);
                        iv[ni].b = imin(width - block, centers[i].x + cfg->ps_range);
                        ++ni;
                    }
                }
                qsort(iv, (size_t)ni, sizeof(interval), interval_cmp);
                int done = -1;
                for (int i = 0; i < ni; ++i) {
                    for (int x = imax(done + 1, iv[i].a); x <= iv[i].b; ++x) {
                        om_match m = {x, y, t,
                                      om_ssd(reference, strides[t0], planes[t] + (ptrdiff_t)y * strides[t] + x,
                                             strides[t], block),
                                      visit++};
                        temporal_order(&m, 1, t, t0, &ordinal);
                        topk_add(&top, m);
                    }
                    done = imax(done, iv[i].b);
                }
            }
            nc = top.size;
            for (int i = 0; i < nc; ++i) topk_add(&global, local[i]);
            memcpy(centers, local, (size_t)nc * sizeof(om_match));
            if (nc == 0) break;
        }
    }
    return 1 + global.size;
}

/* -------------------------------------------------------------- transforms */

/* DctTable<N> (dct8.cpp:69-89): row k = frequency, column i = sample, the
 * orthonormal DCT-II computed in double and rounded to float. */
static float g_dct[7][64 * 64];
static pthread_once_t g_dct_once = PTHREAD_ONCE_INIT;
static const int g_dct_sizes[7] = {1, 2, 4, 8, 12, 16, 32};

static void dct_init(void) {
    const double pi = 3.14159265358979323846264338327950288;
    for (int s = 0; s < 7; ++s) {
        const int n = g_dct_sizes[s];
        const double s0 = sqrt(1.0 / n), s1 = sqrt(2.0 / n);
        for (int k = 0; k < n; ++k)
            for (int i = 0; i < n; ++i)
                g_dct[s][k * n + i] = (float)((k == 0 ? s0 : s1) * cos(pi * ((double)i + 0.5) * (double)k / n));
    }
}

const float* om_dct_table(int n) {
    pthread_once(&g_dct_once, dct_init);
    for (int s = 0; s < 7; ++s)
        if (g_dct_sizes[s] == n) return g_dct[s];
    return NULL;
}

/* HaarScale (dct8.cpp:580-593) */
float om_haar_scale(int n, int j) {
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

static double haar_scale_f64(int n, int j) {
    int e = 0;
    if (j == 0) {
        while ((1 << e) < n) ++e;
    } else {
        while (((j >> e) & 1) == 0) ++e;
        ++e;
    }
    return pow(2.0, -0.5 * e);
}

/* DctLines: count lines of n samples, sample i of line v at
 * base[v * ls + i * ss]; forward y[k] = sum_i T[k][i] x[i], inverse
 * y[i] = sum_k T[k][i] x[k], each an FMA chain in index order. */
static void dct_lines(float* base, int n, ptrdiff_t ls, ptrdiff_t ss, int count, int inverse) {
    if (n <= 1) return;
    const float* T = om_dct_table(n);
    /* 8 lines per pass, lane = line: every line keeps its own FMA chain in
     * index order, so the vector form gives the scalar bits. */
    for (int v0 = 0; v0 < count; v0 += 8) {
        const int lanes = count - v0 < 8 ? count - v0 : 8;
        float x[32 * 8], y[32 * 8];
        for (int i = 0; i < n; ++i)
            for (int l = 0; l < 8; ++l) x[i * 8 + l] = l < lanes ? base[(v0 + l) * ls + i * ss] : 0.f;
        for (int o = 0; o < n; ++o) {
            float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            for (int q = 0; q < n; ++q) {
                const float t = inverse ? T[q * n + o] : T[o * n + q];
                for (int l = 0; l < 8; ++l) acc[l] = fmaf(t, x[q * 8 + l], acc[l]);
            }
            for (int l = 0; l < 8; ++l) y[o * 8 + l] = acc[l];
        }
        for (int i = 0; i < n; ++i)
            for (int l = 0; l < lanes; ++l) base[(v0 + l) * ls + i * ss] = y[i * 8 + l];
    }
}

static void dct2_cube(float* c, int group, int block, int inverse) {
    const int area = block * block;
    dct_lines(c, block, block, 1, group * block, inverse);
    for (int g = 0; g < group; ++g) dct_lines(c + (ptrdiff_t)g * area, block, 1, block, block, inverse);
}

/* HaarLines (dct8.cpp:601-642): level h pairs samples h apart (sum low,
 * difference high); forward scales last, inverse first. */
static void haar_lines(float* base, int n, ptrdiff_t ls, ptrdiff_t ss, int count, int inverse) {
    if (n <= 1) return;
    /* level by level over all lines at once: the same operations per sample */
    if (inverse) {
        for (int j = 0; j < n; ++j) {
            const float f = om_haar_scale(n, j);
            for (int v = 0; v < count; ++v) base[v * ls + j * ss] = base[v * ls + j * ss] * f;
        }
        for (int h = n / 2; h >= 1; h >>= 1)
            for (int i = 0; i < n; i += 2 * h)
                for (int v = 0; v < count; ++v) {
                    float* p = base + v * ls;
                    const float a = p[i * ss], b = p[(i + h) * ss];
                    p[i * ss] = a + b;
                    p[(i + h) * ss] = a - b;
                }
    } else {
        for (int h = 1; h < n; h <<= 1)
            for (int i = 0; i < n; i += 2 * h)
                for (int v = 0; v < count; ++v) {
                    float* p = base + v * ls;
                    const float a = p[i * ss], b = p[(i + h) * ss];
                    p[i * ss] = a + b;
                    p[(i + h) * ss] = a - b;
                }
        for (int j = 0; j < n; ++j) {
            const float f = om_haar_scale(n, j);
            for (int v = 0; v < count; ++v) base[v * ls + j * ss] = base[v * ls + j * ss] * f;
        }
    }
}

/* Bm3dFilterGroup (dct8.cpp:926-1133), the generic path. */
float om_filter_group(float* cube, const float* ref, int group, int block, float sigma, int wiener) {
    const int area = block * block;
    const int total = group * area;
    float* rw = NULL;
    if (wiener && ref) {
        rw = (float*)malloc((size_t)total * sizeof(float));
        memcpy(rw, ref, (size_t)total * sizeof(float));
        dct2_cube(rw, group, block, 0);
        haar_lines(rw, group, 1, area, area, 0);
    }
    dct2_cube(cube, group, block, 0);
    haar_lines(cube, group, 1, area, area, 0);
    int kept = 0;
    float w2sum = 0.f;
    if (rw) {
        const float sig2 = sigma * sigma;
        for (int i = 0; i < total; ++i) {
            float w = 1.f;
            if (i != 0) {
                const float r2 = rw[i] * rw[i];
                const float den = r2 + sig2;
                w = den > 0.f ? r2 / den : 0.f;
            }
            cube[i] = cube[i] * w;
            w2sum = fmaf(w, w, w2sum);
        }
    } else {
        const float thr = 2.7f * sigma;
        for (int i = 0; i < total; ++i) {
            if (i != 0 && fabsf(cube[i]) < thr) {
                cube[i] = 0.f;
            } else {
                ++kept;
            }
        }
    }
    haar_lines(cube, group, 1, area, area, 1);
    dct2_cube(cube, group, block, 1);
    free(rw);
    if (wiener) return 1.f / fmaxf(w2sum, 1e-12f);
    return 1.f / (float)(kept > 1 ? kept : 1);
}

/* ---- FP64 recomputation of the same group: exact cosines and scales ---- */

static void dct_lines_f64(double* base, int n, ptrdiff_t ls, ptrdiff_t ss, int count, int inverse) {
    if (n <= 1) return;
    const double pi = 3.14159265358979323846264338327950288;
    double T[64 * 64];
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i)
            T[k * n + i] = sqrt((k ? 2.0 : 1.0) / n) * cos(pi * ((double)i + 0.5) * (double)k / n);
    double x[64], y[64];
    for (int v = 0; v < count; ++v) {
        double* p = base + v * ls;
        for (int i = 0; i < n; ++i) x[i] = p[i * ss];
        for (int o = 0; o < n; ++o) {
            double acc = 0.0;
            for (int q = 0; q < n; ++q) acc += (inverse ? T[q * n + o] : T[o * n + q]) * x[q];
            y[o] = acc;
        }
        for (int i = 0; i < n; ++i) p[i * ss] = y[i];
    }
}

static void haar_lines_f64(double* base, int n, ptrdiff_t ls, ptrdiff_t ss, int count, int inverse) {
    if (n <= 1) return;
    for (int v = 0; v < count; ++v) {
        double* p = base + v * ls;
        if (inverse) {
            for (int j = 0; j < n; ++j) p[j * ss] *= haar_scale_f64(n, j);
            for (int h = n / 2; h >= 1; h >>= 1)
                for (int i = 0; i < n; i += 2 * h) {
                    const double a = p[i * ss], b = p[(i + h) * ss];
                    p[i * ss] = a + b;
                    p[(i + h) * ss] = a - b;
                }
        } else {
            for (int h = 1; h < n; h <<= 1)
                for (int i = 0; i < n; i += 2 * h) {
                    const double a = p[i * ss], b = p[(i + h) * ss];
                    p[i * ss] = a + b;
                    p[(i + h) * ss] = a - b;
                }
            for (int j = 0; j < n; ++j) p[j * ss] *= haar_scale_f64(n, j);
        }
    }
}

static void dct2_cube_f64(double* c, int group, int block, int inverse) {
    const int area = block * block;
    dct_lines_f64(c, block, block, 1, group * block, inverse);
    for (int g = 0; g < group; ++g) dct_lines_f64(c + (ptrdiff_t)g * area, block, 1, block, block, inverse);
}

double om_filter_group_f64(double* cube, const double* ref, int group, int block, double sigma, int wiener) {
    const int area = block * block;
    const int total = group * area;
    double* rw = NULL;
    if (wiener && ref) {
        rw = (double*)malloc((size_t)total * sizeof(double));
        memcpy(rw, ref, (size_t)total * sizeof(double));
        dct2_cube_f64(rw, group, block, 0);
        haar_lines_f64(rw, group, 1, area, area, 0);
    }
    dct2_cube_f64(cube, group, block, 0);
    haar_lines_f64(cube, group, 1, area, area, 0);
    double weight = 0.0;
    for (int i = 0; i < total; ++i) {
        if (rw) {
            const double den = rw[i] * rw[i] + sigma * sigma;
            const double w = i ? (den > 0 ? rw[i] * rw[i] / den : 0.0) : 1.0;
            cube[i] *= w;
            weight += w * w;
        } else {
            const int keep = i == 0 || fabs(cube[i]) >= 2.7 * sigma;
            if (!keep) cube[i] = 0.0;
            weight += keep;
        }
    }
    haar_lines_f64(cube, group, 1, area, area, 1);
    dct2_cube_f64(cube, group, block, 1);
    free(rw);
    return 1.0 / (weight > 1e-12 ? weight : 1e-12);
}

/* ------------------------------------------------------------ plane passes */

static void pack_patch(float* col, const float* src, ptrdiff_t stride, int x, int y, int block) {
    for (int py = 0; py < block; ++py)
        memcpy(col + py * block, src + (ptrdiff_t)(y + py) * stride + x, (size_t)block * sizeof(float));
}

/* UnpackPatch (pack.cpp:42-87) for an in-bounds patch: num = w*v + num (one
 * rounding), den += w. With a window (block x block weights, not part of the
 * reference's BM3D: the opt-in Kaiser mode of this build) every pixel takes
 * ww = w * win instead of w. */
static void unpack_patch(float* num, float* den, int width, int x, int y, const float* col, int block, float w,
                         const float* win) {
    for (int py = 0; py < block; ++py) {
        float* n = num + (ptrdiff_t)(y + py) * width + x;
        float* d = den + (ptrdiff_t)(y + py) * width + x;
        for (int px = 0; px < block; ++px) {
            const float ww = win ? w * win[py * block + px] : w;
            n[px] = fmaf(ww, col[py * block + px], n[px]);
            d[px] = d[px] + ww;
        }
    }
}

/* Filters the groups of one plane pass into num/den slices. matches of job i
 * are read through get_matches; slices[] maps a match's t to its slice. */
typedef struct pass_ctx {
    const float* const* srcs;
    const ptrdiff_t* sstrides;
    const float* const* refs; /* Wiener reference planes per slot, or NULL */
    const ptrdiff_t* rstrides;
    int width, height;
    const om_stage* st;
    int wiener;
    float* num; /* slices * plane */
    float* den;
    int slices;
    int radius, t0;
    const float* win; /* opt-in aggregation window (block x block), or NULL */
} pass_ctx;

static void filter_commit(pass_ctx* c, const om_match* m, int k, float* cube, float* refcube) {
    const int block = c->st->block, group = c->st->group, area = block * block;
    const size_t plane = (size_t)c->width * (size_t)c->height;
    memset(cube, 0, (size_t)group * area * sizeof(float));
    if (c->wiener) memset(refcube, 0, (size_t)group * area * sizeof(float));
    for (int j = 0; j < k; ++j) {
        const int t = c->radius > 0 ? m[j].t : c->t0;
        pack_patch(cube + (ptrdiff_t)j * area, c->srcs[t], c->sstrides[t], m[j].x, m[j].y, block);
        if (c->wiener) pack_patch(refcube + (ptrdiff_t)j * area, c->refs[t], c->rstrides[t], m[j].x, m[j].y, block);
    }
    const float w = om_filter_group(cube, c->wiener ? refcube : NULL, group, block, c->st->sigma, c->wiener);
    for (int j = 0; j < k; ++j) {
        const int sl = c->radius > 0 ? iclamp(m[j].t - c->t0 + c->radius, 0, c->slices - 1) : 0;
        unpack_patch(c->num + sl * plane, c->den + sl * plane, c->width, m[j].x, m[j].y,
                     cube + (ptrdiff_t)j * area, block, w, c->win);
    }
}

static void finish_plane(float* dst, ptrdiff_t dstride, const float* num, const float* den, const float* src,
                         ptrdiff_t sstride, int width, int height) {
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            const float d = den[(size_t)y * width + x];
            dst[y * dstride + x] = d > 1e-12f ? num[(size_t)y * width + x] / d : src[y * sstride + x];
        }
}

int om_bm3d_plane(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride, int width, int height,
                  const om_stage* st, int wiener, float* dst, ptrdiff_t dstride, int32_t* matches, int32_t* counts) {
    return om_bm3d_plane_matched(src, sstride, ref, rstride, NULL, 0, width, height, st, wiener, dst, dstride, matches,
                                 counts);
}

static int plane_pass(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride,
                      const float* match, ptrdiff_t mstride, int width, int height, const om_stage* st, int wiener,
                      const float* win, float* dst, ptrdiff_t dstride, int32_t* matches, int32_t* counts);

int om_bm3d_plane_matched(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride,
                          const float* match, ptrdiff_t mstride, int width, int height, const om_stage* st,
                          int wiener, float* dst, ptrdiff_t dstride, int32_t* matches, int32_t* counts) {
    return plane_pass(src, sstride, ref, rstride, match, mstride, width, height, st, wiener, NULL, dst, dstride,
                      matches, counts);
}

int om_bm3d_plane_window(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride, int width,
                         int height, const om_stage* st, int wiener, const float* win, float* dst, ptrdiff_t dstride) {
    return plane_pass(src, sstride, ref, rstride, NULL, 0, width, height, st, wiener, win, dst, dstride, NULL, NULL);
}

static int plane_pass(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride,
                      const float* match, ptrdiff_t mstride, int width, int height, const om_stage* st, int wiener,
                      const float* win, float* dst, ptrdiff_t dstride, int32_t* matches, int32_t* counts) {
    if (st->sigma == 0.f) {
        for (int y = 0; y < height; ++y) memcpy(dst + y * dstride, src + y * sstride, (size_t)width * sizeof(float));
        return 0;
    }
    const int block = st->block, group = st->group, area = block * block;
    if (width < block || height < block) return -1;
    const size_t plane = (size_t)width * (size_t)height;
    float* num = (float*)calloc(plane * 2, sizeof(float));
    float* cube = (float*)malloc((size_t)group * area * 2 * sizeof(float));
    if (!num || !cube) {
        free(num);
        free(cube);
        return -1;
    }
    const float* match_src = match ? match : (wiener ? ref : src);
    const ptrdiff_t match_stride = match ? mstride : (wiener ? rstride : sstride);
    pass_ctx c = {&src, &sstride, wiener ? &ref : NULL, &rstride, width, height, st, wiener,
                  num, num + plane, 1, 0, 0, win};
    const int nx = om_grid_count(width, block, st->step), ny = om_grid_count(height, block, st->step);
    om_match m[OM_MAX_GROUP];
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) {
            const int bx = om_grid_pos(i, width, block, st->step), by = om_grid_pos(j, height, block, st->step);
            const int k = om_spatial_match(match_src, match_stride, width, height, bx, by, block, st->bm_range,
                                           group, m, 0);
            const size_t job = (size_t)j * nx + i;
            if (matches) {
                for (int q = 0; q < group; ++q)
                    matches[job * group + q] = q < k ? (int32_t)(((uint32_t)m[q].y << 16) | (uint32_t)m[q].x) : -1;
            }
            if (counts) counts[job] = k;
            filter_commit(&c, m, k, cube, cube + (size_t)group * area);
        }
    }
    finish_plane(dst, dstride, num, num + plane, src, sstride, width, height);
    free(num);
    free(cube);
    return 0;
}

/* temporal_slot_frame (temporal.hpp:19-21) */
static int slot_frame(int center, int slot, int radius, int frames) {
    return center + iclamp(slot - radius, -center, frames - 1 - center);
}

int om_bm3d_plane_fat(const float* const* src, const float* const* ref, int nframes, int n, int width, int height,
                      ptrdiff_t stride, const om_stage* st, int radius, int wiener, float* dst, ptrdiff_t dstride) {
    const int ntemp = 2 * radius + 1;
    const size_t plane = (size_t)width * (size_t)height;
    if (st->sigma == 0.f) { /* temporal_identity (temporal.hpp:24-35) */
        for (int t = 0; t < ntemp; ++t)
            for (int y = 0; y < height; ++y) {
                float* pn = dst + ((ptrdiff_t)(2 * t) * height + y) * dstride;
                float* pd = pn + (ptrdiff_t)height * dstride;
                for (int x = 0; x < width; ++x) {
                    pn[x] = t == radius ? src[n][y * stride + x] : 0.f;
                    pd[x] = t == radius ? 1.f : 0.f;
                }
            }
        return 0;
    }
    const int block = st->block, group = st->group, area = block * block;
    if (width < block || height < block) return -1;
    const float* srcs[2 * OM_MAX_RADIUS + 1];
    const float* refs[2 * OM_MAX_RADIUS + 1];
    ptrdiff_t strides[2 * OM_MAX_RADIUS + 1];
    for (int t = 0; t < ntemp; ++t) {
        const int f = slot_frame(n, t, radius, nframes);
        srcs[t] = src[f];
        refs[t] = wiener ? ref[f] : src[f];
        strides[t] = stride;
    }
    float* num = (float*)calloc(plane * 2 * ntemp, sizeof(float));
    float* cube = (float*)malloc((size_t)group * area * 2 * sizeof(float));
    if (!num || !cube) {
        free(num);
        free(cube);
        return -1;
    }
    pass_ctx c = {srcs, strides, wiener ? refs : NULL, strides, width, height, st, wiener,
                  num, num + plane * ntemp, ntemp, radius, radius, NULL};
    om_search cfg = {block, st->step, group, st->bm_range, radius, st->ps_num, st->ps_range,
                     imax(0, radius - n), radius + imin(radius + 1, nframes - n)};
    const int nx = om_grid_count(width, block, st->step), ny = om_grid_count(height, block, st->step);
    om_match m[OM_MAX_GROUP];
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int bx = om_grid_pos(i, width, block, st->step), by = om_grid_pos(j, height, block, st->step);
            const int k = om_predictive_match(refs, strides, ntemp, width, height, bx, by, radius, &cfg, m);
            if (k <= 0) continue;
            filter_commit(&c, m, k, cube, cube + (size_t)group * area);
        }
    for (int sl = 0; sl < ntemp; ++sl)
        for (int y = 0; y < height; ++y) {
            memcpy(dst + ((ptrdiff_t)(2 * sl) * height + y) * dstride, num + sl * plane + (size_t)y * width,
                   (size_t)width * sizeof(float));
            memcpy(dst + ((ptrdiff_t)(2 * sl + 1) * height + y) * dstride, num + (ntemp + sl) * plane + (size_t)y * width,
                   (size_t)width * sizeof(float));
        }
    free(num);
    free(cube);
    return 0;
}

/* VAggTarget (agg.cpp:151-200): contributions summed in the order given
 * (ascending centres), a single one kept exact at unit weight. */
void om_vaggregate(const float* const* fats, int count, const float* src, int width, int height, ptrdiff_t fstride,
                   ptrdiff_t sstride, int radius, const int* slices, float* dst, ptrdiff_t dstride) {
    (void)radius;
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            float num = 0.f, den = 0.f;
            for (int c = 0; c < count; ++c) {
                const float* base = fats[c] + (ptrdiff_t)(2 * slices[c]) * height * fstride;
                num += base[y * fstride + x];
                den += base[((ptrdiff_t)height + y) * fstride + x];
            }
            float o;
            if (count == 1) {
                o = den == 1.f ? num : (den > 1e-12f ? num / den : src[y * sstride + x]);
            } else {
                o = den > 1e-12f ? (den == 1.f ? num : num / den) : src[y * sstride + x];
            }
            dst[y * dstride + x] = o;
        }
}

int om_bm3d_plane_clip(const float* const* src, const float* const* ref, int nframes, int width, int height,
                       ptrdiff_t stride, const om_stage* st, int radius, int wiener, float* const* dst) {
    const int ntemp = 2 * radius + 1;
    const ptrdiff_t fstride = width;
    const size_t fat_size = (size_t)ntemp * 2 * height * width;
    float* fats = (float*)malloc(fat_size * (size_t)nframes * sizeof(float));
    if (!fats) return -1;
    for (int c = 0; c < nframes; ++c) {
        if (om_bm3d_plane_fat(src, ref, nframes, c, width, height, stride, st, radius, wiener, fats + c * fat_size,
                              fstride) != 0) {
            free(fats);
            return -1;
        }
    }
    for (int n = 0; n < nframes; ++n) {
        const int first = imax(0, n - radius), last = n + imin(radius, nframes - 1 - n);
        const float* list[2 * OM_MAX_RADIUS + 1];
        int sl[2 * OM_MAX_RADIUS + 1];
        for (int c = first; c <= last; ++c) {
            list[c - first] = fats + c * fat_size;
            sl[c - first] = n - c + radius;
        }
        om_vaggregate(list, last - first + 1, src[n], width, height, fstride, stride, radius, sl, dst[n], stride);
    }
    free(fats);
    return 0;
}

/* ------------------------------------------------------- threaded frames */

typedef struct mt_job {
    const float* const* src;
    float* const* dst;
    float* const* basic;
    int nframes, width, height;
    ptrdiff_t stride;
    const om_stage *bs, *fs;
    int two_stage;
    int next;
    int failed;
    pthread_mutex_t mu;
} mt_job;

static void* mt_worker(void* arg) {
    mt_job* j = (mt_job*)arg;
    for (;;) {
        pthread_mutex_lock(&j->mu);
        const int f = j->next++;
        pthread_mutex_unlock(&j->mu);
        if (f >= j->nframes) break;
        int rc;
        if (j->two_stage) {
            rc = om_bm3d_plane(j->src[f], j->stride, NULL, 0, j->width, j->height, j->bs, 0, j->basic[f], j->stride,
                               NULL, NULL);
            if (rc == 0)
                rc = om_bm3d_plane(j->src[f], j->stride, j->basic[f], j->stride, j->width, j->height, j->fs, 1,
                                   j->dst[f], j->stride, NULL, NULL);
        } else {
            rc = om_bm3d_plane(j->src[f], j->stride, NULL, 0, j->width, j->height, j->fs, 0, j->dst[f], j->stride,
                               NULL, NULL);
        }
        if (rc != 0) j->failed = 1;
    }
    return NULL;
}

int om_bm3d_frames_mt(const float* const* src, float* const* dst, float* const* basic_scratch, int nframes,
                      int width, int height, ptrdiff_t stride, const om_stage* basic, const om_stage* fin,
                      int two_stage, int threads) {
    mt_job j = {src, dst, basic_scratch, nframes, width, height, stride, basic, fin, two_stage, 0, 0,
                PTHREAD_MUTEX_INITIALIZER};
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    int started = 0;
    for (int i = 0; i < threads; ++i) {
        if (pthread_create(&tid[i], NULL, mt_worker, &j) != 0) break;
        ++started;
    }
    if (started == 0) mt_worker(&j);
    for (int i = 0; i < started; ++i) pthread_join(tid[i], NULL);
    return j.failed ? -1 : 0;
}

/* One radius-0 stage of one plane with the group filter and the sums in
 * FP64: the groups are those of the FP32 matcher (matched on ref for Wiener,
 * else on src), so the result isolates the arithmetic error of a stage. */
int om_bm3d_plane_f64(const float* src, ptrdiff_t sstride, const float* ref, ptrdiff_t rstride, int width, int height,
                      const om_stage* st, int wiener, double* dst, ptrdiff_t dstride) {
    if (st->sigma == 0.f) {
        for (int y = 0; y < height; ++y)
            for (int x = 0; x < width; ++x) dst[y * dstride + x] = src[y * sstride + x];
        return 0;
    }
    const int block = st->block, group = st->group, area = block * block;
    if (width < block || height < block) return -1;
    const size_t plane = (size_t)width * (size_t)height;
    double* num = (double*)calloc(plane * 2, sizeof(double));
    double* cube = (double*)malloc((size_t)group * area * 2 * sizeof(double));
    if (!num || !cube) {
        free(num);
        free(cube);
        return -1;
    }
    double* den = num + plane;
    double* rcube = cube + (size_t)group * area;
    const float* ms = wiener ? ref : src;
    const ptrdiff_t mst = wiener ? rstride : sstride;
    const int nx = om_grid_count(width, block, st->step), ny = om_grid_count(height, block, st->step);
    om_match m[OM_MAX_GROUP];
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int bx = om_grid_pos(i, width, block, st->step), by = om_grid_pos(j, height, block, st->step);
            const int k = om_spatial_match(ms, mst, width, height, bx, by, block, st->bm_range, group, m, 0);
            memset(cube, 0, (size_t)group * area * 2 * sizeof(double));
            for (int q = 0; q < k; ++q)
                for (int y = 0; y < block; ++y)
                    for (int x = 0; x < block; ++x) {
                        cube[(size_t)q * area + y * block + x] = src[(m[q].y + y) * sstride + m[q].x + x];
                        if (wiener) rcube[(size_t)q * area + y * block + x] = ref[(m[q].y + y) * rstride + m[q].x + x];
                    }
            const double w = om_filter_group_f64(cube, wiener ? rcube : NULL, group, block, (double)st->sigma, wiener);
            for (int q = 0; q < k; ++q)
                for (int y = 0; y < block; ++y)
                    for (int x = 0; x < block; ++x) {
                        const size_t at = (size_t)(m[q].y + y) * width + m[q].x + x;
                        num[at] += w * cube[(size_t)q * area + y * block + x];
                        den[at] += w;
                    }
        }
    for (int y = 0; y < height; ++y)
        for (int x = 0; x < width; ++x) {
            const double d = den[(size_t)y * width + x];
            dst[y * dstride + x] = d > 1e-12 ? num[(size_t)y * width + x] / d : src[y * sstride + x];
        }
    free(num);
    free(cube);
    return 0;
}

/* References of a plane whose groups differ between this build's SSD order
 * and the reference's 8-lane AVX2 order (om_ssd_lanes8): the near-tie rate of
 * the FP32 matcher against the reference CPU plugin's own rounding. */
long om_order_mismatch(const float* plane, ptrdiff_t stride, int width, int height, const om_stage* st, long* refs) {
    const int block = st->block;
    const int nx = om_grid_count(width, block, st->step), ny = om_grid_count(height, block, st->step);
    om_match a[OM_MAX_GROUP], b[OM_MAX_GROUP];
    long bad = 0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const int bx = om_grid_pos(i, width, block, st->step), by = om_grid_pos(j, height, block, st->step);
            const int ka = om_spatial_match(plane, stride, width, height, bx, by, block, st->bm_range, st->group, a, 0);
            const int kb = om_spatial_match(plane, stride, width, height, bx, by, block, st->bm_range, st->group, b, 1);
            int same = ka == kb;
            for (int q = 0; same && q < ka; ++q) same = a[q].x == b[q].x && a[q].y == b[q].y;
            bad += !same;
        }
    if (refs) *refs = (long)nx * ny;
    return bad;
}
