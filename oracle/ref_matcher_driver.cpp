// Drives the reference's own header-only matching code (src/cpu/bm/matcher.hpp:
// match_less, StableTopK, collect_spatial_coords, collect_temporal) with the
// oracle's distance, to pin the oracle's selection logic to the reference.
// TEST INFRASTRUCTURE ONLY: compiled by `make ref` from the reference tree in
// place (nothing copied) into _ref/, loaded by tests/ through ctypes.
#include "cpu/bm/matcher.hpp"

#include <cstddef>
#include <cstdint>

extern "C" float om_ssd(const float* a, ptrdiff_t sa, const float* b, ptrdiff_t sb, int block);

extern "C" int ref_spatial_match(const float* plane, ptrdiff_t stride, int width, int height, int bx, int by,
                                 int block, int bm_range, int group, nss::Match* out) {
    return nss::detail::collect_spatial_coords(width, height, bx, by, block, bm_range, group, out,
                                               [&](int cx, int cy, int x, int y) {
                                                   return om_ssd(plane + cy * stride + cx, stride,
                                                                 plane + y * stride + x, stride, block);
                                               });
}

extern "C" int ref_predictive_match(const float* const* planes, const ptrdiff_t* strides, int ntemp, int width,
                                    int height, int bx, int by, int t0, const int* cfgv, nss::Match* out) {
    nss::SearchConfig cfg;
    cfg.block = cfgv[0];
    cfg.step = cfgv[1];
    cfg.group = cfgv[2];
    cfg.bm_range = cfgv[3];
    cfg.radius = cfgv[4];
    cfg.ps_num = cfgv[5];
    cfg.ps_range = cfgv[6];
    cfg.valid_t_begin = cfgv[7];
    cfg.valid_t_end = cfgv[8];
    const int block = cfg.block;
    int n = ref_spatial_match(planes[t0], strides[t0], width, height, bx, by, block, cfg.bm_range, cfg.group, out);
    const int cx = bx < 0 ? 0 : (bx > width - block ? width - block : bx);
    const int cy = by < 0 ? 0 : (by > height - block ? height - block : by);
    const float* reference = planes[t0] + cy * strides[t0] + cx;
    return nss::detail::collect_temporal(width, height, t0, ntemp, cfg, out, n, [&](int t, int x, int y) {
        return om_ssd(reference, strides[t0], planes[t] + y * strides[t] + x, strides[t], block);
    });
}
