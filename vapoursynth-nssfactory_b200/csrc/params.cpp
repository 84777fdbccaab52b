// Creation-time argument resolution of nss_cuda.BM3D (see params.hpp for the
// reference functions and their order).
#include "params.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>

namespace nssb {
namespace {

constexpr const char* kNs = "nss_cuda";
constexpr int kDefaultBlock = 8, kDefaultGroup = 8, kDefaultStep = 8, kDefaultRange = 9;
constexpr int kDefaultPsNum = 2, kDefaultPsRange = 4;
constexpr float kDefaultSigma = 3.f;

[[noreturn]] void fail(const char* message) {
    throw ArgumentError(std::string(kNs) + ".BM3D: " + message);
}

bool finite_bits(float v) {
    uint32_t u;
    std::memcpy(&u, &v, sizeof u);
    return (u & 0x7f800000u) != 0x7f800000u;
}

bool allowed_block(int v) { return v == 1 || v == 2 || v == 4 || v == 8 || v == 12 || v == 16 || v == 32; }
bool allowed_group(int v) { return v == 1 || v == 2 || v == 4 || v == 8 || v == 16 || v == 32 || v == 64; }

// The call's argument map, read the way the VSMap accessors behave: a missing
// key or a value of another type reports an error and the caller's default
// applies; an int stands for a float (VapourSynth converts on invoke).
class Args {
public:
    Args(const nssb_arg* a, int n) : a_(a), n_(n) {}

    const nssb_arg* find(const char* key) const {
        for (int i = 0; i < n_; ++i)
            if (a_[i].key && std::strcmp(a_[i].key, key) == 0) return &a_[i];
        return nullptr;
    }
    int count(const char* key) const {
        const nssb_arg* e = find(key);
        return e ? e->count : -1;
    }
    int64_t get_int(const char* key, int idx, int* err) const {
        const nssb_arg* e = find(key);
        if (!e || e->type != NSSB_ARG_INT || idx < 0 || idx >= e->count) {
            *err = 1;
            return 0;
        }
        *err = 0;
        return e->ints[idx];
    }
    double get_float(const char* key, int idx, int* err) const {
        const nssb_arg* e = find(key);
        if (!e || idx < 0 || idx >= e->count || (e->type != NSSB_ARG_FLOAT && e->type != NSSB_ARG_INT)) {
            *err = 1;
            return 0;
        }
        *err = 0;
        return e->type == NSSB_ARG_FLOAT ? e->floats[idx] : static_cast<double>(e->ints[idx]);
    }
    const char* get_data(const char* key, int* err) const {
        const nssb_arg* e = find(key);
        if (!e || e->type != NSSB_ARG_DATA || !e->data) {
            *err = 1;
            return nullptr;
        }
        *err = 0;
        return e->data;
    }
    int n() const { return n_; }
    const nssb_arg& at(int i) const { return a_[i]; }

    // map_int (validate.cpp:80-87)
    int map_int(const char* key, int def, int* err_out = nullptr) const {
        int err = 0;
        const int64_t v = get_int(key, 0, &err);
        if (err_out) *err_out = err;
        return err ? def : static_cast<int>(v);
    }
    // map_float_array (validate.cpp:89-106): the last element repeats.
    void float_array(const char* key, float* out, int np, float def) const {
        const int m = count(key);
        for (int i = 0; i < np; ++i) {
            if (m <= 0) {
                out[i] = def;
                continue;
            }
            int err = 0;
            const double v = get_float(key, i < m ? i : m - 1, &err);
            out[i] = err ? def : static_cast<float>(v);
        }
    }
    // map_int_array (validate.cpp:108-125)
    void int_array(const char* key, int* out, int np, int def) const {
        const int m = count(key);
        for (int i = 0; i < np; ++i) {
            if (m <= 0) {
                out[i] = def;
                continue;
            }
            int err = 0;
            const int64_t v = get_int(key, i < m ? i : m - 1, &err);
            out[i] = err ? def : static_cast<int>(v);
        }
    }
    // map_inherit_int (validate.cpp:127-146): a missing plane inherits the previous one.
    void inherit_int(const char* key, int* out, int np, int def) const {
        const int m = count(key);
        for (int i = 0; i < np; ++i) {
            if (m <= 0) {
                out[i] = def;
                continue;
            }
            if (i < m) {
                int err = 0;
                const int64_t v = get_int(key, i, &err);
                out[i] = err ? (i == 0 ? def : out[i - 1]) : static_cast<int>(v);
            } else {
                out[i] = out[i - 1];
            }
        }
    }

private:
    const nssb_arg* a_;
    int n_;
};

int plane_width(const nssb_video_info& vi, int plane) { return vi.width >> (plane ? vi.subsampling_w : 0); }
int plane_height(const nssb_video_info& vi, int plane) { return vi.height >> (plane ? vi.subsampling_h : 0); }
int num_planes(const nssb_video_info& vi) { return vi.color_family == NSSB_GRAY ? 1 : 3; }

// is_const_32f (validate.cpp:47-56)
bool const_32f(const nssb_video_info& vi) {
    if (vi.width < 1 || vi.height < 1 || vi.num_frames < 1 ||
        static_cast<uint64_t>(vi.width) * static_cast<uint64_t>(vi.height) >
            static_cast<uint64_t>(std::numeric_limits<int>::max()) ||
        vi.color_family == 0)
        return false;
    return vi.sample_float == 1 && vi.bits_per_sample == 32 &&
           (vi.color_family == NSSB_GRAY || vi.color_family == NSSB_YUV || vi.color_family == NSSB_RGB);
}

bool same_video(const nssb_video_info& a, const nssb_video_info& b) {
    return a.color_family == b.color_family && a.sample_float == b.sample_float &&
           a.bits_per_sample == b.bits_per_sample && a.subsampling_w == b.subsampling_w &&
           a.subsampling_h == b.subsampling_h && a.width == b.width && a.height == b.height &&
           a.num_frames == b.num_frames;
}

// validate_numeric_args (validate.cpp:13-45), message prefix "nss:" as there.
void validate_numeric(const Args& args) {
    for (int i = 0; i < args.n(); ++i) {
        const nssb_arg& e = args.at(i);
        if (e.type != NSSB_ARG_INT && e.type != NSSB_ARG_FLOAT) continue;
        for (int k = 0; k < e.count; ++k) {
            bool valid;
            if (e.type == NSSB_ARG_INT) {
                const int64_t v = e.ints[k];
                valid = v >= std::numeric_limits<int>::min() && v <= std::numeric_limits<int>::max();
            } else {
                const double v = e.floats[k];
                const double limit = std::numeric_limits<float>::max();
                valid = std::isfinite(v) && v >= -limit && v <= limit;
            }
            if (!valid) {
                char message[256];
                std::snprintf(message, sizeof message, "nss: parameter %s[%d] is not representable as a finite %s",
                              e.key ? e.key : "", k, e.type == NSSB_ARG_INT ? "int" : "float");
                throw ArgumentError(message);
            }
        }
    }
}

// parse_sigma (bm3d_args.cpp:17-25): `user_sigma` keeps the values as the caller gave them.
void parse_sigma(const Args& args, int np, float sigma[3], float user_sigma[3]) {
    args.float_array("sigma", sigma, np, kDefaultSigma);
    std::copy_n(sigma, 3, user_sigma);
    for (int i = 0; i < np; ++i) {
        if (!finite_bits(sigma[i]) || sigma[i] < 0.f) fail("sigma must be finite and non-negative");
        if (sigma[i] != 0.f) sigma[i] = effective_sigma(sigma[i]);
    }
}

// map_adaptive (bm3d_args.cpp:29-37)
void map_adaptive(const Args& args, const char* key, int* out, int np, int fallback, const int* limit) {
    if (args.count(key) <= 0) {
        for (int i = 0; i < np; ++i) out[i] = std::min(fallback, limit[i]);
    } else {
        args.inherit_int(key, out, np, fallback);
    }
}

struct Parsed {
    float sigma[3]{kDefaultSigma, kDefaultSigma, kDefaultSigma};
    int block[3]{8, 8, 8}, group[3]{8, 8, 8}, step[3]{8, 8, 8}, range[3]{9, 9, 9};
    int ps_num[3]{2, 2, 2}, ps_range[3]{4, 4, 4};
    int radius = 0;
    bool chroma = false, final = false;
    float sigma_basic[3]{};
    int block_basic[3]{}, group_basic[3]{}, step_basic[3]{}, ps_num_basic[3]{};
};

// parse_chroma (bm3d_args.cpp:40-57)
void parse_chroma(const Args& args, const nssb_video_info& vi, Parsed& p) {
    const int chroma = args.map_int("chroma", 0);
    if (chroma != 0 && chroma != 1) fail("chroma must be 0 or 1");
    p.chroma = chroma != 0;
    if (!p.chroma) return;
    if (vi.color_family != NSSB_YUV || vi.subsampling_w != 0 || vi.subsampling_h != 0)
        fail("chroma requires a YUV 4:4:4 clip");
    for (int i = 1; i < num_planes(vi); ++i) {
        p.block[i] = p.block[0];
        p.group[i] = p.group[0];
        p.step[i] = p.step[0];
        p.range[i] = p.range[0];
        p.ps_num[i] = p.ps_num[0];
        p.ps_range[i] = p.ps_range[0];
    }
}

// parse_basic_stage (bm3d_args.cpp:61-96)
void parse_basic(const Args& args, const nssb_video_info& vi, bool sigma_basic, bool block_basic, bool group_basic,
                 float user_sigma[3], Parsed& p) {
    const int np = num_planes(vi);
    if (sigma_basic) args.float_array("sigma_basic", user_sigma, np, kDefaultSigma);
    const bool has_block_step = args.count("block_step") > 0;
    const bool has_ps_num = args.count("ps_num") > 0;
    for (int i = 0; i < np; ++i) {
        p.block_basic[i] = p.block[i];
        p.group_basic[i] = p.group[i];
    }
    if (block_basic) args.inherit_int("block_size_basic", p.block_basic, np, kDefaultBlock);
    if (group_basic) args.inherit_int("group_size_basic", p.group_basic, np, kDefaultGroup);
    for (int i = 0; i < np; ++i) {
        const int source = p.chroma ? 0 : i;  // CBM3D: every plane takes plane 0's shape
        p.block_basic[i] = p.block_basic[source];
        p.group_basic[i] = p.group_basic[source];
        if (!finite_bits(user_sigma[i]) || user_sigma[i] < 0.f) fail("sigma_basic must be finite and non-negative");
        p.sigma_basic[i] = user_sigma[i] != 0.f ? effective_sigma(user_sigma[i]) : 0.f;
        if (!allowed_block(p.block_basic[i])) fail("block_size_basic must be one of 1, 2, 4, 8, 12, 16, 32");
        if (!allowed_group(p.group_basic[i])) fail("group_size_basic must be one of 1, 2, 4, 8, 16, 32, 64");
        if (p.block_basic[i] > plane_width(vi, i) || p.block_basic[i] > plane_height(vi, i))
            fail("block_size_basic must not exceed plane dimensions");
        p.step_basic[i] = has_block_step ? p.step[i] : std::min(kDefaultStep, p.block_basic[i]);
        p.ps_num_basic[i] = has_ps_num ? p.ps_num[i] : std::min(kDefaultPsNum, p.group_basic[i]);
        if (p.step_basic[i] > p.block_basic[i]) fail("block_step must be in [1, block_size_basic]");
        if (p.ps_num_basic[i] > p.group_basic[i]) fail("ps_num must be in [1, group_size_basic]");
    }
}

// check_planes (bm3d_args.cpp:99-112)
void check_planes(const nssb_video_info& vi, const Parsed& p) {
    for (int i = 0; i < num_planes(vi); ++i) {
        if (!allowed_block(p.block[i])) fail("block_size must be one of 1, 2, 4, 8, 12, 16, 32");
        if (!allowed_group(p.group[i])) fail("group_size must be one of 1, 2, 4, 8, 16, 32, 64");
        if (p.block[i] > plane_width(vi, i) || p.block[i] > plane_height(vi, i))
            fail("block_size must not exceed plane dimensions");
        if (p.step[i] < 1 || p.step[i] > p.block[i]) fail("block_step must be in [1, block_size]");
        if (p.ps_num[i] < 1 || p.ps_num[i] > p.group[i]) fail("ps_num must be in [1, group_size]");
        if (p.range[i] < 1 || p.range[i] > kMaxRange) fail("bm_range must be in [1, 64]");
        if (p.ps_range[i] < 0 || p.ps_range[i] > kMaxRange) fail("ps_range must be in [0, 64]");
    }
}

// parse_bm3d (bm3d_args.cpp:115-145)
Parsed parse_bm3d(const Args& args, const nssb_video_info& vi, const nssb_video_info* ref) {
    if (!const_32f(vi)) fail("constant Gray/YUV/RGB 32-bit float required");
    if (ref && !same_video(vi, *ref)) fail("ref must match clip");
    Parsed p;
    const int np = num_planes(vi);
    float user_sigma[3];
    parse_sigma(args, np, p.sigma, user_sigma);
    args.inherit_int("block_size", p.block, np, kDefaultBlock);
    args.inherit_int("group_size", p.group, np, kDefaultGroup);
    map_adaptive(args, "block_step", p.step, np, kDefaultStep, p.block);
    args.int_array("bm_range", p.range, np, kDefaultRange);
    map_adaptive(args, "ps_num", p.ps_num, np, kDefaultPsNum, p.group);
    args.int_array("ps_range", p.ps_range, np, kDefaultPsRange);
    p.radius = args.map_int("radius", 0);
    if (p.radius < 0 || p.radius > kMaxRadius) fail("radius must be in [0, 16]");
    parse_chroma(args, vi, p);
    const int final = args.map_int("final", 0);
    if (final != 0 && final != 1) fail("final must be 0 or 1");
    p.final = final != 0;
    const bool sigma_basic = args.count("sigma_basic") > 0;
    const bool block_basic = args.count("block_size_basic") > 0;
    const bool group_basic = args.count("group_size_basic") > 0;
    if (!p.final && (sigma_basic || block_basic || group_basic))
        fail("sigma_basic, block_size_basic and group_size_basic require final=1");
    if (p.final && ref) fail("use only one of final and ref");
    if (p.final) parse_basic(args, vi, sigma_basic, block_basic, group_basic, user_sigma, p);
    check_planes(vi, p);
    return p;
}

// parse_temporal_mode (temporal_args.cpp:10-27); returns true for rolling.
bool parse_temporal_mode(const Args& args, int radius) {
    int err = 0;
    const char* mode = args.get_data("temporal_mode", &err);
    std::string s;
    if (!err && mode) {
        s = mode;
        for (char& c : s)
            if (c >= 'A' && c <= 'Z') c = static_cast<char>(c - 'A' + 'a');
    }
    if (s == "fused") fail("temporal_mode=fused is not supported; use rolling or legacy");
    if (!s.empty() && s != "rolling" && s != "legacy") fail("temporal_mode must be rolling or legacy");
    if (radius <= 0) return false;
    if (s.empty()) return true;  // the device default: finished frames
    return s == "rolling";
}

}  // namespace

float effective_sigma(float user_sigma) {
    // NoiseProfile::bm3d_effective (contracts.hpp:27-29)
    return (user_sigma * (1.f / 255.f)) * 0.75f;
}

Bm3dConfig parse_bm3d_call(const nssb_video_info& clip, const nssb_video_info* ref, const nssb_arg* argv,
                           int nargs) {
    const Args args(argv, nargs);
    validate_numeric(args);
    Bm3dConfig cfg;
    {
        int err = 0;
        const int64_t mb = args.get_int("memory_limit_mb", 0, &err);
        if (!err) {
            if (mb < 1 || mb > 1048576) throw ArgumentError("nss: memory_limit_mb must be in [1, 1048576]");
            cfg.memory_limit_mb = mb;
        }
    }
    const int radius_arg = args.map_int("radius", 0);
    const bool rolling = parse_temporal_mode(args, radius_arg);
    const Parsed p = parse_bm3d(args, clip, ref);
    if (rolling) {
        // parse_rolling with the adaptive cache (temporal_args.cpp:29-56)
        cfg.rolling_chunk = args.map_int("rolling_chunk", 1);
        int limit_err = 0, chunks_err = 0;
        cfg.rolling_cache_limit = args.map_int("rolling_cache_limit", 16, &limit_err);
        cfg.rolling_cache_chunks = args.map_int("rolling_cache_chunks", 1, &chunks_err);
        if (p.radius < 1) fail("rolling mode requires radius > 0");
        if (cfg.rolling_chunk < 1 || cfg.rolling_chunk > 64) fail("rolling_chunk must be in [1, 64]");
        if (limit_err && !chunks_err) cfg.rolling_cache_limit = cfg.rolling_cache_chunks;
        if (cfg.rolling_cache_limit < 1 || cfg.rolling_cache_limit > 64 || cfg.rolling_cache_chunks < 1 ||
            cfg.rolling_cache_chunks > 64)
            fail("rolling_cache_limit must be in [1, 64]");
        if (cfg.rolling_cache_limit < cfg.rolling_cache_chunks)
            fail("rolling_cache_limit must be at least rolling_cache_chunks");
    }
    {
        // parse_backend_args (context.cpp:23-41)
        int err = 0;
        const int64_t device = args.get_int("device_id", 0, &err);
        if (!err) {
            if (device < 0 || device > INT32_MAX) fail("device_id must be >= 0");
            cfg.device_id = static_cast<int>(device);
        }
        const int64_t streams = args.get_int("num_streams", 0, &err);
        if (!err) {
            if (streams < 1 || streams > kMaxStreams) fail("num_streams must be in [1, 16]");
            cfg.num_streams = static_cast<int>(streams);
        }
    }
    cfg.vi = clip;
    cfg.planes = num_planes(clip);
    for (int i = 0; i < cfg.planes; ++i) {
        cfg.plane_w[i] = plane_width(clip, i);
        cfg.plane_h[i] = plane_height(clip, i);
        StageParams& s = cfg.final_stage[i];
        s.sigma = p.sigma[i];
        s.block = p.block[i];
        s.group = p.group[i];
        s.step = p.step[i];
        s.bm_range = p.range[i];
        s.ps_num = p.ps_num[i];
        s.ps_range = p.ps_range[i];
        StageParams& b = cfg.basic_stage[i];
        b = s;
        if (p.final) {
            b.sigma = p.sigma_basic[i];
            b.block = p.block_basic[i];
            b.group = p.group_basic[i];
            b.step = p.step_basic[i];
            b.ps_num = p.ps_num_basic[i];
        }
    }
    cfg.has_ref = ref != nullptr;
    cfg.two_stage = p.final;
    cfg.chroma = p.chroma;
    cfg.radius = p.radius;
    cfg.rolling = rolling;
    cfg.out_vi = clip;
    if (p.radius > 0 && !rolling) cfg.out_vi.height = clip.height * (2 * p.radius + 1) * 2;
    return cfg;
}

}  // namespace nssb
