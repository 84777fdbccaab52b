// The C ABI (include/nss_b200.h): status codes and a per-thread error text,
// no exception crosses it (the reference's checked_create / checked_frame
// boundary, src/frontend/validate.hpp:36-52, src/frontend/ownership.hpp:157-165).
#include "nss_b200.h"

#include "batch.hpp"
#include "server.hpp"
#include "engine.hpp"

#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

struct nssb_bm3d {
    std::unique_ptr<nssb::Engine> engine;
};

struct nssb_batch {
    std::unique_ptr<nssb::BatchEngine> engine;
};

struct nssb_server {
    std::unique_ptr<nssb::Server> server;
};

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& what) {
    g_error = what;
    return code;
}

template <class F>
int guarded(F&& f) {
    try {
        g_error.clear();
        f();
        return NSSB_OK;
    } catch (const nssb::ArgumentError& e) {
        return fail(NSSB_ERR_ARGUMENT, e.what());
    } catch (const nssb::CudaError& e) {
        return fail(NSSB_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(NSSB_ERR_RESOURCE, "nss: resource allocation failed during creation");
    } catch (const std::invalid_argument& e) {
        return fail(NSSB_ERR_STATE, e.what());
    } catch (const std::out_of_range& e) {
        return fail(NSSB_ERR_STATE, e.what());
    } catch (const std::exception& e) {
        return fail(NSSB_ERR_STATE, e.what());
    } catch (...) {
        return fail(NSSB_ERR_STATE, "nss: unexpected failure");
    }
}

// acquire_device (context.cpp:43-60): a creation error, never a render error.
void acquire_device(int device_id, const char* who) {
    int count = 0;
    const cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        throw nssb::ArgumentError(std::string(who) + ": no CUDA device available (" + cudaGetErrorString(e) + ")");
    }
    if (device_id < 0 || device_id >= count)
        throw nssb::ArgumentError(std::string(who) + ": device_id " + std::to_string(device_id) +
                                  " is out of range (" + std::to_string(count) + " devices)");
    cudaDeviceProp prop{};
    NSSB_CUDA(cudaGetDeviceProperties(&prop, device_id));
    if (prop.major != 10 || prop.minor != 0)
        throw nssb::ArgumentError(std::string(who) + ": this build runs on sm_100 (B200) devices only");
}

}  // namespace

extern "C" {

const char* nssb_last_error(void) { return g_error.c_str(); }

const char* nssb_version(void) { return "nss_b200 1.0 (sm_100a)"; }

int nssb_backend_info(int device_id, char* buf, size_t cap) {
    return guarded([&] {
        int count = 0;
        const cudaError_t e = cudaGetDeviceCount(&count);
        std::string s;
        if (e != cudaSuccess || count == 0) {
            (void)cudaGetLastError();
            s = std::string("{\"device_count\": 0, \"error\": \"") + cudaGetErrorString(e) + "\"}";
        } else {
            if (device_id < 0 || device_id >= count) throw nssb::ArgumentError("nss_cuda.Backend: device_id out of range");
            cudaDeviceProp prop{};
            NSSB_CUDA(cudaGetDeviceProperties(&prop, device_id));
            char tmp[512];
            std::snprintf(tmp, sizeof tmp,
                          "{\"device_count\": %d, \"device_id\": %d, \"name\": \"%s\", \"compute_capability\": "
                          "\"%d.%d\", \"sm_count\": %d, \"memory_bytes\": %zu, \"kernels\": \"sm_100a\"}",
                          count, device_id, prop.name, prop.major, prop.minor, prop.multiProcessorCount,
                          (size_t)prop.totalGlobalMem);
            s = tmp;
        }
        if (buf && cap) {
            std::strncpy(buf, s.c_str(), cap - 1);
            buf[cap - 1] = 0;
        }
    });
}

int nssb_bm3d_check(const nssb_video_info* clip, const nssb_video_info* ref, const nssb_arg* args, int nargs,
                    nssb_video_info* out_vi) {
    return guarded([&] {
        if (!clip) throw nssb::ArgumentError("nss_cuda.BM3D: clip missing");
        const nssb::Bm3dConfig cfg = nssb::parse_bm3d_call(*clip, ref, args, nargs);
        if (out_vi) *out_vi = cfg.out_vi;
    });
}

int nssb_bm3d_create(const nssb_video_info* clip, const nssb_video_info* ref, const nssb_arg* args, int nargs,
                     nssb_bm3d** out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!clip || !out) throw nssb::ArgumentError("nss_cuda.BM3D: clip missing");
        const nssb::Bm3dConfig cfg = nssb::parse_bm3d_call(*clip, ref, args, nargs);
        acquire_device(cfg.device_id, "nss_cuda.BM3D");
        auto h = std::make_unique<nssb_bm3d>();
        // the memory plan (plan_planes, group_driver.cpp:571-600): a creation error
        // when the filter's device memory cannot fit memory_limit_mb; this engine
        // keeps whole planes resident, so it fits or it fails -- the limit never
        // changes the output
        if (cfg.memory_limit_mb > 0) {
            const size_t need = nssb::Engine::footprint(cfg, true);
            const int streams = cfg.radius > 0 ? 1 : std::max(1, cfg.num_streams);
            if (need > (size_t)cfg.memory_limit_mb << 20)
                throw nssb::ArgumentError("nss_cuda.BM3D: memory_limit_mb is too small for this clip: each of the " +
                                          std::to_string(streams) + " stream(s) needs at least " +
                                          std::to_string((need / streams >> 20) + 1) + " MiB");
        }
        h->engine = std::make_unique<nssb::Engine>(cfg);
        *out = h.release();
    });
}

void nssb_bm3d_free(nssb_bm3d* h) { delete h; }

int nssb_bm3d_output_info(const nssb_bm3d* h, nssb_video_info* out_vi) {
    return guarded([&] {
        if (!h || !out_vi) throw std::invalid_argument("nss_cuda.BM3D: null handle");
        *out_vi = h->engine->config().out_vi;
    });
}

int nssb_bm3d_frame_window(const nssb_bm3d* h, int n, int* first, int* last) {
    return guarded([&] {
        if (!h || !first || !last) throw std::invalid_argument("nss_cuda.BM3D: null handle");
        h->engine->frame_window(n, first, last);
    });
}

int nssb_bm3d_get_frame(nssb_bm3d* h, int n, const nssb_frame* clip_frames, const nssb_frame* ref_frames, int first,
                        int count, int memory, nssb_frame_out* out) {
    return guarded([&] {
        if (!h || !clip_frames || !out) throw std::invalid_argument("nss_cuda.BM3D: null argument");
        if (memory != NSSB_MEM_HOST && memory != NSSB_MEM_DEVICE)
            throw std::invalid_argument("nss_cuda.BM3D: memory must be NSSB_MEM_HOST or NSSB_MEM_DEVICE");
        h->engine->get_frame(n, clip_frames, ref_frames, first, count, memory, out);
    });
}

int nssb_bm3d_stats(nssb_bm3d* h, int enable_timing, int reset, nssb_kernel_stats* out) {
    return guarded([&] {
        if (!h) throw std::invalid_argument("nss_cuda.BM3D: null handle");
        h->engine->stats(enable_timing, reset, out);
    });
}

int nssb_match_spatial(const float* plane, int64_t stride, int width, int height, int block, int step,
                       int bm_range, int group, int32_t* pos, float* dist, int32_t* count, void* stream) {
    return guarded([&] {
        if (!plane || !pos || !count || width < block || height < block || block < 1 || step < 1 || group < 1 ||
            group > nssb::kMaxGroup || bm_range < 0 || bm_range > nssb::kMaxRange || width > 65535 || height > 65535)
            throw std::invalid_argument("nss_cuda: invalid matching arguments");
        nssb::launch_match_spatial(plane, stride, width, height, block, step, bm_range, group, pos, dist, count,
                                   static_cast<cudaStream_t>(stream));
    });
}

int nssb_bm3d_frame_props(const nssb_bm3d* h, int n, nssb_prop* out, int cap, int* count) {
    if (count) *count = 0;
    return guarded([&] {
        if (!h || !count || cap < 0 || (cap > 0 && !out)) throw std::invalid_argument("nssb_bm3d_frame_props: invalid arguments");
        const nssb::Bm3dConfig& c = h->engine->config();
        if (n < 0 || n >= c.vi.num_frames) throw std::out_of_range("nss_cuda.BM3D: frame number out of range");
        nssb_prop props[7] = {{"_NSSModel", 1}, {"_NSSModelVersion", 3}, {"_NSSNoiseProfile", 1}};
        int k = 3;
        if (c.radius > 0 && !c.rolling) {  // the fat intermediate: one centre's num/den slices
            props[k++] = {"_NSSFatVersion", 2};
            props[k++] = {"_NSSFatRadius", c.radius};
            props[k++] = {"_NSSFatCenter", n};
            props[k++] = {"_NSSFatLayout", 1};
        }
        for (int i = 0; i < k && i < cap; ++i) out[i] = props[i];
        *count = k < cap ? k : cap;
    });
}

int nssb_bm3d_set_window(nssb_bm3d* h, float beta) {
    return guarded([&] {
        if (!h) throw std::invalid_argument("nssb_bm3d_set_window: invalid handle");
        h->engine->set_window(beta);
    });
}

int nssb_bm3d_set_matcher(nssb_bm3d* h, int form) {
    return guarded([&] {
        if (!h) throw std::invalid_argument("nssb_bm3d_set_matcher: invalid handle");
        if (form != NSSB_MATCHER_FP32 && form != NSSB_MATCHER_TENSOR && form != NSSB_MATCHER_AUTO)
            throw std::invalid_argument(
                "nssb_bm3d_set_matcher: form must be NSSB_MATCHER_FP32, NSSB_MATCHER_TENSOR or NSSB_MATCHER_AUTO");
        h->engine->set_matcher(form);
    });
}

int nssb_match_spatial_tc(const float* plane, int64_t stride, int width, int height, int step, int bm_range,
                          int group, int32_t* pos, float* dist, int32_t* count, nssb_tc_stats* stats,
                          void* stream) {
    int timeouts = 0;
    const int rc = guarded([&] {
        if (!plane || !pos || !count || width < 8 || height < 8 || step < 1 || step > 8 || stride < width)
            throw std::invalid_argument("nss_cuda: invalid matching arguments");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        nssb::TcCounters* ctr = nullptr;
        NSSB_CUDA(cudaMallocAsync(&ctr, sizeof(nssb::TcCounters), s));
        NSSB_CUDA(cudaMemsetAsync(ctr, 0, sizeof(nssb::TcCounters), s));
        auto mb = std::make_unique<nssb::MatchBatch>();
        mb->n = 1;
        mb->step = step;
        mb->p[0] = nssb::MatchPlane{plane, stride, pos, dist, count, width, height, 0, 0, 0};
        const bool ok = nssb::launch_match_tc_batch(*mb, bm_range, group, ctr, s);
        nssb::TcCounters host{};
        if (ok) NSSB_CUDA(cudaMemcpyAsync(&host, ctr, sizeof host, cudaMemcpyDeviceToHost, s));
        NSSB_CUDA(cudaFreeAsync(ctr, s));
        NSSB_CUDA(cudaStreamSynchronize(s));
        if (!ok)
            throw std::invalid_argument(
                "nss_cuda: the precision matcher covers 8x8 blocks, bm_range 9 (groups 2/4/8/16) and bm_range "
                "10-64 (groups 2/4/8/16/32)");
        timeouts = (int)host.timeouts;
        if (stats) {
            stats->survivors = (int64_t)host.survivors;
            stats->refs = (int64_t)host.refs;
            uint32_t bits = host.max_ratio_bits;
            std::memcpy(&stats->max_error_ratio, &bits, 4);
            stats->flagged_tiles = (int)host.flagged_tiles;
            stats->timeouts = (int)host.timeouts;
        }
    });
    if (rc == NSSB_OK && timeouts > 0) return fail(NSSB_ERR_TIMEOUT, "nss_cuda: a device wait of the precision matcher gave up");
    return rc;
}

int nssb_match_temporal(const float* const* planes, const int64_t* strides, int ntemp, int t0, int valid_begin,
                        int valid_end, int width, int height, int block, int step, int bm_range, int group,
                        int ps_num, int ps_range, int32_t* pos, int32_t* slot, float* dist, int32_t* count,
                        void* stream) {
    return guarded([&] {
        if (!planes || !strides || !pos || !slot || !dist || !count || ntemp < 1 || ntemp > nssb::kMaxSlots ||
            t0 < 0 || t0 >= ntemp || width < block || height < block || group < 1 || group > nssb::kMaxGroup ||
            ps_num < 1 || ps_num > group || ps_range < 0)
            throw std::invalid_argument("nss_cuda: invalid temporal matching arguments");
        nssb::TemporalPlanes tp{};
        for (int t = 0; t < ntemp; ++t) {
            tp.plane[t] = planes[t];
            tp.stride[t] = strides[t];
        }
        auto s = static_cast<cudaStream_t>(stream);
        nssb::launch_match_spatial(planes[t0], strides[t0], width, height, block, step, bm_range, group, pos, dist,
                                   count, s);
        nssb::launch_match_temporal(tp, ntemp, t0, valid_begin, valid_end, width, height, block, step, group, ps_num,
                                    ps_range, pos, slot, dist, count, s);
    });
}

int nssb_bm3d_plane_stage(const float* src, const float* ref, float* dst, int64_t stride, int width, int height,
                          float sigma, int block, int group, int step, int bm_range, void* stream) {
    return guarded([&] {
        if (!src || !dst || width < block || height < block || block < 1 || step < 1 || step > block ||
            group < 1 || group > nssb::kMaxGroup || bm_range < 0 || bm_range > nssb::kMaxRange)
            throw std::invalid_argument("nss_cuda: invalid stage arguments");
        nssb::StageParams sp;
        sp.sigma = sigma;
        sp.block = block;
        sp.group = group;
        sp.step = step;
        sp.bm_range = bm_range;
        nssb::Engine::plane_stage(src, ref, dst, stride, width, height, sp, static_cast<cudaStream_t>(stream));
    });
}

int nssb_bm3d_plane_stage_noalloc(const float* src, const float* ref, float* dst, int64_t stride, int width,
                                  int height, float sigma, int block, int group, int step, int bm_range,
                                  void* stream) {
    return guarded([&] {
        if (!src || !dst || width < block || height < block || block < 1 || step < 1 || step > block ||
            group < 1 || group > nssb::kMaxGroup || bm_range < 0 || bm_range > nssb::kMaxRange || stride < width)
            throw std::invalid_argument("nss_cuda: invalid stage arguments");
        nssb::StageParams sp;
        sp.sigma = sigma;
        sp.block = block;
        sp.group = group;
        sp.step = step;
        sp.bm_range = bm_range;
        nssb::plane_stage_noalloc(src, ref, dst, stride, width, height, sp, static_cast<cudaStream_t>(stream));
    });
}

int nssb_batch_create(int device_id, const nssb_arg* args, int nargs, nssb_batch** out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!out) throw std::invalid_argument("nssb_batch_create: out missing");
        nssb::BatchOptions opt;
        for (int i = 0; i < nargs; ++i) {
            const nssb_arg& a = args[i];
            const std::string key = a.key ? a.key : "";
            int* slot = key == "match_form"          ? &opt.fixed.match.form
                        : key == "match_parts"       ? &opt.fixed.match.parts
                        : key == "match_persistent"  ? &opt.fixed.match.persistent
                        : key == "group_warps"       ? &opt.fixed.group.warps
                        : key == "group_ctas_per_sm" ? &opt.fixed.group.ctas_per_sm
                                                     : nullptr;
            if (key == "chunk_frames") slot = &opt.chunk_frames;
            if (key != "autotune" && key != "graph" && !slot)
                throw nssb::ArgumentError("nss_batch: unknown argument " + key);
            if (a.type != NSSB_ARG_INT || a.count != 1 || !a.ints)
                throw nssb::ArgumentError("nss_batch: " + key + " must be one int");
            const int64_t v = a.ints[0];
            if (key == "autotune") opt.autotune = v != 0;
            else if (key == "graph") opt.graphs = v != 0;
            else *slot = (int)v;
        }
        const nssb::LaunchTunes& f = opt.fixed;
        if (f.match.form != 0 && f.match.form != 1)
            throw nssb::ArgumentError("nss_batch: match_form must be 0 or 1");
        if (f.match.parts != 1 && f.match.parts != 2 && f.match.parts != 4)
            throw nssb::ArgumentError("nss_batch: match_parts must be 1, 2 or 4");
        if (f.group.warps != 2 && f.group.warps != 4 && f.group.warps != 8)
            throw nssb::ArgumentError("nss_batch: group_warps must be 2, 4 or 8");
        if (opt.chunk_frames < 0) throw nssb::ArgumentError("nss_batch: chunk_frames must not be negative");
        if (f.group.ctas_per_sm < 1 || f.group.ctas_per_sm > 64)
            throw nssb::ArgumentError("nss_batch: group_ctas_per_sm must be in [1, 64]");
        acquire_device(device_id, "nss_batch");
        auto h = std::make_unique<nssb_batch>();
        h->engine = std::make_unique<nssb::BatchEngine>(device_id, opt);
        *out = h.release();
    });
}

int nssb_batch_run(nssb_batch* b, const nssb_batch_item* items, int n) {
    return guarded([&] {
        if (!b || (n > 0 && !items) || n < 0) throw std::invalid_argument("nssb_batch_run: invalid arguments");
        std::vector<nssb::BatchItem> list((size_t)n);
        for (int i = 0; i < n; ++i) {
            const nssb_batch_item& it = items[i];
            if (!it.node) throw std::invalid_argument("nssb_batch_run: item without node");
            list[i] = nssb::BatchItem{&it.node->engine->config(), it.clip, it.ref, it.memory, it.out};
        }
        b->engine->run(list.data(), n);
    });
}

int nssb_batch_get_info(nssb_batch* b, nssb_batch_info* out) {
    return guarded([&] {
        if (!b || !out) throw std::invalid_argument("nssb_batch_get_info: invalid arguments");
        b->engine->info(out);
    });
}

void nssb_batch_free(nssb_batch* b) { delete b; }

int nssb_server_create(int device_id, const nssb_arg* args, int nargs, nssb_server** out) {
    if (out) *out = nullptr;
    return guarded([&] {
        if (!out) throw std::invalid_argument("nssb_server_create: out missing");
        nssb::ServerOptions opt;
        for (int i = 0; i < nargs; ++i) {
            const nssb_arg& a = args[i];
            const std::string key = a.key ? a.key : "";
            if (key != "memory_budget_mb" && key != "max_tick_mpx" && key != "workers")
                throw nssb::ArgumentError("nss_server: unknown argument " + key);
            if (a.type != NSSB_ARG_INT || a.count != 1 || !a.ints)
                throw nssb::ArgumentError("nss_server: " + key + " must be one int");
            const int64_t v = a.ints[0];
            if (v < 0 || (key != "memory_budget_mb" && v < 1) || (key == "workers" && v > 64))
                throw nssb::ArgumentError("nss_server: " + key + " out of range");
            if (key == "memory_budget_mb") opt.budget_bytes = (size_t)v << 20;
            else if (key == "max_tick_mpx") opt.max_tick_mpx = (double)v;
            else opt.workers = (int)v;
        }
        acquire_device(device_id, "nss_server");
        auto h = std::make_unique<nssb_server>();
        h->server = std::make_unique<nssb::Server>(device_id, opt);
        *out = h.release();
    });
}

int nssb_server_submit(nssb_server* s, const nssb_serve_request* req, int64_t* ticket) {
    if (ticket) *ticket = 0;
    return guarded([&] {
        if (!s || !req || !ticket) throw std::invalid_argument("nssb_server_submit: invalid arguments");
        *ticket = s->server->submit(*req);
    });
}

int nssb_server_wait(nssb_server* s, int64_t ticket, int64_t timeout_ms, nssb_serve_result* out) {
    int timed_out = 0;
    const int rc = guarded([&] {
        if (!s) throw std::invalid_argument("nssb_server_wait: invalid arguments");
        timed_out = !s->server->wait(ticket, timeout_ms, out);
    });
    if (rc == NSSB_OK && timed_out) return fail(NSSB_ERR_TIMEOUT, "nssb_server_wait: timed out");
    return rc;
}

int nssb_server_get_stats(nssb_server* s, nssb_server_stats* out) {
    return guarded([&] {
        if (!s || !out) throw std::invalid_argument("nssb_server_get_stats: invalid arguments");
        s->server->stats(out);
    });
}

void nssb_server_free(nssb_server* s) { delete s; }

}  // extern "C"
