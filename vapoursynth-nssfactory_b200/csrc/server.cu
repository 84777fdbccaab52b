// Serving form (see server.hpp).
#include "server.hpp"

#include <algorithm>
#include <cstring>
#include <sstream>

namespace nssb {

namespace {

double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Engines with equal keys are interchangeable (everything but the frame count).
std::string engine_key(const Bm3dConfig& c, int memory) {
    std::ostringstream os;
    os << c.vi.color_family << '/' << c.vi.subsampling_w << c.vi.subsampling_h << '/' << c.vi.width << 'x'
       << c.vi.height << '/' << c.radius << c.rolling << c.two_stage << c.has_ref << c.chroma << '/' << memory;
    for (int p = 0; p < c.planes; ++p)
        for (const StageParams* s : {&c.basic_stage[p], &c.final_stage[p]}) {
            uint32_t bits;
            std::memcpy(&bits, &s->sigma, 4);
            os << ',' << bits << '/' << s->block << '/' << s->group << '/' << s->step << '/' << s->bm_range << '/'
               << s->ps_num << '/' << s->ps_range;
        }
    return os.str();
}

int64_t plane_pitch(int w) { return (int64_t)((w + 31) / 32 * 32); }

// Device copies of a host request's frames: clip (+ ref) and outputs.
size_t staging_bytes(const Bm3dConfig& c, int frames, bool ref) {
    size_t frame = 0;
    for (int p = 0; p < c.planes; ++p) frame += (size_t)plane_pitch(c.plane_w[p]) * c.plane_h[p] * 4;
    return frame * frames * (ref ? 3 : 2);
}

double frame_mpx(const Bm3dConfig& c) {
    double px = 0;
    for (int p = 0; p < c.planes; ++p) px += (double)c.plane_w[p] * c.plane_h[p];
    return px / 1e6;
}

}  // namespace

Server::Server(int device, const ServerOptions& opt) : device_(device), opt_(opt) {
    NSSB_CUDA(cudaSetDevice(device_));
    if (opt_.budget_bytes == 0) {
        // what the library's pool keeps from earlier work goes back first, so
        // the free memory measured includes it
        dev_pool_trim(device_);
        size_t free_b = 0, total_b = 0;
        NSSB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        opt_.budget_bytes = free_b / 10 * 8;
    }
    BatchOptions bo;
    bo.autotune = false;  // layouts change every tick: fixed shapes, no capture
    bo.graphs = false;
    bo.plan_per_stream = true;
    bo.fixed.match.parts = 2;
    bo.fixed.group.warps = 8;
    bo.fixed.group.ctas_per_sm = 16;
    batch_ = std::make_unique<BatchEngine>(device_, bo);
    st_.budget_bytes = (int64_t)opt_.budget_bytes;
    dispatcher_ = std::thread([this] { dispatcher(); });
    for (int i = 0; i < std::max(1, opt_.workers); ++i) workers_.emplace_back([this] { worker(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        stop_ = true;
        while (!queue_.empty()) {
            Ptr r = queue_.front();
            queue_.pop_front();
            r->complete = true;
            r->status = NSSB_ERR_STATE;
            r->error = "nss_server: stopped before the request was admitted";
            r->finished = Clock::now();
            ++st_.failed;
        }
    }
    cv_.notify_all();
    done_cv_.notify_all();
    if (dispatcher_.joinable()) dispatcher_.join();
    for (auto& w : workers_)
        if (w.joinable()) w.join();
    idle_.clear();
    batch_.reset();
}

int64_t Server::submit(const nssb_serve_request& req) {
    if (!req.clip || !req.out) throw std::invalid_argument("nssb_server_submit: clip and out are required");
    if (req.vi.num_frames < 1) throw std::invalid_argument("nssb_server_submit: a request needs at least one frame");
    if (req.memory != NSSB_MEM_HOST && req.memory != NSSB_MEM_DEVICE)
        throw std::invalid_argument("nssb_server_submit: memory must be NSSB_MEM_HOST or NSSB_MEM_DEVICE");
    auto r = std::make_shared<Request>();
    r->cfg = parse_bm3d_call(req.vi, req.ref ? &req.vi : nullptr, req.args, req.nargs);
    if (r->cfg.radius > 0 && !r->cfg.rolling)
        throw ArgumentError("nss_server: temporal_mode legacy gives no finished frames and is not served");
    r->cfg.device_id = device_;
    r->frames = req.vi.num_frames;
    r->memory = req.memory;
    r->clip.assign(req.clip, req.clip + r->frames);
    if (req.ref) r->ref.assign(req.ref, req.ref + r->frames);
    r->out.assign(req.out, req.out + r->frames);
    r->key = engine_key(r->cfg, NSSB_MEM_DEVICE);  // temporal engines always work on device frames
    if (r->cfg.radius == 0) {
        std::vector<BatchItem> items((size_t)r->frames, BatchItem{&r->cfg, nullptr, nullptr, r->memory, nullptr});
        r->footprint = BatchPlan::footprint(items.data(), r->frames);
    } else {
        // a pooled engine working on device frames + the request's frames staged on the device
        r->footprint = Engine::footprint(r->cfg, false);
        if (r->memory == NSSB_MEM_HOST) r->footprint += staging_bytes(r->cfg, r->frames, !r->ref.empty());
    }
    r->submitted = Clock::now();
    {
        std::lock_guard<std::mutex> lock(mu_);
        if (stop_) throw std::invalid_argument("nss_server: stopping");
        r->id = next_id_++;
        queue_.push_back(r);
        live_[r->id] = r;
        ++st_.submitted;
    }
    cv_.notify_all();
    return r->id;
}

void Server::admit_locked() {
    while (!queue_.empty()) {
        const Ptr& r = queue_.front();
        while (!idle_.empty() && reserved_ + idle_total_ + r->footprint > opt_.budget_bytes) {
            idle_total_ -= idle_.begin()->second.bytes;
            idle_.erase(idle_.begin());  // the least recently returned engine
        }
        if (reserved_ + idle_total_ + r->footprint > opt_.budget_bytes && active_ > 0) break;
        Ptr a = r;
        queue_.pop_front();
        reserved_ += a->footprint;
        ++active_;
        a->admitted = Clock::now();
        st_.peak_active = std::max(st_.peak_active, active_);
        st_.peak_reserved_bytes = std::max(st_.peak_reserved_bytes, (int64_t)(reserved_ + idle_total_));
        if (a->cfg.radius == 0) spatial_.push_back(a);
        else temporal_.push_back(a);
        cv_.notify_all();
    }
}

void Server::complete_locked(const Ptr& r, int status, const std::string& error) {
    if (r->complete) return;
    r->complete = true;
    r->status = status;
    r->error = error;
    r->finished = Clock::now();
    reserved_ -= r->footprint;
    --active_;
    if (status == NSSB_OK) {
        ++st_.completed;
        st_.frames += r->frames;
    } else {
        ++st_.failed;
    }
    done_cv_.notify_all();
    cv_.notify_all();
}

// Continuous batching of the admitted radius-0 requests.
void Server::dispatcher() {
    std::unique_lock<std::mutex> lk(mu_);
    (void)cudaSetDevice(device_);
    for (;;) {
        admit_locked();
        std::vector<std::pair<Ptr, int>> tick;
        double mpx = 0;
        for (const Ptr& r : spatial_) {
            const double f = frame_mpx(r->cfg);
            while (r->next < r->frames && (tick.empty() || mpx + f <= opt_.max_tick_mpx)) {
                tick.emplace_back(r, r->next++);
                mpx += f;
            }
        }
        if (tick.empty()) {
            if (stop_ && spatial_.empty() && queue_.empty()) break;
            cv_.wait(lk);
            continue;
        }
        lk.unlock();
        std::vector<BatchItem> items;
        items.reserve(tick.size());
        for (auto& t : tick) {
            Request& r = *t.first;
            items.push_back(BatchItem{&r.cfg, &r.clip[t.second], r.ref.empty() ? nullptr : &r.ref[t.second],
                                      r.memory, &r.out[t.second]});
        }
        int status = NSSB_OK;
        std::string error;
        try {
            batch_->run(items.data(), (int)items.size());
        } catch (const CudaError& e) {
            status = NSSB_ERR_CUDA;
            error = e.what();
        } catch (const std::bad_alloc&) {
            status = NSSB_ERR_RESOURCE;
            error = "nss_server: device memory exhausted";
        } catch (const std::exception& e) {
            status = NSSB_ERR_STATE;
            error = e.what();
        }
        lk.lock();
        ++st_.ticks;
        st_.tick_frames += (int64_t)tick.size();
        for (auto& t : tick) {
            Request& r = *t.first;
            if (status != NSSB_OK) complete_locked(t.first, status, error);
            else if (++r.done == r.frames) complete_locked(t.first, NSSB_OK, std::string());
        }
        spatial_.erase(std::remove_if(spatial_.begin(), spatial_.end(), [](const Ptr& r) { return r->complete; }),
                       spatial_.end());
    }
}

std::unique_ptr<Engine> Server::take_engine(const Request& r) {
    {
        std::lock_guard<std::mutex> lock(mu_);
        for (auto it = idle_.begin(); it != idle_.end(); ++it) {
            if (it->first == r.key) {
                std::unique_ptr<Engine> e = std::move(it->second.engine);
                idle_total_ -= it->second.bytes;
                idle_.erase(it);
                ++st_.engines_reused;
                return e;
            }
        }
        ++st_.engines_created;
    }
    return std::make_unique<Engine>(r.cfg);
}

void Server::return_engine(const std::string& key, std::unique_ptr<Engine> e, size_t bytes) {
    std::lock_guard<std::mutex> lock(mu_);
    idle_.emplace_back(key, Idle{std::move(e), bytes});
    idle_total_ += bytes;
}

// One radius > 0 request at a time per worker, on a pooled engine.
void Server::worker() {
    (void)cudaSetDevice(device_);
    cudaStream_t stream = nullptr;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) return;
    struct Release {
        cudaStream_t s;
        ~Release() { (void)cudaStreamDestroy(s); }
    } release{stream};
    for (;;) {
        Ptr r;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !temporal_.empty(); });
            if (temporal_.empty()) {
                if (stop_) return;
                continue;
            }
            r = temporal_.front();
            temporal_.pop_front();
        }
        int status = NSSB_OK;
        std::string error;
        std::unique_ptr<Engine> e;
        void* stage = nullptr;
        try {
            e = take_engine(*r);
            e->reset_clip(r->frames);
            const Bm3dConfig& c = r->cfg;
            const bool host = r->memory == NSSB_MEM_HOST;
            std::vector<nssb_frame> dclip(r->clip), dref(r->ref);
            std::vector<nssb_frame_out> dout(r->out);
            if (host) {
                // the whole clip goes to the device once; outputs come back as they finish
                stage = dev_alloc(staging_bytes(c, r->frames, !r->ref.empty()));
                char* at = static_cast<char*>(stage);
                auto place = [&](auto& frame, const auto* src, cudaMemcpyKind kind) {
                    for (int p = 0; p < c.planes; ++p) {
                        const int64_t pitch = plane_pitch(c.plane_w[p]);
                        float* dst = reinterpret_cast<float*>(at);
                        at += (size_t)pitch * c.plane_h[p] * 4;
                        if (src)
                            NSSB_CUDA(cudaMemcpy2DAsync(dst, pitch * 4, src->planes[p], src->strides[p] * 4,
                                                        c.plane_w[p] * 4, c.plane_h[p], kind, stream));
                        frame.planes[p] = dst;
                        frame.strides[p] = pitch;
                    }
                };
                for (int f = 0; f < r->frames; ++f) {
                    place(dclip[f], &r->clip[f], cudaMemcpyHostToDevice);
                    if (!r->ref.empty()) place(dref[f], &r->ref[f], cudaMemcpyHostToDevice);
                    place(dout[f], static_cast<const nssb_frame*>(nullptr), cudaMemcpyHostToDevice);
                }
                NSSB_CUDA(cudaStreamSynchronize(stream));
            }
            for (int f = 0; f < r->frames; ++f) {
                e->get_frame(f, dclip.data(), dref.empty() ? nullptr : dref.data(), 0, r->frames, NSSB_MEM_DEVICE,
                             &dout[f]);
                if (host)
                    for (int p = 0; p < c.planes; ++p)
                        NSSB_CUDA(cudaMemcpy2DAsync(r->out[f].planes[p], r->out[f].strides[p] * 4, dout[f].planes[p],
                                                    dout[f].strides[p] * 4, c.plane_w[p] * 4, c.plane_h[p],
                                                    cudaMemcpyDeviceToHost, stream));
                std::lock_guard<std::mutex> lock(mu_);
                ++st_.temporal_frames;
            }
            NSSB_CUDA(cudaStreamSynchronize(stream));
        } catch (const CudaError& ex) {
            status = NSSB_ERR_CUDA;
            error = ex.what();
        } catch (const std::bad_alloc&) {
            status = NSSB_ERR_RESOURCE;
            error = "nss_server: device memory exhausted";
        } catch (const std::exception& ex) {
            status = NSSB_ERR_STATE;
            error = ex.what();
        }
        (void)cudaStreamSynchronize(stream);
        if (stage) dev_free(stage);
        if (e && status == NSSB_OK) return_engine(r->key, std::move(e), Engine::footprint(r->cfg, false));
        e.reset();
        std::lock_guard<std::mutex> lock(mu_);
        complete_locked(r, status, error);
    }
}

bool Server::wait(int64_t ticket, int64_t timeout_ms, nssb_serve_result* out) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = live_.find(ticket);
    if (it == live_.end()) throw std::invalid_argument("nssb_server_wait: unknown or already collected ticket");
    Ptr r = it->second;
    auto ready = [&] { return r->complete; };
    if (timeout_ms < 0) done_cv_.wait(lk, ready);
    else if (!done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) return false;
    if (out) {
        *out = nssb_serve_result{};
        out->status = r->status;
        out->frames = r->frames;
        const auto adm = r->admitted.time_since_epoch().count() ? r->admitted : r->finished;
        out->queue_ms = ms_between(r->submitted, adm);
        out->latency_ms = ms_between(r->submitted, r->finished);
        out->footprint_bytes = (int64_t)r->footprint;
        std::strncpy(out->error, r->error.c_str(), sizeof(out->error) - 1);
    }
    live_.erase(ticket);
    return true;
}

void Server::stats(nssb_server_stats* out) {
    std::lock_guard<std::mutex> lock(mu_);
    st_.queued = (int64_t)queue_.size();
    st_.active = active_;
    st_.reserved_bytes = (int64_t)(reserved_ + idle_total_);
    if (out) *out = st_;
}

}  // namespace nssb
