// Serving form: a request loop over one GPU. Requests -- short clips of any
// resolution, sigma and radius with the BM3D arguments of nss_cuda.BM3D --
// are admitted in arrival order while their device footprint fits the memory
// budget (and one at a time when nothing else runs, so an oversized request
// still progresses). Admitted radius-0 requests feed a continuous batch: each
// tick renders the pending frames of every admitted radius-0 request through
// the batched form (one launch per kernel over all of them), and requests
// that arrive during a tick join the next one. Radius > 0 requests run on
// worker threads, each on a pooled engine with its own stream, whose window
// frames and rolling sums stay on the device for the request; their kernels
// overlap the ticks on the GPU. Outputs do not depend on what else runs.
// No reference counterpart (the reference serves frames through
// VapourSynth's frame threads and its SlotPool, src/cuda/runtime/stream_pool.hpp:62-140).
#pragma once

#include "batch.hpp"
#include "engine.hpp"
#include "nss_b200.h"

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace nssb {

struct ServerOptions {
    size_t budget_bytes = 0;   // 0: 80 % of the device memory free at creation
    double max_tick_mpx = 64;  // pixels (all planes) a tick renders at most
    int workers = 8;           // radius > 0 requests in flight
};

class Server {
public:
    Server(int device, const ServerOptions& opt);
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    // Validates the arguments (creation errors as nss_cuda.BM3D reports them)
    // and queues the request; returns its ticket.
    int64_t submit(const nssb_serve_request& req);
    // Waits up to timeout_ms (< 0: forever); false on timeout.
    bool wait(int64_t ticket, int64_t timeout_ms, nssb_serve_result* out);
    void stats(nssb_server_stats* out);

private:
    using Clock = std::chrono::steady_clock;
    struct Request {
        int64_t id = 0;
        Bm3dConfig cfg;
        std::string key;  // engine pool key
        std::vector<nssb_frame> clip, ref;
        std::vector<nssb_frame_out> out;
        int memory = NSSB_MEM_HOST;
        int frames = 0, next = 0, done = 0;
        size_t footprint = 0;
        Clock::time_point submitted, admitted, finished;
        int status = NSSB_OK;
        std::string error;
        bool complete = false;
    };
    using Ptr = std::shared_ptr<Request>;

    void dispatcher();
    void worker();
    void admit_locked();
    void complete_locked(const Ptr& r, int status, const std::string& error);
    std::unique_ptr<Engine> take_engine(const Request& r);
    void return_engine(const std::string& key, std::unique_ptr<Engine> e, size_t bytes);

    int device_;
    ServerOptions opt_;
    std::unique_ptr<BatchEngine> batch_;
    std::mutex mu_;
    std::condition_variable cv_;       // dispatcher and workers: new work, completions, stop
    std::condition_variable done_cv_;  // waiters
    bool stop_ = false;
    int64_t next_id_ = 1;
    std::deque<Ptr> queue_;                  // submitted, not admitted
    std::vector<Ptr> spatial_;               // admitted radius-0 requests with frames left
    std::deque<Ptr> temporal_;               // admitted radius > 0 requests waiting for a worker
    std::map<int64_t, Ptr> live_;            // not yet collected by wait()
    size_t reserved_ = 0;
    int64_t active_ = 0;
    struct Idle {
        std::unique_ptr<Engine> engine;
        size_t bytes;
    };
    std::deque<std::pair<std::string, Idle>> idle_;  // engine pool, least recently returned first
    size_t idle_total_ = 0;
    nssb_server_stats st_{};
    std::thread dispatcher_;
    std::vector<std::thread> workers_;
};

}  // namespace nssb
