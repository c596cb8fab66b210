// Serving loop: continuous batching of verify requests on one device.
//
// No reference counterpart (the reference serves one synchronous call per
// caller batch, src/cpu/src/ufsecp_gpu_impl.cpp:317-408).  Requests (each one
// or more ECDSA / BIP-340 jobs in host memory) are submitted from any thread
// and return at once with an id.  One scheduler thread owns `slots` batch
// slots (each its own stream, pinned staging and CUDA graphs, batch.h):
// whenever a slot is free it packs the oldest pending requests, up to
// max_launch_items items, into one persistent-queue launch, so requests that
// arrive while others run are admitted as soon as a slot and memory free up,
// and their launches overlap on the device.  A request larger than
// max_launch_items is cut into pieces that ride in successive launches.
// Admission is bounded by a memory budget: the slots' fixed staging (pinned +
// device, reserved at start) plus the staged bytes of the items of every launch
// in flight stay within memory_budget_bytes.  Decompressed keys and their
// 1P..8P tables stay resident in a device key table shared by all slots
// (pubcache.cuh, keytable.h), so repeated keys skip decompression and table
// set-up.  The verdicts of a request are the per-kind verify's, whatever it is
// batched with.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "backend.h"
#include "batch.h"
#include "keytable.h"
#include "ufsecp/ufsecp_cancel.h"

namespace uf {

struct ServerConfig {
    uint32_t slots = 8;
    uint32_t max_launch_items = 1u << 16;
    uint64_t memory_budget_bytes = 8ull << 30;
    uint32_t batch_window_us = 0;     // wait this long for more work before launching a small batch
    uint32_t key_cache_log2 = 18;     // resident key table of 2^k slots (576 B each); 0 = none
};

struct ServerStats {
    uint64_t requests_done = 0;
    uint64_t items_done = 0;
    uint64_t launches = 0;
    double p50_us = 0, p99_us = 0, max_us = 0, mean_us = 0;
    double busy_s = 0;                // wall time with at least one launch in flight
    double span_s = 0;                // first submit to last completion
    uint64_t peak_budget_bytes = 0;   // reserved staging + item bytes in flight, at most the budget
    uint64_t reserved_bytes = 0;      // the slots' fixed staging (pinned + device)
    uint32_t peak_slots_in_flight = 0;
    uint64_t pending_requests = 0;
    uint64_t cache_lookups = 0, cache_hits = 0;   // resident key cache, since start
};

class Server {
public:
    explicit Server(Backend* be) : be_(be) {}
    ~Server();
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    int start(const ServerConfig& cfg);
    // Thread-safe.  The jobs' host buffers must stay valid until wait() for
    // this id has returned kOk; the verdicts are written into jobs[j].out.
    int submit(const VerifyJob* jobs, size_t n_jobs, uint64_t* id) { return submit(jobs, n_jobs, nullptr, id); }
    // Thread-safe.  `cancel` (may be null; copied) is polled by the scheduler
    // before every launch that would take a piece of this request; once it
    // answers non-zero the pieces not launched yet are dropped and the request
    // ends with kErrCancelled, its verdict bytes cleared.  The predicate is
    // called on the scheduler thread and must not call into the server.
    int submit(const VerifyJob* jobs, size_t n_jobs, const ufsecp_cancel_token* cancel, uint64_t* id);
    // Thread-safe.  kOk once the request is complete (its record is then
    // released), kErrGpuQueue on timeout, kErrBadInput for an unknown id; a
    // launch failure is returned as its error code, after the request's
    // verdict bytes were cleared (fail closed).
    int wait(uint64_t id, uint32_t timeout_ms);
    // Thread-safe.  Abandons a request: pieces not launched yet are dropped,
    // pieces on the device finish (a kernel is not stopped) and cancel waits
    // for them, at most timeout_ms.  kOk: the server has forgotten the request
    // and touches its buffers no more; the verdict bytes are cleared unless the
    // request had completed before the call.  kErrGpuQueue: pieces were still
    // in flight at the timeout (nothing more will be launched for it; call
    // cancel or wait again).  kErrBadInput: unknown id.
    int cancel(uint64_t id, uint32_t timeout_ms);
    // Latency percentiles over the requests completed since the last reset.
    void stats(ServerStats* out, bool reset);

private:
    using Clock = std::chrono::steady_clock;

    struct Request {
        uint64_t id = 0;
        std::vector<VerifyJob> jobs;
        size_t items = 0;
        size_t next_job = 0, next_item = 0;      // first piece not yet launched
        uint32_t pieces_in_flight = 0;
        bool all_launched = false, done = false;
        bool abandoned = false;                  // cancel() was called before completion
        bool has_token = false;
        ufsecp_cancel_token token{};
        int status = kOk;
        Clock::time_point t_submit;
    };
    struct Launch {
        std::unique_ptr<BatchSlot> slot;
        std::vector<VerifyJob> jobs;       // pieces of requests, in order
        std::vector<Request*> owners;      // owner of each piece
        size_t bytes = 0;
        bool busy = false;
    };

    void loop();
    bool admit(Launch& L);               // under mu_
    void complete(Launch& L, int rc);    // under mu_
    void finalize(Request* r);           // under mu_: r is done; clears its verdicts unless it succeeded
    void drop_pending(Request* r);       // under mu_: r's pieces not launched yet are dropped
    // pinned + device staging of one item, and its key-table slot index and to-do entry
    static size_t bytes_per_item(int kind) { return 2 * (32 + (kind == 0 ? 33 : 32) + 64 + 1) + 8; }

    Backend* be_;
    ServerConfig cfg_;
    std::thread thread_;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_;
    bool stop_ = false, started_ = false;
    uint64_t next_id_ = 1;
    std::deque<Request*> pending_;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs_;
    std::vector<Launch> launches_;
    uint64_t budget_used_ = 0, reserved_ = 0;
    KeyTable keys_;                  // resident key table shared by the slots
    // statistics
    std::vector<double> lat_us_;
    uint64_t items_done_ = 0, n_launches_ = 0, peak_budget_ = 0;
    uint32_t peak_in_flight_ = 0;
    double busy_s_ = 0;
    bool have_first_ = false;
    Clock::time_point t_first_submit_, t_last_done_, t_busy_since_;
    uint32_t in_flight_ = 0;
};

}  // namespace uf
