// Mixed-batch slot implementation (see batch.h).
#include "batch.h"

#include <string.h>

#include <algorithm>
#include <vector>

#include "backend.h"
#include "nvtx.h"

namespace uf {

namespace {
uint32_t bucket(size_t n) {
    if (n == 0) return 0;
    uint32_t b = BatchSlot::kMinBucket;
    while (b < n) b <<= 1;
    return b;
}
}  // namespace

cudaError_t HostBuf::ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    release();
    size_t want = std::max(bytes, cap * 2);
    want = (want + 4095) & ~size_t{4095};
    cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        (void)cudaGetLastError();
        return e;
    }
    cap = want;
    return cudaSuccess;
}

void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

BatchSlot::~BatchSlot() {
    if (!be_) return;
    cudaSetDevice(be_->device());
    if (stream_) cudaStreamSynchronize(stream_);
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
    if (stream2_) cudaStreamSynchronize(stream2_);
    if (done_) cudaEventDestroy(done_);
    if (fork_) cudaEventDestroy(fork_);
    if (join_) cudaEventDestroy(join_);
    if (stream2_) cudaStreamDestroy(stream2_);
    if (d_head_) cudaFree(d_head_);
    pinned_.release();
    big_pinned_.release();
    dev_.release();
    big_dev_.release();
    if (stream_) cudaStreamDestroy(stream_);
}

int BatchSlot::init(Backend* be, bool use_graphs) {
    be_ = be;
    use_graphs_ = use_graphs;
    cudaError_t e = cudaSetDevice(be->device());
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&stream2_, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join_, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done_, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&d_head_, 256);
    if (e == cudaSuccess && use_graphs) {
        // the graph buckets all bind this one staging pair, sized for the largest bucket
        const QueueLayout maxl(kGraphMaxItems, kGraphMaxItems);
        e = pinned_.ensure(maxl.host_bytes);
        if (e == cudaSuccess) e = dev_.ensure(maxl.total);
    }
    if (e != cudaSuccess) return be->cuda_error(e, "batch slot init");
    return kOk;
}

// Small layouts run two lanes per signature (the backend's tuned limit); the
// choice is part of the graph key, so a changed limit never replays a graph
// captured with the other kernels.
bool BatchSlot::two_lanes(const QueueArgs& a) const {
    return (uint64_t)a.cap_e + a.cap_s <= be_->queue_pair_items();
}

uint64_t BatchSlot::graph_key(const QueueArgs& a) const {
    return ((uint64_t)a.cap_e << 32) | a.cap_s | (two_lanes(a) ? (1ull << 63) : 0);
}

QueueArgs BatchSlot::args_for(uint8_t* d) const {
    QueueArgs a;
    a.counts = reinterpret_cast<const uint32_t*>(d);
    a.cap_e = layout_.cap_e;
    a.cap_s = layout_.cap_s;
    a.e_msgs = d + layout_.e_msgs;
    a.s_msgs = d + layout_.s_msgs;
    a.e_sigs = d + layout_.e_sigs;
    a.s_sigs = d + layout_.s_sigs;
    a.s_pubs = d + layout_.s_pubs;
    a.e_pubs = d + layout_.e_pubs;
    a.e_out = d + layout_.e_out;
    a.s_out = d + layout_.s_out;
    a.cache = cache_;
    a.cache_mask = cache_mask_;
    a.cache_stats = cache_stats_;
    if (cache_) {
        a.e_slot = reinterpret_cast<uint32_t*>(d + layout_.e_slot);
        a.s_slot = reinterpret_cast<uint32_t*>(d + layout_.s_slot);
        a.todo = reinterpret_cast<uint32_t*>(d + layout_.todo);
        a.todo_count = reinterpret_cast<uint32_t*>(d) + 2;
    }
    return a;
}

int BatchSlot::run_direct(const QueueArgs& a) {
    uint8_t* h = staged_big_ ? (uint8_t*)big_pinned_.p : (uint8_t*)pinned_.p;
    uint8_t* d = staged_big_ ? (uint8_t*)big_dev_.p : (uint8_t*)dev_.p;
    cudaError_t e = cudaMemcpyAsync(d, h, layout_.in_bytes, cudaMemcpyHostToDevice, stream_);
    if (e == cudaSuccess)
        e = two_lanes(a) ? launch_verify_queue_pair(a, be_->gtab(), d_head_, be_->queue_pair_grid(), stream_, stream2_,
                                                    fork_, join_)
                         : launch_verify_queue(a, be_->gtab(), d_head_, be_->queue_grid(), stream_, stream2_, fork_,
                                               join_);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h + layout_.e_out, d + layout_.e_out, layout_.out_bytes, cudaMemcpyDeviceToHost, stream_);
    if (e != cudaSuccess) return be_->cuda_error(e, "batch enqueue");
    return kOk;
}

int BatchSlot::run_graph(const QueueArgs& a, uint64_t key) {
    auto it = graphs_.find(key);
    if (it == graphs_.end()) {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaError_t e = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return be_->cuda_error(e, "graph capture");
        const int rc = run_direct(a);
        e = cudaStreamEndCapture(stream_, &g);
        if (rc != kOk) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess) return be_->cuda_error(e, "graph instantiate");
        it = graphs_.emplace(key, exec).first;
    }
    cudaError_t e = cudaGraphLaunch(it->second, stream_);
    if (e != cudaSuccess) return be_->cuda_error(e, "graph launch");
    return kOk;
}

int BatchSlot::enqueue(const VerifyJob* jobs, size_t n_jobs) {
    NvtxRange range("batch slot: pack + launch");
    if (const int rc = be_->fault_point("batch enqueue")) return rc;
    size_t n_e = 0, n_s = 0;
    for (size_t j = 0; j < n_jobs; ++j) (jobs[j].kind == 0 ? n_e : n_s) += jobs[j].count;
    cudaError_t e = cudaSetDevice(be_->device());
    if (e != cudaSuccess) return be_->cuda_error(e, "cudaSetDevice");
    // the staging is reused: the previous launch (finished or abandoned after
    // an error) must be off it first; normally it is complete already
    if ((e = cudaEventSynchronize(done_)) != cudaSuccess) return be_->cuda_error(e, "batch slot");
    const bool graph = use_graphs_ && n_e <= kGraphMaxItems && n_s <= kGraphMaxItems;
    if (graph) {
        layout_ = QueueLayout(bucket(n_e), bucket(n_s));
        staged_big_ = false;
    } else {
        layout_ = QueueLayout((uint32_t)n_e, (uint32_t)n_s);
        staged_big_ = true;
        if ((e = big_pinned_.ensure(layout_.host_bytes)) != cudaSuccess) return be_->cuda_error(e, "cudaHostAlloc");
        if ((e = big_dev_.ensure(layout_.total)) != cudaSuccess) return be_->cuda_error(e, "cudaMalloc");
    }
    uint8_t* h = staged_big_ ? (uint8_t*)big_pinned_.p : (uint8_t*)pinned_.p;
    uint32_t* hdr = reinterpret_cast<uint32_t*>(h);
    hdr[0] = (uint32_t)n_e;
    hdr[1] = (uint32_t)n_s;
    hdr[2] = 0;   // the key table's to-do count
    size_t oe = 0, os = 0;
    for (size_t j = 0; j < n_jobs; ++j) {
        const VerifyJob& J = jobs[j];
        if (J.count == 0) continue;
        if (J.kind == 0) {
            memcpy(h + layout_.e_msgs + 32 * oe, J.msgs, 32 * J.count);
            memcpy(h + layout_.e_sigs + 64 * oe, J.sigs, 64 * J.count);
            memcpy(h + layout_.e_pubs + 33 * oe, J.pubs, 33 * J.count);
            oe += J.count;
        } else {
            memcpy(h + layout_.s_msgs + 32 * os, J.msgs, 32 * J.count);
            memcpy(h + layout_.s_sigs + 64 * os, J.sigs, 64 * J.count);
            memcpy(h + layout_.s_pubs + 32 * os, J.pubs, 32 * J.count);
            os += J.count;
        }
    }
    uint8_t* d = staged_big_ ? (uint8_t*)big_dev_.p : (uint8_t*)dev_.p;
    const QueueArgs a = args_for(d);
    last_graph_ = graph;
    const int rc = graph ? run_graph(a, graph_key(a)) : run_direct(a);
    if (rc != kOk) return rc;
    if ((e = cudaEventRecord(done_, stream_)) != cudaSuccess) return be_->cuda_error(e, "event record");
    return kOk;
}

int BatchSlot::prewarm(uint32_t max_items) {
    if (!use_graphs_) return kOk;
    std::vector<uint32_t> caps = {0};
    for (uint32_t b = kMinBucket; b <= kGraphMaxItems; b <<= 1) caps.push_back(b);
    cudaError_t e = cudaSetDevice(be_->device());
    if (e != cudaSuccess) return be_->cuda_error(e, "cudaSetDevice");
    for (uint32_t ce : caps) {
        for (uint32_t cs : caps) {
            if ((ce == 0 && cs == 0) || (uint64_t)ce + cs > 2ull * std::max(max_items, kMinBucket)) continue;
            layout_ = QueueLayout(ce, cs);
            staged_big_ = false;
            uint32_t* hdr = reinterpret_cast<uint32_t*>(pinned_.p);
            hdr[0] = 0;
            hdr[1] = 0;
            hdr[2] = 0;
            const QueueArgs a = args_for((uint8_t*)dev_.p);
            const int rc = run_graph(a, graph_key(a));
            if (rc != kOk) return rc;
        }
    }
    if ((e = cudaStreamSynchronize(stream_)) != cudaSuccess) return be_->cuda_error(e, "prewarm");
    return kOk;
}

bool BatchSlot::ready() { return cudaEventQuery(done_) != cudaErrorNotReady; }

int BatchSlot::finish(const VerifyJob* jobs, size_t n_jobs) {
    NvtxRange range("batch slot: verdicts out");
    cudaError_t e = cudaEventSynchronize(done_);
    if (e != cudaSuccess) return be_->cuda_error(e, "batch");
    const uint8_t* h = staged_big_ ? (const uint8_t*)big_pinned_.p : (const uint8_t*)pinned_.p;
    size_t oe = 0, os = 0;
    for (size_t j = 0; j < n_jobs; ++j) {
        const VerifyJob& J = jobs[j];
        if (J.count == 0) continue;
        if (J.kind == 0) {
            memcpy(J.out, h + layout_.e_out + oe, J.count);
            oe += J.count;
        } else {
            memcpy(J.out, h + layout_.s_out + os, J.count);
            os += J.count;
        }
    }
    return kOk;
}

}  // namespace uf
