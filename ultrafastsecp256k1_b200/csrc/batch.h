// Mixed ECDSA / BIP-340 batches: packing, one-launch execution, CUDA graphs.
//
// No reference counterpart (the reference verifies one caller batch per
// synchronous call with per-call cudaMalloc / cudaFree,
// src/gpu/src/gpu_backend_cuda.cu:972-1028).  A BatchSlot owns one stream, a
// pinned host staging buffer and its device twin laid out as QueueLayout
// (kernels.h).  enqueue() packs any number of caller jobs into the staging
// buffer, then issues  H2D copy -> queue-head reset -> persistent queue kernel
// -> D2H copy  on the slot's stream.  For staging layouts up to
// kGraphMaxItems per kind the sequence is a CUDA graph captured once per
// capacity bucket (powers of two from 256) and replayed; the kernel reads the
// live item counts from the copied header, so a bucket's graph serves every
// fill level.  Larger layouts take the same sequence as direct calls.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <map>
#include <vector>

#include "backend.h"
#include "kernels.h"

namespace uf {

struct VerifyJob {
    int kind;             // 0 ECDSA (33-byte keys), 1 BIP-340 (32-byte x-only keys), 2 BIP-340 by RLC
    size_t count;
    const uint8_t* msgs;  // count x 32, host memory
    const uint8_t* pubs;
    const uint8_t* sigs;  // count x 64
    uint8_t* out;         // count verdict bytes, host memory
};

class BatchSlot {
public:
    static constexpr uint32_t kGraphMaxItems = 1u << 16;
    static constexpr uint32_t kMinBucket = 256;

    BatchSlot() = default;
    ~BatchSlot();
    BatchSlot(const BatchSlot&) = delete;
    BatchSlot& operator=(const BatchSlot&) = delete;

    // Creates the stream, completion event and queue head on the backend's device.
    int init(Backend* be, bool use_graphs = true);
    // Packs `jobs` and enqueues the work; returns immediately.  The jobs' host
    // buffers must stay valid until finish() returns.
    int enqueue(const VerifyJob* jobs, size_t n_jobs);
    // Captures and runs (with zero items) the graph of every capacity bucket
    // pair whose total is at most max_items, so that later launches of any
    // shape find their graph instantiated and their kernels loaded.
    int prewarm(uint32_t max_items);
    // True once the enqueued work has completed on the device.
    bool ready();
    // Waits for the enqueued work and writes every job's verdicts.
    int finish(const VerifyJob* jobs, size_t n_jobs);

    // Resident key table for the queue kernels (kernels.h QueueArgs,
    // pubcache.cuh); set before the first enqueue: captured graphs keep the
    // pointers.
    void set_cache(PubCacheSlot* slots, uint32_t mask, unsigned long long* stats) {
        cache_ = slots;
        cache_mask_ = mask;
        cache_stats_ = stats;
    }
    cudaStream_t stream() const { return stream_; }
    size_t staged_bytes() const { return layout_.total; }
    size_t graphs_cached() const { return graphs_.size(); }
    bool last_used_graph() const { return last_graph_; }

private:
    int run_direct(const QueueArgs& a);
    bool two_lanes(const QueueArgs& a) const;
    uint64_t graph_key(const QueueArgs& a) const;
    int run_graph(const QueueArgs& a, uint64_t key);
    QueueArgs args_for(uint8_t* dev_base) const;

    Backend* be_ = nullptr;
    bool use_graphs_ = true;
    cudaStream_t stream_ = nullptr;
    cudaStream_t stream2_ = nullptr;           // the BIP-340 queue's branch
    cudaEvent_t fork_ = nullptr, join_ = nullptr;
    cudaEvent_t done_ = nullptr;
    unsigned int* d_head_ = nullptr;
    HostBuf pinned_;                 // graph-bucket staging (fixed size, graphs bind it)
    DevBuf dev_;
    HostBuf big_pinned_;             // direct-path staging (grows)
    DevBuf big_dev_;
    QueueLayout layout_;
    bool staged_big_ = false;
    bool last_graph_ = false;
    std::map<uint64_t, cudaGraphExec_t> graphs_;
    PubCacheSlot* cache_ = nullptr;
    uint32_t cache_mask_ = 0;
    unsigned long long* cache_stats_ = nullptr;
};

}  // namespace uf
