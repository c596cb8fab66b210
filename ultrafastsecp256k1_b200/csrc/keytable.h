// Host owner of a resident key table (device slots of pubcache.cuh).
//
// One table per user of the queue kernels: the context's synchronous mixed-job
// calls (Backend::verify_jobs) and each server.  Layout in device memory:
// 2^log2 slots of kPubCacheSlotBytes, then two 64-bit counters (lookups,
// hits).  Slots are never evicted; clear() empties the table.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "kernels.h"

namespace uf {

class Backend;

class KeyTable {
public:
    static constexpr uint32_t kMinLog2 = 8, kMaxLog2 = 24;

    KeyTable() = default;
    ~KeyTable() { release(); }
    KeyTable(const KeyTable&) = delete;
    KeyTable& operator=(const KeyTable&) = delete;

    // Allocates and zeroes 2^log2 slots on the backend's device (synchronous).
    int create(Backend* be, uint32_t log2);
    void release();
    bool on() const { return d_ != nullptr; }
    uint32_t log2() const { return log2_; }
    size_t bytes() const { return on() ? slot_count() * kPubCacheSlotBytes + 256 : 0; }
    size_t slot_count() const { return size_t{1} << log2_; }
    PubCacheSlot* slots() const { return (PubCacheSlot*)d_; }
    uint32_t mask() const { return (uint32_t)(slot_count() - 1); }
    unsigned long long* counters() const {
        return on() ? (unsigned long long*)((uint8_t*)d_ + slot_count() * kPubCacheSlotBytes) : nullptr;
    }
    // Empties every slot and the counters, ordered on `s`.
    cudaError_t clear(cudaStream_t s);
    // Lookups and hits since creation / the last clear (synchronous read).
    cudaError_t read_counters(uint64_t* lookups, uint64_t* hits) const;

private:
    void* d_ = nullptr;
    uint32_t log2_ = 0;
    int dev_ = -1;
};

}  // namespace uf
