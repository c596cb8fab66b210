// Resident key table owner (keytable.h).
#include "keytable.h"

#include "backend.h"

namespace uf {

int KeyTable::create(Backend* be, uint32_t log2) {
    release();
    if (log2 < kMinLog2 || log2 > kMaxLog2) return be->set_error(kErrBadInput, "key table: log2 slots must be 8..24");
    log2_ = log2;
    dev_ = be->device();
    const size_t n = slot_count() * kPubCacheSlotBytes + 256;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n);
    if (e == cudaSuccess) e = cudaMemset(p, 0, n);
    if (e != cudaSuccess) {
        if (p) cudaFree(p);
        log2_ = 0;
        return be->cuda_error(e, "key table");
    }
    d_ = p;
    return kOk;
}

void KeyTable::release() {
    if (d_) {
        int cur = -1;
        cudaGetDevice(&cur);
        if (dev_ >= 0 && cur != dev_) cudaSetDevice(dev_);
        cudaFree(d_);
        if (cur >= 0 && cur != dev_) cudaSetDevice(cur);
    }
    d_ = nullptr;
    log2_ = 0;
}

cudaError_t KeyTable::clear(cudaStream_t s) {
    if (!d_) return cudaSuccess;
    return cudaMemsetAsync(d_, 0, bytes(), s);
}

cudaError_t KeyTable::read_counters(uint64_t* lookups, uint64_t* hits) const {
    *lookups = *hits = 0;
    if (!d_) return cudaSuccess;
    unsigned long long c[2] = {0, 0};
    const cudaError_t e = cudaMemcpy(c, counters(), sizeof(c), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) {
        *lookups = c[0];
        *hits = c[1];
    }
    return e;
}

}  // namespace uf
