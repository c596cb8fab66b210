// Persistent work-queue verify kernel for mixed ECDSA / BIP-340 batches.
//
// No reference counterpart: the reference launches one kernel per batch call
// (src/gpu/src/gpu_backend_cuda.cu:972, :1085).  Here many caller batches of
// both kinds are packed into one staging region (see QueueLayout in
// kernels.h): per kind contiguous msg / key / signature arrays, ECDSA items
// first.  ONE launch of a grid sized to the resident capacity (SMs x
// blocks/SM) drains it: each warp claims 32 consecutive items with one
// atomicAdd on a queue head in device memory and verifies them, until the
// queue is empty.  Every claimed chunk except at most one is of a single kind,
// so the two verify paths do not diverge inside a warp.  There are no waits: a
// warp that finds the queue empty exits.
//
// The item counts are read from a header in device memory (copied with the
// inputs), so a CUDA graph captured for one capacity bucket replays unchanged
// for any fill level of that bucket.  The queue head is the kernel's scratch
// memory; the launch sequence zeroes it before the kernel.
#include "kernels.h"
#include "verify.cuh"
#include "dev_tables.cuh"

namespace uf {

__global__ void __launch_bounds__(kVerifyThreads)
k_verify_queue(QueueArgs a, const uint4* __restrict__ gt, unsigned int* __restrict__ head) {
    extern __shared__ uint4 smem_tab[];
    const SmemTab tab{smem_tab + threadIdx.x, blockDim.x};
    const GlobalGT g{gt};
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t n_e = min(a.counts[0], a.cap_e), n_s = min(a.counts[1], a.cap_s);
    const uint32_t total = n_e + n_s;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(head, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        const uint32_t i = base + lane;
        if (i < total) {
            uint32_t mw[8], sw[16];
            if (i < n_e) {
                load_words8(mw, a.e_msgs + 32ull * i);
                load_words8(sw, a.e_sigs + 64ull * i);
                load_words8(sw + 8, a.e_sigs + 64ull * i + 32);
                a.e_out[i] = ecdsa_verify_one(mw, a.e_pubs + 33ull * i, sw, tab, g) ? 1 : 0;
            } else {
                const uint32_t j = i - n_e;
                uint32_t pw[8];
                load_words8(mw, a.s_msgs + 32ull * j);
                load_words8(sw, a.s_sigs + 64ull * j);
                load_words8(sw + 8, a.s_sigs + 64ull * j + 32);
                load_words8(pw, a.s_pubs + 32ull * j);
                a.s_out[j] = schnorr_verify_one(mw, pw, sw, tab, g) ? 1 : 0;
            }
        }
    }
}

cudaError_t launch_verify_queue(const QueueArgs& a, const void* d_gtab, unsigned int* d_head, int grid,
                                cudaStream_t s) {
    const size_t smem = kVerifyThreads * kVerifySmemPerThread;
    if (grid <= 0) grid = 1;
    cudaError_t e = cudaMemsetAsync(d_head, 0, sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    k_verify_queue<<<grid, kVerifyThreads, smem, s>>>(a, reinterpret_cast<const uint4*>(d_gtab), d_head);
    return cudaGetLastError();
}

int verify_queue_occupancy() {
    int blocks = 0;
    const size_t smem = kVerifyThreads * kVerifySmemPerThread;
    cudaFuncSetAttribute(k_verify_queue, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_verify_queue, kVerifyThreads, smem);
    return blocks;
}

}  // namespace uf
