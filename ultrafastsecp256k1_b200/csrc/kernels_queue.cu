// Persistent work-queue verify kernels for mixed ECDSA / BIP-340 batches.
//
// No reference counterpart: the reference launches one kernel per batch call
// (src/gpu/src/gpu_backend_cuda.cu:972, :1085).  Here many caller batches of
// both kinds are packed into one staging region (see QueueLayout in
// kernels.h): per kind contiguous msg / key / signature arrays.  Each kind has
// its own queue kernel (so a warp never holds both verify paths, and each
// kernel's code stays small for the instruction cache) and its own queue head;
// the two launches run as parallel branches (fork / join events), so a mixed
// request costs one verify latency, not two.  A grid sized to the resident
// capacity (SMs x blocks/SM) drains each queue: each warp claims 32
// consecutive items with one atomicAdd on its queue head and verifies them,
// until the queue is empty.  There are no waits: a warp that finds its queue
// empty exits.
//
// The item counts are read from a header in device memory (copied with the
// inputs), so a CUDA graph captured for one capacity bucket replays unchanged
// for any fill level of that bucket.  The queue heads are the kernels'
// scratch memory; the launch sequence zeroes them first.
#include "kernels.h"
#include "verify.cuh"
#include "dev_tables.cuh"

namespace uf {

// kKind 0 ECDSA, 1 BIP-340.  kCached: keys are looked up in / added to the
// resident cache (a.cache); per warp the lookups and hits are added to
// a.cache_stats.
template <bool kCached, int kKind>
__global__ void __launch_bounds__(kVerifyThreads, 3)
k_verify_queue(QueueArgs a, const uint4* __restrict__ gt, unsigned int* __restrict__ head) {
    extern __shared__ uint4 smem_tab[];
    const SmemTab tab{smem_tab + threadIdx.x, blockDim.x};
    const GlobalGT g{gt};
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t total = kKind == 0 ? min(a.counts[0], a.cap_e) : min(a.counts[1], a.cap_s);
    unsigned long long lookups = 0, hits = 0;     // kCached: this thread's counts
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(head + kKind, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        const uint32_t i = base + lane;
        if (i < total) {
            uint32_t mw[8], sw[16];
            bool ok, hit = false;
            if (kKind == 0) {
                load_words8(mw, a.e_msgs + 32ull * i);
                load_words8(sw, a.e_sigs + 64ull * i);
                load_words8(sw + 8, a.e_sigs + 64ull * i + 32);
                if (kCached)
                    ok = ecdsa_verify_one(mw, a.e_pubs + 33ull * i, sw, tab, g,
                                          CountingPubCache{PubCache{a.cache, a.cache_mask}, &hit});
                else
                    ok = ecdsa_verify_one(mw, a.e_pubs + 33ull * i, sw, tab, g);
                a.e_out[i] = ok ? 1 : 0;
            } else {
                uint32_t pw[8];
                load_words8(mw, a.s_msgs + 32ull * i);
                load_words8(sw, a.s_sigs + 64ull * i);
                load_words8(sw + 8, a.s_sigs + 64ull * i + 32);
                load_words8(pw, a.s_pubs + 32ull * i);
                if (kCached)
                    ok = schnorr_verify_one(mw, pw, sw, tab, g, CountingPubCache{PubCache{a.cache, a.cache_mask}, &hit});
                else
                    ok = schnorr_verify_one(mw, pw, sw, tab, g);
                a.s_out[i] = ok ? 1 : 0;
            }
            if (kCached) {
                lookups++;
                hits += hit ? 1 : 0;
            }
        }
    }
    if (kCached && a.cache_stats) {
        // one pair of atomics per warp (all lanes leave the loop together)
        for (int o = 16; o > 0; o >>= 1) {
            lookups += __shfl_down_sync(0xFFFFFFFFu, lookups, o);
            hits += __shfl_down_sync(0xFFFFFFFFu, hits, o);
        }
        if (lane == 0 && lookups) {
            atomicAdd(&a.cache_stats[0], lookups);
            atomicAdd(&a.cache_stats[1], hits);
        }
    }
}

template <bool kCached, int kKind>
static void launch_kind(const QueueArgs& a, const uint4* gt, unsigned int* head, int grid, size_t smem,
                        cudaStream_t s) {
    k_verify_queue<kCached, kKind><<<grid, kVerifyThreads, smem, s>>>(a, gt, head);
}

cudaError_t launch_verify_queue(const QueueArgs& a, const void* d_gtab, unsigned int* d_head, int grid,
                                cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join) {
    const size_t smem = kVerifyThreads * kVerifySmemPerThread;
    if (grid <= 0) grid = 1;
    const uint4* gt = reinterpret_cast<const uint4*>(d_gtab);
    cudaError_t e = cudaMemsetAsync(d_head, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    const bool both = a.cap_e > 0 && a.cap_s > 0;
    if (both) {
        // BIP-340 queue on the second stream, in parallel with the ECDSA queue
        if ((e = cudaEventRecord(fork, s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s2, fork, 0)) != cudaSuccess) return e;
    }
    if (a.cap_e > 0) {
        if (a.cache) launch_kind<true, 0>(a, gt, d_head, grid, smem, s);
        else launch_kind<false, 0>(a, gt, d_head, grid, smem, s);
    }
    if (a.cap_s > 0) {
        cudaStream_t ss = both ? s2 : s;
        if (a.cache) launch_kind<true, 1>(a, gt, d_head, grid, smem, ss);
        else launch_kind<false, 1>(a, gt, d_head, grid, smem, ss);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (both) {
        if ((e = cudaEventRecord(join, s2)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, join, 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

int verify_queue_occupancy() {
    const size_t smem = kVerifyThreads * kVerifySmemPerThread;
    int lo = 1 << 30;
    auto probe = [&](auto f) {
        int b = 0;
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, kVerifyThreads, smem);
        lo = b < lo ? b : lo;
    };
    probe(k_verify_queue<false, 0>);
    probe(k_verify_queue<false, 1>);
    probe(k_verify_queue<true, 0>);
    probe(k_verify_queue<true, 1>);
    return lo;
}

}  // namespace uf
