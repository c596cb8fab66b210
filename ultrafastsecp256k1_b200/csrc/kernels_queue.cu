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
//
// With the resident key table (pubcache.cuh) two passes run before the queue
// kernels: k_key_resolve gives every item its key's slot (claiming slots for
// new keys), k_key_build builds the claimed slots' tables; the queue kernels
// then copy an item's table instead of decompressing its key and building the
// table, so every lane of a warp runs the same instruction stream.
#include "kernels.h"
#include "verify.cuh"
#include "dev_tables.cuh"

namespace uf {

// One thread per item slot of both kinds (ECDSA items first, cap_e of them,
// then BIP-340): parse the key, find or claim its slot, record the slot index.
// Keys that fail to parse (prefix, x >= p) get kNoSlot: their verdict is 0
// either way.  Per warp one pair of atomics adds the lookups and the hits
// (keys found in a slot that was not claimed in this pass).
__global__ void __launch_bounds__(128)
k_key_resolve(QueueArgs a) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n_e = min(a.counts[0], a.cap_e), n_s = min(a.counts[1], a.cap_s);
    bool looked = false, hit = false;
    const bool is_e = t < a.cap_e;
    const uint32_t i = is_e ? t : t - a.cap_e;
    if (is_e ? i < n_e : (t < a.cap_e + a.cap_s && i < n_s)) {
        Fe x;
        bool odd = false, ok;
        if (is_e) {
            const uint8_t* pub = a.e_pubs + 33ull * i;
            ok = pub[0] == 0x02 || pub[0] == 0x03;
            odd = pub[0] == 0x03;
            be32_to_limbs(x.v, pub + 1);
        } else {
            uint32_t pw[8];
            load_words8(pw, a.s_pubs + 32ull * i);
            words_be_to_limbs(x.v, pw);
            ok = true;
        }
        ok = ok && limbs_lt_p(x.v);
        uint32_t slot = kNoSlot;
        if (ok) {
            bool claimed;
            slot = key_resolve(a.cache, a.cache_mask, x, odd, &claimed);
            if (claimed) a.todo[atomicAdd(a.todo_count, 1u)] = slot;
            looked = true;
            hit = slot != kNoSlot && !claimed;
        }
        (is_e ? a.e_slot : a.s_slot)[i] = slot;
    }
    if (a.cache_stats) {
        const uint32_t nl = __reduce_add_sync(0xFFFFFFFFu, looked ? 1u : 0u);
        const uint32_t nh = __reduce_add_sync(0xFFFFFFFFu, hit ? 1u : 0u);
        if ((threadIdx.x & 31u) == 0 && nl) {
            atomicAdd(&a.cache_stats[0], (unsigned long long)nl);
            atomicAdd(&a.cache_stats[1], (unsigned long long)nh);
        }
    }
}

// Grid-stride over this launch's to-do list: decompress the slot's key and
// build its 1P..8P table in place (READY), or mark an x off the curve BAD.
// Every thread runs the same instruction stream (no verify lanes wait).
__global__ void __launch_bounds__(128)
k_key_build(QueueArgs a) {
    const uint32_t n = *a.todo_count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        PubCacheSlot* slot = a.cache + a.todo[k];
        Fe x, y;
        for (int q = 0; q < 8; ++q) x.v[q] = slot->key[q];
        if (!lift_x_parity(y, x, slot->key[8] != 0)) {
            slot_publish(*slot, kSlotBad);
            continue;
        }
        SlotTab st{slot};
        build_ptable(st, x, y);
        slot_publish(*slot, kSlotReady);
    }
}

cudaError_t launch_key_passes(const QueueArgs& a, int grid, cudaStream_t s) {
    const uint64_t items = (uint64_t)a.cap_e + a.cap_s;
    if (!a.cache || items == 0) return cudaSuccess;
    k_key_resolve<<<(unsigned)((items + 127) / 128), 128, 0, s>>>(a);
    k_key_build<<<grid > 0 ? grid : 1, 128, 0, s>>>(a);
    return cudaGetLastError();
}

// kKind 0 ECDSA, 1 BIP-340.  kCached: the item's key table comes from its
// resolved slot (a.e_slot / a.s_slot) when that slot is ready.
template <bool kCached, int kKind>
__global__ void __launch_bounds__(kVerifyThreads, 3)
k_verify_queue(QueueArgs a, const uint4* __restrict__ gt, unsigned int* __restrict__ head) {
    extern __shared__ uint4 smem_tab[];
    const SmemTab tab{smem_tab + threadIdx.x, blockDim.x};
    const GlobalGT g{gt};
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t total = kKind == 0 ? min(a.counts[0], a.cap_e) : min(a.counts[1], a.cap_s);
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(head + kKind, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        const uint32_t i = base + lane;
        if (i < total) {
            uint32_t mw[8], sw[16];
            bool ok;
            if (kKind == 0) {
                load_words8(mw, a.e_msgs + 32ull * i);
                load_words8(sw, a.e_sigs + 64ull * i);
                load_words8(sw + 8, a.e_sigs + 64ull * i + 32);
                if (kCached) {
                    const uint32_t si = a.e_slot[i];
                    ok = ecdsa_verify_one(mw, a.e_pubs + 33ull * i, sw, tab, g,
                                          SlotPubCache{si == kNoSlot ? nullptr : a.cache + si});
                } else {
                    ok = ecdsa_verify_one(mw, a.e_pubs + 33ull * i, sw, tab, g);
                }
                a.e_out[i] = ok ? 1 : 0;
            } else {
                uint32_t pw[8];
                load_words8(mw, a.s_msgs + 32ull * i);
                load_words8(sw, a.s_sigs + 64ull * i);
                load_words8(sw + 8, a.s_sigs + 64ull * i + 32);
                load_words8(pw, a.s_pubs + 32ull * i);
                if (kCached) {
                    const uint32_t si = a.s_slot[i];
                    ok = schnorr_verify_one(mw, pw, sw, tab, g, SlotPubCache{si == kNoSlot ? nullptr : a.cache + si});
                } else {
                    ok = schnorr_verify_one(mw, pw, sw, tab, g);
                }
                a.s_out[i] = ok ? 1 : 0;
            }
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
    if ((e = launch_key_passes(a, grid, s)) != cudaSuccess) return e;
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
