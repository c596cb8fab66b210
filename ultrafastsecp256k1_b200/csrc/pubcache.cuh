// Device-resident cache of decompressed public keys and their P tables.
//
// No reference counterpart (the reference CPU keeps a 1024-slot lift_x cache,
// src/cpu/src/schnorr.cpp:275, and rebuilds every GPU table per signature).
// The serving path keeps, per distinct key (x, y parity), the 1P..8P affine
// table the verify kernels build, so a repeated key skips its square root, its
// table additions and the table's inversion.  Open addressing over a
// power-of-two slot array, 4 probes.  A slot is published once: a thread that
// wins EMPTY -> WRITING (atomicCAS) writes key and table, then stores READY
// with release order; readers load the state with acquire order and use only
// READY slots whose key matches, so a reader never sees a half-written table.
// Slots are never evicted; when the probe window is full the key is simply
// not cached.  Only keys that decompressed are inserted.
#pragma once
#include "common.cuh"
#include "fe.cuh"

namespace uf {

#if defined(__CUDACC__)
#define UF_MEMBER __host__ __device__ __forceinline__
#else
#define UF_MEMBER inline
#endif

// No cache: every key is decompressed and its table built.
struct NoPubCache {
    template <class Tab>
    UF_MEMBER bool fetch(const Fe&, bool, Tab&) const { return false; }
    template <class Tab>
    UF_MEMBER void put(const Fe&, bool, const Tab&) const {}
};

}  // namespace uf

#if defined(__CUDACC__)
#include <cuda/atomic>

namespace uf {

struct alignas(64) PubCacheSlot {
    uint32_t state;      // 0 empty, 1 being written, 2 ready
    uint32_t key[9];     // x limbs, parity
    uint32_t pad[6];
    uint4 tab[32];       // entry k: x (2 x uint4), y (2 x uint4)
};
static_assert(sizeof(PubCacheSlot) == 576, "slot layout");

constexpr int kPubCacheProbes = 4;

struct PubCache {
    PubCacheSlot* slots;
    uint32_t mask;       // slot count - 1

    __device__ __forceinline__ static uint32_t hash(const Fe& x, bool odd) {
        uint32_t h = x.v[0] * 0x9E3779B1u ^ x.v[1] * 0x85EBCA77u ^ x.v[5] * 0xC2B2AE3Du ^ (odd ? 0x27D4EB2Fu : 0u);
        return h ^ (h >> 15);
    }
    __device__ __forceinline__ static bool same(const PubCacheSlot& s, const Fe& x, bool odd) {
        uint32_t d = s.key[8] ^ (odd ? 1u : 0u);
        for (int k = 0; k < 8; ++k) d |= s.key[k] ^ x.v[k];
        return d == 0;
    }

    // out of line: called once per signature, and inlining it would raise the
    // verify kernels' register count
    template <class Tab>
    __device__ __noinline__ bool fetch(const Fe& x, bool odd, Tab& tab) const {
        const uint32_t h = hash(x, odd);
        for (int p = 0; p < kPubCacheProbes; ++p) {
            PubCacheSlot& s = slots[(h + p) & mask];
            const uint32_t st = cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(s.state)
                                    .load(cuda::memory_order_acquire);
            if (st == 0) return false;
            if (st != 2 || !same(s, x, odd)) continue;
            for (int k = 0; k < 8; ++k) {
                const uint4 a = s.tab[4 * k], b = s.tab[4 * k + 1], c = s.tab[4 * k + 2], d = s.tab[4 * k + 3];
                Fe tx, ty;
                tx.v[0] = a.x; tx.v[1] = a.y; tx.v[2] = a.z; tx.v[3] = a.w;
                tx.v[4] = b.x; tx.v[5] = b.y; tx.v[6] = b.z; tx.v[7] = b.w;
                ty.v[0] = c.x; ty.v[1] = c.y; ty.v[2] = c.z; ty.v[3] = c.w;
                ty.v[4] = d.x; ty.v[5] = d.y; ty.v[6] = d.z; ty.v[7] = d.w;
                tab.store(k, tx, ty);
            }
            return true;
        }
        return false;
    }

    template <class Tab>
    __device__ __noinline__ void put(const Fe& x, bool odd, const Tab& tab) const {
        const uint32_t h = hash(x, odd);
        for (int p = 0; p < kPubCacheProbes; ++p) {
            PubCacheSlot& s = slots[(h + p) & mask];
            if (atomicCAS(&s.state, 0u, 1u) != 0u) {
                if (cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(s.state).load(cuda::memory_order_acquire) ==
                        2 && same(s, x, odd))
                    return;   // already cached
                continue;
            }
            for (int k = 0; k < 8; ++k) s.key[k] = x.v[k];
            s.key[8] = odd ? 1u : 0u;
            for (int k = 0; k < 8; ++k) {
                Fe tx, ty;
                tab.load(k, tx, ty);
                s.tab[4 * k] = make_uint4(tx.v[0], tx.v[1], tx.v[2], tx.v[3]);
                s.tab[4 * k + 1] = make_uint4(tx.v[4], tx.v[5], tx.v[6], tx.v[7]);
                s.tab[4 * k + 2] = make_uint4(ty.v[0], ty.v[1], ty.v[2], ty.v[3]);
                s.tab[4 * k + 3] = make_uint4(ty.v[4], ty.v[5], ty.v[6], ty.v[7]);
            }
            cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(s.state).store(2u, cuda::memory_order_release);
            return;
        }
    }
};

// PubCache that also records whether its last fetch hit.
struct CountingPubCache {
    PubCache c;
    bool* hit;
    template <class Tab>
    __device__ __forceinline__ bool fetch(const Fe& x, bool odd, Tab& tab) const {
        const bool h = c.fetch(x, odd, tab);
        *hit = h;
        return h;
    }
    template <class Tab>
    __device__ __forceinline__ void put(const Fe& x, bool odd, const Tab& tab) const { c.put(x, odd, tab); }
};

}  // namespace uf
#endif  // __CUDACC__
