// Device-resident table of decompressed public keys and their P tables.
//
// No reference counterpart (the reference CPU keeps a 1024-slot lift_x cache,
// src/cpu/src/schnorr.cpp:275, and rebuilds every GPU table per signature).
// Per distinct key (x, y parity) a slot holds the 1P..8P affine table the
// verify kernels would otherwise build per signature, so a repeated key skips
// its square root, its table additions and the table's inversion.
//
// The table is filled in separate passes ahead of the verify kernels, so that
// the verify warps never mix lanes that build a table with lanes that copy one
// (the per-lane lookup inside the verify made 73 % of warps pay both):
//
//   resolve (one thread per item): parse the key, hash it, probe up to
//     kKeyProbes slots.  An empty slot is claimed (EMPTY -> CLAIMED by
//     atomicCAS), its key written, then published KEYED (release); the slot
//     joins this launch's to-do list.  A CLAIMED slot is another thread's key
//     being written: the prober waits for KEYED, up to kKeyWaitIters polls
//     (then it gives up: the item is verified without the table).  A KEYED /
//     READY / BAD slot with the same key is the item's slot; another key moves
//     on to the next probe.  The item's slot index (or kNoSlot) is stored.
//   build (one thread per to-do entry): lift_x of the slot's key; an x off the
//     curve publishes BAD, otherwise the table is built in the slot and
//     published READY (release).
//   verify: an item whose slot is READY (acquire) copies the table; BAD is a
//     known invalid key (verdict 0 without a square root); kNoSlot or a slot a
//     concurrent launch has not built yet is verified the plain way.
//
// Slots are never evicted; when the probe window is full the key is simply
// not cached.  The verdicts never depend on the table.
#pragma once
#include "common.cuh"
#include "fe.cuh"

namespace uf {

#if defined(__CUDACC__)
#define UF_MEMBER __host__ __device__ __forceinline__
#else
#define UF_MEMBER inline
#endif

// fetch() results: the key's table was loaded / no table (verify the plain
// way) / the key is known not to be on the curve.
enum : int { kKeyTable = 1, kKeyNone = 0, kKeyBad = -1 };

// No cache: every key is decompressed and its table built.
struct NoPubCache {
    template <class Tab>
    UF_MEMBER int fetch(Tab&) const { return kKeyNone; }
};

constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

}  // namespace uf

#if defined(__CUDACC__)
#include <cuda/atomic>

namespace uf {

struct alignas(64) PubCacheSlot {
    uint32_t state;      // kSlotEmpty .. kSlotBad
    uint32_t key[9];     // x limbs, parity
    uint32_t pad[6];
    uint4 tab[32];       // entry k: x (2 x uint4), y (2 x uint4)
};
static_assert(sizeof(PubCacheSlot) == 576, "slot layout");

enum : uint32_t { kSlotEmpty = 0, kSlotClaimed = 1, kSlotKeyed = 2, kSlotReady = 3, kSlotBad = 4 };
constexpr int kKeyProbes = 8;
constexpr int kKeyWaitIters = 1 << 14;

__device__ __forceinline__ uint32_t slot_state(const PubCacheSlot& s) {
    return cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(const_cast<uint32_t&>(s.state))
        .load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void slot_publish(PubCacheSlot& s, uint32_t st) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(s.state).store(st, cuda::memory_order_release);
}

__device__ __forceinline__ uint32_t key_hash(const Fe& x, bool odd) {
    uint32_t h = x.v[0] * 0x9E3779B1u ^ x.v[1] * 0x85EBCA77u ^ x.v[5] * 0xC2B2AE3Du ^ (odd ? 0x27D4EB2Fu : 0u);
    return h ^ (h >> 15);
}

__device__ __forceinline__ bool slot_has_key(const PubCacheSlot& s, const Fe& x, bool odd) {
    uint32_t d = s.key[8] ^ (odd ? 1u : 0u);
    for (int k = 0; k < 8; ++k) d |= s.key[k] ^ x.v[k];
    return d == 0;
}

// Resolve pass for one key.  Returns the slot index or kNoSlot; *claimed is
// set when this thread claimed the slot (its table is then built by the
// build pass of the same launch).
__device__ __forceinline__ uint32_t key_resolve(PubCacheSlot* slots, uint32_t mask, const Fe& x, bool odd,
                                                bool* claimed) {
    *claimed = false;
    const uint32_t h = key_hash(x, odd);
    for (int p = 0; p < kKeyProbes; ++p) {
        const uint32_t idx = (h + (uint32_t)p) & mask;
        PubCacheSlot& s = slots[idx];
        uint32_t st = slot_state(s);
        if (st == kSlotEmpty) {
            st = atomicCAS(&s.state, kSlotEmpty, kSlotClaimed);
            if (st == kSlotEmpty) {
                for (int k = 0; k < 8; ++k) s.key[k] = x.v[k];
                s.key[8] = odd ? 1u : 0u;
                slot_publish(s, kSlotKeyed);
                *claimed = true;
                return idx;
            }
        }
        // another thread's key is being written into this slot: wait (bounded)
        for (int it = 0; st == kSlotClaimed && it < kKeyWaitIters; ++it) {
            __nanosleep(64);
            st = slot_state(s);
        }
        if (st == kSlotClaimed) return kNoSlot;
        if (slot_has_key(s, x, odd)) return idx;
    }
    return kNoSlot;
}

// Read-only probe (no slot is claimed): the slot index holding the key when it
// is READY (its table built) or BAD (known off the curve), else kNoSlot.
// For callers that only need the decompressed key (entry 0 of the table is
// the key's point itself) and build nothing.
__device__ __forceinline__ uint32_t key_lookup(const PubCacheSlot* slots, uint32_t mask, const Fe& x, bool odd) {
    const uint32_t h = key_hash(x, odd);
    for (int p = 0; p < kKeyProbes; ++p) {
        const uint32_t idx = (h + (uint32_t)p) & mask;
        const PubCacheSlot& s = slots[idx];
        const uint32_t st = slot_state(s);
        if (st == kSlotEmpty) return kNoSlot;
        if ((st == kSlotReady || st == kSlotBad) && slot_has_key(s, x, odd)) return idx;
    }
    return kNoSlot;
}

// The verify kernels' view of an item's slot (resolved before the launch).
struct SlotPubCache {
    const PubCacheSlot* slot;   // null: no slot
    template <class Tab>
    __device__ __noinline__ int fetch(Tab& tab) const {
        if (!slot) return kKeyNone;
        const uint32_t st = slot_state(*slot);
        if (st == kSlotBad) return kKeyBad;
        if (st != kSlotReady) return kKeyNone;
        for (int k = 0; k < 8; ++k) {
            const uint4 a = slot->tab[4 * k], b = slot->tab[4 * k + 1], c = slot->tab[4 * k + 2],
                        d = slot->tab[4 * k + 3];
            Fe tx, ty;
            tx.v[0] = a.x; tx.v[1] = a.y; tx.v[2] = a.z; tx.v[3] = a.w;
            tx.v[4] = b.x; tx.v[5] = b.y; tx.v[6] = b.z; tx.v[7] = b.w;
            ty.v[0] = c.x; ty.v[1] = c.y; ty.v[2] = c.z; ty.v[3] = c.w;
            ty.v[4] = d.x; ty.v[5] = d.y; ty.v[6] = d.z; ty.v[7] = d.w;
            tab.store(k, tx, ty);
        }
        return kKeyTable;
    }
};

// A slot's table as the Tab of build_ptable (the build pass writes it in place).
struct SlotTab {
    PubCacheSlot* slot;
    __device__ __forceinline__ void store(int k, const Fe& x, const Fe& y) const {
        uint4* q = slot->tab + 4 * k;
        q[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
        q[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
        q[2] = make_uint4(y.v[0], y.v[1], y.v[2], y.v[3]);
        q[3] = make_uint4(y.v[4], y.v[5], y.v[6], y.v[7]);
    }
    __device__ __forceinline__ void load(int k, Fe& x, Fe& y) const {
        const uint4* q = slot->tab + 4 * k;
        const uint4 a = q[0], b = q[1], c = q[2], d = q[3];
        x.v[0] = a.x; x.v[1] = a.y; x.v[2] = a.z; x.v[3] = a.w;
        x.v[4] = b.x; x.v[5] = b.y; x.v[6] = b.z; x.v[7] = b.w;
        y.v[0] = c.x; y.v[1] = c.y; y.v[2] = c.z; y.v[3] = c.w;
        y.v[4] = d.x; y.v[5] = d.y; y.v[6] = d.z; y.v[7] = d.w;
    }
};

}  // namespace uf
#endif  // __CUDACC__
