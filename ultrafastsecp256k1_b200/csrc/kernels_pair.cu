// Two lanes per signature, for small calls.
//
// No reference counterpart (the reference verifies one signature per
// thread).  A call of a few thousand signatures occupies a few warps per SM,
// so its time is one thread's verify latency, not the device's throughput.
// Here lanes 2t and 2t+1 verify signature t together: both parse the
// signature, decompress the key, compute the scalars and build the 1P..8P
// table (the same instruction stream, so the warp does not diverge), then
// each runs the main loop over half of the four GLV streams (dual_mul_half:
// lane 2t the a1*G and b1*P streams, lane 2t+1 the a2*(lambda G) and
// b2*(lambda P) streams, with the full 128 doublings each).  Lane 2t+1's
// partial sum reaches lane 2t through warp shuffles; one general addition
// gives R and lane 2t applies the same final check as the one-lane kernels
// (ecdsa_check_x / schnorr_check).  Each lane's loop has 33 + 7 instead of
// 66 + 14 table additions: a shorter critical path for 1.6x the work, which
// pays only while the device has idle capacity.  The autotuner sets the call
// size up to which it is used (tuning keys <kind>_pair_items).
//
// Verdict semantics are those of ecdsa_verify_one / schnorr_verify_one
// (compact ECDSA with low-S required, strict BIP-340); the opaque consensus
// form stays on the one-lane kernel.
#include "kernels.h"
#include "verify.cuh"
#include "dev_tables.cuh"

namespace uf {
namespace {

constexpr int kPairThreads = 128;

// Jacobian point across the lane pair (lane ^ 1); every lane of the warp calls it.
__device__ __forceinline__ Jac shfl_partner(const Jac& a) {
    Jac b;
    UF_UNROLL
    for (int k = 0; k < 8; ++k) {
        b.X.v[k] = __shfl_xor_sync(0xFFFFFFFFu, a.X.v[k], 1);
        b.Y.v[k] = __shfl_xor_sync(0xFFFFFFFFu, a.Y.v[k], 1);
        b.Z.v[k] = __shfl_xor_sync(0xFFFFFFFFu, a.Z.v[k], 1);
    }
    b.inf = __shfl_xor_sync(0xFFFFFFFFu, a.inf ? 1 : 0, 1) != 0;
    return b;
}

// One item verified by a lane pair (both lanes of the pair call it with the
// same item; `valid` false for a pair without an item).  Every lane of the warp
// must call it: it ends with warp shuffles.  The verdict is meaningful on the
// even lane (half 0).
// kKind 0: ECDSA (compact r || s, low-S), 1: BIP-340.
// `cache` (SlotPubCache / NoPubCache) may supply the key's table (both lanes
// copy it into their own shared-memory columns) or know the key to be off the
// curve.
template <int kKind, class Cache>
__device__ __forceinline__ bool pair_item(const uint8_t* msg, const uint8_t* pub, const uint8_t* sig, bool valid,
                                          int half, const SmemTab& tab, const GlobalGT& g, const Cache& cache) {
    bool ok = valid, have_tab = false;
    Sc r, s, a, b;        // r kept for the ECDSA check
    uint32_t rb[8];       // BIP-340: r as limbs
    Fe px, py;
    if (ok) {
        uint32_t mw[8], sw[16];
        load_words8(mw, msg);
        load_words8(sw, sig);
        load_words8(sw + 8, sig + 32);
        if (kKind == 0) {
            // as ecdsa_verify_one / ecdsa_verify_rs (src/cpu/src/impl/ufsecp_ecdsa.cpp:244-272)
            words_be_to_limbs(r.v, sw);
            words_be_to_limbs(s.v, sw + 8);
            ok = !sc_is_zero(r) && limbs_lt_n(r.v) && !sc_is_zero(s) && limbs_lt_n(s.v) && sc_is_low(s.v);
            const uint8_t prefix = pub[0];
            ok = ok && (prefix == 0x02 || prefix == 0x03);
            if (ok) {
                be32_to_limbs(px.v, pub + 1);
                ok = limbs_lt_p(px.v);
            }
            if (ok) {
                const int c = cache.fetch(tab);
                have_tab = c == kKeyTable;
                ok = c != kKeyBad && (have_tab || lift_x_parity(py, px, prefix == 0x03));
            }
            if (ok) {
                Sc z, w;
                words_be_to_limbs(z.v, mw);
                sc_reduce_once(z);
                sc_inv(w, s);
                sc_mul(a, z, w);     // u1
                sc_mul(b, r, w);     // u2
            }
        } else {
            // as schnorr_verify_one (src/cpu/src/schnorr.cpp:542-612)
            uint32_t pw[8];
            load_words8(pw, pub);
            words_be_to_limbs(rb, sw);
            words_be_to_limbs(a.v, sw + 8);        // s
            ok = limbs_lt_p(rb) && !sc_is_zero(a) && limbs_lt_n(a.v);
            if (ok) {
                words_be_to_limbs(px.v, pw);
                ok = limbs_lt_p(px.v);
            }
            if (ok) {
                const int c = cache.fetch(tab);
                have_tab = c == kKeyTable;
                ok = c != kKeyBad && (have_tab || lift_x_parity(py, px, false));
            }
            if (ok) {
                uint32_t rbe[8], pbe[8], mbe[8], h[8];
                UF_UNROLL
                for (int k = 0; k < 8; ++k) {
                    rbe[k] = bswap32(sw[k]);
                    pbe[k] = bswap32(pw[k]);
                    mbe[k] = bswap32(mw[k]);
                }
                bip340_challenge(h, rbe, pbe, mbe);
                Sc e;
                UF_UNROLL
                for (int k = 0; k < 8; ++k) e.v[k] = h[7 - k];
                sc_reduce_once(e);
                sc_neg(b, e);        // R = s G - e P
            }
        }
    }
    Jac R;
    jac_set_inf(R);
    if (ok) dual_mul_half(R, a, px, py, b, tab, g, half, have_tab);
    const Jac other = shfl_partner(R);     // every lane of the warp arrives here
    if (ok && half == 0) {
        jac_add(R, other);
        ok = kKind == 0 ? ecdsa_check_x(R, r) : schnorr_check(R, rb);
    }
    return ok;
}

// Two threads per item; the grid covers 2n threads exactly (no grid-stride
// loop, so every lane of a warp reaches the shuffles once).
template <int kKind>
__global__ void __launch_bounds__(kPairThreads)
k_verify_pair(const uint8_t* __restrict__ msgs, const uint8_t* __restrict__ pubs, const uint8_t* __restrict__ sigs,
              uint32_t n, const uint4* __restrict__ gt, uint8_t* __restrict__ out, int collect) {
    extern __shared__ uint4 smem_tab[];
    const SmemTab tab{smem_tab + threadIdx.x, blockDim.x};
    const GlobalGT g{gt};
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t i = tid >> 1;
    const int half = (int)(tid & 1u);
    const bool valid = i < n;
    const uint32_t j = valid ? i : 0;      // an in-bounds index for the (unused) pointers
    const bool ok = pair_item<kKind>(msgs + 32ull * j, pubs + (kKind == 0 ? 33ull : 32ull) * j, sigs + 64ull * j,
                                     valid, half, tab, g, NoPubCache());
    if (valid && half == 0) {
        if (collect) {
            if (ok) out[i] = 0;
        } else {
            out[i] = ok ? 1 : 0;
        }
    }
}

// The work-queue form (the per-kind queues of kernels_queue.cu): each warp
// claims 16 items and verifies them with its 16 lane pairs, until its queue is
// empty.  The claim is warp-uniform, so every lane reaches the shuffles of each
// round.  With the key table (a.cache) an item's table comes from its resolved
// slot.
template <int kKind>
__global__ void __launch_bounds__(kPairThreads)
k_verify_queue_pair(QueueArgs a, const uint4* __restrict__ gt, unsigned int* __restrict__ head) {
    extern __shared__ uint4 smem_tab[];
    const SmemTab tab{smem_tab + threadIdx.x, blockDim.x};
    const GlobalGT g{gt};
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t total = kKind == 0 ? min(a.counts[0], a.cap_e) : min(a.counts[1], a.cap_s);
    const uint8_t* msgs = kKind == 0 ? a.e_msgs : a.s_msgs;
    const uint8_t* pubs = kKind == 0 ? a.e_pubs : a.s_pubs;
    const uint8_t* sigs = kKind == 0 ? a.e_sigs : a.s_sigs;
    uint8_t* out = kKind == 0 ? a.e_out : a.s_out;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(head + kKind, 16u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        const uint32_t i = base + (lane >> 1);
        const bool valid = i < total;
        const uint32_t j = valid ? i : 0;
        const uint32_t si = a.cache && valid ? (kKind == 0 ? a.e_slot : a.s_slot)[i] : kNoSlot;
        const bool ok = pair_item<kKind>(msgs + 32ull * j, pubs + (kKind == 0 ? 33ull : 32ull) * j, sigs + 64ull * j,
                                         valid, (int)(lane & 1u), tab, g,
                                         SlotPubCache{si == kNoSlot ? nullptr : a.cache + si});
        if (valid && (lane & 1u) == 0) out[i] = ok ? 1 : 0;
    }
}

}  // namespace

cudaError_t launch_verify_pair(int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs, uint32_t n,
                               const void* d_gtab, uint8_t* out, int collect, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t smem = kPairThreads * kVerifySmemPerThread;
    const uint64_t threads = 2ull * n;
    const int grid = (int)((threads + kPairThreads - 1) / kPairThreads);
    const uint4* gt = reinterpret_cast<const uint4*>(d_gtab);
    if (kind == 0)
        k_verify_pair<0><<<grid, kPairThreads, smem, s>>>(msgs, pubs, sigs, n, gt, out, collect);
    else
        k_verify_pair<1><<<grid, kPairThreads, smem, s>>>(msgs, pubs, sigs, n, gt, out, collect);
    return cudaGetLastError();
}

cudaError_t launch_verify_queue_pair(const QueueArgs& a, const void* d_gtab, unsigned int* d_head, int grid,
                                     cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join) {
    const size_t smem = kPairThreads * kVerifySmemPerThread;
    if (grid <= 0) grid = 1;
    const uint4* gt = reinterpret_cast<const uint4*>(d_gtab);
    cudaError_t e = cudaMemsetAsync(d_head, 0, 2 * sizeof(unsigned int), s);
    if (e != cudaSuccess) return e;
    if ((e = launch_key_passes(a, grid, s)) != cudaSuccess) return e;
    const bool both = a.cap_e > 0 && a.cap_s > 0;
    if (both) {
        if ((e = cudaEventRecord(fork, s)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s2, fork, 0)) != cudaSuccess) return e;
    }
    if (a.cap_e > 0) k_verify_queue_pair<0><<<grid, kPairThreads, smem, s>>>(a, gt, d_head);
    if (a.cap_s > 0) k_verify_queue_pair<1><<<grid, kPairThreads, smem, both ? s2 : s>>>(a, gt, d_head);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (both) {
        if ((e = cudaEventRecord(join, s2)) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, join, 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Opts the two-lane kernels in to their dynamic shared memory; returns the
// smallest resident-block count per SM among them (the queue form's grid).
int verify_pair_occupancy() {
    const size_t smem = kPairThreads * kVerifySmemPerThread;
    int lo = 1 << 30;
    auto probe = [&](auto f) {
        int blocks = 0;
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, f, kPairThreads, smem);
        lo = blocks < lo ? blocks : lo;
    };
    probe(k_verify_pair<0>);
    probe(k_verify_pair<1>);
    probe(k_verify_queue_pair<0>);
    probe(k_verify_queue_pair<1>);
    return lo;
}

}  // namespace uf
