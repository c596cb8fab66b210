// Launch wrappers for the sm_100a kernels (C++ linkage, used by the backend).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "common.cuh"
#include "ufsecp/ufsecp_gpu_ext.h"

namespace uf {

// Byte size of the per-context generator tables: 2^(UF_GWIN-1) multiples of G
// and of lambda*G, affine, 64 bytes each.
constexpr size_t kGTableEntries = size_t{1} << (UF_GWIN - 1);   // per table (G, lambda G)
constexpr size_t kGTableBytes = 2 * kGTableEntries * 64;

// Threads per block of the per-signature verify kernels and the dynamic
// shared memory each block needs (8 table points x 64 bytes per thread).
constexpr int kVerifyThreads = 128;
constexpr size_t kVerifySmemPerThread = 8 * 64;

cudaError_t launch_gtable_init(void* d_gtab, cudaStream_t s);
// The same tables for wbits-bit windows (2^(wbits-1) multiples each, 2^wbits * 64 bytes).
cudaError_t launch_gtable_init_w(void* d_gtab, int wbits, cudaStream_t s);

// One signature per thread, grid-stride.  kind 0 = ECDSA (pubs: 33-byte SEC1
// compressed), 1 = BIP-340 (pubs: 32-byte x-only).  msgs 32 B, sigs 64 B, all
// contiguous; msgs / x-only pubs / sigs must be 16-byte aligned.  out[i] = 1
// for a valid signature, 0 otherwise.  With collect != 0 a valid signature
// writes 0 and an invalid one leaves out[i] untouched.  Variants 0..5 are the
// same kernel built with different code-size choices (kernels_verify.cu).
constexpr int kVerifyVariants = 12;
// G-window bits of each variant's generator tables (9: 3-bit P / 18-bit G
// windows, 10: 5-bit P, 11: 16-bit G; the others 4 / UF_GWIN).
constexpr int kVariantGWin[kVerifyVariants] = {UF_GWIN, UF_GWIN, UF_GWIN, UF_GWIN, UF_GWIN, UF_GWIN,
                                               UF_GWIN, UF_GWIN, UF_GWIN, 18, UF_GWIN, 16};
constexpr int kVariantPWin[kVerifyVariants] = {4, 4, 4, 4, 4, 4, 4, 4, 4, 3, 5, 4};
typedef cudaError_t (*verify_launcher)(int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs,
                                       uint32_t n, const void* d_gtab, uint8_t* out, int collect, int grid,
                                       cudaStream_t s);
typedef int (*verify_occupancy_fn)(int kind);
cudaError_t launch_verify_v0(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v1(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v2(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v3(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v4(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v5(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v6(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v7(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v8(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
int verify_occupancy_v0(int kind);
int verify_occupancy_v1(int kind);
int verify_occupancy_v2(int kind);
int verify_occupancy_v3(int kind);
int verify_occupancy_v4(int kind);
int verify_occupancy_v5(int kind);
int verify_occupancy_v6(int kind);
int verify_occupancy_v7(int kind);
int verify_occupancy_v8(int kind);
cudaError_t launch_verify_v9(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                             int, int, cudaStream_t);
cudaError_t launch_verify_v10(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                              int, int, cudaStream_t);
cudaError_t launch_verify_v11(int, const uint8_t*, const uint8_t*, const uint8_t*, uint32_t, const void*, uint8_t*,
                              int, int, cudaStream_t);
int verify_occupancy_v9(int kind);
int verify_occupancy_v10(int kind);
int verify_occupancy_v11(int kind);

// The same verify with block-wide batch inversion (kernels_verify_grp.cu):
// the table, final-Z and ECDSA s inversions are shared by the `group` (64 or
// 128) threads of a block.  `grid` resident blocks from verify_grp_occupancy,
// which also opts the kernels in to their shared memory.
cudaError_t launch_verify_grp(int group, int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs,
                              uint32_t n, const void* d_gtab, uint8_t* out, int collect, int grid, cudaStream_t s);
int verify_grp_occupancy(int group, int kind);

// Per-item batch operations (kernels_ops.cu); device pointers, asynchronous.
cudaError_t launch_xonly_validate(const uint8_t* keys32, uint32_t n, uint8_t* out, int sms, cudaStream_t s);
cudaError_t launch_pubkey_validate(const uint8_t* pubs33, uint32_t n, uint8_t* out, int sms, cudaStream_t s);
cudaError_t launch_commitment_verify(const uint8_t* internal_x, const uint8_t* tweak, const uint8_t* tweaked_x,
                                     const uint8_t* parity, uint32_t n, const void* d_gtab, uint8_t* out, int sms,
                                     cudaStream_t s);
cudaError_t launch_tagged_hash(const uint8_t tag_hash[32], const uint8_t* msgs, const uint32_t* lens,
                               uint32_t fixed_len, uint32_t stride, uint32_t n, uint8_t* out32, int sms,
                               cudaStream_t s);

// Mixed-batch staging layout shared by host (pinned) and device buffers:
//   [header 256 B: n_e, n_s, to-do count][e_msgs cap_e*32][s_msgs cap_s*32]
//   [e_sigs cap_e*64][s_sigs cap_s*64][s_pubs cap_s*32][e_pubs cap_e*33]
//   [e_out cap_e][s_out cap_s]
// then, on the device only, the key table's per-launch scratch:
//   [e_slot cap_e*4][s_slot cap_s*4][todo (cap_e+cap_s)*4]
// Every region starts 256-byte aligned.  in_bytes covers header + inputs (one
// host->device copy), out_bytes the verdicts (one device->host copy),
// host_bytes the pinned staging, total the device buffer.
struct QueueLayout {
    uint32_t cap_e = 0, cap_s = 0;
    size_t e_msgs, s_msgs, e_sigs, s_sigs, s_pubs, e_pubs, e_out, s_out, e_slot, s_slot, todo, in_bytes, out_bytes,
        host_bytes, total;
    static size_t up(size_t x) { return (x + 255) & ~size_t{255}; }
    QueueLayout() = default;
    QueueLayout(uint32_t ce, uint32_t cs) : cap_e(ce), cap_s(cs) {
        e_msgs = 256;
        s_msgs = up(e_msgs + (size_t)ce * 32);
        e_sigs = up(s_msgs + (size_t)cs * 32);
        s_sigs = up(e_sigs + (size_t)ce * 64);
        s_pubs = up(s_sigs + (size_t)cs * 64);
        e_pubs = up(s_pubs + (size_t)cs * 32);
        e_out = up(e_pubs + (size_t)ce * 33);
        s_out = up(e_out + (size_t)ce);
        e_slot = up(s_out + (size_t)cs);
        s_slot = up(e_slot + (size_t)ce * 4);
        todo = up(s_slot + (size_t)cs * 4);
        total = up(todo + ((size_t)ce + cs) * 4);
        in_bytes = e_out;
        out_bytes = e_slot - e_out;
        host_bytes = e_slot;
    }
};

struct PubCacheSlot;
struct QueueArgs {
    const uint32_t* counts;  // device header: n_e, n_s, to-do count
    uint32_t cap_e, cap_s;   // region capacities: the kernel never reads past them
    const uint8_t *e_msgs, *e_pubs, *e_sigs, *s_msgs, *s_pubs, *s_sigs;
    uint8_t *e_out, *s_out;
    // optional resident key table (pubcache.cuh): slots, slot count - 1, two
    // counters (lookups, hits); the launch's per-item slot indices and to-do
    // list (device-only regions of the layout) and its to-do counter (header
    // word 2, zeroed by the host copy); null cache = no table
    PubCacheSlot* cache = nullptr;
    uint32_t cache_mask = 0;
    unsigned long long* cache_stats = nullptr;
    uint32_t *e_slot = nullptr, *s_slot = nullptr, *todo = nullptr, *todo_count = nullptr;
};
constexpr size_t kPubCacheSlotBytes = 576;

// Zeroes the two queue heads (d_head[0] ECDSA, d_head[1] BIP-340), then
// launches the per-kind persistent queue kernels (`grid` resident blocks
// each) over the items described by `a`: kinds with capacity 0 are skipped;
// with both kinds, the BIP-340 kernel runs on s2 between a fork event recorded
// on s and a join event s waits for (kernels_queue.cu).  With a key table
// (a.cache) the resolve and build passes (pubcache.cuh) run first, on s.
cudaError_t launch_verify_queue(const QueueArgs& a, const void* d_gtab, unsigned int* d_head, int grid,
                                cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join);
int verify_queue_occupancy();
// The key table's resolve and build passes alone (launch_verify_queue and
// launch_verify_queue_pair call it when a.cache is set); `grid` resident blocks
// for the build pass.
cudaError_t launch_key_passes(const QueueArgs& a, int grid, cudaStream_t s);

// Two lanes per signature (kernels_pair.cu), kind 0 ECDSA (compact) or 1
// BIP-340, for small calls; verify_pair_occupancy() also opts the kernels in
// to their shared memory (call once per device).
cudaError_t launch_verify_pair(int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs, uint32_t n,
                               const void* d_gtab, uint8_t* out, int collect, cudaStream_t s);
int verify_pair_occupancy();
// The work-queue form of the two-lane kernels (no key cache), same contract as
// launch_verify_queue; `grid` from verify_pair_occupancy().
cudaError_t launch_verify_queue_pair(const QueueArgs& a, const void* d_gtab, unsigned int* d_head, int grid,
                                     cudaStream_t s, cudaStream_t s2, cudaEvent_t fork, cudaEvent_t join);

// Allocation-free mixed verification (kernels_noalloc.cu): the jobs' buffers
// are device-accessible memory the caller owns; the queue head and the job
// table live in a static device array of the library (kNoAllocScratchBytes,
// 49,408 bytes), nothing is allocated.  The descriptor table is built
// straight into a per-thread staging array (no large stack frame).  On a
// failed launch every job's verdict bytes are cleared with cudaMemsetAsync.
constexpr size_t kNoAllocJobLimit = 1024;
constexpr size_t kNoAllocHeaderBytes = 256;
constexpr size_t kNoAllocJobBytes = 48;
constexpr size_t kNoAllocScratchBytes = kNoAllocHeaderBytes + kNoAllocJobLimit * kNoAllocJobBytes;
cudaError_t verify_jobs_noalloc(int device, const ufsecp_gpu_ext_job_t* jobs, size_t n_jobs, const void* d_gtab,
                                cudaStream_t s, int* limit_hit);

// Batch signer (workload generator): kind 0 = ECDSA (pubs 33 B), 1 = BIP-340
// (pubs 32 B x-only, auxs 32 B aux_rand).  ok[i] = 0 for an invalid key.
cudaError_t launch_sign(int kind, const uint8_t* msgs, const uint8_t* sks, const uint8_t* auxs, uint32_t n,
                        const void* d_gtab, uint8_t* pubs, uint8_t* sigs, uint8_t* ok, int grid, cudaStream_t s);

// Building-block probes for the tests (op codes in ufsecp_gpu_ext.h).
cudaError_t launch_diag(uint32_t op, const uint8_t* in, uint32_t n, uint8_t* out,
                        const void* d_gtab, cudaStream_t s);

// Field multiply / square / add / sub as the verify kernels compile them
// (diag op 11): a | b (64 B) -> a*b | a^2 | a+b | a-b | 4a | 8a (192 B, normalized).
cudaError_t launch_field_diag(const uint8_t* in, uint32_t n, uint8_t* out, int sms, cudaStream_t s);

// Integer multiply-add issue-rate probe: every thread runs `iters` rounds of
// 16 independent 32-bit IMADs.  Returns a checksum so the work is not elided.
cudaError_t launch_imad_peak(uint32_t* d_sink, int blocks, int threads, int iters, cudaStream_t s);

// Building-block throughput probe (op codes in ufsecp_gpu_ext.h), one per
// verify-kernel variant.
typedef cudaError_t (*probe_launcher)(int op, int blocks, int threads, int iters, uint32_t* sink, cudaStream_t s);
cudaError_t launch_probe_v0(int, int, int, int, uint32_t*, cudaStream_t);
cudaError_t launch_probe_v1(int, int, int, int, uint32_t*, cudaStream_t);
cudaError_t launch_probe_v2(int, int, int, int, uint32_t*, cudaStream_t);
cudaError_t launch_probe_v3(int, int, int, int, uint32_t*, cudaStream_t);
cudaError_t launch_probe_v4(int, int, int, int, uint32_t*, cudaStream_t);
cudaError_t launch_probe_v5(int, int, int, int, uint32_t*, cudaStream_t);
cudaError_t launch_probe_v6(int, int, int, int, uint32_t*, cudaStream_t);
cudaError_t launch_probe_v7(int, int, int, int, uint32_t*, cudaStream_t);
cudaError_t launch_probe_v8(int, int, int, int, uint32_t*, cudaStream_t);

}  // namespace uf
