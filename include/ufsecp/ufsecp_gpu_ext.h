/* ufsecp_gpu_ext.h -- B200 extensions of the verify ABI (additive).
 *
 * These entry points have no counterpart in the reference header; they expose
 * what a B200 deployment needs beyond the synchronous host-buffer calls of
 * ufsecp_gpu.h: verification over buffers already resident in device memory
 * (asynchronous on a caller stream), the context's stream for event timing,
 * and probes used by the test-suite and the benchmark.  All of them use the
 * same context and error codes as ufsecp_gpu.h. */
#ifndef UFSECP_GPU_EXT_H
#define UFSECP_GPU_EXT_H

#include "ufsecp_gpu.h"
#include "ufsecp_cancel.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Device-resident verify.  All pointers are device pointers (cudaMalloc or
 * torch CUDA storage) of the same layout as the host calls; msgs, x-only keys
 * and signatures must be 16-byte aligned.  The launch is enqueued on `stream`
 * (a cudaStream_t; NULL = the context's stream) and the call returns without
 * waiting; d_out[i] = 1 / 0 once the stream reaches that point.  Calls of at
 * least 262,144 items are cut into launches of 131,072 that alternate between
 * `stream` and a second stream forked from it and joined back into it, so one
 * launch's last partial wave overlaps the next; the work stays ordered on
 * `stream`. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_ecdsa_verify_device(ufsecp_gpu_ctx* ctx, const uint8_t* d_msg_hashes32,
                                                             const uint8_t* d_pubkeys33, const uint8_t* d_sigs64,
                                                             size_t count, uint8_t* d_out_results, void* stream);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_schnorr_verify_device(ufsecp_gpu_ctx* ctx, const uint8_t* d_msg_hashes32,
                                                               const uint8_t* d_pubkeys_x32, const uint8_t* d_sigs64,
                                                               size_t count, uint8_t* d_out_results, void* stream);

/* Mixed ECDSA / BIP-340 batches in one launch.  Each job is one caller batch
 * with the layouts of ufsecp_gpu_ecdsa_verify_batch (kind 0: 33-byte
 * compressed keys) or ufsecp_gpu_schnorr_verify_batch (kind 1: 32-byte x-only
 * keys), host buffers.  All jobs are packed into pinned staging and verified
 * by one persistent work-queue kernel (warps claim 32-item chunks from a
 * device queue head); layouts up to 65,536 items per kind replay a CUDA graph
 * captured per capacity bucket.  Synchronous, like the reference calls; the
 * verdicts equal those of the per-kind calls item for item.  Kind 2 is
 * BIP-340 (the kind 1 layouts) checked by random linear combination: all
 * kind 2 items of the call are verified by one RLC batch verify (the
 * ufsecp_gpu_ext_schnorr_verify_rlc engine, locate step and bisection down to
 * per-item verdicts, weights seeded by a digest of the items XOR fresh random
 * bytes) in segments of `reserved` items (0 = 16384), after the kind 0 / 1
 * jobs; for batches expected to be (nearly) all valid, where one MSM check
 * per segment replaces the per-signature verifies.  Its verdicts equal the
 * per-signature verify's.  Gating as the reference ABI: NULL ctx ->
 * NULL_ARG, no jobs -> OK, every out buffer is cleared first, NULL buffers of
 * a non-empty job -> NULL_ARG, kind > 2 or a total above 2^26 -> BAD_INPUT.
 * ufsecp_gpu_ext_verify_jobs_noalloc and the serving loop take kinds 0 and 1
 * only. */
typedef struct {
    uint32_t kind;                /* 0 = ECDSA, 1 = BIP-340, 2 = BIP-340 by RLC */
    uint32_t reserved;            /* kind 2: RLC segment length (0 = 16384); else 0 */
    size_t count;
    const uint8_t* msg_hashes32;  /* count * 32 */
    const uint8_t* pubkeys;       /* count * 33 (ECDSA) or count * 32 (BIP-340) */
    const uint8_t* sigs64;        /* count * 64 */
    uint8_t* out_results;         /* count bytes: 1 valid, 0 invalid */
} ufsecp_gpu_ext_job_t;

UFSECP_API ufsecp_error_t ufsecp_gpu_ext_verify_jobs(ufsecp_gpu_ctx* ctx, const ufsecp_gpu_ext_job_t* jobs,
                                                     size_t n_jobs);

/* One host-buffer batch over several contexts (no reference counterpart):
 * the items are cut into n_ctx contiguous shares (the first count % n_ctx
 * shares one item longer), each verified on its own context, in its own host
 * thread, by ufsecp_gpu_ecdsa_verify_batch (kind 0, 33-byte keys) or
 * ufsecp_gpu_schnorr_verify_batch (kind 1, 32-byte x-only keys).  Verdicts
 * are per item, so no data crosses between devices; with one context per GPU
 * the shares run on all of them at once.  The contexts must be distinct and
 * not used by other threads during the call.  Gating as the single-context
 * calls: NULL ctxs or a NULL context -> NULL_ARG, count 0 -> OK, n_ctx 0, a
 * context listed twice, kind > 1 or count > 2^26 -> BAD_INPUT; the verdict
 * buffer is cleared first and again after any share fails, whose code is
 * returned (the first failing share's). */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_verify_batch_sharded(ufsecp_gpu_ctx* const* ctxs, size_t n_ctx,
                                                              uint32_t kind, const uint8_t* msg_hashes32,
                                                              const uint8_t* pubkeys, const uint8_t* sigs64,
                                                              size_t count, uint8_t* out_results);

/* Host-side fault injection, for testing fail-closed behaviour (no
 * reference counterpart; nothing faults on the device).  Once armed, the
 * (after + 1)-th fault point the context crosses fails, and the injector
 * disarms itself: kind 1 as if a CUDA call returned cudaErrorMemoryAllocation
 * (UFSECP_ERR_GPU_MEMORY), 2 as if a launch returned cudaErrorLaunchFailure
 * (UFSECP_ERR_GPU_LAUNCH), 3 as if the host ran out of memory (std::bad_alloc,
 * UFSECP_ERR_GPU_MEMORY); kind 0 disarms.  Fault points: every chunk launch
 * of the host-buffer verify calls, every device-buffer verify call, every
 * mixed-job or served launch and every RLC round.  The failing step is not
 * made; the call returns the error with its result bytes cleared. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_inject_fault(ufsecp_gpu_ctx* ctx, uint32_t after, int kind);

/* Resident key table of ufsecp_gpu_ext_verify_jobs (no reference
 * counterpart).  Per distinct public key (x, parity) a device slot keeps the
 * decompressed key's 1P..8P table, so a key seen before skips its square root,
 * table additions and the table's inversion; an x off the curve is remembered
 * as such.  Before the verify kernels, a resolve pass gives each item its key's
 * slot and a build pass fills the new slots, so the verify warps never mix
 * lanes that build a table with lanes that copy one.  Verdicts never depend on
 * the table.  log2_slots: 0 = off; 8..24 = an empty table of 2^log2_slots
 * slots of 576 bytes (a table of that size is emptied in place, another size
 * is made on the next verify_jobs call).  Default: 18
 * (151 MB), from the tuning file's key_table_log2 or the environment
 * variable UFSECP_B200_KEY_TABLE when set.  Slots are never evicted: when a
 * key's probe window is full it is verified without the table.
 * key_table_stats: out[0] lookups (items whose key parsed) and out[1] hits
 * (items whose key already had a slot, claimed by an earlier item) since the
 * table was made, out[2] its slot count (0 = off or not made yet). */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_set_key_table(ufsecp_gpu_ctx* ctx, uint32_t log2_slots);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_key_table_stats(ufsecp_gpu_ctx* ctx, uint64_t out[3]);

/* Allocation-free variant of ufsecp_gpu_ext_verify_jobs, for callers that
 * cannot call cudaMalloc (GPU memory owned by another allocator or framework,
 * a fixed device-memory budget, or a policy that the verifier must not
 * allocate).  No counterpart in the reference.  The jobs' buffers are DEVICE
 * (device-accessible) memory the caller owns: msgs / signatures / x-only keys
 * 16-byte aligned, outputs one byte per item.  The call allocates nothing: the
 * work-queue kernel's scratch (queue head and job table, 49,408 bytes) is a
 * static device array of the library, at most UFSECP_GPU_EXT_NOALLOC_MAX_JOBS
 * jobs per call (more -> UFSECP_ERR_BAD_INPUT with an explanatory
 * last_error_msg).  The first call on a device looks up that array's device
 * address; make that first call before any stream capture.  The job table is
 * copied to the device from the library's own pageable host staging, so the
 * call may wait until those bytes are staged; it then enqueues the kernel on
 * `stream` (NULL = the context's stream) and returns; the verdicts are ready
 * when the stream reaches that point.  If the copy or the launch fails, every
 * job's verdict bytes are cleared on `stream` and the error is returned.  All
 * calls share the array and the queue head is reset by every call, so calls
 * whose work overlaps on the GPU race: serialise them (one stream, or wait for
 * the previous call). */
#define UFSECP_GPU_EXT_NOALLOC_MAX_JOBS 1024
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_verify_jobs_noalloc(ufsecp_gpu_ctx* ctx, const ufsecp_gpu_ext_job_t* jobs,
                                                             size_t n_jobs, void* stream);

/* BIP-340 batch verification by random linear combination (RLC).
 * Counterpart of the reference's CPU batch verify (schnorr_batch_verify,
 * src/cpu/src/batch_verify.cpp:324-424) with per-item verdicts: the items are
 * cut into batches of batch_size (0 = one batch, the last batch ragged); every
 * batch is checked by ONE multi-scalar multiplication
 *     sum a_i R_i + sum (a_i e_i) P_i - (sum a_i s_i) G == infinity
 * with 128-bit weights a_i = SHA-256(seed32 || le32 i)[0:16] (never 0);
 * failing batches are bisected and small failing pieces verified one by one,
 * so out_results[i] equals ufsecp_gpu_schnorr_verify_batch's verdict for every
 * item (a false accept needs a 2^-128 event).  out_batch_ok (may be NULL)
 * receives one byte per batch: 1 when all its items are valid.  window_bits:
 * 0 = chosen per batch length, else 4..16 (Pippenger window).  seed32 should
 * be unpredictable to whoever produced the signatures.  Up to 2^24 items per
 * call.  Host buffers, synchronous; the _device form takes 16-byte aligned
 * device buffers and runs on `stream` (NULL = the context's stream), returning
 * when the verdicts are written (it reads each round's result on the host). */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_schnorr_verify_rlc(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                            const uint8_t* pubkeys_x32, const uint8_t* sigs64,
                                                            size_t count, size_t batch_size, const uint8_t* seed32,
                                                            int window_bits, uint8_t* out_results,
                                                            uint8_t* out_batch_ok);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_schnorr_verify_rlc_device(ufsecp_gpu_ctx* ctx, const uint8_t* d_msg_hashes32,
                                                                   const uint8_t* d_pubkeys_x32,
                                                                   const uint8_t* d_sigs64, size_t count,
                                                                   size_t batch_size, const uint8_t* seed32,
                                                                   int window_bits, uint8_t* d_out_results,
                                                                   uint8_t* out_batch_ok, void* stream);
/* Counters of the context's last RLC call: out[0] MSM rounds (the first check,
 * one per bisection level and one per locate step), out[1] segments checked
 * (locate rounds included), out[2] items verified one by one (bisection
 * leaves and locate candidates), out[3] window bits of the first round.
 * rlc_located: failing segments the locate step resolved. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_rlc_stats(ufsecp_gpu_ctx* ctx, uint64_t out[4]);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_rlc_located(ufsecp_gpu_ctx* ctx, uint64_t* located);
/* Items of the last RLC call whose x-only key was resident in the context's
 * key table (ufsecp_gpu_ext_set_key_table; keys enter it through
 * ufsecp_gpu_ext_verify_jobs): their lift_x square root was skipped. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_rlc_key_hits(ufsecp_gpu_ctx* ctx, uint64_t* hits);

/* Locate step of RLC verification (on = 1, the default; 0 = bisection only).
 * A failing batch S with sum T = sum a_i D_i != infinity (D_i = R_i + e_i P_i
 * - s_i G, infinity exactly for a valid item) first gets one more
 * multi-scalar multiplication with every weight a_i multiplied by its position
 * j_i = i - start + 1, T' = sum j_i a_i D_i.  With one invalid item j,
 * T' = j T, and a baby-step giant-step search over the multiples 1 .. |S| of T
 * (one block per segment) finds j; the candidate is verified by the plain
 * kernel and, when invalid, resolves S in two rounds instead of one per
 * bisection level.  With two or more invalid items no multiple matches (but
 * for a 2^-128 event over the weights) and S is bisected as before; verdicts
 * never depend on the search.  Segments of at most 65,535 items. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_set_rlc_locate(ufsecp_gpu_ctx* ctx, int on);

/* Input binding of the reference-shaped batch API's seed: the SHA-256 tree
 * digest of n BIP-340 items (host buffers, layouts as above).  Per item
 * d_i = SHA-256(r || s || x(P) || m) (the 128 bytes the reference hashes per
 * entry, src/cpu/src/batch_verify.cpp:361-369); then, while more than one
 * digest remains, groups of 16 consecutive digests are replaced by the
 * SHA-256 of their concatenation (a short last group hashes what it has);
 * out32 = SHA-256(root || le32 n).  ufsecp_gpu_ext_schnorr_batch_verify and
 * _identify_invalid take their RLC seed as this digest XOR 32 fresh random
 * bytes, as the reference mixes its input hash with CSPRNG bytes (:355-380). */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_rlc_input_digest(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                          const uint8_t* pubkeys_x32, const uint8_t* sigs64,
                                                          size_t count, uint8_t out32[32]);

/* The reference's batch API on the GPU, same rows, gating and results:
 * ufsecp_schnorr_batch_verify (src/cpu/src/impl/ufsecp_taproot.cpp:703) and
 * ufsecp_schnorr_batch_identify_invalid (:849).  Rows are [x-only key 32 |
 * msg 32 | sig 64] = 128 bytes, n <= 2^20.  The first row (in index order)
 * with x >= p returns UFSECP_ERR_BAD_PUBKEY, with r >= p or s outside [1, n-1]
 * UFSECP_ERR_BAD_SIG.  batch_verify returns UFSECP_OK when every row is valid
 * and UFSECP_ERR_VERIFY_FAIL otherwise; identify_invalid writes the indices
 * of the invalid rows, ascending (at most *invalid_count of them), and sets
 * *invalid_count to their total.  One RLC batch of all rows with a fresh
 * random seed, bisected on failure. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_schnorr_batch_verify(ufsecp_gpu_ctx* ctx, const uint8_t* entries, size_t n);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_schnorr_batch_identify_invalid(ufsecp_gpu_ctx* ctx, const uint8_t* entries,
                                                                        size_t n, size_t* invalid_out,
                                                                        size_t* invalid_count);

/* Serving loop: continuous batching of verify requests (no counterpart in the
 * reference, which serves one synchronous call per batch).  A request is one
 * or more jobs (ECDSA and / or BIP-340, host buffers, layouts as above).
 * submit() returns at once with an id; a scheduler thread packs the oldest
 * pending requests into persistent-queue launches on `slots` streams as soon
 * as a slot and the memory budget allow (up to max_launch_items items per
 * launch; larger requests ride in several launches), so work that arrives
 * while other launches run overlaps with them on the device.  The request's
 * buffers must stay valid until wait() on its id returned UFSECP_OK; its
 * verdicts are then in out_results and equal the per-kind verify calls' for
 * every item, whatever it was batched with.  wait() returns
 * UFSECP_ERR_GPU_QUEUE on timeout (the request stays pending).  While a server
 * runs, its context belongs to the server's thread: make no other call on that
 * context.  Destroy the server (it finishes the pending requests) before the
 * context.  With key_cache_log2 set, decompressed keys with their 1P..8P
 * tables stay resident in a device key table shared by the slots (the design
 * of ufsecp_gpu_ext_set_key_table), so a key seen before skips its square
 * root, table additions and inversion (verdicts are unchanged).  The memory
 * budget covers the slots' fixed staging (pinned + device) and the key table,
 * reserved at creation (fewer slots are made if they do not fit), plus the
 * staged bytes of the items in flight; pending requests wait for room.
 * Config NULL = defaults: 8 slots, 65,536 items per launch, an 8 GiB budget,
 * no batch window, a key table of 2^18 slots. */
typedef struct ufsecp_gpu_ext_server ufsecp_gpu_ext_server;
typedef struct {
    uint32_t slots;                 /* streams / launches in flight, 1..64 */
    uint32_t max_launch_items;      /* 1..65536 */
    uint64_t memory_budget_bytes;
    uint32_t batch_window_us;       /* 0: launch as soon as a slot is free */
    uint32_t key_cache_log2;        /* resident key table of 2^k slots, 576 B each:
                                       0 or 1 = none, else 8..24 (NULL config: 18) */
} ufsecp_gpu_ext_server_config_t;
typedef struct {
    uint64_t requests_done, items_done, launches;
    uint64_t peak_budget_bytes;               /* slot staging + item bytes in flight, <= the budget */
    uint64_t reserved_bytes;                  /* the slots' fixed staging (pinned + device) */
    uint64_t pending_requests;
    uint32_t peak_slots_in_flight, reserved;
    double p50_us, p99_us, max_us, mean_us;   /* submit -> verdicts written, completed requests */
    double busy_s, span_s;                    /* time with a launch in flight; first submit -> last completion */
    uint64_t cache_lookups, cache_hits;       /* resident key cache since creation */
} ufsecp_gpu_ext_server_stats_t;

UFSECP_API ufsecp_error_t ufsecp_gpu_ext_server_create(ufsecp_gpu_ctx* ctx,
                                                       const ufsecp_gpu_ext_server_config_t* config,
                                                       ufsecp_gpu_ext_server** server_out);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_server_submit(ufsecp_gpu_ext_server* server,
                                                       const ufsecp_gpu_ext_job_t* jobs, size_t n_jobs,
                                                       uint64_t* request_id);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_server_wait(ufsecp_gpu_ext_server* server, uint64_t request_id,
                                                     uint32_t timeout_ms);
/* Cancellation (the token type is the reference's, include/ufsecp/ufsecp_cancel.h).
 * submit_cancellable: as submit, with a token (may be NULL; copied) that the
 * scheduler polls before every launch that would take a piece of the request;
 * once it answers non-zero no further piece is launched, pieces already on
 * the device finish, and the request ends with UFSECP_ERR_CANCELLED, its
 * verdict bytes cleared (wait() returns that code).  The predicate runs on
 * the server's scheduler thread and must not call into the server.
 * cancel: abandons a request, typically after wait() timed out.  Pieces not
 * launched yet are dropped; pieces on the device finish (a kernel is not
 * stopped) and cancel waits for them, at most timeout_ms.  UFSECP_OK: the
 * server has forgotten the request and touches its buffers no more, so the
 * caller may free them; the verdict bytes are cleared unless the request had
 * completed before the call.  UFSECP_ERR_GPU_QUEUE: pieces were still on the
 * device at the timeout (nothing more is launched for it; call cancel or wait
 * again before freeing the buffers).  UFSECP_ERR_BAD_INPUT: unknown id.  A
 * request that fails on the GPU ends with its error code and its verdict
 * bytes cleared as well (fail closed). */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_server_submit_cancellable(ufsecp_gpu_ext_server* server,
                                                                   const ufsecp_gpu_ext_job_t* jobs, size_t n_jobs,
                                                                   const ufsecp_cancel_token* cancel,
                                                                   uint64_t* request_id);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_server_cancel(ufsecp_gpu_ext_server* server, uint64_t request_id,
                                                       uint32_t timeout_ms);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_server_stats(ufsecp_gpu_ext_server* server,
                                                      ufsecp_gpu_ext_server_stats_t* out, int reset);
UFSECP_API void ufsecp_gpu_ext_server_destroy(ufsecp_gpu_ext_server* server);

/* Engine hook provider: the GPU side of the reference engine's column-verify
 * accelerator hook (secp256k1::GpuColumnsVerifyHook,
 * src/cpu/include/secp256k1/batch_verify.hpp:143-168; the reference's own
 * provider is src/gpu/src/gpu_engine_hook.cpp:81-104).  Same signature and
 * return contract: kind 0 = ECDSA opaque little-endian columns (keys =
 * compressed pubkeys), kind 1 = BIP-340 columns (keys = x-only); returns 1 when
 * every row is valid, 0 when at least one is invalid (out_results fully
 * written), -1 to decline (no CUDA device, bad arguments or any GPU error) so
 * that the engine runs its CPU path.  Uses one process-wide context on device
 * 0, created on first use and serialised by a mutex.  Install it with
 * secp256k1::install_gpu_columns_verify_hook(&ufsecp_gpu_ext_engine_columns_hook). */
UFSECP_API int ufsecp_gpu_ext_engine_columns_hook(int kind, const uint8_t* digests32, const uint8_t* keys,
                                                  const uint8_t* sigs64, size_t count,
                                                  uint8_t* out_results) UFSECP_NOEXCEPT;
/* Arms host-side fault injection on the hook's process-wide context (made here
 * if needed), as ufsecp_gpu_ext_inject_fault does for a caller's context:
 * the hook then declines the failing call and the engine answers on its CPU
 * path.  UFSECP_ERR_GPU_UNAVAILABLE without a device. */
UFSECP_API int ufsecp_gpu_ext_engine_hook_inject_fault(uint32_t after, int kind);
/* Calls the hook handled on the GPU / declined, since load. */
UFSECP_API void ufsecp_gpu_ext_engine_hook_counters(uint64_t* handled, uint64_t* declined);
/* Destroys the hook's process-wide context (the next call creates it again). */
UFSECP_API void ufsecp_gpu_ext_engine_hook_release(void);

/* Batch signing for synthetic workloads (device pointers, asynchronous on
 * `stream`): kind 0 = ECDSA, RFC 6979 nonce, low-S compact r||s, 33-byte
 * compressed pubkeys out; kind 1 = BIP-340 with aux_rand (d_aux32), 32-byte
 * x-only pubkeys out.  d_ok[i] = 0 when sk[i] is 0 or >= n.  Output bytes are
 * those of the reference's CPU signers ufsecp_ecdsa_sign / ufsecp_schnorr_sign. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_sign_device(ufsecp_gpu_ctx* ctx, uint32_t kind, const uint8_t* d_msgs32,
                                                     const uint8_t* d_privkeys32, const uint8_t* d_aux32,
                                                     size_t count, uint8_t* d_pubkeys_out, uint8_t* d_sigs64_out,
                                                     uint8_t* d_ok, void* stream);

/* The context's own stream (cudaStream_t), on which every host-buffer call of
 * ufsecp_gpu.h enqueues its copies and kernels. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_stream(ufsecp_gpu_ctx* ctx, void** stream_out);

/* SM count of the context's device, and blocks per SM the ECDSA (kind 0) /
 * BIP-340 (kind 1) verify kernels reach. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_device_props(ufsecp_gpu_ctx* ctx, int* sm_count, int* ecdsa_blocks_per_sm,
                                                      int* schnorr_blocks_per_sm);

/* Verify-kernel variant per signature kind (0 ECDSA, 1 BIP-340).  The
 * variants compute the same verdicts; 0..8 differ in how much of the field /
 * point arithmetic is inlined (instruction-cache footprint vs. call overhead),
 * 9..11 in window widths with variant 4's code: 9 = 3-bit P windows (a 4-entry
 * table) with 18-bit G windows, 10 = 5-bit P windows (16 entries), 11 = 16-bit
 * G windows (the default is 4-bit P and 20-bit G windows); the generator
 * tables of another G width (16 / 4 MB) are made when such a variant is chosen.
 * ultrafastsecp256k1_b200.autotune measures them and writes the tuning file
 * read at context creation (UFSECP_B200_TUNING).  The tuning may also name a
 * small-launch variant per kind, used by verify calls of at most `items`
 * items (latency-bound launches with a few warps per SM, where inlining the
 * field arithmetic wins; the chunks of a larger call keep the main variant); set_variant applies its variant to every launch size and
 * clears the small-launch one.  get_small_variant reports -1 when none. */
#define UFSECP_EXT_VERIFY_VARIANTS 12
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_set_variant(ufsecp_gpu_ctx* ctx, int kind, int variant);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_get_variant(ufsecp_gpu_ctx* ctx, int kind, int* variant_out,
                                                     int* blocks_per_sm_out);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_get_small_variant(ufsecp_gpu_ctx* ctx, int kind, int* variant_out,
                                                           uint32_t* items_out);
/* variant -1 removes the small-launch variant of `kind`. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_set_small_variant(ufsecp_gpu_ctx* ctx, int kind, int variant,
                                                           uint32_t items);

/* Lanes per signature (kind 0 ECDSA, 1 BIP-340): with lanes = 2, calls of at
 * most `items` items run two threads per signature, each over half of the
 * four GLV streams, their partial sums added at the end: a shorter verify
 * latency for 1.6x the arithmetic, which pays while the device has idle
 * capacity (small calls).  lanes = 1 turns it off.  The tuning file sets it
 * per kind (ecdsa_pair_items / schnorr_pair_items); set_variant turns it off.
 * The opaque-row / column surfaces always use one lane. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_set_lanes(ufsecp_gpu_ctx* ctx, int kind, int lanes, uint32_t items);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_get_lanes(ufsecp_gpu_ctx* ctx, int kind, int* lanes_out,
                                                   uint32_t* items_out);

/* Inversion group per kind (0 ECDSA, 1 BIP-340): 1 = every signature runs its
 * own inversions (the variant kernels above); 64 or 128 = kernels whose
 * blocks of that many threads share each modular inversion by Montgomery's
 * trick (the P table's Z product, BIP-340's final Z, ECDSA's s^-1: one
 * inversion per block and site instead of one per warp).  Applies to the main
 * verify launches, not to the two-lane or small-launch paths.  The tuning file
 * sets it per kind (ecdsa_inv_group / schnorr_inv_group, chosen by the
 * autotuner); UFSECP_B200_INV_GROUP overrides both kinds; set_variant resets
 * the kind to 1.  Verdicts do not depend on it. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_set_inversion_group(ufsecp_gpu_ctx* ctx, int kind, int group);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_get_inversion_group(ufsecp_gpu_ctx* ctx, int kind, int* group_out);

/* RLC bucket chunk: the number of bucket points one thread sums before the
 * per-bucket merge.  The tuning file sets it per batch size (rlc_chunk_<n>;
 * the nearest tuned size in log scale applies, else 16).  set: 2..256 fixes it
 * for every segment length, 0 restores the tuned values (the environment
 * variable UFSECP_B200_RLC_CHUNK sets the same override at context creation).
 * get: the chunk a segment of `len` items uses.  Verdicts do not depend on it. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_set_rlc_chunk(ufsecp_gpu_ctx* ctx, uint32_t chunk);
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_get_rlc_chunk(ufsecp_gpu_ctx* ctx, uint32_t len, uint32_t* chunk_out);

/* Measured 32-bit integer multiply-add issue rate of the device (ops / s):
 * every thread of a full grid runs 16 independent mad.lo.u32 chains. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_imad_peak(ufsecp_gpu_ctx* ctx, double* ops_per_s);

/* Building-block throughput probe: launches blocks x threads threads, each
 * running `iters` rounds of one operation on register-resident values, and
 * returns the launch time in milliseconds (CUDA events).  op: 1 two fe_mul
 * chains, 2 two fe_sqr chains, 3 fe_inv, 4 sqrt exponentiation, 5 Jacobian
 * doubling, 6 Jacobian + affine add, 7 scalar inverse, 8 GLV split,
 * 9 BIP-340 challenge hash; integer multiply-add forms, 8 per round with
 * data-dependent multipliers: 10 mad.lo.u32, 11 mad.hi.u32, 12 mad.wide.u32,
 * 13 mad.lo.cc / madc.hi.cc carry chain, 14 operand-scanning step
 * (32x32 + 32 + 32 -> 64); 15 two 256x256 PTX products (no reduction),
 * 16 two inlined field multiplies (no call). */
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_probe(ufsecp_gpu_ctx* ctx, int op, int blocks, int threads, int iters,
                                               float* ms_out);

/* Device arithmetic probes (one item per thread), host buffers in and out.
 * op  in -> out bytes per item
 *  1  a|b (64) -> a*b mod p (32)         2  a (32) -> a^2 mod p (32)
 *  3  a (32) -> a^-1 mod p (32)          4  a (32) -> ok (1) | sqrt (32)
 *  5  a|b (64) -> a*b mod n (32)         6  a (32) -> a^-1 mod n (32)
 *  7  k (32) -> |k1| (16) | |k2| (16) | neg1 | neg2    (GLV split)
 *  8  k (32) -> (k*G).x | (k*G).y (64), zeros for infinity
 *  9  a|x|b (96) -> finite (1) | x (32) | y (32) of a*G + b*P, P = lift_x(x)
 * 10  r|p|m (96) -> BIP-340 challenge digest (32)
 * 11  a|b (64) -> a*b | a^2 | a+b | a-b | 4a | 8a mod p (192), through the field code
 *     of the verify kernels (PTX carry chains), inputs any 256-bit values
 * All values big-endian. */
#define UFSECP_EXT_DIAG_FE_MUL    1
#define UFSECP_EXT_DIAG_FE_SQR    2
#define UFSECP_EXT_DIAG_FE_INV    3
#define UFSECP_EXT_DIAG_FE_SQRT   4
#define UFSECP_EXT_DIAG_SC_MUL    5
#define UFSECP_EXT_DIAG_SC_INV    6
#define UFSECP_EXT_DIAG_GLV       7
#define UFSECP_EXT_DIAG_GEN_MUL   8
#define UFSECP_EXT_DIAG_DUAL_MUL  9
#define UFSECP_EXT_DIAG_CHALLENGE 10
#define UFSECP_EXT_DIAG_FE_PTX    11
UFSECP_API ufsecp_error_t ufsecp_gpu_ext_diag(ufsecp_gpu_ctx* ctx, uint32_t op, const uint8_t* in, size_t n,
                                              uint8_t* out);

#ifdef __cplusplus
}
#endif

#endif /* UFSECP_GPU_EXT_H */
