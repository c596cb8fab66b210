/* ufsecp_gpu.h -- drop-in GPU C ABI of the B200 batch signature-verify library.
 *
 * Every declaration replaces the function of the same name in the reference
 * header include/ufsecp/ufsecp_gpu.h (UltrafastSecp256k1 v4.5.0); the line of
 * the reference declaration is given beside each one.  Names, argument order,
 * types, strides and error codes are identical, so a program built against the
 * reference header links against libufsecp_gpu.so unchanged.
 *
 * Implemented on the sm_100a kernels of this library:
 *   discovery / lifecycle / errors: backend_count, backend_name, is_available,
 *     device_count, device_info, ctx_create, ctx_destroy, is_ready, last_error,
 *     last_error_msg, error_str;
 *   verification: ecdsa_verify_batch, schnorr_verify_batch, ecdsa_verify_collect,
 *     schnorr_verify_collect, ecdsa_verify_opaque_rows, ecdsa_verify_lbtc_rows,
 *     ecdsa_verify_lbtc_columns, schnorr_verify_lbtc_columns;
 *   adjacent operations on the same math: msm, xonly_validate, pubkey_validate,
 *     commitment_verify, tagged_hash, tagged_hash_var.
 * Every other operation of the reference surface (key generation, ECDH,
 * hashing, BIP-324 / BIP-352, ZK, FROST, recovery) is present for link
 * compatibility and returns UFSECP_ERR_GPU_UNSUPPORTED (104), which the
 * reference header allows for operations a backend does not implement.
 *
 * Conventions (as the reference C ABI layer, src/cpu/src/ufsecp_gpu_impl.cpp):
 *   - NULL ctx -> UFSECP_ERR_NULL_ARG; count == 0 -> UFSECP_OK, buffers untouched;
 *     count > 2^26 -> UFSECP_ERR_BAD_INPUT; result buffers are cleared to 0
 *     before the NULL-buffer check and again after any non-OK backend return.
 *   - Invalid signatures / keys are verdicts (out[i] = 0), not errors.
 *   - Calls are synchronous: results are in the caller's buffer on return.
 *   - A context is single-thread; use one per thread or lock externally.
 *   - Verdicts follow the reference CPU verify (ufsecp_ecdsa_verify /
 *     ufsecp_schnorr_verify): strict r, s ranges, low-S required for ECDSA,
 *     strict x < p for keys and BIP-340 r. */
#ifndef UFSECP_GPU_H
#define UFSECP_GPU_H

#include "ufsecp_version.h"
#include "ufsecp_error.h"

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#  define UFSECP_NOEXCEPT noexcept
extern "C" {
#else
#  define UFSECP_NOEXCEPT
#endif

#define UFSECP_ERR_GPU_UNAVAILABLE  100
#define UFSECP_ERR_GPU_DEVICE       101
#define UFSECP_ERR_GPU_LAUNCH       102
#define UFSECP_ERR_GPU_MEMORY       103
#define UFSECP_ERR_GPU_UNSUPPORTED  104
#define UFSECP_ERR_GPU_BACKEND      105
#define UFSECP_ERR_GPU_QUEUE        106

#define UFSECP_GPU_BACKEND_NONE     0
#define UFSECP_GPU_BACKEND_CUDA     1
#define UFSECP_GPU_BACKEND_OPENCL   2
#define UFSECP_GPU_BACKEND_METAL    3

typedef struct ufsecp_gpu_ctx ufsecp_gpu_ctx;

/* ---- discovery (reference ufsecp_gpu.h:109-132) ------------------------- */

/* ref :109 -- number of compiled-in backends (1: CUDA); fills ids if given. */
UFSECP_API uint32_t ufsecp_gpu_backend_count(uint32_t* backend_ids, uint32_t max_ids) UFSECP_NOEXCEPT;
/* ref :112 -- "CUDA", "OpenCL", "Metal" or "none". */
UFSECP_API const char* ufsecp_gpu_backend_name(uint32_t backend_id);
/* ref :115 -- 1 when the backend is compiled in and a device exists. */
UFSECP_API int ufsecp_gpu_is_available(uint32_t backend_id) UFSECP_NOEXCEPT;
/* ref :118 -- device count of a backend (0 if unavailable). */
UFSECP_API uint32_t ufsecp_gpu_device_count(uint32_t backend_id) UFSECP_NOEXCEPT;

/* ref :121-129 -- same layout. */
typedef struct {
    char     name[128];
    uint64_t global_mem_bytes;
    uint32_t compute_units;
    uint32_t max_clock_mhz;
    uint32_t max_threads_per_block;
    uint32_t backend_id;
    uint32_t device_index;
} ufsecp_gpu_device_info_t;

/* ref :132 */
UFSECP_API ufsecp_error_t ufsecp_gpu_device_info(uint32_t backend_id, uint32_t device_index,
                                                 ufsecp_gpu_device_info_t* info_out);

/* ---- lifecycle (reference ufsecp_gpu.h:146-167) ------------------------- */

/* ref :146 -- creates the device context: stream, generator tables, buffers. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ctx_create(ufsecp_gpu_ctx** ctx_out, uint32_t backend_id, uint32_t device_index);
/* ref :152 */
UFSECP_API void ufsecp_gpu_ctx_destroy(ufsecp_gpu_ctx* ctx);
/* ref :158 */
UFSECP_API int ufsecp_gpu_is_ready(const ufsecp_gpu_ctx* ctx) UFSECP_NOEXCEPT;
/* ref :161 */
UFSECP_API ufsecp_error_t ufsecp_gpu_last_error(const ufsecp_gpu_ctx* ctx);
/* ref :167 -- borrowed string, valid until the next call on the same ctx. */
UFSECP_API const char* ufsecp_gpu_last_error_msg(const ufsecp_gpu_ctx* ctx);

/* ---- the verify path ------------------------------------------------------ */

/* ref :200 -- ECDSA: msg_hashes32 count*32 B, pubkeys33 count*33 B (SEC1
 * compressed), sigs64 count*64 B (compact r||s big-endian); out_results
 * count bytes, 1 = valid. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ecdsa_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                        const uint8_t* pubkeys33, const uint8_t* sigs64,
                                                        size_t count, uint8_t* out_results);
/* ref :254 -- BIP-340: msg_hashes32 count*32 B, pubkeys_x32 count*32 B
 * (x-only), sigs64 count*64 B (R.x||s); out_results count bytes. */
UFSECP_API ufsecp_error_t ufsecp_gpu_schnorr_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                          const uint8_t* pubkeys_x32, const uint8_t* sigs64,
                                                          size_t count, uint8_t* out_results);
/* ref :326 -- same verdict as ecdsa_verify_batch, collapsed in place: the
 * caller seeds key_buffer with non-zero bytes; valid rows become 0, invalid
 * rows keep their byte. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ecdsa_verify_collect(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                          const uint8_t* pubkeys33, const uint8_t* sigs64,
                                                          size_t count, uint8_t* key_buffer);
/* ref :345 -- BIP-340 sibling of ecdsa_verify_collect. */
UFSECP_API ufsecp_error_t ufsecp_gpu_schnorr_verify_collect(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                            const uint8_t* pubkeys_x32, const uint8_t* sigs64,
                                                            size_t count, uint8_t* key_buffer);

/* ref :228 / :236 / :278 / :299 -- consensus row / column surfaces.
 * opaque_rows (lbtc_rows is an alias): rows [msg 32 | compressed pubkey 33 |
 * opaque signature 64 | tail], stride >= 129 bytes (else BAD_INPUT); the
 * signature is the libsecp in-memory layout, r then s as 32 little-endian
 * bytes each, r and s in [1, n-1], high-S accepted (normalised), the verdicts
 * of the reference CPU's ufsecp_ecdsa_verify_opaque_rows
 * (src/cpu/src/impl/ufsecp_ecdsa.cpp:412).  ecdsa_lbtc_columns: the same
 * verdicts from three column arrays.  schnorr_lbtc_columns: the BIP-340
 * verdicts of ufsecp_gpu_schnorr_verify_batch on the same columns. */
UFSECP_API ufsecp_error_t ufsecp_gpu_ecdsa_verify_opaque_rows(ufsecp_gpu_ctx* ctx, const uint8_t* rows, size_t stride,
                                                              size_t count, uint8_t* out_results);
UFSECP_API ufsecp_error_t ufsecp_gpu_ecdsa_verify_lbtc_rows(ufsecp_gpu_ctx* ctx, const uint8_t* rows, size_t stride,
                                                            size_t count, uint8_t* out_results);
UFSECP_API ufsecp_error_t ufsecp_gpu_ecdsa_verify_lbtc_columns(ufsecp_gpu_ctx* ctx, const uint8_t* digests32,
                                                               const uint8_t* pubkeys33, const uint8_t* sigs64,
                                                               size_t count, uint8_t* out_results);
UFSECP_API ufsecp_error_t ufsecp_gpu_schnorr_verify_lbtc_columns(ufsecp_gpu_ctx* ctx, const uint8_t* digests32,
                                                                 const uint8_t* xonly32, const uint8_t* sigs64,
                                                                 size_t count, uint8_t* out_results);

/* ref :607 -- short English description of any ufsecp error code. */
UFSECP_API const char* ufsecp_gpu_error_str(ufsecp_error_t err);

/* ---- other operations of the reference surface ---------------------------
 * Present for link compatibility; they return UFSECP_ERR_GPU_UNSUPPORTED. */
/* ref :182 */
UFSECP_API ufsecp_error_t ufsecp_gpu_generator_mul_batch(ufsecp_gpu_ctx* ctx, const uint8_t* scalars32, size_t count,
                                                         uint8_t* out_pubkeys33);
/* ref :364 */
UFSECP_API ufsecp_error_t ufsecp_gpu_ecdh_batch(ufsecp_gpu_ctx* ctx, const uint8_t* privkeys32,
                                                const uint8_t* peer_pubkeys33, size_t count, uint8_t* out_secrets32);
/* ref :380 */
UFSECP_API ufsecp_error_t ufsecp_gpu_hash160_pubkey_batch(ufsecp_gpu_ctx* ctx, const uint8_t* pubkeys33, size_t count,
                                                          uint8_t* out_hash160);
/* ref :397 */
UFSECP_API ufsecp_error_t ufsecp_gpu_msm(ufsecp_gpu_ctx* ctx, const uint8_t* scalars32, const uint8_t* points33,
                                         size_t n, uint8_t* out_result33);
/* ref :419 */
UFSECP_API ufsecp_error_t ufsecp_gpu_xonly_validate(ufsecp_gpu_ctx* ctx, const uint8_t* keys32, size_t n,
                                                    uint8_t* results);
/* ref :439 */
UFSECP_API ufsecp_error_t ufsecp_gpu_commitment_verify(ufsecp_gpu_ctx* ctx, const uint8_t* internal_x32,
                                                       const uint8_t* tweak32, const uint8_t* tweaked_x32,
                                                       const uint8_t* parity, size_t n, uint8_t* results);
/* ref :460 */
UFSECP_API ufsecp_error_t ufsecp_gpu_tagged_hash(ufsecp_gpu_ctx* ctx, const uint8_t* tag_hash32, const uint8_t* msgs,
                                                 size_t msg_len, size_t n, uint8_t* out32);
/* ref :477 */
UFSECP_API ufsecp_error_t ufsecp_gpu_pubkey_validate(ufsecp_gpu_ctx* ctx, const uint8_t* pubkeys33, size_t n,
                                                     uint8_t* results);
/* ref :496 */
UFSECP_API ufsecp_error_t ufsecp_gpu_tagged_hash_var(ufsecp_gpu_ctx* ctx, const uint8_t* tag_hash32,
                                                     const uint8_t* msgs, const uint32_t* msg_lens, size_t stride,
                                                     size_t n, uint8_t* out32);
/* ref :516 */
UFSECP_API ufsecp_error_t ufsecp_gpu_hash256(ufsecp_gpu_ctx* ctx, const uint8_t* inputs, size_t input_len, size_t n,
                                             uint8_t* out32);
/* ref :538 */
UFSECP_API ufsecp_error_t ufsecp_gpu_hash256_var(ufsecp_gpu_ctx* ctx, const uint8_t* inputs,
                                                 const uint32_t* input_lens, size_t stride, size_t n, uint8_t* out32);
/* ref :569 */
UFSECP_API ufsecp_error_t ufsecp_gpu_frost_verify_partial_batch(
    ufsecp_gpu_ctx* ctx, const uint8_t* z_i32, const uint8_t* D_i33, const uint8_t* E_i33, const uint8_t* Y_i33,
    const uint8_t* rho_i32, const uint8_t* lambda_ie32, const uint8_t* negate_R, const uint8_t* negate_key,
    size_t count, uint8_t* out_results);
/* ref :596 */
UFSECP_API ufsecp_error_t ufsecp_gpu_ecrecover_batch(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                     const uint8_t* sigs64, const int* recids, size_t count,
                                                     uint8_t* out_pubkeys33, uint8_t* out_valid);
/* ref :629 */
UFSECP_API ufsecp_error_t ufsecp_gpu_zk_knowledge_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t* proofs64,
                                                               const uint8_t* pubkeys65, const uint8_t* messages32,
                                                               size_t count, uint8_t* out_results);
/* ref :655 */
UFSECP_API ufsecp_error_t ufsecp_gpu_zk_dleq_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t* proofs64,
                                                          const uint8_t* G_pts65, const uint8_t* H_pts65,
                                                          const uint8_t* P_pts65, const uint8_t* Q_pts65, size_t count,
                                                          uint8_t* out_results);
/* ref :681 */
UFSECP_API ufsecp_error_t ufsecp_gpu_bulletproof_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t* proofs324,
                                                              const uint8_t* commitments65,
                                                              const uint8_t* H_generator65, size_t count,
                                                              uint8_t* out_results);
/* ref :710 */
UFSECP_API ufsecp_error_t ufsecp_gpu_bip324_aead_encrypt_batch(ufsecp_gpu_ctx* ctx, const uint8_t* keys32,
                                                               const uint8_t* nonces12, const uint8_t* plaintexts,
                                                               const uint32_t* sizes, uint32_t max_payload,
                                                               size_t count, uint8_t* wire_out);
/* ref :736 */
UFSECP_API ufsecp_error_t ufsecp_gpu_bip324_aead_decrypt_batch(ufsecp_gpu_ctx* ctx, const uint8_t* keys32,
                                                               const uint8_t* nonces12, const uint8_t* wire_in,
                                                               const uint32_t* sizes, uint32_t max_payload,
                                                               size_t count, uint8_t* plaintext_out,
                                                               uint8_t* out_valid);
#define UFSECP_ECDSA_SNARK_WITNESS_BYTES 760
/* ref :767 */
UFSECP_API ufsecp_error_t ufsecp_gpu_zk_ecdsa_snark_witness_batch(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                                  const uint8_t* pubkeys33, const uint8_t* sigs64,
                                                                  size_t count, uint8_t* out_witnesses);
#define UFSECP_SCHNORR_SNARK_WITNESS_BYTES 472
/* ref :794 */
UFSECP_API ufsecp_error_t ufsecp_gpu_zk_schnorr_snark_witness_batch(ufsecp_gpu_ctx* ctx, const uint8_t* msgs32,
                                                                    const uint8_t* pubkeys_x32, const uint8_t* sigs64,
                                                                    size_t count, uint8_t* out_witnesses);
#define UFSECP_BIP352_SCAN_PLAN_BYTES 264
/* ref :825 */
UFSECP_API ufsecp_error_t ufsecp_bip352_prepare_scan_plan(const uint8_t scan_privkey32[32], uint8_t plan264_out[264]);
/* ref :861 */
UFSECP_API ufsecp_error_t ufsecp_gpu_bip352_scan_batch(ufsecp_gpu_ctx* ctx, const uint8_t scan_privkey32[32],
                                                       const uint8_t spend_pubkey33[33],
                                                       const uint8_t* tweak_pubkeys33, size_t n_tweaks,
                                                       uint64_t* prefix64_out);

#ifdef __cplusplus
}
#endif

#endif /* UFSECP_GPU_H */
