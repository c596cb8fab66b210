// extern "C" surface: ufsecp_gpu.h (the reference's GPU ABI) and
// ufsecp_gpu_ext.h (B200 additions).
//
// Argument gating, output clearing and exception mapping follow the
// reference's C ABI layer src/cpu/src/ufsecp_gpu_impl.cpp: batch cap 2^26
// (:76), bad_alloc -> GPU_MEMORY / other exceptions -> INTERNAL (:79-81),
// clear-before and clear-after-failure of result buffers (:117-140, :317-336).
#include <cuda_runtime.h>
#include <string.h>

#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <random>
#include <algorithm>

#include <thread>
#include <vector>

#include "backend.h"
#include "batch.h"
#include "rlc.h"
#include "server.h"
#include "ufsecp/ufsecp_gpu.h"
#include "ufsecp/ufsecp_gpu_ext.h"

struct ufsecp_gpu_ctx {
    std::unique_ptr<uf::Backend> backend;
    uint32_t backend_id;
    uint32_t device_index;
    uf::RlcStats rlc_stats;      // of the last RLC call
};

struct ufsecp_gpu_ext_server {
    std::unique_ptr<uf::Server> server;
};

namespace {

constexpr size_t kMaxBatch = size_t{1} << 26;

bool clear_out(uint8_t* out, size_t count, size_t stride) {
    if (!out || count == 0) return true;
    if (count > std::numeric_limits<size_t>::max() / stride) return false;
    memset(out, 0, count * stride);
    return true;
}

ufsecp_error_t finish(ufsecp_error_t rc, uint8_t* out, size_t count, size_t stride) {
    if (rc != UFSECP_OK) clear_out(out, count, stride);
    return rc;
}

int cuda_device_count() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    return n;
}

// Shared gating of the result-bearing verify calls.
template <class F>
ufsecp_error_t gated_verify(ufsecp_gpu_ctx* ctx, const uint8_t* a, const uint8_t* b, const uint8_t* c, size_t count,
                            uint8_t* out, F&& run) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (count > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (!clear_out(out, count, 1)) return UFSECP_ERR_BAD_INPUT;
    if (!a || !b || !c || !out) return UFSECP_ERR_NULL_ARG;
    try {
        return finish(run(), out, count, 1);
    } catch (const std::bad_alloc&) {
        return finish(UFSECP_ERR_GPU_MEMORY, out, count, 1);
    } catch (...) {
        return finish(UFSECP_ERR_INTERNAL, out, count, 1);
    }
}

template <class F>
ufsecp_error_t gated_collect(ufsecp_gpu_ctx* ctx, const uint8_t* a, const uint8_t* b, const uint8_t* c, size_t count,
                             uint8_t* key_buffer, F&& run) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (!a || !b || !c || !key_buffer) return UFSECP_ERR_NULL_ARG;
    if (count > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    try {
        return run();
    } catch (const std::bad_alloc&) {
        return UFSECP_ERR_GPU_MEMORY;
    } catch (...) {
        return UFSECP_ERR_INTERNAL;
    }
}

// Runs a result-bearing call, re-clearing its output on failure.
template <class F>
ufsecp_error_t guarded_out(uint8_t* out, size_t count, size_t stride, F&& run) {
    try {
        return finish(run(), out, count, stride);
    } catch (const std::bad_alloc&) {
        return finish(UFSECP_ERR_GPU_MEMORY, out, count, stride);
    } catch (...) {
        return finish(UFSECP_ERR_INTERNAL, out, count, stride);
    }
}

template <class F>
ufsecp_error_t guarded_call(F&& run) {
    try {
        return run();
    } catch (const std::bad_alloc&) {
        return UFSECP_ERR_GPU_MEMORY;
    } catch (...) {
        return UFSECP_ERR_INTERNAL;
    }
}

void fresh_seed(uint8_t seed[32]);

ufsecp_error_t unsupported(ufsecp_gpu_ctx* ctx, size_t count) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    ctx->backend->set_error(UFSECP_ERR_GPU_UNSUPPORTED, "operation not implemented by the B200 verify backend");
    return UFSECP_ERR_GPU_UNSUPPORTED;
}

}  // namespace

extern "C" {

// ---- discovery -------------------------------------------------------------

uint32_t ufsecp_gpu_backend_count(uint32_t* backend_ids, uint32_t max_ids) noexcept {
    if (backend_ids && max_ids > 0) backend_ids[0] = UFSECP_GPU_BACKEND_CUDA;
    return 1;
}

const char* ufsecp_gpu_backend_name(uint32_t backend_id) {
    switch (backend_id) {
        case UFSECP_GPU_BACKEND_CUDA: return "CUDA";
        case UFSECP_GPU_BACKEND_OPENCL: return "OpenCL";
        case UFSECP_GPU_BACKEND_METAL: return "Metal";
        default: return "none";
    }
}

int ufsecp_gpu_is_available(uint32_t backend_id) noexcept {
    return backend_id == UFSECP_GPU_BACKEND_CUDA && cuda_device_count() > 0 ? 1 : 0;
}

uint32_t ufsecp_gpu_device_count(uint32_t backend_id) noexcept {
    return backend_id == UFSECP_GPU_BACKEND_CUDA ? (uint32_t)cuda_device_count() : 0u;
}

ufsecp_error_t ufsecp_gpu_device_info(uint32_t backend_id, uint32_t device_index, ufsecp_gpu_device_info_t* info_out) {
    if (!info_out) return UFSECP_ERR_NULL_ARG;
    if (backend_id != UFSECP_GPU_BACKEND_CUDA) return UFSECP_ERR_GPU_UNAVAILABLE;
    const int n = cuda_device_count();
    if (n == 0) return UFSECP_ERR_GPU_UNAVAILABLE;
    if ((int)device_index >= n) return UFSECP_ERR_GPU_DEVICE;
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, (int)device_index) != cudaSuccess) {
        (void)cudaGetLastError();
        return UFSECP_ERR_GPU_DEVICE;
    }
    memset(info_out, 0, sizeof(*info_out));
    strncpy(info_out->name, p.name, sizeof(info_out->name) - 1);
    info_out->global_mem_bytes = p.totalGlobalMem;
    info_out->compute_units = (uint32_t)p.multiProcessorCount;
    int clk_khz = 0;
    cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, (int)device_index);
    info_out->max_clock_mhz = (uint32_t)(clk_khz / 1000);
    info_out->max_threads_per_block = (uint32_t)p.maxThreadsPerBlock;
    info_out->backend_id = UFSECP_GPU_BACKEND_CUDA;
    info_out->device_index = device_index;
    return UFSECP_OK;
}

// ---- lifecycle -------------------------------------------------------------

ufsecp_error_t ufsecp_gpu_ctx_create(ufsecp_gpu_ctx** ctx_out, uint32_t backend_id, uint32_t device_index) {
    if (!ctx_out) return UFSECP_ERR_NULL_ARG;
    *ctx_out = nullptr;
    if (backend_id != UFSECP_GPU_BACKEND_CUDA) return UFSECP_ERR_GPU_UNAVAILABLE;
    try {
        auto be = std::make_unique<uf::Backend>();
        const int rc = be->init((int)device_index);
        if (rc != UFSECP_OK) return rc;
        auto* ctx = new (std::nothrow) ufsecp_gpu_ctx;
        if (!ctx) return UFSECP_ERR_INTERNAL;
        ctx->backend = std::move(be);
        ctx->backend_id = backend_id;
        ctx->device_index = device_index;
        *ctx_out = ctx;
        return UFSECP_OK;
    } catch (const std::bad_alloc&) {
        return UFSECP_ERR_GPU_MEMORY;
    } catch (...) {
        return UFSECP_ERR_INTERNAL;
    }
}

void ufsecp_gpu_ctx_destroy(ufsecp_gpu_ctx* ctx) {
    if (ctx) {
        ctx->backend.reset();
        delete ctx;
    }
}

int ufsecp_gpu_is_ready(const ufsecp_gpu_ctx* ctx) noexcept {
    return ctx && ctx->backend && ctx->backend->ready() ? 1 : 0;
}

ufsecp_error_t ufsecp_gpu_last_error(const ufsecp_gpu_ctx* ctx) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->last_error();
}

const char* ufsecp_gpu_last_error_msg(const ufsecp_gpu_ctx* ctx) {
    if (!ctx) return "NULL GPU context";
    return ctx->backend->last_error_msg();
}

const char* ufsecp_gpu_error_str(ufsecp_error_t err) {
    switch (err) {
        case UFSECP_OK: return "OK";
        case UFSECP_ERR_NULL_ARG: return "NULL argument";
        case UFSECP_ERR_BAD_KEY: return "invalid private key";
        case UFSECP_ERR_BAD_PUBKEY: return "invalid public key";
        case UFSECP_ERR_BAD_SIG: return "invalid signature";
        case UFSECP_ERR_BAD_INPUT: return "bad input";
        case UFSECP_ERR_VERIFY_FAIL: return "verification failed";
        case UFSECP_ERR_ARITH: return "arithmetic error";
        case UFSECP_ERR_SELFTEST: return "self-test failed";
        case UFSECP_ERR_INTERNAL: return "internal error";
        case UFSECP_ERR_BUF_TOO_SMALL: return "buffer too small";
        case UFSECP_ERR_NOT_FOUND: return "not found";
        case UFSECP_ERR_DEPRECATED_API: return "deprecated API";
        case UFSECP_ERR_CANCELLED: return "cancelled";
        case UFSECP_ERR_GPU_UNAVAILABLE: return "GPU backend unavailable";
        case UFSECP_ERR_GPU_DEVICE: return "GPU device not found or init failed";
        case UFSECP_ERR_GPU_LAUNCH: return "GPU kernel launch failed";
        case UFSECP_ERR_GPU_MEMORY: return "GPU memory allocation or copy failed";
        case UFSECP_ERR_GPU_UNSUPPORTED: return "operation not supported on this GPU backend";
        case UFSECP_ERR_GPU_BACKEND: return "GPU driver / runtime error";
        case UFSECP_ERR_GPU_QUEUE: return "GPU queue / stream error";
        default: return "unknown error";
    }
}

// ---- verify ----------------------------------------------------------------

ufsecp_error_t ufsecp_gpu_ecdsa_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32, const uint8_t* pubkeys33,
                                             const uint8_t* sigs64, size_t count, uint8_t* out_results) {
    return gated_verify(ctx, msg_hashes32, pubkeys33, sigs64, count, out_results, [&] {
        return ctx->backend->verify_host(0, msg_hashes32, pubkeys33, sigs64, count, out_results, false);
    });
}

ufsecp_error_t ufsecp_gpu_schnorr_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                               const uint8_t* pubkeys_x32, const uint8_t* sigs64, size_t count,
                                               uint8_t* out_results) {
    return gated_verify(ctx, msg_hashes32, pubkeys_x32, sigs64, count, out_results, [&] {
        return ctx->backend->verify_host(1, msg_hashes32, pubkeys_x32, sigs64, count, out_results, false);
    });
}

ufsecp_error_t ufsecp_gpu_ecdsa_verify_collect(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                               const uint8_t* pubkeys33, const uint8_t* sigs64, size_t count,
                                               uint8_t* key_buffer) {
    return gated_collect(ctx, msg_hashes32, pubkeys33, sigs64, count, key_buffer, [&] {
        return ctx->backend->verify_host(0, msg_hashes32, pubkeys33, sigs64, count, key_buffer, true);
    });
}

ufsecp_error_t ufsecp_gpu_schnorr_verify_collect(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                 const uint8_t* pubkeys_x32, const uint8_t* sigs64, size_t count,
                                                 uint8_t* key_buffer) {
    return gated_collect(ctx, msg_hashes32, pubkeys_x32, sigs64, count, key_buffer, [&] {
        return ctx->backend->verify_host(1, msg_hashes32, pubkeys_x32, sigs64, count, key_buffer, true);
    });
}

ufsecp_error_t ufsecp_gpu_ecdsa_verify_opaque_rows(ufsecp_gpu_ctx* ctx, const uint8_t* rows, size_t stride,
                                                   size_t count, uint8_t* out_results) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (count > kMaxBatch || stride < 129u) return UFSECP_ERR_BAD_INPUT;
    if (!rows || !out_results) return UFSECP_ERR_NULL_ARG;
    clear_out(out_results, count, 1);
    try {
        return finish(ctx->backend->verify_host_strided(2, rows, stride, rows + 32, stride, rows + 65, stride, count,
                                                        out_results, false),
                      out_results, count, 1);
    } catch (const std::bad_alloc&) {
        return finish(UFSECP_ERR_GPU_MEMORY, out_results, count, 1);
    } catch (...) {
        return finish(UFSECP_ERR_INTERNAL, out_results, count, 1);
    }
}

ufsecp_error_t ufsecp_gpu_ecdsa_verify_lbtc_rows(ufsecp_gpu_ctx* ctx, const uint8_t* rows, size_t stride, size_t count,
                                                 uint8_t* out_results) {
    return ufsecp_gpu_ecdsa_verify_opaque_rows(ctx, rows, stride, count, out_results);
}

ufsecp_error_t ufsecp_gpu_ecdsa_verify_lbtc_columns(ufsecp_gpu_ctx* ctx, const uint8_t* digests32,
                                                    const uint8_t* pubkeys33, const uint8_t* sigs64, size_t count,
                                                    uint8_t* out_results) {
    return gated_verify(ctx, digests32, pubkeys33, sigs64, count, out_results, [&] {
        return ctx->backend->verify_host(2, digests32, pubkeys33, sigs64, count, out_results, false);
    });
}

ufsecp_error_t ufsecp_gpu_schnorr_verify_lbtc_columns(ufsecp_gpu_ctx* ctx, const uint8_t* digests32,
                                                      const uint8_t* xonly32, const uint8_t* sigs64, size_t count,
                                                      uint8_t* out_results) {
    return gated_verify(ctx, digests32, xonly32, sigs64, count, out_results, [&] {
        return ctx->backend->verify_host(1, digests32, xonly32, sigs64, count, out_results, false);
    });
}

// ---- the rest of the reference surface: not implemented here -----------------

ufsecp_error_t ufsecp_gpu_generator_mul_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_ecdh_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_hash160_pubkey_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_msm(ufsecp_gpu_ctx* ctx, const uint8_t* scalars32, const uint8_t* points33, size_t n,
                              uint8_t* out_result33) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n == 0) return UFSECP_OK;
    if (n > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (!clear_out(out_result33, 1, 33)) return UFSECP_ERR_BAD_INPUT;
    if (!scalars32 || !points33 || !out_result33) return UFSECP_ERR_NULL_ARG;
    return guarded_out(out_result33, 1, 33, [&]() -> int {
        uf::Backend& be = *ctx->backend;
        if (!be.ready()) return be.set_error(UFSECP_ERR_GPU_DEVICE, "context not ready");
        if (n > uf::RlcVerifier::kMaxItems) return be.set_error(UFSECP_ERR_BAD_INPUT, "MSM: more than 2^24 points");
        cudaError_t e = cudaSetDevice(be.device());
        if (e != cudaSuccess) return be.cuda_error(e, "cudaSetDevice");
        int status = 0;
        const int rc = be.rlc().msm_host(scalars32, points33, (uint32_t)n, out_result33, &status);
        if (rc != UFSECP_OK) return rc;
        if (status == UFSECP_ERR_BAD_INPUT) return be.set_error(status, "scalar >= n");
        if (status == UFSECP_ERR_BAD_PUBKEY) return be.set_error(status, "invalid point in array");
        if (status == UFSECP_ERR_ARITH) return be.set_error(status, "MSM result is infinity");
        be.clear_error();
        return UFSECP_OK;
    });
}
ufsecp_error_t ufsecp_gpu_xonly_validate(ufsecp_gpu_ctx* ctx, const uint8_t* keys32, size_t n, uint8_t* results) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n == 0) return UFSECP_OK;
    if (n > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (!clear_out(results, n, 1)) return UFSECP_ERR_BAD_INPUT;
    if (!keys32 || !results) return UFSECP_ERR_NULL_ARG;
    return guarded_out(results, n, 1, [&] { return ctx->backend->xonly_validate(keys32, n, results); });
}
ufsecp_error_t ufsecp_gpu_commitment_verify(ufsecp_gpu_ctx* ctx, const uint8_t* internal_x32, const uint8_t* tweak32,
                                            const uint8_t* tweaked_x32, const uint8_t* parity, size_t n,
                                            uint8_t* results) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n == 0) return UFSECP_OK;
    if (n > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (!clear_out(results, n, 1)) return UFSECP_ERR_BAD_INPUT;
    if (!internal_x32 || !tweak32 || !tweaked_x32 || !parity || !results) return UFSECP_ERR_NULL_ARG;
    return guarded_out(results, n, 1, [&] {
        return ctx->backend->commitment_verify(internal_x32, tweak32, tweaked_x32, parity, n, results);
    });
}
ufsecp_error_t ufsecp_gpu_tagged_hash(ufsecp_gpu_ctx* ctx, const uint8_t* tag_hash32, const uint8_t* msgs,
                                      size_t msg_len, size_t n, uint8_t* out32) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n == 0) return UFSECP_OK;
    if (n > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (msg_len == 0 || msg_len > 256) return UFSECP_ERR_BAD_INPUT;
    if (!clear_out(out32, n, 32)) return UFSECP_ERR_BAD_INPUT;
    if (!tag_hash32 || !msgs || !out32) return UFSECP_ERR_NULL_ARG;
    return guarded_out(out32, n, 32, [&] {
        return ctx->backend->tagged_hash(tag_hash32, msgs, nullptr, msg_len, msg_len, n, out32);
    });
}
ufsecp_error_t ufsecp_gpu_pubkey_validate(ufsecp_gpu_ctx* ctx, const uint8_t* pubkeys33, size_t n, uint8_t* results) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n == 0) return UFSECP_OK;
    if (n > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (!clear_out(results, n, 1)) return UFSECP_ERR_BAD_INPUT;
    if (!pubkeys33 || !results) return UFSECP_ERR_NULL_ARG;
    return guarded_out(results, n, 1, [&] { return ctx->backend->pubkey_validate(pubkeys33, n, results); });
}
ufsecp_error_t ufsecp_gpu_tagged_hash_var(ufsecp_gpu_ctx* ctx, const uint8_t* tag_hash32, const uint8_t* msgs,
                                          const uint32_t* msg_lens, size_t stride, size_t n, uint8_t* out32) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n == 0) return UFSECP_OK;
    if (n > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (stride == 0 || stride > 256) return UFSECP_ERR_BAD_INPUT;
    if (!clear_out(out32, n, 32)) return UFSECP_ERR_BAD_INPUT;
    if (!tag_hash32 || !msgs || !msg_lens || !out32) return UFSECP_ERR_NULL_ARG;
    return guarded_out(out32, n, 32, [&] {
        return ctx->backend->tagged_hash(tag_hash32, msgs, msg_lens, 0, stride, n, out32);
    });
}
ufsecp_error_t ufsecp_gpu_hash256(ufsecp_gpu_ctx* ctx, const uint8_t*, size_t, size_t n, uint8_t*) {
    return unsupported(ctx, n);
}
ufsecp_error_t ufsecp_gpu_hash256_var(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint32_t*, size_t, size_t n,
                                      uint8_t*) {
    return unsupported(ctx, n);
}
ufsecp_error_t ufsecp_gpu_frost_verify_partial_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*,
                                                     const uint8_t*, const uint8_t*, const uint8_t*, const uint8_t*,
                                                     const uint8_t*, const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_ecrecover_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*, const int*,
                                          size_t count, uint8_t*, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_zk_knowledge_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*,
                                                    const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_zk_dleq_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*, const uint8_t*,
                                               const uint8_t*, const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_bulletproof_verify_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*,
                                                   const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_bip324_aead_encrypt_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*,
                                                    const uint8_t*, const uint32_t*, uint32_t, size_t count,
                                                    uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_bip324_aead_decrypt_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*,
                                                    const uint8_t*, const uint32_t*, uint32_t, size_t count, uint8_t*,
                                                    uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_zk_ecdsa_snark_witness_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*,
                                                       const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_gpu_zk_schnorr_snark_witness_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*,
                                                         const uint8_t*, size_t count, uint8_t*) {
    return unsupported(ctx, count);
}
ufsecp_error_t ufsecp_bip352_prepare_scan_plan(const uint8_t*, uint8_t*) { return UFSECP_ERR_GPU_UNSUPPORTED; }
ufsecp_error_t ufsecp_gpu_bip352_scan_batch(ufsecp_gpu_ctx* ctx, const uint8_t*, const uint8_t*, const uint8_t*,
                                            size_t n_tweaks, uint64_t*) {
    return unsupported(ctx, n_tweaks);
}

// ---- B200 extensions -------------------------------------------------------

ufsecp_error_t ufsecp_gpu_ext_ecdsa_verify_device(ufsecp_gpu_ctx* ctx, const uint8_t* d_msg_hashes32,
                                                  const uint8_t* d_pubkeys33, const uint8_t* d_sigs64, size_t count,
                                                  uint8_t* d_out_results, void* stream) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (count > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (!d_msg_hashes32 || !d_pubkeys33 || !d_sigs64 || !d_out_results) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->verify_device(0, d_msg_hashes32, d_pubkeys33, d_sigs64, count, d_out_results,
                                       (cudaStream_t)stream);
}

ufsecp_error_t ufsecp_gpu_ext_schnorr_verify_device(ufsecp_gpu_ctx* ctx, const uint8_t* d_msg_hashes32,
                                                    const uint8_t* d_pubkeys_x32, const uint8_t* d_sigs64,
                                                    size_t count, uint8_t* d_out_results, void* stream) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (count > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (!d_msg_hashes32 || !d_pubkeys_x32 || !d_sigs64 || !d_out_results) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->verify_device(1, d_msg_hashes32, d_pubkeys_x32, d_sigs64, count, d_out_results,
                                       (cudaStream_t)stream);
}

ufsecp_error_t ufsecp_gpu_ext_verify_jobs(ufsecp_gpu_ctx* ctx, const ufsecp_gpu_ext_job_t* jobs, size_t n_jobs) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n_jobs == 0) return UFSECP_OK;
    if (!jobs) return UFSECP_ERR_NULL_ARG;
    size_t total = 0;
    for (size_t j = 0; j < n_jobs; ++j) {
        if (jobs[j].out_results) clear_out(jobs[j].out_results, jobs[j].count, 1);
        total += jobs[j].count;
    }
    for (size_t j = 0; j < n_jobs; ++j) {
        const ufsecp_gpu_ext_job_t& J = jobs[j];
        if (J.count == 0) continue;
        if (!J.msg_hashes32 || !J.pubkeys || !J.sigs64 || !J.out_results) return UFSECP_ERR_NULL_ARG;
        if (J.kind > 2) return UFSECP_ERR_BAD_INPUT;
    }
    if (total > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    int rc;
    try {
        std::vector<uf::VerifyJob> v(n_jobs);
        uint32_t segment = 0;
        for (size_t j = 0; j < n_jobs; ++j) {
            v[j] = uf::VerifyJob{(int)jobs[j].kind, jobs[j].count, jobs[j].msg_hashes32, jobs[j].pubkeys,
                                 jobs[j].sigs64, jobs[j].out_results};
            // the first kind 2 job that names a segment length sets it for the call
            if (jobs[j].kind == 2 && jobs[j].count && !segment) segment = jobs[j].reserved;
        }
        uint8_t rand32[32];
        fresh_seed(rand32);
        rc = ctx->backend->verify_jobs(v.data(), n_jobs, segment, rand32);
    } catch (const std::bad_alloc&) {
        rc = UFSECP_ERR_GPU_MEMORY;
    } catch (...) {
        rc = UFSECP_ERR_INTERNAL;
    }
    // fail closed: no verdict of a failed call may read as valid
    if (rc != UFSECP_OK)
        for (size_t j = 0; j < n_jobs; ++j) clear_out(jobs[j].out_results, jobs[j].count, 1);
    return (ufsecp_error_t)rc;
}

ufsecp_error_t ufsecp_gpu_ext_verify_batch_sharded(ufsecp_gpu_ctx* const* ctxs, size_t n_ctx, uint32_t kind,
                                                  const uint8_t* msg_hashes32, const uint8_t* pubkeys,
                                                  const uint8_t* sigs64, size_t count, uint8_t* out_results) {
    if (!ctxs) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (n_ctx == 0 || kind > 1 || count > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    for (size_t k = 0; k < n_ctx; ++k) {
        if (!ctxs[k]) return UFSECP_ERR_NULL_ARG;
        for (size_t q = 0; q < k; ++q)
            if (ctxs[q] == ctxs[k]) return UFSECP_ERR_BAD_INPUT;
    }
    if (!clear_out(out_results, count, 1)) return UFSECP_ERR_BAD_INPUT;
    if (!msg_hashes32 || !pubkeys || !sigs64 || !out_results) return UFSECP_ERR_NULL_ARG;
    const size_t ps = kind == 0 ? 33 : 32;
    std::vector<ufsecp_error_t> rc(n_ctx, UFSECP_OK);
    try {
        std::vector<std::thread> th;
        struct JoinAll {
            std::vector<std::thread>& v;
            ~JoinAll() {
                for (std::thread& x : v)
                    if (x.joinable()) x.join();
            }
        } join_all{th};
        size_t off = 0;
        for (size_t k = 0; k < n_ctx; ++k) {
            const size_t share = count / n_ctx + (k < count % n_ctx ? 1 : 0);
            if (share)
                th.emplace_back([&, k, off, share]() {
                    rc[k] = kind == 0 ? ufsecp_gpu_ecdsa_verify_batch(ctxs[k], msg_hashes32 + 32 * off,
                                                                      pubkeys + ps * off, sigs64 + 64 * off, share,
                                                                      out_results + off)
                                      : ufsecp_gpu_schnorr_verify_batch(ctxs[k], msg_hashes32 + 32 * off,
                                                                        pubkeys + ps * off, sigs64 + 64 * off, share,
                                                                        out_results + off);
                });
            off += share;
        }
    } catch (const std::bad_alloc&) {
        clear_out(out_results, count, 1);
        return UFSECP_ERR_GPU_MEMORY;
    } catch (...) {
        clear_out(out_results, count, 1);
        return UFSECP_ERR_INTERNAL;
    }
    for (size_t k = 0; k < n_ctx; ++k)
        if (rc[k] != UFSECP_OK) {
            clear_out(out_results, count, 1);
            return rc[k];
        }
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_inject_fault(ufsecp_gpu_ctx* ctx, uint32_t after, int kind) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (kind < 0 || kind > 3) return ctx->backend->set_error(UFSECP_ERR_BAD_INPUT, "fault kind must be 0..3");
    ctx->backend->arm_fault(after, kind);
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_set_key_table(ufsecp_gpu_ctx* ctx, uint32_t log2_slots) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    return guarded_call([&]() -> ufsecp_error_t {
        cudaError_t e = cudaSetDevice(ctx->backend->device());
        if (e != cudaSuccess) return ctx->backend->cuda_error(e, "cudaSetDevice");
        return ctx->backend->set_key_table(log2_slots);
    });
}

ufsecp_error_t ufsecp_gpu_ext_key_table_stats(ufsecp_gpu_ctx* ctx, uint64_t out[3]) {
    if (!ctx || !out) return UFSECP_ERR_NULL_ARG;
    return guarded_call([&]() -> ufsecp_error_t {
        cudaError_t e = cudaSetDevice(ctx->backend->device());
        if (e != cudaSuccess) return ctx->backend->cuda_error(e, "cudaSetDevice");
        return ctx->backend->key_table_stats(&out[0], &out[1], &out[2]);
    });
}

ufsecp_error_t ufsecp_gpu_ext_verify_jobs_noalloc(ufsecp_gpu_ctx* ctx, const ufsecp_gpu_ext_job_t* jobs,
                                                  size_t n_jobs, void* stream) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n_jobs == 0) return UFSECP_OK;
    if (!jobs) return UFSECP_ERR_NULL_ARG;
    uf::Backend& be = *ctx->backend;
    if (n_jobs > uf::kNoAllocJobLimit)
        return be.set_error(UFSECP_ERR_BAD_INPUT,
                            "more than 1024 jobs: the allocation-free path's static scratch holds 1024 job descriptors");
    size_t total = 0;
    for (size_t j = 0; j < n_jobs; ++j) {
        const ufsecp_gpu_ext_job_t& J = jobs[j];
        if (J.kind > 1) return be.set_error(UFSECP_ERR_BAD_INPUT, "job kind must be 0 (ECDSA) or 1 (BIP-340)");
        if (J.count == 0) continue;
        if (!J.msg_hashes32 || !J.pubkeys || !J.sigs64 || !J.out_results) return UFSECP_ERR_NULL_ARG;
        if (((uintptr_t)J.msg_hashes32 | (uintptr_t)J.sigs64 | (J.kind == 1 ? (uintptr_t)J.pubkeys : 0)) & 15u)
            return be.set_error(UFSECP_ERR_BAD_INPUT, "device inputs must be 16-byte aligned");
        total += J.count;
    }
    if (total > kMaxBatch) return be.set_error(UFSECP_ERR_BAD_INPUT, "more than 2^26 items");
    if (!be.ready()) return be.set_error(UFSECP_ERR_GPU_DEVICE, "context not ready");
    cudaError_t e = cudaSetDevice(be.device());
    int limit = 0;
    if (e == cudaSuccess)
        e = uf::verify_jobs_noalloc(be.device(), jobs, n_jobs, be.gtab(),
                                    stream ? (cudaStream_t)stream : be.stream(), &limit);
    if (limit) return be.set_error(UFSECP_ERR_BAD_INPUT, "job limits of the allocation-free path exceeded");
    if (e != cudaSuccess) return be.cuda_error(e, "allocation-free verify");
    be.clear_error();
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_sign_device(ufsecp_gpu_ctx* ctx, uint32_t kind, const uint8_t* d_msgs32,
                                          const uint8_t* d_privkeys32, const uint8_t* d_aux32, size_t count,
                                          uint8_t* d_pubkeys_out, uint8_t* d_sigs64_out, uint8_t* d_ok, void* stream) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (kind > 1 || count > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    if (!d_msgs32 || !d_privkeys32 || (kind == 1 && !d_aux32) || !d_pubkeys_out || !d_sigs64_out || !d_ok)
        return UFSECP_ERR_NULL_ARG;
    return ctx->backend->sign_device((int)kind, d_msgs32, d_privkeys32, d_aux32, count, d_pubkeys_out, d_sigs64_out,
                                     d_ok, (cudaStream_t)stream);
}

ufsecp_error_t ufsecp_gpu_ext_stream(ufsecp_gpu_ctx* ctx, void** stream_out) {
    if (!ctx || !stream_out) return UFSECP_ERR_NULL_ARG;
    *stream_out = (void*)ctx->backend->stream();
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_device_props(ufsecp_gpu_ctx* ctx, int* sm_count, int* ecdsa_blocks_per_sm,
                                           int* schnorr_blocks_per_sm) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    const int sms = ctx->backend->sms();
    if (sm_count) *sm_count = sms;
    if (ecdsa_blocks_per_sm) *ecdsa_blocks_per_sm = sms ? ctx->backend->verify_grid(0) / sms : 0;
    if (schnorr_blocks_per_sm) *schnorr_blocks_per_sm = sms ? ctx->backend->verify_grid(1) / sms : 0;
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_set_variant(ufsecp_gpu_ctx* ctx, int kind, int variant) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->set_variant(kind, variant);
}

ufsecp_error_t ufsecp_gpu_ext_get_variant(ufsecp_gpu_ctx* ctx, int kind, int* variant_out, int* blocks_per_sm_out) {
    if (!ctx || !variant_out) return UFSECP_ERR_NULL_ARG;
    if (kind < 0 || kind > 1) return UFSECP_ERR_BAD_INPUT;
    *variant_out = ctx->backend->variant(kind);
    if (blocks_per_sm_out) *blocks_per_sm_out = ctx->backend->blocks_per_sm(kind, *variant_out);
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_get_small_variant(ufsecp_gpu_ctx* ctx, int kind, int* variant_out,
                                                uint32_t* items_out) {
    if (!ctx || !variant_out) return UFSECP_ERR_NULL_ARG;
    if (kind < 0 || kind > 1) return UFSECP_ERR_BAD_INPUT;
    *variant_out = ctx->backend->small_variant(kind);
    if (items_out) *items_out = *variant_out >= 0 ? ctx->backend->small_items(kind) : 0;
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_set_small_variant(ufsecp_gpu_ctx* ctx, int kind, int variant, uint32_t items) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->set_small_variant(kind, variant, items);
}

ufsecp_error_t ufsecp_gpu_ext_set_lanes(ufsecp_gpu_ctx* ctx, int kind, int lanes, uint32_t items) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->set_lanes(kind, lanes, items);
}

ufsecp_error_t ufsecp_gpu_ext_get_lanes(ufsecp_gpu_ctx* ctx, int kind, int* lanes_out, uint32_t* items_out) {
    if (!ctx || !lanes_out) return UFSECP_ERR_NULL_ARG;
    if (kind < 0 || kind > 1) return UFSECP_ERR_BAD_INPUT;
    const uint32_t items = ctx->backend->pair_items(kind);
    *lanes_out = items ? 2 : 1;
    if (items_out) *items_out = items;
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_set_inversion_group(ufsecp_gpu_ctx* ctx, int kind, int group) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->set_inversion_group(kind, group);
}

ufsecp_error_t ufsecp_gpu_ext_get_inversion_group(ufsecp_gpu_ctx* ctx, int kind, int* group_out) {
    if (!ctx || !group_out) return UFSECP_ERR_NULL_ARG;
    if (kind < 0 || kind > 1) return UFSECP_ERR_BAD_INPUT;
    *group_out = ctx->backend->inversion_group(kind);
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_set_rlc_locate(ufsecp_gpu_ctx* ctx, int on) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (on != 0 && on != 1) return ctx->backend->set_error(UFSECP_ERR_BAD_INPUT, "locate must be 0 or 1");
    ctx->backend->set_rlc_locate(on != 0);
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_set_rlc_chunk(ufsecp_gpu_ctx* ctx, uint32_t chunk) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->set_rlc_chunk(chunk);
}

ufsecp_error_t ufsecp_gpu_ext_get_rlc_chunk(ufsecp_gpu_ctx* ctx, uint32_t len, uint32_t* chunk_out) {
    if (!ctx || !chunk_out) return UFSECP_ERR_NULL_ARG;
    *chunk_out = ctx->backend->rlc_chunk(len);
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_imad_peak(ufsecp_gpu_ctx* ctx, double* ops_per_s) {
    if (!ctx || !ops_per_s) return UFSECP_ERR_NULL_ARG;
    return ctx->backend->imad_peak(ops_per_s);
}

ufsecp_error_t ufsecp_gpu_ext_probe(ufsecp_gpu_ctx* ctx, int op, int blocks, int threads, int iters, float* ms_out) {
    if (!ctx || !ms_out) return UFSECP_ERR_NULL_ARG;
    if (op < 1 || op > 16 || blocks < 1 || threads < 1 || threads > 1024 || iters < 1) return UFSECP_ERR_BAD_INPUT;
    return ctx->backend->probe(op, blocks, threads, iters, ms_out);
}

ufsecp_error_t ufsecp_gpu_ext_diag(ufsecp_gpu_ctx* ctx, uint32_t op, const uint8_t* in, size_t n, uint8_t* out) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n == 0) return UFSECP_OK;
    if (!in || !out) return UFSECP_ERR_NULL_ARG;
    static const int in_sz[12] = {0, 64, 32, 32, 32, 64, 32, 32, 32, 96, 96, 64};
    static const int out_sz[12] = {0, 32, 32, 32, 33, 32, 32, 34, 64, 65, 32, 192};
    if (op < 1 || op > 11 || n > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    return ctx->backend->diag(op, in, n, out, (size_t)in_sz[op], (size_t)out_sz[op]);
}

}  // extern "C"

// ---- RLC batch verification ------------------------------------------------

namespace {

constexpr size_t kMaxRlcItems = size_t{1} << 24;
constexpr size_t kMaxRefBatch = size_t{1} << 20;   // the reference batch API's cap

// 32 bytes from the host's random device; the reference batch API mixes them
// into a digest of the batch's inputs (RlcVerifier::verify_entries).
void fresh_seed(uint8_t seed[32]) {
    std::random_device rd;
    for (int k = 0; k < 8; ++k) {
        const uint32_t v = rd();
        memcpy(seed + 4 * k, &v, 4);
    }
}

template <class F>
ufsecp_error_t guarded(F&& run) {
    try {
        return run();
    } catch (const std::bad_alloc&) {
        return UFSECP_ERR_GPU_MEMORY;
    } catch (...) {
        return UFSECP_ERR_INTERNAL;
    }
}

// Shared body of the two reference-shaped batch calls: gate + verdicts.
ufsecp_error_t rows_verdicts(ufsecp_gpu_ctx* ctx, const uint8_t* entries, size_t n, std::vector<uint8_t>& verdicts) {
    uf::Backend& be = *ctx->backend;
    if (!be.ready()) return be.set_error(UFSECP_ERR_GPU_DEVICE, "context not ready");
    cudaError_t e = cudaSetDevice(be.device());
    if (e != cudaSuccess) return be.cuda_error(e, "cudaSetDevice");
    uint8_t seed[32];
    fresh_seed(seed);
    verdicts.assign(n, 0);
    int gate = 0;
    uint32_t where = 0;
    ctx->rlc_stats = uf::RlcStats{};
    const int rc = be.rlc().verify_entries(entries, (uint32_t)n, seed, verdicts.data(), &gate, &where,
                                           &ctx->rlc_stats);
    if (rc != UFSECP_OK) return rc;
    if (gate == UFSECP_ERR_BAD_PUBKEY) return be.set_error(gate, "non-canonical pubkey (x>=p) in batch");
    if (gate == UFSECP_ERR_BAD_SIG) return be.set_error(gate, "invalid Schnorr sig in batch");
    be.clear_error();
    return UFSECP_OK;
}

}  // namespace

extern "C" {

ufsecp_error_t ufsecp_gpu_ext_schnorr_verify_rlc(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                                 const uint8_t* pubkeys_x32, const uint8_t* sigs64, size_t count,
                                                 size_t batch_size, const uint8_t* seed32, int window_bits,
                                                 uint8_t* out_results, uint8_t* out_batch_ok) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (count > kMaxRlcItems) return ctx->backend->set_error(UFSECP_ERR_BAD_INPUT, "RLC: more than 2^24 items");
    clear_out(out_results, count, 1);
    const size_t n_batches = batch_size == 0 || batch_size >= count ? 1 : (count + batch_size - 1) / batch_size;
    clear_out(out_batch_ok, n_batches, 1);
    if (!msg_hashes32 || !pubkeys_x32 || !sigs64 || !seed32 || !out_results) return UFSECP_ERR_NULL_ARG;
    const ufsecp_error_t rc = guarded([&]() -> ufsecp_error_t {
        uf::Backend& be = *ctx->backend;
        if (!be.ready()) return be.set_error(UFSECP_ERR_GPU_DEVICE, "context not ready");
        cudaError_t e = cudaSetDevice(be.device());
        if (e != cudaSuccess) return be.cuda_error(e, "cudaSetDevice");
        ctx->rlc_stats = uf::RlcStats{};
        const int r = be.rlc().verify_host(msg_hashes32, pubkeys_x32, sigs64, (uint32_t)count,
                                           (uint32_t)std::min(batch_size, count), seed32, window_bits, out_results,
                                           out_batch_ok, &ctx->rlc_stats);
        if (r != UFSECP_OK) return (ufsecp_error_t)r;
        be.clear_error();
        return UFSECP_OK;
    });
    if (rc != UFSECP_OK) {   // fail closed, exceptions included
        clear_out(out_results, count, 1);
        clear_out(out_batch_ok, n_batches, 1);
    }
    return rc;
}

ufsecp_error_t ufsecp_gpu_ext_schnorr_verify_rlc_device(ufsecp_gpu_ctx* ctx, const uint8_t* d_msg_hashes32,
                                                        const uint8_t* d_pubkeys_x32, const uint8_t* d_sigs64,
                                                        size_t count, size_t batch_size, const uint8_t* seed32,
                                                        int window_bits, uint8_t* d_out_results,
                                                        uint8_t* out_batch_ok, void* stream) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (count == 0) return UFSECP_OK;
    if (count > kMaxRlcItems) return ctx->backend->set_error(UFSECP_ERR_BAD_INPUT, "RLC: more than 2^24 items");
    if (!d_msg_hashes32 || !d_pubkeys_x32 || !d_sigs64 || !seed32 || !d_out_results) return UFSECP_ERR_NULL_ARG;
    return guarded([&]() -> ufsecp_error_t {
        uf::Backend& be = *ctx->backend;
        if (!be.ready()) return be.set_error(UFSECP_ERR_GPU_DEVICE, "context not ready");
        cudaError_t e = cudaSetDevice(be.device());
        if (e != cudaSuccess) return be.cuda_error(e, "cudaSetDevice");
        ctx->rlc_stats = uf::RlcStats{};
        const int rc = be.rlc().verify(d_msg_hashes32, d_pubkeys_x32, d_sigs64, (uint32_t)count,
                                       (uint32_t)std::min(batch_size, count), seed32, window_bits, d_out_results,
                                       out_batch_ok, stream ? (cudaStream_t)stream : be.stream(), &ctx->rlc_stats);
        if (rc != UFSECP_OK) return rc;
        be.clear_error();
        return UFSECP_OK;
    });
}

ufsecp_error_t ufsecp_gpu_ext_rlc_input_digest(ufsecp_gpu_ctx* ctx, const uint8_t* msg_hashes32,
                                               const uint8_t* pubkeys_x32, const uint8_t* sigs64, size_t count,
                                               uint8_t out32[32]) {
    if (!ctx || !out32) return UFSECP_ERR_NULL_ARG;
    if (count > kMaxRlcItems) return ctx->backend->set_error(UFSECP_ERR_BAD_INPUT, "RLC: more than 2^24 items");
    if (count && (!msg_hashes32 || !pubkeys_x32 || !sigs64)) return UFSECP_ERR_NULL_ARG;
    return guarded([&]() -> ufsecp_error_t {
        uf::Backend& be = *ctx->backend;
        if (!be.ready()) return be.set_error(UFSECP_ERR_GPU_DEVICE, "context not ready");
        cudaError_t e = cudaSetDevice(be.device());
        if (e != cudaSuccess) return be.cuda_error(e, "cudaSetDevice");
        const int rc = be.rlc().input_digest_host(msg_hashes32, pubkeys_x32, sigs64, (uint32_t)count, out32);
        if (rc != UFSECP_OK) return rc;
        be.clear_error();
        return UFSECP_OK;
    });
}

ufsecp_error_t ufsecp_gpu_ext_rlc_stats(ufsecp_gpu_ctx* ctx, uint64_t out[4]) {
    if (!ctx || !out) return UFSECP_ERR_NULL_ARG;
    out[0] = ctx->rlc_stats.rounds;
    out[1] = ctx->rlc_stats.segments;
    out[2] = ctx->rlc_stats.leaf_items;
    out[3] = (uint64_t)ctx->rlc_stats.window_bits;
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_rlc_located(ufsecp_gpu_ctx* ctx, uint64_t* located) {
    if (!ctx || !located) return UFSECP_ERR_NULL_ARG;
    *located = ctx->rlc_stats.located;
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_rlc_key_hits(ufsecp_gpu_ctx* ctx, uint64_t* hits) {
    if (!ctx || !hits) return UFSECP_ERR_NULL_ARG;
    *hits = ctx->rlc_stats.key_hits;
    return UFSECP_OK;
}

ufsecp_error_t ufsecp_gpu_ext_schnorr_batch_verify(ufsecp_gpu_ctx* ctx, const uint8_t* entries, size_t n) {
    if (!ctx) return UFSECP_ERR_NULL_ARG;
    if (n == 0) return UFSECP_OK;
    if (!entries) return UFSECP_ERR_NULL_ARG;
    if (n > kMaxRefBatch) return ctx->backend->set_error(UFSECP_ERR_BAD_INPUT, "batch count too large");
    return guarded([&]() -> ufsecp_error_t {
        std::vector<uint8_t> v;
        const ufsecp_error_t rc = rows_verdicts(ctx, entries, n, v);
        if (rc != UFSECP_OK) return rc;
        for (size_t i = 0; i < n; ++i)
            if (!v[i]) return ctx->backend->set_error(UFSECP_ERR_VERIFY_FAIL, "batch verify failed");
        return UFSECP_OK;
    });
}

ufsecp_error_t ufsecp_gpu_ext_schnorr_batch_identify_invalid(ufsecp_gpu_ctx* ctx, const uint8_t* entries, size_t n,
                                                             size_t* invalid_out, size_t* invalid_count) {
    if (!ctx || !entries || !invalid_out || !invalid_count) return UFSECP_ERR_NULL_ARG;
    if (n > kMaxRefBatch) return ctx->backend->set_error(UFSECP_ERR_BAD_INPUT, "batch count too large");
    return guarded([&]() -> ufsecp_error_t {
        const size_t cap = *invalid_count;
        std::vector<uint8_t> v;
        if (n) {
            const ufsecp_error_t rc = rows_verdicts(ctx, entries, n, v);
            if (rc != UFSECP_OK) return rc;
        }
        size_t total = 0;
        for (size_t i = 0; i < n; ++i) {
            if (v[i]) continue;
            if (total < cap) invalid_out[total] = i;
            ++total;
        }
        *invalid_count = total;
        return UFSECP_OK;
    });
}

// ---- serving loop -------------------------------------------------------------

ufsecp_error_t ufsecp_gpu_ext_server_create(ufsecp_gpu_ctx* ctx, const ufsecp_gpu_ext_server_config_t* config,
                                            ufsecp_gpu_ext_server** server_out) {
    if (!ctx || !server_out) return UFSECP_ERR_NULL_ARG;
    *server_out = nullptr;
    return guarded([&]() -> ufsecp_error_t {
        uf::ServerConfig cfg;
        if (config) {
            cfg.slots = config->slots;
            cfg.max_launch_items = config->max_launch_items;
            cfg.memory_budget_bytes = config->memory_budget_bytes;
            cfg.batch_window_us = config->batch_window_us;
            cfg.key_cache_log2 = config->key_cache_log2 <= 1 ? 0 : config->key_cache_log2;   // NULL: the default
        }
        cudaError_t e = cudaSetDevice(ctx->backend->device());
        if (e != cudaSuccess) return ctx->backend->cuda_error(e, "cudaSetDevice");
        std::unique_ptr<ufsecp_gpu_ext_server> s(new ufsecp_gpu_ext_server());
        s->server.reset(new uf::Server(ctx->backend.get()));
        const int rc = s->server->start(cfg);
        if (rc != UFSECP_OK) return rc;
        *server_out = s.release();
        return UFSECP_OK;
    });
}

ufsecp_error_t ufsecp_gpu_ext_server_submit(ufsecp_gpu_ext_server* server, const ufsecp_gpu_ext_job_t* jobs,
                                            size_t n_jobs, uint64_t* request_id) {
    return ufsecp_gpu_ext_server_submit_cancellable(server, jobs, n_jobs, nullptr, request_id);
}

ufsecp_error_t ufsecp_gpu_ext_server_submit_cancellable(ufsecp_gpu_ext_server* server,
                                                        const ufsecp_gpu_ext_job_t* jobs, size_t n_jobs,
                                                        const ufsecp_cancel_token* cancel, uint64_t* request_id) {
    if (!server || !request_id || (n_jobs && !jobs)) return UFSECP_ERR_NULL_ARG;
    size_t total = 0;
    for (size_t j = 0; j < n_jobs; ++j) {
        const ufsecp_gpu_ext_job_t& J = jobs[j];
        if (J.kind > 1) return UFSECP_ERR_BAD_INPUT;
        if (J.count == 0) continue;
        if (!J.msg_hashes32 || !J.pubkeys || !J.sigs64 || !J.out_results) return UFSECP_ERR_NULL_ARG;
        total += J.count;
    }
    if (total > kMaxBatch) return UFSECP_ERR_BAD_INPUT;
    return guarded([&]() -> ufsecp_error_t {
        std::vector<uf::VerifyJob> v;
        v.reserve(n_jobs);
        for (size_t j = 0; j < n_jobs; ++j) {
            clear_out(jobs[j].out_results, jobs[j].count, 1);
            v.push_back(uf::VerifyJob{(int)jobs[j].kind, jobs[j].count, jobs[j].msg_hashes32, jobs[j].pubkeys,
                                      jobs[j].sigs64, jobs[j].out_results});
        }
        return server->server->submit(v.data(), v.size(), cancel, request_id);
    });
}

ufsecp_error_t ufsecp_gpu_ext_server_cancel(ufsecp_gpu_ext_server* server, uint64_t request_id, uint32_t timeout_ms) {
    if (!server) return UFSECP_ERR_NULL_ARG;
    return guarded([&]() -> ufsecp_error_t { return server->server->cancel(request_id, timeout_ms); });
}

ufsecp_error_t ufsecp_gpu_ext_server_wait(ufsecp_gpu_ext_server* server, uint64_t request_id, uint32_t timeout_ms) {
    if (!server) return UFSECP_ERR_NULL_ARG;
    return guarded([&]() -> ufsecp_error_t { return server->server->wait(request_id, timeout_ms); });
}

ufsecp_error_t ufsecp_gpu_ext_server_stats(ufsecp_gpu_ext_server* server, ufsecp_gpu_ext_server_stats_t* out,
                                           int reset) {
    if (!server || !out) return UFSECP_ERR_NULL_ARG;
    uf::ServerStats s;
    server->server->stats(&s, reset != 0);
    memset(out, 0, sizeof(*out));
    out->requests_done = s.requests_done;
    out->items_done = s.items_done;
    out->launches = s.launches;
    out->peak_budget_bytes = s.peak_budget_bytes;
    out->reserved_bytes = s.reserved_bytes;
    out->pending_requests = s.pending_requests;
    out->peak_slots_in_flight = s.peak_slots_in_flight;
    out->p50_us = s.p50_us;
    out->p99_us = s.p99_us;
    out->max_us = s.max_us;
    out->mean_us = s.mean_us;
    out->busy_s = s.busy_s;
    out->span_s = s.span_s;
    out->cache_lookups = s.cache_lookups;
    out->cache_hits = s.cache_hits;
    return UFSECP_OK;
}

void ufsecp_gpu_ext_server_destroy(ufsecp_gpu_ext_server* server) {
    try {
        delete server;
    } catch (...) {
    }
}

}  // extern "C"

// ---- engine hook provider ------------------------------------------------------

namespace {

std::mutex g_hook_mu;
std::unique_ptr<ufsecp_gpu_ctx> g_hook_ctx;   // process-wide context of the hook (device 0)
bool g_hook_probed = false;
uint64_t g_hook_handled = 0, g_hook_declined = 0;

}  // namespace

extern "C" {

int ufsecp_gpu_ext_engine_columns_hook(int kind, const uint8_t* digests32, const uint8_t* keys,
                                       const uint8_t* sigs64, size_t count, uint8_t* out_results) noexcept {
    try {
        std::lock_guard<std::mutex> lk(g_hook_mu);
        if (!g_hook_probed) {
            g_hook_probed = true;
            if (cuda_device_count() > 0) {
                std::unique_ptr<ufsecp_gpu_ctx> c(new ufsecp_gpu_ctx());
                c->backend_id = UFSECP_GPU_BACKEND_CUDA;
                c->device_index = 0;
                c->backend.reset(new uf::Backend());
                if (c->backend->init(0) == UFSECP_OK && c->backend->ready()) g_hook_ctx = std::move(c);
            }
        }
        const bool usable = g_hook_ctx && (kind == 0 || kind == 1) && digests32 && keys && sigs64 && out_results &&
                            count > 0 && count <= kMaxBatch;
        if (!usable) {
            ++g_hook_declined;
            return -1;
        }
        int rc;
        try {
            rc = g_hook_ctx->backend->verify_host(kind == 0 ? 2 : 1, digests32, keys, sigs64, count, out_results,
                                                  false);
        } catch (...) {
            rc = UFSECP_ERR_INTERNAL;
        }
        if (rc != UFSECP_OK) {
            ++g_hook_declined;
            return -1;   // operational error: the engine falls back to its CPU path
        }
        ++g_hook_handled;
        for (size_t i = 0; i < count; ++i)
            if (out_results[i] == 0) return 0;
        return 1;
    } catch (...) {
        return -1;
    }
}

void ufsecp_gpu_ext_engine_hook_counters(uint64_t* handled, uint64_t* declined) {
    std::lock_guard<std::mutex> lk(g_hook_mu);
    if (handled) *handled = g_hook_handled;
    if (declined) *declined = g_hook_declined;
}

int ufsecp_gpu_ext_engine_hook_inject_fault(uint32_t after, int kind) {
    if (kind < 0 || kind > 3) return UFSECP_ERR_BAD_INPUT;
    std::lock_guard<std::mutex> lk(g_hook_mu);
    if (!g_hook_probed) {
        g_hook_probed = true;
        if (cuda_device_count() > 0) {
            std::unique_ptr<ufsecp_gpu_ctx> c(new ufsecp_gpu_ctx());
            c->backend_id = UFSECP_GPU_BACKEND_CUDA;
            c->device_index = 0;
            c->backend.reset(new uf::Backend());
            if (c->backend->init(0) == UFSECP_OK && c->backend->ready()) g_hook_ctx = std::move(c);
        }
    }
    if (!g_hook_ctx) return UFSECP_ERR_GPU_UNAVAILABLE;
    g_hook_ctx->backend->arm_fault(after, kind);
    return UFSECP_OK;
}

void ufsecp_gpu_ext_engine_hook_release(void) {
    std::lock_guard<std::mutex> lk(g_hook_mu);
    g_hook_ctx.reset();
    g_hook_probed = false;
}

}  // extern "C"
