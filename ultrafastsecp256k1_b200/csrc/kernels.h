// Launch wrappers for the sm_100a kernels (C++ linkage, used by the backend).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace uf {

// Byte size of the per-context generator tables: 128 multiples of G and of
// lambda*G, affine, 64 bytes each.
constexpr size_t kGTableBytes = 2 * 128 * 64;

// Threads per block of the per-signature verify kernels and the dynamic
// shared memory each block needs (8 table points x 64 bytes per thread).
constexpr int kVerifyThreads = 128;
constexpr size_t kVerifySmemPerThread = 8 * 64;

cudaError_t launch_gtable_init(void* d_gtab, cudaStream_t s);

// One signature per thread, grid-stride.  kind 0 = ECDSA (pubs: 33-byte SEC1
// compressed), 1 = BIP-340 (pubs: 32-byte x-only).  msgs 32 B, sigs 64 B, all
// contiguous; msgs / x-only pubs / sigs must be 16-byte aligned.  out[i] = 1
// for a valid signature, 0 otherwise.  With collect != 0 a valid signature
// writes 0 and an invalid one leaves out[i] untouched.  Variants 0..5 are the
// same kernel built with different code-size choices (kernels_verify.cu).
constexpr int kVerifyVariants = 6;
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
int verify_occupancy_v0(int kind);
int verify_occupancy_v1(int kind);
int verify_occupancy_v2(int kind);
int verify_occupancy_v3(int kind);
int verify_occupancy_v4(int kind);
int verify_occupancy_v5(int kind);

// Batch signer (workload generator): kind 0 = ECDSA (pubs 33 B), 1 = BIP-340
// (pubs 32 B x-only, auxs 32 B aux_rand).  ok[i] = 0 for an invalid key.
cudaError_t launch_sign(int kind, const uint8_t* msgs, const uint8_t* sks, const uint8_t* auxs, uint32_t n,
                        const void* d_gtab, uint8_t* pubs, uint8_t* sigs, uint8_t* ok, int grid, cudaStream_t s);

// Building-block probes for the tests (op codes in ufsecp_gpu_ext.h).
cudaError_t launch_diag(uint32_t op, const uint8_t* in, uint32_t n, uint8_t* out,
                        const void* d_gtab, cudaStream_t s);

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

}  // namespace uf
