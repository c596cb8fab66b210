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

// One signature per thread, grid-stride.  Inputs: msgs 32 B, pubs 33 B
// (ECDSA, SEC1 compressed) or 32 B (BIP-340 x-only), sigs 64 B, all
// contiguous; msgs / x-only pubs / sigs must be 16-byte aligned.  out[i] = 1
// for a valid signature, 0 otherwise.  With collect != 0 a valid signature
// writes 0 and an invalid one leaves out[i] untouched.
cudaError_t launch_ecdsa_verify(const uint8_t* msgs, const uint8_t* pubs33, const uint8_t* sigs,
                                uint32_t n, const void* d_gtab, uint8_t* out, int collect,
                                int grid, cudaStream_t s);
cudaError_t launch_schnorr_verify(const uint8_t* msgs, const uint8_t* xonly32, const uint8_t* sigs,
                                  uint32_t n, const void* d_gtab, uint8_t* out, int collect,
                                  int grid, cudaStream_t s);

// Batch signer (workload generator): kind 0 = ECDSA (pubs 33 B), 1 = BIP-340
// (pubs 32 B x-only, auxs 32 B aux_rand).  ok[i] = 0 for an invalid key.
cudaError_t launch_sign(int kind, const uint8_t* msgs, const uint8_t* sks, const uint8_t* auxs, uint32_t n,
                        const void* d_gtab, uint8_t* pubs, uint8_t* sigs, uint8_t* ok, int grid, cudaStream_t s);

// Blocks per SM the verify kernels reach (occupancy query).
int verify_blocks_per_sm(int kind);

// Building-block probes for the tests (op codes in ufsecp_gpu_ext.h).
cudaError_t launch_diag(uint32_t op, const uint8_t* in, uint32_t n, uint8_t* out,
                        const void* d_gtab, cudaStream_t s);

// Integer multiply-add issue-rate probe: every thread runs `iters` rounds of
// 16 independent 32-bit IMADs.  Returns a checksum so the work is not elided.
cudaError_t launch_imad_peak(uint32_t* d_sink, int blocks, int threads, int iters, cudaStream_t s);

// Building-block throughput probe (op codes in ufsecp_gpu_ext.h).
cudaError_t launch_probe(int op, int blocks, int threads, int iters, uint32_t* sink, cudaStream_t s);

}  // namespace uf
