// Per-signature verify kernels (the plain form: one signature per thread).
//
// The reference's ecdsa_verify_batch_kernel / schnorr_verify_batch_kernel
// (src/cuda/src/secp256k1.cu:153, :232) re-designed for B200; ecmult.cuh has the
// scalar-multiplication design.  Memory layout per block:
//   * dynamic shared memory holds each thread's 1P..8P table as
//     [entry][quad][thread] uint4, so a warp's data-dependent table reads are
//     bank-conflict free (each thread owns its own bank column);
//   * the 1..2^(UF_GWIN-1) multiples of G and lambda*G (64 MB for 20-bit
//     windows) stay in global memory, served from L2 through the read-only path;
//   * Booth digits live in a small per-thread local array indexed uniformly
//     across the warp (coalesced, L1 resident).
//
// This file is compiled several times (UF_VARIANT 0..11) with different
// code-size choices (UF_NOINLINE_POINT / UF_NOINLINE_FIELD, see common.cuh)
// and, for variants 9..11, other window widths (UF_PWIN P-window bits, 3 / 5;
// UF_GWIN G-window bits, 18 / 16, over generator tables of that width); the
// backend picks a variant per signature kind (tuned per device).
#include "kernels.h"
#include "verify.cuh"
#include "dev_tables.cuh"

#ifndef UF_VARIANT
#define UF_VARIANT 0
#endif
// Block size and the minimum resident blocks per SM asked of the register
// allocator.  The default is 128 threads with no register cap (3 blocks per SM:
// registers and the 512-byte per-thread table both limit it); 64-thread blocks
// capped at 128 registers fit 7 blocks, 14 warps per SM.
#ifndef UF_PLAIN_THREADS
#define UF_PLAIN_THREADS kVerifyThreads
#endif
#ifdef UF_MIN_BLOCKS
#define UF_BOUNDS __launch_bounds__(UF_PLAIN_THREADS, UF_MIN_BLOCKS)
#else
#define UF_BOUNDS __launch_bounds__(UF_PLAIN_THREADS)
#endif
// UF_TAB7: 1P kept in registers, 448 bytes of shared memory per thread.
#ifdef UF_TAB7
#define UF_TAB_T SmemTab7
#define UF_SMEM_PER_THREAD ((size_t)(kPTab - 1) * 64)
#else
#define UF_TAB_T const SmemTab
#define UF_SMEM_PER_THREAD ((size_t)kPTab * 64)   // 2^(UF_PWIN-1) table points of 64 bytes
#endif
#define UF_CAT2(a, b) a##b
#define UF_CAT(a, b) UF_CAT2(a, b)

namespace uf {
namespace UF_CAT(vk, UF_VARIANT) {

// kKind: 0 ECDSA (compact r || s), 1 BIP-340, 2 ECDSA (opaque little-endian r, s; high-S accepted)
template <int kKind>
__global__ void UF_BOUNDS
k_verify(const uint8_t* __restrict__ msgs, const uint8_t* __restrict__ pubs, const uint8_t* __restrict__ sigs,
         uint32_t n, const uint4* __restrict__ gt, uint8_t* __restrict__ out, int collect) {
    extern __shared__ uint4 smem_tab[];
    UF_TAB_T tab{smem_tab + threadIdx.x, blockDim.x};
    const GlobalGT g{gt};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t mw[8], sw[16];
        load_words8(mw, msgs + 32ull * i);
        load_words8(sw, sigs + 64ull * i);
        load_words8(sw + 8, sigs + 64ull * i + 32);
        bool ok;
        if (kKind == 0) {
            ok = ecdsa_verify_one(mw, pubs + 33ull * i, sw, tab, g);
        } else if (kKind == 2) {
            ok = ecdsa_verify_opaque_one(mw, pubs + 33ull * i, sw, tab, g);
        } else {
            uint32_t pw[8];
            load_words8(pw, pubs + 32ull * i);
            ok = schnorr_verify_one(mw, pw, sw, tab, g);
        }
        if (collect) {
            if (ok) out[i] = 0;
        } else {
            out[i] = ok ? 1 : 0;
        }
    }
}

}  // namespace vkN

cudaError_t UF_CAT(launch_verify_v, UF_VARIANT)(int kind, const uint8_t* msgs, const uint8_t* pubs,
                                                const uint8_t* sigs, uint32_t n, const void* d_gtab, uint8_t* out,
                                                int collect, int grid, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    // the shared-memory opt-in was set per device by verify_occupancy_v*() at context creation
    const size_t smem = UF_PLAIN_THREADS * UF_SMEM_PER_THREAD;
    const int need = (int)((n + UF_PLAIN_THREADS - 1) / UF_PLAIN_THREADS);
    if (grid <= 0 || grid > need) grid = need;
    const uint4* gt = reinterpret_cast<const uint4*>(d_gtab);
    if (kind == 0)
        UF_CAT(vk, UF_VARIANT)::k_verify<0><<<grid, UF_PLAIN_THREADS, smem, s>>>(msgs, pubs, sigs, n, gt, out, collect);
    else if (kind == 2)
        UF_CAT(vk, UF_VARIANT)::k_verify<2><<<grid, UF_PLAIN_THREADS, smem, s>>>(msgs, pubs, sigs, n, gt, out, collect);
    else
        UF_CAT(vk, UF_VARIANT)::k_verify<1><<<grid, UF_PLAIN_THREADS, smem, s>>>(msgs, pubs, sigs, n, gt, out, collect);
    return cudaGetLastError();
}

int UF_CAT(verify_occupancy_v, UF_VARIANT)(int kind) {
    int blocks = 0;
    const size_t smem = UF_PLAIN_THREADS * UF_SMEM_PER_THREAD;
    if (kind != 1) {
        // the opaque ECDSA instance shares kind 0's shape; opt both in
        auto f2 = UF_CAT(vk, UF_VARIANT)::k_verify<2>;
        cudaFuncSetAttribute(f2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        auto f = UF_CAT(vk, UF_VARIANT)::k_verify<0>;
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, f, UF_PLAIN_THREADS, smem);
    } else {
        auto f = UF_CAT(vk, UF_VARIANT)::k_verify<1>;
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, f, UF_PLAIN_THREADS, smem);
    }
    return blocks;
}

}  // namespace uf
