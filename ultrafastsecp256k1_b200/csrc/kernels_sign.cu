// Batch signing kernel: the synthetic-workload generator (not on the verify
// path).  One signature per thread with the signers of sign.cuh; the
// generator multiplications use the context's G tables.
#include "kernels.h"
#include "sign.cuh"
#include "dev_tables.cuh"

namespace uf {

__global__ void __launch_bounds__(128)
k_sign(int kind, const uint8_t* __restrict__ msgs, const uint8_t* __restrict__ sks, const uint8_t* __restrict__ auxs,
       uint32_t n, const uint4* __restrict__ gt, uint8_t* __restrict__ pubs, uint8_t* __restrict__ sigs,
       uint8_t* __restrict__ ok) {
    const GlobalGT g{gt};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint8_t m[32], k[32], a[32], pub[33], sig[64];
        for (int j = 0; j < 32; ++j) { m[j] = msgs[32ull * i + j]; k[j] = sks[32ull * i + j]; }
        bool good;
        if (kind == 0) {
            good = ecdsa_sign_one(pub, sig, m, k, g);
            for (int j = 0; j < 33; ++j) pubs[33ull * i + j] = pub[j];
        } else {
            for (int j = 0; j < 32; ++j) a[j] = auxs[32ull * i + j];
            good = schnorr_sign_one(pub, sig, m, k, a, g);
            for (int j = 0; j < 32; ++j) pubs[32ull * i + j] = pub[j];
        }
        for (int j = 0; j < 64; ++j) sigs[64ull * i + j] = sig[j];
        ok[i] = good ? 1 : 0;
    }
}

cudaError_t launch_sign(int kind, const uint8_t* msgs, const uint8_t* sks, const uint8_t* auxs, uint32_t n,
                        const void* d_gtab, uint8_t* pubs, uint8_t* sigs, uint8_t* ok, int grid, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const int need = (int)((n + 127) / 128);
    if (grid <= 0 || grid > need) grid = need;
    k_sign<<<grid, 128, 0, s>>>(kind, msgs, sks, auxs, n, reinterpret_cast<const uint4*>(d_gtab), pubs, sigs, ok);
    return cudaGetLastError();
}

}  // namespace uf
