// Launchers of the RLC kernels that run one serial chain per segment or
// window (rlc_serial.cu): few threads, so latency-bound, and compiled with the
// field and point operations inlined (the wide kernels of rlc.cu keep them out
// of line for the instruction cache).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rlc_dev.cuh"

namespace uf {

// Running sums over each (segment, window)'s buckets in sub-ranges, their
// combination per window, and Horner over the windows per segment:
// segok[s] = 1 when segment s's sum is infinity, | 2 when it holds an item
// that failed to parse; segpt[s] = the sum.
cudaError_t launch_rlc_windows(const rlcdev::RoundGeo& g, const uint4* buckets, uint4* wu, uint4* wt, uint4* wins,
                               const uint32_t* segbad, uint8_t* segok, uint4* segpt, cudaStream_t s);

// Buckets of two or more chunks: the sum of their chunk partials (mixed
// additions when the partials are affine, else Jacobian), by a thread per
// bucket, or by a warp per bucket of more than kHeavyChunks chunks (their keys
// listed in heavy[1..heavy[0]] by the first kernel).
cudaError_t launch_rlc_bucket_merge(bool affine, const uint32_t* coff, uint32_t K, const uint4* partials,
                                    uint4* buckets, uint32_t* heavy, int heavy_grid, cudaStream_t s);

}  // namespace uf
