// The RLC kernels with one serial chain per bucket, segment or window: the
// merge of a bucket's chunk sums, the running sums, the window combination
// and Horner.  The last three run a few thousand threads at most, so a
// chain's latency, not the issue rate, sets their time, and the merge's
// chains are short and uneven.  This file is compiled with the field and
// point operations inlined, so that the independent products inside a
// doubling or an addition overlap (measured faster for these kernels, slower
// for the wide kernels of rlc.cu).
#include "rlc_serial.h"

#include "point.cuh"

namespace uf {

namespace {

using namespace rlcdev;

// One thread per (segment, window, sub-range j of m buckets):
// T_j = sum_b bucket_b, U_j = sum_b (b - j m + 1) bucket_b by running sums.
__global__ void __launch_bounds__(128)
k_rlc_wpart(RoundGeo g, const uint4* __restrict__ buckets, uint4* __restrict__ wu, uint4* __restrict__ wt) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.n_seg * (uint32_t)(g.W * g.S)) return;
    const uint32_t sw = q / (uint32_t)g.S, j = q - sw * (uint32_t)g.S;
    const int m = g.B / g.S;
    const uint4* base = buckets + kJacQ * ((uint64_t)sw * g.B + (uint64_t)j * m);
    Jac run, tot, b;
    jac_set_inf(run);
    jac_set_inf(tot);
    for (int k = m - 1; k >= 0; --k) {
        load_jac(base + kJacQ * k, b);
        jac_add(run, b);
        jac_add(tot, run);
    }
    store_jac(wu + kJacQ * (uint64_t)q, tot);
    store_jac(wt + kJacQ * (uint64_t)q, run);
}

// One thread per (segment, window): window sum = sum_j U_j + m sum_j j T_j.
__global__ void __launch_bounds__(128)
k_rlc_wcomb(RoundGeo g, const uint4* __restrict__ wu, const uint4* __restrict__ wt, uint4* __restrict__ wins) {
    const uint32_t sw = blockIdx.x * blockDim.x + threadIdx.x;
    if (sw >= g.n_seg * (uint32_t)g.W) return;
    const uint64_t q0 = (uint64_t)sw * g.S;
    Jac acc, run, jt, p;
    jac_set_inf(acc);
    jac_set_inf(run);
    jac_set_inf(jt);
    for (int j = g.S - 1; j >= 1; --j) {
        load_jac(wt + kJacQ * (q0 + j), p);
        jac_add(run, p);
        jac_add(jt, run);
    }
    for (int m = g.B / g.S; m > 1; m >>= 1) jac_dbl(jt);
    for (int j = 0; j < g.S; ++j) {
        load_jac(wu + kJacQ * (q0 + j), p);
        jac_add(acc, p);
    }
    jac_add(acc, jt);
    store_jac(wins + kJacQ * (uint64_t)sw, acc);
}

// One thread per segment: Horner over the windows; ok = 1 if the sum is
// infinity, | 2 if the segment holds an item that failed to parse.
__global__ void __launch_bounds__(64)
k_rlc_finish(RoundGeo g, const uint4* __restrict__ wins, const uint32_t* __restrict__ segbad,
             uint8_t* __restrict__ segok, uint4* __restrict__ segpt) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.n_seg) return;
    const uint4* base = wins + kJacQ * (uint64_t)s * g.W;
    Jac acc, w;
    load_jac(base + kJacQ * (g.W - 1), acc);
    for (int k = g.W - 2; k >= 0; --k) {
        for (int d = 0; d < g.c; ++d) jac_dbl(acc);
        load_jac(base + kJacQ * k, w);
        jac_add(acc, w);
    }
    segok[s] = (uint8_t)((acc.inf ? 1 : 0) | (segbad[s] ? 2 : 0));
    store_jac(segpt + kJacQ * (uint64_t)s, acc);
}

// Buckets with 0 or >= 2 chunks: infinity, or the sum of their partials.
// A bucket of more than kHeavyChunks chunks (skewed digits: the top windows
// of a locate round's j-scaled magnitudes put most points of a segment into a
// few buckets) is left to k_rlc_bucket_heavy: its key goes to `heavy`.
// Adds a chunk partial: affine (Z = 1, from the affine chunk trees) or Jacobian.
template <bool kAff>
__device__ __forceinline__ void add_partial(Jac& acc, const uint4* q) {
    Jac p;
    load_jac(q, p);
    if (!kAff) jac_add(acc, p);
    else if (!p.inf) jac_add_aff(acc, p.X, p.Y);
}

template <bool kAff>
__global__ void __launch_bounds__(128)
k_rlc_bucket_fin(const uint32_t* __restrict__ coff, uint32_t K, const uint4* __restrict__ partials,
                 uint4* __restrict__ buckets, uint32_t* __restrict__ heavy) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= K) return;
    const uint32_t c0 = coff[k], c1 = coff[k + 1];
    if (c1 - c0 == 1) return;
    if (c1 - c0 > kHeavyChunks) {
        heavy[1 + atomicAdd(&heavy[0], 1u)] = k;
        return;
    }
    Jac acc;
    jac_set_inf(acc);
    for (uint32_t c = c0; c < c1; ++c) add_partial<kAff>(acc, partials + kJacQ * (uint64_t)c);
    store_jac(buckets + kJacQ * (uint64_t)k, acc);
}

// Jacobian point from lane `src` of the warp (every lane calls it).
__device__ __forceinline__ Jac shfl_jac(const Jac& a, int src) {
    Jac b;
    for (int k = 0; k < 8; ++k) {
        b.X.v[k] = __shfl_sync(0xFFFFFFFFu, a.X.v[k], src);
        b.Y.v[k] = __shfl_sync(0xFFFFFFFFu, a.Y.v[k], src);
        b.Z.v[k] = __shfl_sync(0xFFFFFFFFu, a.Z.v[k], src);
    }
    b.inf = __shfl_sync(0xFFFFFFFFu, a.inf ? 1 : 0, src) != 0;
    return b;
}

// One warp per heavy bucket (heavy[0] of them, keys in heavy[1..]): lane l
// sums partials l, l + 32, ..., then the 32 lane sums meet in a shuffle tree:
// about chunks / 32 + 5 serial additions instead of chunks.
template <bool kAff>
__global__ void __launch_bounds__(128)
k_rlc_bucket_heavy(const uint32_t* __restrict__ coff, const uint4* __restrict__ partials,
                   uint4* __restrict__ buckets, const uint32_t* __restrict__ heavy) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < heavy[0]; w += warps) {
        const uint32_t k = heavy[1 + w];
        const uint32_t c0 = coff[k], c1 = coff[k + 1];
        Jac acc;
        jac_set_inf(acc);
        for (uint32_t c = c0 + lane; c < c1; c += 32) add_partial<kAff>(acc, partials + kJacQ * (uint64_t)c);
        for (int o = 16; o > 0; o >>= 1) {
            const Jac other = shfl_jac(acc, (int)(lane ^ (uint32_t)o));
            jac_add(acc, other);
        }
        if (lane == 0) store_jac(buckets + kJacQ * (uint64_t)k, acc);
    }
}

inline unsigned grid_of(uint64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

cudaError_t launch_rlc_windows(const RoundGeo& g, const uint4* buckets, uint4* wu, uint4* wt, uint4* wins,
                               const uint32_t* segbad, uint8_t* segok, uint4* segpt, cudaStream_t s) {
    const uint64_t n_seg = g.n_seg;
    k_rlc_wpart<<<grid_of(n_seg * g.W * g.S, 128), 128, 0, s>>>(g, buckets, wu, wt);
    k_rlc_wcomb<<<grid_of(n_seg * g.W, 128), 128, 0, s>>>(g, wu, wt, wins);
    k_rlc_finish<<<grid_of(n_seg, 64), 64, 0, s>>>(g, wins, segbad, segok, segpt);
    return cudaGetLastError();
}

cudaError_t launch_rlc_bucket_merge(bool affine, const uint32_t* coff, uint32_t K, const uint4* partials,
                                    uint4* buckets, uint32_t* heavy, int heavy_grid, cudaStream_t s) {
    if (affine) {
        k_rlc_bucket_fin<true><<<grid_of(K, 128), 128, 0, s>>>(coff, K, partials, buckets, heavy);
        k_rlc_bucket_heavy<true><<<heavy_grid, 128, 0, s>>>(coff, partials, buckets, heavy);
    } else {
        k_rlc_bucket_fin<false><<<grid_of(K, 128), 128, 0, s>>>(coff, K, partials, buckets, heavy);
        k_rlc_bucket_heavy<false><<<heavy_grid, 128, 0, s>>>(coff, partials, buckets, heavy);
    }
    return cudaGetLastError();
}

}  // namespace uf
