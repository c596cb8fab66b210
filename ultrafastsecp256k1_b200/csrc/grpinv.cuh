// Montgomery batch inversion across the threads of a block.
//
// Role in the reference: batch_inverse_montgomery
// (src/cuda/include/batch_inversion.cuh:194) and the shared-Z trick inside
// shamir_double_mul_glv (src/cuda/include/secp256k1.cuh:3730-3760); on the CPU
// the ECDSA batch s^-1 arena (src/cpu/src/batch_verify.cpp:594-609).  Here the
// group is the G threads of one block, each with its own value (a signature's
// table Z product, its final Z, or its ECDSA s): one modular inversion serves
// all G of them.
//
// SIMT shapes the design: a per-lane inversion costs a warp one inversion's
// instruction stream whatever the lane count, so sharing an inversion inside a
// warp saves nothing.  Sharing it across the block's warps does: warp 0 alone
// runs the prefix products, the one (variable-time safegcd) inversion and the
// back-substitution while the other warps wait at the barrier and their SM
// issue slots go to other blocks.  Per value that is about 24 / 32 field
// multiplies plus 1 / (G / 32) of an inversion for warp 0, instead of one
// inversion per warp.
//
//   1. every thread stores its value in shared memory ([word][thread] words);
//   2. warp 0, lane l holding values q l .. q l + q - 1 (q = G / 32): local
//      prefix products, a warp scan (Hillis-Steele, shuffles) of the lanes'
//      products and a suffix scan, the inverse of the block's product
//      (computed by every lane on the same value: no divergence), then the
//      inverse of each value as (inverse of the prefix through it) x (prefix
//      before it);
//   3. every thread reads its inverse back.
//
// Every thread of the block must call group_invert the same number of times
// (barriers inside).  A thread with nothing to invert passes one.  A zero value
// would zero the product and with it every inverse of the block, so a zero is
// replaced by one and reported: the caller treats that item as failed (no
// correct verify ever passes zero: table and accumulator Z of finite points
// and ECDSA s are non-zero).
#pragma once
#include "common.cuh"
#include "fe.cuh"
#include "fn.cuh"
#include "point.cuh"

namespace uf {

// Field (mod p) and scalar (mod n) operations for group_invert.
struct GrpFieldOps {
    typedef Fe T;
    __device__ __forceinline__ static void mul(Fe& r, const Fe& a, const Fe& b) { fe_mul(r, a, b); }
    __device__ __forceinline__ static void inv(Fe& r, const Fe& a) { fe_inv(r, a); }
    __device__ __forceinline__ static bool is_zero(const Fe& a) { return fe_is_zero(a); }
};
struct GrpScalarOps {
    typedef Sc T;
    __device__ __forceinline__ static void mul(Sc& r, const Sc& a, const Sc& b) { sc_mul(r, a, b); }
    __device__ __forceinline__ static void inv(Sc& r, const Sc& a) { sc_inv(r, a); }
    __device__ __forceinline__ static bool is_zero(const Sc& a) { return sc_is_zero(a); }
};

template <class V>
__device__ __forceinline__ void grp_one(V& r) {
    r.v[0] = 1;
    UF_UNROLL
    for (int i = 1; i < 8; ++i) r.v[i] = 0;
}

template <class V>
__device__ __forceinline__ V grp_shfl_up(const V& a, int d) {
    V r;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_up_sync(0xFFFFFFFFu, a.v[i], d);
    return r;
}

template <class V>
__device__ __forceinline__ V grp_shfl_down(const V& a, int d) {
    V r;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_down_sync(0xFFFFFFFFu, a.v[i], d);
    return r;
}

template <class V>
__device__ __forceinline__ V grp_shfl(const V& a, int src) {
    V r;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = __shfl_sync(0xFFFFFFFFu, a.v[i], src);
    return r;
}

// Warp 0's part: the values of the block in sh are replaced by their
// inverses.  Out of line, so that its registers do not add to the pressure of
// the verify code around it.
template <class Ops, int G>
__device__ __noinline__ void grp_warp0(uint32_t* sh) {
    typedef typename Ops::T V;
    constexpr int Q = G / 32;     // values per lane of warp 0
    const int t = threadIdx.x;
    V a[Q], p[Q];
    UF_UNROLL
    for (int j = 0; j < Q; ++j) {
        UF_UNROLL
        for (int i = 0; i < 8; ++i) a[j].v[i] = sh[i * G + Q * t + j];
    }
    p[0] = a[0];
    UF_UNROLL
    for (int j = 1; j < Q; ++j) Ops::mul(p[j], p[j - 1], a[j]);
    // inclusive prefix and suffix products of the lanes' products
    V incl = p[Q - 1], suf = p[Q - 1];
    UF_UNROLL
    for (int d = 1; d < 32; d <<= 1) {
        const V o = grp_shfl_up(incl, d);
        if (t >= d) Ops::mul(incl, incl, o);
        const V u = grp_shfl_down(suf, d);
        if (t + d < 32) Ops::mul(suf, suf, u);
    }
    V excl = grp_shfl_up(incl, 1), sexcl = grp_shfl_down(suf, 1);
    if (t == 0) grp_one(excl);
    if (t == 31) grp_one(sexcl);
    V total = grp_shfl(incl, 31), q;
    Ops::inv(q, total);               // the same value in every lane: one inversion
    Ops::mul(q, q, sexcl);            // inverse of the prefix through this lane's last value
    for (int j = Q - 1; j >= 0; --j) {
        V before = excl, r;
        if (j > 0) Ops::mul(before, excl, p[j - 1]);
        Ops::mul(r, q, before);       // a[j]^-1
        if (j > 0) Ops::mul(q, q, a[j]);
        UF_UNROLL
        for (int i = 0; i < 8; ++i) sh[i * G + Q * t + j] = r.v[i];
    }
}

// x <- x^-1 for every thread of the block (G = blockDim.x, a multiple of 32,
// at most 128).  sh: 8 * G words of shared memory.  Returns false when this
// thread's value was zero (x is then left as one).
template <class Ops, int G>
__device__ __forceinline__ bool group_invert(typename Ops::T& x, uint32_t* sh) {
    static_assert(G % 32 == 0 && G >= 32 && G <= 128, "group: 1..4 warps");
    const int t = threadIdx.x;
    const bool zero = Ops::is_zero(x);
    if (zero) grp_one(x);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) sh[i * G + t] = x.v[i];
    __syncthreads();
    if (t < 32) grp_warp0<Ops, G>(sh);
    __syncthreads();
    UF_UNROLL
    for (int i = 0; i < 8; ++i) x.v[i] = sh[i * G + t];
    __syncthreads();                      // the next call may overwrite sh
    return !zero;
}

}  // namespace uf
