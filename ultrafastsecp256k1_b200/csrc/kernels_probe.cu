// Throughput probes of the verify path's building blocks, one copy per
// verify-kernel variant (the same field / point code generation) (field mul / sqr,
// inversions, sqrt, point doubling and mixed add, GLV split, the challenge
// hash).  Each thread runs `iters` rounds on values held in registers; the
// host times the launch with CUDA events and reports operations per second,
// which is how the kernel design is checked against the IMAD issue rate.
#include "kernels.h"
#include "verify.cuh"

#ifndef UF_VARIANT
#define UF_VARIANT 0
#endif
#define UF_CAT2(a, b) a##b
#define UF_CAT(a, b) UF_CAT2(a, b)

namespace uf {
namespace UF_CAT(pk, UF_VARIANT) {

__device__ __forceinline__ void seed_fe(Fe& a, uint32_t s) {
    for (int i = 0; i < 8; ++i) {
        s = s * 1664525u + 1013904223u;
        a.v[i] = s;
    }
    a.v[7] &= 0x7FFFFFFFu;
}

__global__ void k_probe(int op, int iters, uint32_t* sink) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    Fe a, b, c, d;
    seed_fe(a, tid * 4 + 1);
    seed_fe(b, tid * 4 + 2);
    seed_fe(c, tid * 4 + 3);
    seed_fe(d, tid * 4 + 4);
    uint32_t acc = 0;
    switch (op) {
        case 1:  // two independent fe_mul chains
            for (int i = 0; i < iters; ++i) { fe_mul(a, a, b); fe_mul(c, c, d); }
            break;
        case 2:  // two independent fe_sqr chains
            for (int i = 0; i < iters; ++i) { fe_sqr(a, a); fe_sqr(c, c); }
            break;
        case 3:  // field inverse (divsteps)
            for (int i = 0; i < iters; ++i) { fe_inv(a, a); a.v[0] |= 1; }
            break;
        case 4:  // square-root exponentiation
            for (int i = 0; i < iters; ++i) fe_sqrt_candidate(a, a);
            break;
        case 5: {  // Jacobian doubling
            Jac P;
            P.X = a; P.Y = b; P.Z = c; P.inf = false;
            for (int i = 0; i < iters; ++i) jac_dbl(P);
            a = P.X;
            break;
        }
        case 6: {  // Jacobian + affine
            Jac P;
            P.X = a; P.Y = b; P.Z = c; P.inf = false;
            for (int i = 0; i < iters; ++i) jac_add_aff(P, d, b);
            a = P.X;
            break;
        }
        case 7: {  // scalar inverse mod n
            Sc s;
            for (int k = 0; k < 8; ++k) s.v[k] = a.v[k];
            for (int i = 0; i < iters; ++i) { sc_inv(s, s); s.v[0] |= 1; }
            a.v[0] = s.v[0];
            break;
        }
        case 8: {  // GLV split
            Sc s;
            for (int k = 0; k < 8; ++k) s.v[k] = a.v[k];
            GlvSplit g;
            for (int i = 0; i < iters; ++i) { glv_split(g, s); s.v[0] ^= g.k1[0]; }
            a.v[0] = s.v[0];
            break;
        }
        case 9: {  // BIP-340 challenge (2 compressions)
            uint32_t h[8];
            for (int i = 0; i < iters; ++i) { bip340_challenge(h, a.v, b.v, c.v); a.v[0] ^= h[0]; }
            break;
        }
#if defined(__CUDA_ARCH__)
        // Integer multiply-add forms, 8 independent chains per thread, 8 ops
        // per round; every multiplier comes from the previous round's result
        // so that no product is loop-invariant: the issue cost of each form.
        case 10:  // mad.lo.u32
            for (int i = 0; i < iters; ++i)
                for (int k = 0; k < 8; ++k)
                    asm("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a.v[k]) : "r"(b.v[k]), "r"(c.v[k]));
            break;
        case 11:  // mad.hi.u32
            for (int i = 0; i < iters; ++i)
                for (int k = 0; k < 8; ++k)
                    asm("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a.v[k]) : "r"(b.v[k]), "r"(c.v[k]));
            break;
        case 12: {  // mad.wide.u32: w = lo(w) * b + w
            uint64_t w[8];
            for (int k = 0; k < 8; ++k) w[k] = ((uint64_t)c.v[k] << 32) | a.v[k];
            for (int i = 0; i < iters; ++i)
                for (int k = 0; k < 8; ++k)
                    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(w[k]) : "r"((uint32_t)w[k]), "r"(b.v[k]));
            for (int k = 0; k < 8; ++k) a.v[k] = (uint32_t)w[k] ^ (uint32_t)(w[k] >> 32);
            break;
        }
        case 13:  // carry-chained mad.lo.cc / madc.hi.cc pairs, multiplier = last round's top limb
            for (int i = 0; i < iters; ++i) {
                const uint32_t m = a.v[7];
                asm("mad.lo.cc.u32 %0, %8, %9, %0;\n\t"
                    "madc.hi.cc.u32 %1, %8, %9, %1;\n\t"
                    "madc.lo.cc.u32 %2, %10, %9, %2;\n\t"
                    "madc.hi.cc.u32 %3, %10, %9, %3;\n\t"
                    "madc.lo.cc.u32 %4, %11, %9, %4;\n\t"
                    "madc.hi.cc.u32 %5, %11, %9, %5;\n\t"
                    "madc.lo.cc.u32 %6, %12, %9, %6;\n\t"
                    "madc.hi.u32 %7, %12, %9, %7;"
                    : "+r"(a.v[0]), "+r"(a.v[1]), "+r"(a.v[2]), "+r"(a.v[3]), "+r"(a.v[4]), "+r"(a.v[5]),
                      "+r"(a.v[6]), "+r"(a.v[7])
                    : "r"(b.v[0]), "r"(m), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]));
            }
            break;
        case 14: {  // operand-scanning step: w = lo(w) * b + hi(w) + lo(w)
            uint64_t w[8];
            for (int k = 0; k < 8; ++k) w[k] = ((uint64_t)c.v[k] << 32) | a.v[k];
            for (int i = 0; i < iters; ++i)
                for (int k = 0; k < 8; ++k) w[k] = (uint64_t)(uint32_t)w[k] * b.v[k] + (w[k] >> 32) + (uint32_t)w[k];
            for (int k = 0; k < 8; ++k) a.v[k] = (uint32_t)w[k] ^ (uint32_t)(w[k] >> 32);
            break;
        }
        case 15:  // two independent 256x256 PTX products, low halves fed back (no reduction, no call)
            for (int i = 0; i < iters; ++i) {
                uint32_t t[16], u[16];
                mul256_sel_ptx(t, a.v, b.v);
                mul256_sel_ptx(u, c.v, d.v);
                for (int k = 0; k < 8; ++k) { a.v[k] = t[k] ^ t[k + 8]; c.v[k] = u[k] ^ u[k + 8]; }
            }
            break;
        case 16:  // two independent inlined field multiplies (product + reduction, no call)
            for (int i = 0; i < iters; ++i) { a = fe_mul_c(a, b); c = fe_mul_c(c, d); }
            break;
#endif
        default:
            break;
    }
    for (int i = 0; i < 8; ++i) acc ^= a.v[i] ^ c.v[i];
    if (acc == 0x9E3779B9u) sink[0] = acc;   // keeps the work observable
}

}  // namespace pkN

// Compiled once per verify-kernel variant (same code-size flags), see build.py.
cudaError_t UF_CAT(launch_probe_v, UF_VARIANT)(int op, int blocks, int threads, int iters, uint32_t* sink,
                                               cudaStream_t s) {
    UF_CAT(pk, UF_VARIANT)::k_probe<<<blocks, threads, 0, s>>>(op, iters, sink);
    return cudaGetLastError();
}

}  // namespace uf
