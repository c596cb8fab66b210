// Field arithmetic mod p = 2^256 - 2^32 - 977 on 8 x 32-bit limbs.
//
// Role in the reference: Fp mul/sqr/add/sub of src/cuda/include/secp256k1.cuh
// (field_mul :1522, field_sqr :1536, reduce_512_to_256 :1290, field_add/sub
// :1072/:1139) and the 8x32 hybrid mul of secp256k1_32_hybrid_final.cuh:15-103.
// Written here from the arithmetic, for sm_100a's 32-bit integer pipe:
//
//  * values are "weakly reduced": any 256-bit integer congruent to the field
//    element (so [0, 2^256)); fe_normalize() makes them canonical;
//  * products are reduced with the fold 2^256 = K (mod p), K = 2^32 + 977:
//    t = H*2^256 + L  ->  L + 977*H + (H << 32), then a second, small fold;
//  * add/sub fold their carry/borrow with K as well (at most twice).
#pragma once
#include "common.cuh"
#include "fe_ptx.cuh"
#include "fe_ptx_sqr.cuh"

namespace uf {

struct Fe { uint32_t v[8]; };

#define UF_P0 0xFFFFFC2Fu
#define UF_P1 0xFFFFFFFEu

UF_HD void fe_set_u32(Fe& r, uint32_t a) {
    r.v[0] = a;
    UF_UNROLL
    for (int i = 1; i < 8; ++i) r.v[i] = 0;
}

UF_HD void fe_p(Fe& r) {
    r.v[0] = UF_P0; r.v[1] = UF_P1;
    UF_UNROLL
    for (int i = 2; i < 8; ++i) r.v[i] = 0xFFFFFFFFu;
}

// v += c*K (c in {0,1}); returns the carry out of limb 7.
UF_HD uint32_t fe_add_k(uint32_t v[8], uint32_t c) {
    uint64_t t = (uint64_t)v[0] + 977u * c;
    v[0] = lo32(t);
    t = (uint64_t)v[1] + c + (t >> 32);
    v[1] = lo32(t);
    UF_UNROLL
    for (int i = 2; i < 8; ++i) {
        t = (uint64_t)v[i] + (t >> 32);
        v[i] = lo32(t);
    }
    return hi32(t);
}

// v -= c*K (c in {0,1}); returns the borrow out of limb 7.
UF_HD uint32_t fe_sub_k(uint32_t v[8], uint32_t c) {
    uint64_t t = (uint64_t)v[0] - 977u * c;
    v[0] = lo32(t);
    uint32_t br = (uint32_t)(t >> 63);
    t = (uint64_t)v[1] - c - br;
    v[1] = lo32(t);
    br = (uint32_t)(t >> 63);
    UF_UNROLL
    for (int i = 2; i < 8; ++i) {
        t = (uint64_t)v[i] - br;
        v[i] = lo32(t);
        br = (uint32_t)(t >> 63);
    }
    return br;
}

UF_HD void fe_add(Fe& r, const Fe& a, const Fe& b) {
#if defined(__CUDA_ARCH__) && defined(UF_PTX_MUL)
    uint32_t tp[8];
    fe_add_ptx(tp, a.v, b.v);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = tp[i];
    return;
#endif
    uint64_t t = 0;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        t = (uint64_t)a.v[i] + b.v[i] + (t >> 32);
        r.v[i] = lo32(t);
    }
    uint32_t c = hi32(t);
    c = fe_add_k(r.v, c);   // a+b-2^256+K
    fe_add_k(r.v, c);       // only when the first fold wrapped: result is tiny
}

UF_HD void fe_sub(Fe& r, const Fe& a, const Fe& b) {
#if defined(__CUDA_ARCH__) && defined(UF_PTX_MUL)
    uint32_t tp[8];
    fe_sub_ptx(tp, a.v, b.v);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = tp[i];
    return;
#endif
    uint32_t br = 0;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        uint64_t t = (uint64_t)a.v[i] - b.v[i] - br;
        r.v[i] = lo32(t);
        br = (uint32_t)(t >> 63);
    }
    br = fe_sub_k(r.v, br);   // a-b+2^256-K = a-b+p
    fe_sub_k(r.v, br);        // only when b > p and a tiny: a-b+2p
}

UF_HD void fe_neg(Fe& r, const Fe& a) {
    Fe z;
    fe_set_u32(z, 0);
    fe_sub(r, z, a);
}

UF_HD void fe_dbl(Fe& r, const Fe& a) { fe_add(r, a, a); }

// s[0..7] + top * 2^256 (top < 2^45) -> weakly reduced r (second, small fold).
UF_HD void fe_fold_top(Fe& r, uint32_t s[8], uint64_t s8) {
    const uint64_t m = s8 * 977u;           // < 2^55
    uint64_t c = (uint64_t)s[0] + lo32(m);
    s[0] = lo32(c);
    c >>= 32;
    c += (uint64_t)s[1] + hi32(m) + lo32(s8);
    s[1] = lo32(c);
    c >>= 32;
    c += (uint64_t)s[2] + hi32(s8);
    s[2] = lo32(c);
    c >>= 32;
    UF_UNROLL
    for (int j = 3; j < 8; ++j) {
        c += s[j];
        s[j] = lo32(c);
        c >>= 32;
    }
    fe_add_k(s, (uint32_t)c);
    UF_UNROLL
    for (int j = 0; j < 8; ++j) r.v[j] = s[j];
}

// Reduce a 512-bit product t[0..15] to a weakly reduced field element.
UF_HD void fe_reduce512(Fe& r, const uint32_t t[16]) {
    uint32_t s[8];
#if defined(__CUDA_ARCH__) && defined(UF_PTX_MUL)
    fold_top_ptx(s, fold_977_ptx(s, t));
    UF_UNROLL
    for (int j = 0; j < 8; ++j) r.v[j] = s[j];
    return;
#else
    uint64_t c = (uint64_t)t[8] * 977u + t[0];
    s[0] = lo32(c);
    c >>= 32;
    UF_UNROLL
    for (int j = 1; j < 8; ++j) {
        c += (uint64_t)t[8 + j] * 977u + t[j] + t[7 + j];
        s[j] = lo32(c);
        c >>= 32;
    }
    const uint64_t s8 = c + t[15];          // < 2^45: weight 2^256
    fe_fold_top(r, s, s8);
#endif
}

// 256x256 -> 512 schoolbook product (operand scanning, 64-bit accumulators:
// each step is one 32x32+32+32 multiply-add, which the sm_100a backend maps
// onto the integer multiply-add pipe).
UF_HD void mul256(uint32_t t[16], const uint32_t a[8], const uint32_t b[8]) {
    uint64_t c = 0;
    UF_UNROLL
    for (int j = 0; j < 8; ++j) {
        c = (uint64_t)a[j] * b[0] + (c >> 32);
        t[j] = lo32(c);
    }
    t[8] = hi32(c);
    UF_UNROLL
    for (int i = 1; i < 8; ++i) {
        c = 0;
        UF_UNROLL
        for (int j = 0; j < 8; ++j) {
            c = (uint64_t)a[j] * b[i] + t[i + j] + (c >> 32);
            t[i + j] = lo32(c);
        }
        t[i + 8] = hi32(c);
    }
}

// Squaring: 28 cross products doubled + 8 diagonal squares.
UF_HD void sqr256(uint32_t t[16], const uint32_t a[8]) {
    // cross products sum_{i<j} a_i a_j 2^(32(i+j))
    UF_UNROLL
    for (int k = 0; k < 16; ++k) t[k] = 0;
    UF_UNROLL
    for (int i = 0; i < 7; ++i) {
        uint64_t c = 0;
        UF_UNROLL
        for (int j = i + 1; j < 8; ++j) {
            c = (uint64_t)a[i] * a[j] + t[i + j] + (c >> 32);
            t[i + j] = lo32(c);
        }
        t[i + 8] = hi32(c);
    }
    // double (t < 2^511 so the top bit shifts out as zero)
    t[15] = (t[14] >> 31);
    UF_UNROLL
    for (int k = 14; k > 0; --k) t[k] = (t[k] << 1) | (t[k - 1] >> 31);
    t[0] <<= 1;
    // add diagonal squares
    uint64_t c = 0;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        const uint64_t sq = (uint64_t)a[i] * a[i];
        c = (uint64_t)t[2 * i] + lo32(sq) + (c >> 32);
        t[2 * i] = lo32(c);
        c = (uint64_t)t[2 * i + 1] + hi32(sq) + (c >> 32);
        t[2 * i + 1] = lo32(c);
    }
}

// By-value cores, so that an out-of-line build (UF_NOINLINE_FIELD) passes
// operands in registers rather than through the stack.
// UF_PTX_MUL selects the PTX carry-chain product / square of fe_ptx.cuh and
// fe_ptx_sqr.cuh on the device (and the PTX add / sub above).
UF_HD Fe fe_mul_c(Fe a, Fe b) {
    uint32_t t[16];
    Fe r;
#if defined(__CUDA_ARCH__) && defined(UF_PTX_MUL)
    mul256_sel_ptx(t, a.v, b.v);
#else
    mul256(t, a.v, b.v);
#endif
    fe_reduce512(r, t);
    return r;
}

UF_HD Fe fe_sqr_c(Fe a) {
    uint32_t t[16];
    Fe r;
#if defined(__CUDA_ARCH__) && defined(UF_PTX_MUL)
    sqr256_ptx(t, a.v);
#else
    sqr256(t, a.v);
#endif
    fe_reduce512(r, t);
    return r;
}

UF_FIELD_FN Fe fe_mul_v(Fe a, Fe b) { return fe_mul_c(a, b); }
UF_FIELD_FN Fe fe_sqr_v(Fe a) { return fe_sqr_c(a); }

// n >= 1 squarings in one out-of-line call (the square-root chain's runs of
// up to 88 squarings pay one call, not one per squaring).
UF_FIELD_FN Fe fe_sqr_n_v(Fe a, int n) {
    UF_NOUNROLL
    for (int i = 0; i < n; ++i) a = fe_sqr_c(a);
    return a;
}

UF_HD void fe_mul(Fe& r, const Fe& a, const Fe& b) { r = fe_mul_v(a, b); }
UF_HD void fe_sqr(Fe& r, const Fe& a) { r = fe_sqr_v(a); }

// r = a * m for a small m (< 2^22).
UF_HD void fe_mul_small(Fe& r, const Fe& a, uint32_t m) {
    uint64_t c = 0;
    uint32_t s[8];
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        c = (uint64_t)a.v[i] * m + (c >> 32);
        s[i] = lo32(c);
    }
    const uint64_t top = c >> 32;           // < 2^22, weight 2^256
    const uint64_t k = top * 977u;
    c = (uint64_t)s[0] + lo32(k);
    s[0] = lo32(c);
    c = (uint64_t)s[1] + hi32(k) + (uint32_t)top + (c >> 32);
    s[1] = lo32(c);
    UF_UNROLL
    for (int i = 2; i < 8; ++i) {
        c = (uint64_t)s[i] + (c >> 32);
        s[i] = lo32(c);
    }
    fe_add_k(s, hi32(c));
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = s[i];
}

// r = a * 2^k mod p for k = 1..8 (a shift and one fold on the device).
template <int k>
UF_HD void fe_mul_pow2(Fe& r, const Fe& a) {
#if defined(__CUDA_ARCH__) && defined(UF_PTX_MUL)
    uint32_t t[8];
    fe_shl_ptx<k>(t, a.v);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = t[i];
#else
    fe_mul_small(r, a, 1u << k);
#endif
}

// Canonical representative in [0, p).
UF_HD void fe_normalize(Fe& a) {
    uint32_t t[8];
    UF_UNROLL
    for (int i = 0; i < 8; ++i) t[i] = a.v[i];
    const uint32_t ge = fe_add_k(t, 1);     // a >= p  <=>  a + K >= 2^256
    UF_UNROLL
    for (int i = 0; i < 8; ++i) a.v[i] = ge ? t[i] : a.v[i];
}

UF_HD bool fe_is_zero(const Fe& a) {
    // weakly reduced zero is 0 or p
    uint32_t z = 0, q = (a.v[0] ^ UF_P0) | (a.v[1] ^ UF_P1);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) z |= a.v[i];
    UF_UNROLL
    for (int i = 2; i < 8; ++i) q |= ~a.v[i];
    return z == 0 || q == 0;
}

UF_HD bool fe_equal(const Fe& a, const Fe& b) {
    Fe d;
    fe_sub(d, a, b);
    return fe_is_zero(d);
}

// x < p for a raw 256-bit integer (strict BIP-340 / SEC1 parse).
UF_HD bool limbs_lt_p(const uint32_t v[8]) {
    uint32_t t[8];
    UF_UNROLL
    for (int i = 0; i < 8; ++i) t[i] = v[i];
    return fe_add_k(t, 1) == 0;
}

UF_HD void fe_sqr_n(Fe& r, const Fe& a, int n) { r = fe_sqr_n_v(a, n); }

// a^((p+1)/4): the square root when a is a square.  (p+1)/4 is, from the top,
// 223 one-bits, a zero, 22 ones, four zeros, two ones, two zeros; the chain
// builds x^(2^k - 1) blocks (253 squarings, 13 multiplications).
UF_COLD void fe_sqrt_candidate(Fe& r, const Fe& a) {
    Fe x2, x3, x6, x9, x11, x22, x44, x88, x176, x220, x223, t;
    fe_sqr(t, a);        fe_mul(x2, t, a);
    fe_sqr(t, x2);       fe_mul(x3, t, a);
    fe_sqr_n(t, x3, 3);  fe_mul(x6, t, x3);
    fe_sqr_n(t, x6, 3);  fe_mul(x9, t, x3);
    fe_sqr_n(t, x9, 2);  fe_mul(x11, t, x2);
    fe_sqr_n(t, x11, 11); fe_mul(x22, t, x11);
    fe_sqr_n(t, x22, 22); fe_mul(x44, t, x22);
    fe_sqr_n(t, x44, 44); fe_mul(x88, t, x44);
    fe_sqr_n(t, x88, 88); fe_mul(x176, t, x88);
    fe_sqr_n(t, x176, 44); fe_mul(x220, t, x44);
    fe_sqr_n(t, x220, 3); fe_mul(x223, t, x3);
    fe_sqr_n(t, x223, 23); fe_mul(t, t, x22);
    fe_sqr_n(t, t, 6);   fe_mul(t, t, x2);
    fe_sqr_n(r, t, 2);
}

// Returns true and a root iff a is a square mod p.
UF_HDI bool fe_sqrt(Fe& r, const Fe& a) {
    Fe y, chk;
    fe_sqrt_candidate(y, a);
    fe_sqr(chk, y);
    r = y;
    return fe_equal(chk, a);
}

}  // namespace uf
