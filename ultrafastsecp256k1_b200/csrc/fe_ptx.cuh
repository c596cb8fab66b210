// Field building blocks in PTX carry chains (device only): the 256 x 256 ->
// 512-bit product (rows below, and one level of Karatsuba on 128-bit halves,
// the form the field multiply uses), the two folds of the reduction by
// 2^256 = 2^32 + 977 (mod p), and add / sub / small shifts whose folds touch
// only the limbs a fold reaches in the common case.
//
// Row product: operand scanning, one row per limb b[i] of the multiplier.  Within a row the
// products a[j]*b[i] are split by the parity of j, because lo(a[j] b[i]) lands
// on limb i+j and hi(a[j] b[i]) on i+j+1: the even products (j = 0,2,4,6) then
// touch limbs i..i+7 exactly once each and form ONE unbroken carry chain
//   mad.lo.cc, madc.hi.cc, madc.lo.cc, ..., madc.hi.cc, addc
// and the odd products (j = 1,3,5,7) form a second chain over limbs i+1..i+8.
// That is 16 multiply-adds and 1 add per row, 8 rows.  Carry bounds: after
// rows 0..i the accumulator holds a * (b mod 2^(32(i+1))) < 2^(32(i+9)), so
// limb i+8 is zero before row i's even chain deposits its carry there, and the
// odd chain of row i never carries out of limb i+8.
//
// The reference's GPU field multiply is also an 8x32 mad.lo.cc / madc.hi.cc
// product (src/cuda/include/secp256k1_32_hybrid_final.cuh:15-103, a column-wise
// Comba arrangement); this is the row-wise even/odd arrangement instead.
#pragma once
#include "common.cuh"

#if defined(__CUDA_ARCH__)
namespace uf {

#define UF_ROW_EVEN(T0, T1, T2, T3, T4, T5, T6, T7, T8, BI)                                      \
    asm("mad.lo.cc.u32 %0, %9, %13, %0;\n\t"                                                     \
        "madc.hi.cc.u32 %1, %9, %13, %1;\n\t"                                                    \
        "madc.lo.cc.u32 %2, %10, %13, %2;\n\t"                                                   \
        "madc.hi.cc.u32 %3, %10, %13, %3;\n\t"                                                   \
        "madc.lo.cc.u32 %4, %11, %13, %4;\n\t"                                                   \
        "madc.hi.cc.u32 %5, %11, %13, %5;\n\t"                                                   \
        "madc.lo.cc.u32 %6, %12, %13, %6;\n\t"                                                   \
        "madc.hi.cc.u32 %7, %12, %13, %7;\n\t"                                                   \
        "addc.u32 %8, %8, 0;"                                                                    \
        : "+r"(T0), "+r"(T1), "+r"(T2), "+r"(T3), "+r"(T4), "+r"(T5), "+r"(T6), "+r"(T7), "+r"(T8) \
        : "r"(a[0]), "r"(a[2]), "r"(a[4]), "r"(a[6]), "r"(BI))

#define UF_ROW_ODD(T1, T2, T3, T4, T5, T6, T7, T8, BI)                                           \
    asm("mad.lo.cc.u32 %0, %8, %12, %0;\n\t"                                                     \
        "madc.hi.cc.u32 %1, %8, %12, %1;\n\t"                                                    \
        "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"                                                    \
        "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"                                                    \
        "madc.lo.cc.u32 %4, %10, %12, %4;\n\t"                                                   \
        "madc.hi.cc.u32 %5, %10, %12, %5;\n\t"                                                   \
        "madc.lo.cc.u32 %6, %11, %12, %6;\n\t"                                                   \
        "madc.hi.u32 %7, %11, %12, %7;"                                                          \
        : "+r"(T1), "+r"(T2), "+r"(T3), "+r"(T4), "+r"(T5), "+r"(T6), "+r"(T7), "+r"(T8)          \
        : "r"(a[1]), "r"(a[3]), "r"(a[5]), "r"(a[7]), "r"(BI))

__device__ __forceinline__ void mul256_ptx(uint32_t t[16], const uint32_t a[8], const uint32_t b[8]) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0, t8 = 0, t9 = 0, t10 = 0, t11 = 0,
             t12 = 0, t13 = 0, t14 = 0, t15 = 0;
    UF_ROW_EVEN(t0, t1, t2, t3, t4, t5, t6, t7, t8, b[0]);
    UF_ROW_ODD(t1, t2, t3, t4, t5, t6, t7, t8, b[0]);
    UF_ROW_EVEN(t1, t2, t3, t4, t5, t6, t7, t8, t9, b[1]);
    UF_ROW_ODD(t2, t3, t4, t5, t6, t7, t8, t9, b[1]);
    UF_ROW_EVEN(t2, t3, t4, t5, t6, t7, t8, t9, t10, b[2]);
    UF_ROW_ODD(t3, t4, t5, t6, t7, t8, t9, t10, b[2]);
    UF_ROW_EVEN(t3, t4, t5, t6, t7, t8, t9, t10, t11, b[3]);
    UF_ROW_ODD(t4, t5, t6, t7, t8, t9, t10, t11, b[3]);
    UF_ROW_EVEN(t4, t5, t6, t7, t8, t9, t10, t11, t12, b[4]);
    UF_ROW_ODD(t5, t6, t7, t8, t9, t10, t11, t12, b[4]);
    UF_ROW_EVEN(t5, t6, t7, t8, t9, t10, t11, t12, t13, b[5]);
    UF_ROW_ODD(t6, t7, t8, t9, t10, t11, t12, t13, b[5]);
    UF_ROW_EVEN(t6, t7, t8, t9, t10, t11, t12, t13, t14, b[6]);
    UF_ROW_ODD(t7, t8, t9, t10, t11, t12, t13, t14, b[6]);
    UF_ROW_EVEN(t7, t8, t9, t10, t11, t12, t13, t14, t15, b[7]);
    UF_ROW_ODD(t8, t9, t10, t11, t12, t13, t14, t15, b[7]);
    t[0] = t0; t[1] = t1; t[2] = t2; t[3] = t3; t[4] = t4; t[5] = t5; t[6] = t6; t[7] = t7;
    t[8] = t8; t[9] = t9; t[10] = t10; t[11] = t11; t[12] = t12; t[13] = t13; t[14] = t14; t[15] = t15;
}

#undef UF_ROW_EVEN
#undef UF_ROW_ODD

// 128 x 128 -> 256-bit product (4 x 4 limbs), the same even / odd row chains
// as mul256_ptx: after rows 0..i the value is below 2^(32(i+5)), so limb i+4
// is zero before row i's even chain deposits its carry there.
#define UF_ROW4_EVEN(T0, T1, T2, T3, T4, BI)                                                     \
    asm("mad.lo.cc.u32 %0, %5, %7, %0;\n\t"                                                      \
        "madc.hi.cc.u32 %1, %5, %7, %1;\n\t"                                                     \
        "madc.lo.cc.u32 %2, %6, %7, %2;\n\t"                                                     \
        "madc.hi.cc.u32 %3, %6, %7, %3;\n\t"                                                     \
        "addc.u32 %4, %4, 0;"                                                                    \
        : "+r"(T0), "+r"(T1), "+r"(T2), "+r"(T3), "+r"(T4)                                       \
        : "r"(a[0]), "r"(a[2]), "r"(BI))
#define UF_ROW4_ODD(T1, T2, T3, T4, BI)                                                          \
    asm("mad.lo.cc.u32 %0, %4, %6, %0;\n\t"                                                      \
        "madc.hi.cc.u32 %1, %4, %6, %1;\n\t"                                                     \
        "madc.lo.cc.u32 %2, %5, %6, %2;\n\t"                                                     \
        "madc.hi.u32 %3, %5, %6, %3;"                                                            \
        : "+r"(T1), "+r"(T2), "+r"(T3), "+r"(T4)                                                 \
        : "r"(a[1]), "r"(a[3]), "r"(BI))

__device__ __forceinline__ void mul128_ptx(uint32_t t[8], const uint32_t a[4], const uint32_t b[4]) {
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0;
    UF_ROW4_EVEN(t0, t1, t2, t3, t4, b[0]);
    UF_ROW4_ODD(t1, t2, t3, t4, b[0]);
    UF_ROW4_EVEN(t1, t2, t3, t4, t5, b[1]);
    UF_ROW4_ODD(t2, t3, t4, t5, b[1]);
    UF_ROW4_EVEN(t2, t3, t4, t5, t6, b[2]);
    UF_ROW4_ODD(t3, t4, t5, t6, b[2]);
    UF_ROW4_EVEN(t3, t4, t5, t6, t7, b[3]);
    UF_ROW4_ODD(t4, t5, t6, t7, b[3]);
    t[0] = t0; t[1] = t1; t[2] = t2; t[3] = t3; t[4] = t4; t[5] = t5; t[6] = t6; t[7] = t7;
}

#undef UF_ROW4_EVEN
#undef UF_ROW4_ODD

// s = x mod 2^128 + x >> 128 (4 limbs) and its carry bit c.
__device__ __forceinline__ void kara_sum_ptx(uint32_t sa[4], uint32_t& ca, const uint32_t a[8]) {
    asm("add.cc.u32 %0, %5, %9;\n\t"
        "addc.cc.u32 %1, %6, %10;\n\t"
        "addc.cc.u32 %2, %7, %11;\n\t"
        "addc.cc.u32 %3, %8, %12;\n\t"
        "addc.u32 %4, 0, 0;"
        : "=r"(sa[0]), "=r"(sa[1]), "=r"(sa[2]), "=r"(sa[3]), "=r"(ca)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]));
}

// Karatsuba combination: t = z0 + (m - z0 - z2) 2^128 + z2 2^256 where
// m = (sa + ca 2^128)(sb + cb 2^128) = p + ca sb 2^128 + cb sa 2^128 + ca cb 2^256
// and p = sa sb (all exact; m - z0 - z2 < 2^257).
__device__ __forceinline__ void kara_combine_ptx(uint32_t t[16], const uint32_t z0[8], const uint32_t z2[8],
                                                 uint32_t p[8], const uint32_t sa[4], const uint32_t sb[4],
                                                 uint32_t ca, uint32_t cb) {
    // m[0..8] = p + (ca ? sb : 0) 2^128 + (cb ? sa : 0) 2^128 + ca cb 2^256
    const uint32_t ma = 0u - ca, mb = 0u - cb;
    uint32_t m8;
    asm("add.cc.u32 %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.cc.u32 %2, %2, %7;\n\t"
        "addc.cc.u32 %3, %3, %8;\n\t"
        "addc.u32 %4, 0, 0;"
        : "+r"(p[4]), "+r"(p[5]), "+r"(p[6]), "+r"(p[7]), "=r"(m8)
        : "r"(sb[0] & ma), "r"(sb[1] & ma), "r"(sb[2] & ma), "r"(sb[3] & ma));
    asm("add.cc.u32 %0, %0, %5;\n\t"
        "addc.cc.u32 %1, %1, %6;\n\t"
        "addc.cc.u32 %2, %2, %7;\n\t"
        "addc.cc.u32 %3, %3, %8;\n\t"
        "addc.u32 %4, %4, %9;"
        : "+r"(p[4]), "+r"(p[5]), "+r"(p[6]), "+r"(p[7]), "+r"(m8)
        : "r"(sa[0] & mb), "r"(sa[1] & mb), "r"(sa[2] & mb), "r"(sa[3] & mb), "r"(ca & cb));
    // z1 = m - z0 - z2 (nonnegative, below 2^257)
    asm("sub.cc.u32 %0, %0, %9;\n\t"
        "subc.cc.u32 %1, %1, %10;\n\t"
        "subc.cc.u32 %2, %2, %11;\n\t"
        "subc.cc.u32 %3, %3, %12;\n\t"
        "subc.cc.u32 %4, %4, %13;\n\t"
        "subc.cc.u32 %5, %5, %14;\n\t"
        "subc.cc.u32 %6, %6, %15;\n\t"
        "subc.cc.u32 %7, %7, %16;\n\t"
        "subc.u32 %8, %8, 0;"
        : "+r"(p[0]), "+r"(p[1]), "+r"(p[2]), "+r"(p[3]), "+r"(p[4]), "+r"(p[5]), "+r"(p[6]), "+r"(p[7]),
          "+r"(m8)
        : "r"(z0[0]), "r"(z0[1]), "r"(z0[2]), "r"(z0[3]), "r"(z0[4]), "r"(z0[5]), "r"(z0[6]), "r"(z0[7]));
    asm("sub.cc.u32 %0, %0, %9;\n\t"
        "subc.cc.u32 %1, %1, %10;\n\t"
        "subc.cc.u32 %2, %2, %11;\n\t"
        "subc.cc.u32 %3, %3, %12;\n\t"
        "subc.cc.u32 %4, %4, %13;\n\t"
        "subc.cc.u32 %5, %5, %14;\n\t"
        "subc.cc.u32 %6, %6, %15;\n\t"
        "subc.cc.u32 %7, %7, %16;\n\t"
        "subc.u32 %8, %8, 0;"
        : "+r"(p[0]), "+r"(p[1]), "+r"(p[2]), "+r"(p[3]), "+r"(p[4]), "+r"(p[5]), "+r"(p[6]), "+r"(p[7]),
          "+r"(m8)
        : "r"(z2[0]), "r"(z2[1]), "r"(z2[2]), "r"(z2[3]), "r"(z2[4]), "r"(z2[5]), "r"(z2[6]), "r"(z2[7]));
    // t = z0 | z2, then + z1 at limb 4
    t[0] = z0[0]; t[1] = z0[1]; t[2] = z0[2]; t[3] = z0[3];
    asm("add.cc.u32 %0, %12, %20;\n\t"
        "addc.cc.u32 %1, %13, %21;\n\t"
        "addc.cc.u32 %2, %14, %22;\n\t"
        "addc.cc.u32 %3, %15, %23;\n\t"
        "addc.cc.u32 %4, %16, %24;\n\t"
        "addc.cc.u32 %5, %17, %25;\n\t"
        "addc.cc.u32 %6, %18, %26;\n\t"
        "addc.cc.u32 %7, %19, %27;\n\t"
        "addc.cc.u32 %8, %29, %28;\n\t"
        "addc.cc.u32 %9, %30, 0;\n\t"
        "addc.cc.u32 %10, %31, 0;\n\t"
        "addc.u32 %11, %32, 0;"
        : "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7]), "=r"(t[8]), "=r"(t[9]), "=r"(t[10]), "=r"(t[11]),
          "=r"(t[12]), "=r"(t[13]), "=r"(t[14]), "=r"(t[15])
        : "r"(z0[4]), "r"(z0[5]), "r"(z0[6]), "r"(z0[7]), "r"(z2[0]), "r"(z2[1]), "r"(z2[2]), "r"(z2[3]),
          "r"(p[0]), "r"(p[1]), "r"(p[2]), "r"(p[3]), "r"(p[4]), "r"(p[5]), "r"(p[6]), "r"(p[7]),
          "r"(m8), "r"(z2[4]), "r"(z2[5]), "r"(z2[6]), "r"(z2[7]));
}

// 256 x 256 -> 512 by one level of Karatsuba on 128-bit halves:
// a = a0 + a1 2^128, b = b0 + b1 2^128, z0 = a0 b0, z2 = a1 b1,
// m = (a0 + a1)(b0 + b1) with the two sums' carry bits ca, cb handled as
// m = sa sb + ca sb 2^128 + cb sa 2^128 + ca cb 2^256 (sa, sb their low 128
// bits), z1 = m - z0 - z2 = a0 b1 + a1 b0 < 2^257, t = z0 + z1 2^128 + z2 2^256.
// Three 4 x 4 products (96 multiply-adds) instead of 128, for about 60 adds,
// which run on the integer ALU pipe rather than the multiply-add one.
__device__ __forceinline__ void mul256_kara_ptx(uint32_t t[16], const uint32_t a[8], const uint32_t b[8]) {
    uint32_t z0[8], z2[8], p[8], sa[4], sb[4], ca, cb;
    mul128_ptx(z0, a, b);
    mul128_ptx(z2, a + 4, b + 4);
    kara_sum_ptx(sa, ca, a);
    kara_sum_ptx(sb, cb, b);
    mul128_ptx(p, sa, sb);
    kara_combine_ptx(t, z0, z2, p, sa, sb, ca, cb);
}

// The product the field multiply uses: Karatsuba (measured on B200: 157
// instead of 178 IMAD issue slots per product, field multiply 253 -> 230),
// or the plain rows with UF_MUL_ROWS.
__device__ __forceinline__ void mul256_sel_ptx(uint32_t t[16], const uint32_t a[8], const uint32_t b[8]) {
#if defined(UF_MUL_ROWS)
    mul256_ptx(t, a, b);
#else
    mul256_kara_ptx(t, a, b);
#endif
}

// First fold of the reduction mod p for the 512-bit t = H*2^256 + L:
// s[0..7] + top*2^256 = L + 977*H + (H << 32), with top < 2^32 + 978.
// Order matters for the carry bounds: L + 977*H < 2^266 fits limbs 0..8, then
// adding H << 32 can carry once more into a 33rd top bit.
__device__ __forceinline__ uint64_t fold_977_ptx(uint32_t s[8], const uint32_t t[16]) {
    uint32_t s0 = t[0], s1 = t[1], s2 = t[2], s3 = t[3], s4 = t[4], s5 = t[5], s6 = t[6], s7 = t[7], s8 = 0, s9;
    // + 977*H, even then odd limbs of H (each one carry chain)
    asm("mad.lo.cc.u32 %0, %9, 977, %0;\n\t"
        "madc.hi.cc.u32 %1, %9, 977, %1;\n\t"
        "madc.lo.cc.u32 %2, %10, 977, %2;\n\t"
        "madc.hi.cc.u32 %3, %10, 977, %3;\n\t"
        "madc.lo.cc.u32 %4, %11, 977, %4;\n\t"
        "madc.hi.cc.u32 %5, %11, 977, %5;\n\t"
        "madc.lo.cc.u32 %6, %12, 977, %6;\n\t"
        "madc.hi.cc.u32 %7, %12, 977, %7;\n\t"
        "addc.u32 %8, %8, 0;"
        : "+r"(s0), "+r"(s1), "+r"(s2), "+r"(s3), "+r"(s4), "+r"(s5), "+r"(s6), "+r"(s7), "+r"(s8)
        : "r"(t[8]), "r"(t[10]), "r"(t[12]), "r"(t[14]));
    asm("mad.lo.cc.u32 %0, %8, 977, %0;\n\t"
        "madc.hi.cc.u32 %1, %8, 977, %1;\n\t"
        "madc.lo.cc.u32 %2, %9, 977, %2;\n\t"
        "madc.hi.cc.u32 %3, %9, 977, %3;\n\t"
        "madc.lo.cc.u32 %4, %10, 977, %4;\n\t"
        "madc.hi.cc.u32 %5, %10, 977, %5;\n\t"
        "madc.lo.cc.u32 %6, %11, 977, %6;\n\t"
        "madc.hi.u32 %7, %11, 977, %7;"
        : "+r"(s1), "+r"(s2), "+r"(s3), "+r"(s4), "+r"(s5), "+r"(s6), "+r"(s7), "+r"(s8)
        : "r"(t[9]), "r"(t[11]), "r"(t[13]), "r"(t[15]));
    // + (H << 32)
    asm("add.cc.u32 %0, %0, %9;\n\t"
        "addc.cc.u32 %1, %1, %10;\n\t"
        "addc.cc.u32 %2, %2, %11;\n\t"
        "addc.cc.u32 %3, %3, %12;\n\t"
        "addc.cc.u32 %4, %4, %13;\n\t"
        "addc.cc.u32 %5, %5, %14;\n\t"
        "addc.cc.u32 %6, %6, %15;\n\t"
        "addc.cc.u32 %7, %7, %16;\n\t"
        "addc.u32 %8, 0, 0;"
        : "+r"(s1), "+r"(s2), "+r"(s3), "+r"(s4), "+r"(s5), "+r"(s6), "+r"(s7), "+r"(s8), "=r"(s9)
        : "r"(t[8]), "r"(t[9]), "r"(t[10]), "r"(t[11]), "r"(t[12]), "r"(t[13]), "r"(t[14]), "r"(t[15]));
    s[0] = s0; s[1] = s1; s[2] = s2; s[3] = s3; s[4] = s4; s[5] = s5; s[6] = s6; s[7] = s7;
    return ((uint64_t)s9 << 32) | s8;
}

// Second fold: s[0..7] + top * 2^256 -> weakly reduced s, for the top
// (< 2^32 + 978) that fold_977_ptx returns.  top * K (K = 2^32 + 977) lands on
// limbs 0..2: lo(tl*977) on 0, hi(tl*977) + tl on 1, th on 2 (top = th*2^32 +
// tl).  The common path is those seven carry-chained instructions.  Three rare
// cases take the branch: th = 1 (top >= 2^32, its 977 * 2^32 still to add),
// a carry out of limb 2 (limb 2 was 0xFFFFFFFF), and a wrap past 2^256, which
// is folded once more as + K (the value is then below 2^65, so it cannot wrap
// again).
__device__ __forceinline__ void fold_top_ptx(uint32_t s[8], uint64_t top) {
    const uint32_t tl = (uint32_t)top, th = (uint32_t)(top >> 32);
    uint32_t c;
    asm("mad.lo.cc.u32 %0, %4, 977, %0;\n\t"
        "madc.hi.cc.u32 %1, %4, 977, %1;\n\t"
        "addc.cc.u32 %2, %2, %5;\n\t"
        "addc.u32 %3, 0, 0;"
        : "+r"(s[0]), "+r"(s[1]), "+r"(s[2]), "=r"(c)
        : "r"(tl), "r"(th));
    asm("add.cc.u32 %0, %0, %3;\n\t"
        "addc.cc.u32 %1, %1, 0;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(s[1]), "+r"(s[2]), "+r"(c)
        : "r"(tl));
    if (__builtin_expect((c | th) != 0, 0)) {
        uint32_t w;
        asm("mad.lo.cc.u32 %0, %8, 977, %0;\n\t"   // th * 977 * 2^32 on limb 1
            "addc.cc.u32 %1, %1, 0;\n\t"
            "addc.cc.u32 %2, %2, %9;\n\t"          // the carry out of limb 2
            "addc.cc.u32 %3, %3, 0;\n\t"
            "addc.cc.u32 %4, %4, 0;\n\t"
            "addc.cc.u32 %5, %5, 0;\n\t"
            "addc.cc.u32 %6, %6, 0;\n\t"
            "addc.u32 %7, 0, 0;"
            : "+r"(s[1]), "+r"(s[2]), "+r"(s[3]), "+r"(s[4]), "+r"(s[5]), "+r"(s[6]), "+r"(s[7]), "=r"(w)
            : "r"(th), "r"(c));
        if (w) {   // wrapped past 2^256: + K (the value is now below 2^65: limbs 3..7 are zero)
            asm("add.cc.u32 %0, %0, 977;\n\t"
                "addc.cc.u32 %1, %1, 1;\n\t"
                "addc.u32 %2, %2, 0;"
                : "+r"(s[0]), "+r"(s[1]), "+r"(s[2]));
        }
    }
}

// r += c * K (K = 2^32 + 977) for the carry word c < 2^22 of a value that
// overflowed 2^256 by c: c * 977 on limb 0 and c on limb 1.  A carry out of
// limb 1 (limb 1 all ones) continues on the rare path; wrapping past 2^256
// again leaves a value below c * K < 2^55 (limbs 2..7 zero), so the last
// + K stays in limbs 0..1.
__device__ __forceinline__ void fold_k_ptx(uint32_t r[8], uint32_t c) {
    uint32_t c2;
    asm("mad.lo.cc.u32 %0, %3, 977, %0;\n\t"
        "addc.cc.u32 %1, %1, %3;\n\t"
        "addc.u32 %2, 0, 0;"
        : "+r"(r[0]), "+r"(r[1]), "=r"(c2)
        : "r"(c));
    if (__builtin_expect(c2 != 0, 0)) {
        asm("add.cc.u32 %0, %0, 1;\n\t"
            "addc.cc.u32 %1, %1, 0;\n\t"
            "addc.cc.u32 %2, %2, 0;\n\t"
            "addc.cc.u32 %3, %3, 0;\n\t"
            "addc.cc.u32 %4, %4, 0;\n\t"
            "addc.cc.u32 %5, %5, 0;\n\t"
            "addc.u32 %6, 0, 0;"
            : "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "=r"(c2));
        if (c2) {
            asm("add.cc.u32 %0, %0, 977;\n\t"
                "addc.u32 %1, %1, 1;"
                : "+r"(r[0]), "+r"(r[1]));
        }
    }
}

// r = a * 2^k mod p (weakly reduced in and out), k = 1..8: a funnel shift of
// the limbs and one fold of the k bits shifted out.
template <int k>
__device__ __forceinline__ void fe_shl_ptx(uint32_t r[8], const uint32_t a[8]) {
    static_assert(k >= 1 && k <= 8, "shift of 1..8 bits");
    const uint32_t top = a[7] >> (32 - k);
#pragma unroll
    for (int i = 7; i > 0; --i) r[i] = __funnelshift_l(a[i - 1], a[i], k);
    r[0] = a[0] << k;
    fold_k_ptx(r, top);
}

// r = a + b mod p (weakly reduced in and out).  The carry out of the 256-bit
// add is folded back as +K (K = 2^32 + 977) on limbs 0..1; carrying further
// (limb 1 all ones) and wrapping past 2^256 again (only when the sum is below
// K) take rare branches.
__device__ __forceinline__ void fe_add_ptx(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
    uint32_t c;
    asm("add.cc.u32 %0, %9, %17;\n\t"
        "addc.cc.u32 %1, %10, %18;\n\t"
        "addc.cc.u32 %2, %11, %19;\n\t"
        "addc.cc.u32 %3, %12, %20;\n\t"
        "addc.cc.u32 %4, %13, %21;\n\t"
        "addc.cc.u32 %5, %14, %22;\n\t"
        "addc.cc.u32 %6, %15, %23;\n\t"
        "addc.cc.u32 %7, %16, %24;\n\t"
        "addc.u32 %8, 0, 0;"
        : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]), "=&r"(r[6]), "=&r"(r[7]),
          "=&r"(c)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
          "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
    fold_k_ptx(r, c);
}

// r = a - b mod p (weakly reduced in and out).  A borrow out of the 256-bit
// subtraction is folded as -K (adds p) on limbs 0..1; borrowing further (limb
// 1 zero) and a second borrow (possible only when b > p and a is tiny, one
// more -K) take rare branches.
__device__ __forceinline__ void fe_sub_ptx(uint32_t r[8], const uint32_t a[8], const uint32_t b[8]) {
    uint32_t br;
    asm("sub.cc.u32 %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32 %8, 0, 0;"
        : "=&r"(r[0]), "=&r"(r[1]), "=&r"(r[2]), "=&r"(r[3]), "=&r"(r[4]), "=&r"(r[5]), "=&r"(r[6]), "=&r"(r[7]),
          "=&r"(br)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]),
          "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
    // br is 0 or 0xFFFFFFFF: subtract K & br (977 on limb 0, 1 on limb 1); a
    // borrow out of limb 1 (limb 1 was 0) continues on the rare path
    const uint32_t k0 = br & 977u, k1 = br & 1u;
    uint32_t b2;
    asm("sub.cc.u32 %0, %0, %3;\n\t"
        "subc.cc.u32 %1, %1, %4;\n\t"
        "subc.u32 %2, 0, 0;"
        : "+r"(r[0]), "+r"(r[1]), "=r"(b2)
        : "r"(k0), "r"(k1));
    if (__builtin_expect(b2 != 0, 0)) {
        asm("sub.cc.u32 %0, %0, 1;\n\t"
            "subc.cc.u32 %1, %1, 0;\n\t"
            "subc.cc.u32 %2, %2, 0;\n\t"
            "subc.cc.u32 %3, %3, 0;\n\t"
            "subc.cc.u32 %4, %4, 0;\n\t"
            "subc.cc.u32 %5, %5, 0;\n\t"
            "subc.u32 %6, 0, 0;"
            : "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]), "=r"(b2));
        if (b2) {   // a second borrow (b > p and a tiny): the value is 2^256 - (K - x) with
                    // x < K, limbs 2..7 all ones and limb 1 >= 2^32 - 3: - K stays in limbs 0..1
            asm("sub.cc.u32 %0, %0, 977;\n\t"
                "subc.u32 %1, %1, 1;"
                : "+r"(r[0]), "+r"(r[1]));
        }
    }
}

}  // namespace uf
#endif
