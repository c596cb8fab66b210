// Scalar arithmetic mod n (the group order) and the GLV split.
//
// Role in the reference: Scalar parse / from_bytes / mul / inverse
// (src/cpu/src/scalar.cpp, GPU scalar_mul_mod_n secp256k1.cuh:726,
// scalar_inverse :823) and glv_decompose (src/cpu/src/glv.cpp:397,
// secp256k1.cuh:986).  Only a handful of scalar operations run per
// signature, so these favour simplicity: products are reduced by folding with
// C = 2^256 - n (129 bits); inverses use the divstep inverse of safegcd.cuh.
//
// GLV: lambda is the cube root of unity mod n with lambda*(x, y) = (beta*x, y).
// k = k1 + k2*lambda with |k1|, |k2| < 2^128, computed as in the GLV paper
// (Gallant, Lambert, Vanstone 2001, section 4) from the short lattice basis
// (a1, b1), (a2, b2) of {(a, b): a + b*lambda = 0 mod n}:
//   c1 = round(k * b2 / n), c2 = round(-k * b1 / n)   (as (k*g) >> 384 with
//   g1 = round(2^384 b2 / n), g2 = round(-2^384 b1 / n)),
//   k2 = -c1*b1 - c2*b2,  k1 = k - k2*lambda   (mod n).
// All constants below were derived for this file from the curve parameters.
#pragma once
#include "common.cuh"
#include "fe.cuh"
#include "safegcd.cuh"

namespace uf {

struct Sc { uint32_t v[8]; };

UF_HD void sc_n(uint32_t n[8]) {
    n[0] = 0xD0364141u; n[1] = 0xBFD25E8Cu; n[2] = 0xAF48A03Bu; n[3] = 0xBAAEDCE6u;
    n[4] = 0xFFFFFFFEu; n[5] = 0xFFFFFFFFu; n[6] = 0xFFFFFFFFu; n[7] = 0xFFFFFFFFu;
}

UF_HD void modinfo_n(ModInfo& mi) {
    sc_n(mi.m);
    mi.m30[0] = 0x10364141; mi.m30[1] = 0x3F497A33; mi.m30[2] = 0x348A03BB;
    mi.m30[3] = 0x2BB739AB; mi.m30[4] = 0x3FFFFEBA; mi.m30[5] = 0x3FFFFFFF;
    mi.m30[6] = 0x3FFFFFFF; mi.m30[7] = 0x3FFFFFFF; mi.m30[8] = 0x0000FFFF;
    mi.minv30 = 0x2A774EC1u;
}

UF_HD void modinfo_p(ModInfo& mi) {
    mi.m[0] = 0xFFFFFC2Fu; mi.m[1] = 0xFFFFFFFEu;
    for (int i = 2; i < 8; ++i) mi.m[i] = 0xFFFFFFFFu;
    mi.m30[0] = 0x3FFFFC2F; mi.m30[1] = 0x3FFFFFFB;
    for (int i = 2; i < 8; ++i) mi.m30[i] = 0x3FFFFFFF;
    mi.m30[8] = 0x0000FFFF;
    mi.minv30 = 0x2DDACACFu;
}

UF_HD bool sc_is_zero(const Sc& a) { return is_zero256(a.v); }

// raw < n
UF_HD bool limbs_lt_n(const uint32_t v[8]) {
    uint32_t n[8];
    sc_n(n);
    return lt256(v, n);
}

// a - n when a >= n (a < 2^256 < 2n, so once is enough)
UF_HD void sc_reduce_once(Sc& a) {
    uint32_t n[8], t[8], br = 0;
    sc_n(n);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        const uint64_t d = (uint64_t)a.v[i] - n[i] - br;
        t[i] = lo32(d);
        br = (uint32_t)(d >> 63);
    }
    UF_UNROLL
    for (int i = 0; i < 8; ++i) a.v[i] = br ? a.v[i] : t[i];
}

UF_HD void sc_neg(Sc& r, const Sc& a) {
    if (sc_is_zero(a)) { r = a; return; }
    uint32_t n[8], br = 0;
    sc_n(n);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        const uint64_t d = (uint64_t)n[i] - a.v[i] - br;
        r.v[i] = lo32(d);
        br = (uint32_t)(d >> 63);
    }
}

UF_HD void sc_add(Sc& r, const Sc& a, const Sc& b) {
    uint64_t t = 0;
    uint32_t s[8];
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        t = (uint64_t)a.v[i] + b.v[i] + (t >> 32);
        s[i] = lo32(t);
    }
    // a + b < 2n; if it carried out, subtracting n (mod 2^256) is the answer
    const uint32_t carry = hi32(t);
    uint32_t n[8], d[8], br = 0;
    sc_n(n);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        const uint64_t x = (uint64_t)s[i] - n[i] - br;
        d[i] = lo32(x);
        br = (uint32_t)(x >> 63);
    }
    const bool take = carry || !br;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = take ? d[i] : s[i];
}

// 512-bit value -> mod n.  2^256 = C (mod n), C = 2^256 - n < 2^129.
UF_HDI void sc_reduce512(Sc& r, const uint32_t t_in[16]) {
    const uint32_t C[5] = {0x2FC9BEBFu, 0x402DA173u, 0x50B75FC4u, 0x45512319u, 0x00000001u};
    uint32_t x[16];
    UF_UNROLL
    for (int i = 0; i < 16; ++i) x[i] = t_in[i];
    for (int round = 0; round < 6; ++round) {
        uint32_t hz = 0;
        UF_UNROLL
        for (int i = 8; i < 16; ++i) hz |= x[i];
        if (hz == 0) break;
        uint32_t y[16];
        UF_UNROLL
        for (int i = 0; i < 16; ++i) y[i] = i < 8 ? x[i] : 0;
        UF_UNROLL
        for (int i = 0; i < 8; ++i) {
            uint64_t c = 0;
            UF_UNROLL
            for (int j = 0; j < 5; ++j) {
                c = (uint64_t)x[8 + i] * C[j] + y[i + j] + (c >> 32);
                y[i + j] = lo32(c);
            }
            uint32_t carry = hi32(c);
            UF_UNROLL
            for (int k = i + 5; k < 16; ++k) {
                const uint64_t s = (uint64_t)y[k] + carry;
                y[k] = lo32(s);
                carry = hi32(s);
            }
        }
        UF_UNROLL
        for (int i = 0; i < 16; ++i) x[i] = y[i];
    }
    UF_UNROLL
    for (int i = 0; i < 8; ++i) r.v[i] = x[i];
    sc_reduce_once(r);
}

UF_HDI void sc_mul(Sc& r, const Sc& a, const Sc& b) {
    uint32_t t[16];
    mul256(t, a.v, b.v);
    sc_reduce512(r, t);
}

UF_HDI void sc_inv(Sc& r, const Sc& a) {
    ModInfo mi;
    modinfo_n(mi);
    modinv_var(r.v, a.v, mi);
}

// s <= n/2 (BIP-62 low-S, src/cpu/src/ecdsa.cpp:114-124)
UF_HD bool sc_is_low(const uint32_t s[8]) {
    const uint32_t h[8] = {0x681B20A0u, 0xDFE92F46u, 0x57A4501Du, 0x5D576E73u,
                           0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0x7FFFFFFFu};
    return !lt256(h, s);
}

// round((k * g) / 2^384) for a 256-bit k and g: the top 128 bits (+ rounding).
UF_HD void mulshift384(uint32_t out[4], const uint32_t k[8], const uint32_t g[8]) {
    uint32_t t[16];
    mul256(t, k, g);
    const uint32_t rnd = t[11] >> 31;       // bit 383
    uint64_t c = (uint64_t)t[12] + rnd;
    out[0] = lo32(c);
    UF_UNROLL
    for (int i = 1; i < 4; ++i) {
        c = (uint64_t)t[12 + i] + (c >> 32);
        out[i] = lo32(c);
    }
}

struct GlvSplit {
    uint32_t k1[4], k2[4];   // magnitudes, < 2^128
    bool neg1, neg2;         // k = (-1)^neg1 k1 + (-1)^neg2 k2 * lambda (mod n)
};

UF_HDI void glv_split(GlvSplit& out, const Sc& k) {
    const uint32_t G1[8] = {0x45DBB031u, 0xE893209Au, 0x71E8CA7Fu, 0x3DAA8A14u,
                            0x9284EB15u, 0xE86C90E4u, 0xA7D46BCDu, 0x3086D221u};
    const uint32_t G2[8] = {0x8AC47F71u, 0x1571B4AEu, 0x9DF506C6u, 0x221208ACu,
                            0x0ABFE4C4u, 0x6F547FA9u, 0x010E8828u, 0xE4437ED6u};
    const Sc MB1 = {{0x0ABFE4C3u, 0x6F547FA9u, 0x010E8828u, 0xE4437ED6u, 0, 0, 0, 0}};
    const Sc MB2 = {{0x3DB1562Cu, 0xD765CDA8u, 0x0774346Du, 0x8A280AC5u,
                     0xFFFFFFFEu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}};
    const Sc LAM = {{0x1B23BD72u, 0xDF02967Cu, 0x20816678u, 0x122E22EAu,
                     0x8812645Au, 0xA5261C02u, 0xC05C30E0u, 0x5363AD4Cu}};
    uint32_t c1w[4], c2w[4];
    mulshift384(c1w, k.v, G1);
    mulshift384(c2w, k.v, G2);
    Sc c1 = {{c1w[0], c1w[1], c1w[2], c1w[3], 0, 0, 0, 0}};
    Sc c2 = {{c2w[0], c2w[1], c2w[2], c2w[3], 0, 0, 0, 0}};
    Sc t1, t2, k2, k1;
    sc_mul(t1, c1, MB1);
    sc_mul(t2, c2, MB2);
    sc_add(k2, t1, t2);
    sc_mul(t1, k2, LAM);
    sc_neg(t1, t1);
    sc_add(k1, k, t1);
    // map to signed magnitudes: values above n/2 are negative
    out.neg1 = !sc_is_low(k1.v);
    out.neg2 = !sc_is_low(k2.v);
    if (out.neg1) sc_neg(k1, k1);
    if (out.neg2) sc_neg(k2, k2);
    UF_UNROLL
    for (int i = 0; i < 4; ++i) { out.k1[i] = k1.v[i]; out.k2[i] = k2.v[i]; }
}

}  // namespace uf
