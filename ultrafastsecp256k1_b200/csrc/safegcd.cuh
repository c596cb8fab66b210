// Variable-time modular inversion by Bernstein-Yang divsteps ("safegcd"),
// in 30-bit signed limbs so that every product fits the 32x32->64 integer
// multiply of sm_100a.
//
// Role in the reference: the CPU inverses Scalar::inverse (src/cpu/src/scalar.cpp:841,
// 30-bit variant :850-1120) and fe_inverse_safegcd_impl (src/cpu/src/field.cpp:2848).
// The reference GPU path uses Fermat chains instead (secp256k1.cuh:823, :2614-2706);
// this file gives the GPU the divstep algorithm (Bernstein & Yang, "Fast
// constant-time gcd computation and modular inversion", 2019), variable-time
// variant (inputs here are public).
//
// Code form followed: libsecp256k1's variable-time modular inversion,
// src/modinv32_impl.h (secp256k1_modinv32_divsteps_30_var,
// secp256k1_modinv32_update_de_30) and, for the 6-bit inverse step of
// f^-1 mod 2^6 (w = f g (f f - 2)), src/modinv64_impl.h.  divsteps30_var and
// update_de30 below take their statement structure from those functions
// (the trailing-zero batched loop, the swap / negate, the md / me correction
// that makes the division by 2^30 exact); the limb conversion helpers are
// this file's own.  That code is distributed under the MIT licence:
//
//   Copyright (c) 2020 Peter Dettman (libsecp256k1 modinv32 / modinv64)
//   Permission is hereby granted, free of charge, to any person obtaining a
//   copy of this software and associated documentation files (the
//   "Software"), to deal in the Software without restriction, including
//   without limitation the rights to use, copy, modify, merge, publish,
//   distribute, sublicense, and/or sell copies of the Software, and to permit
//   persons to whom the Software is furnished to do so, subject to the
//   following conditions: The above copyright notice and this permission
//   notice shall be included in all copies or substantial portions of the
//   Software.  THE SOFTWARE IS PROVIDED "AS IS", WITHOUT WARRANTY OF ANY
//   KIND, EXPRESS OR IMPLIED, INCLUDING BUT NOT LIMITED TO THE WARRANTIES OF
//   MERCHANTABILITY, FITNESS FOR A PARTICULAR PURPOSE AND NONINFRINGEMENT.
//   IN NO EVENT SHALL THE AUTHORS OR COPYRIGHT HOLDERS BE LIABLE FOR ANY
//   CLAIM, DAMAGES OR OTHER LIABILITY, WHETHER IN AN ACTION OF CONTRACT, TORT
//   OR OTHERWISE, ARISING FROM, OUT OF OR IN CONNECTION WITH THE SOFTWARE OR
//   THE USE OR OTHER DEALINGS IN THE SOFTWARE.
//
// Algorithm:
//   state f = M, g = x, d = 0, e = 1, with invariants d*x = f, e*x = g (mod M)
//   and delta = 1 (kept as eta = -delta).  Batches of 30 divsteps are run on
//   the low 32 bits of f, g, accumulating a 2x2 transition matrix T with
//   [f', g'] = T [f, g] / 2^30; T is then applied to the full f, g (exact
//   division) and to d, e (mod M, an M-multiple makes the division exact).
//   When g = 0, f = +-1 and x^-1 = +-d.
#pragma once
#include "common.cuh"

namespace uf {

struct ModInfo {
    uint32_t m[8];      // modulus, 8 x 32 little-endian
    int32_t m30[9];     // modulus in signed 30-bit limbs
    uint32_t minv30;    // M^-1 mod 2^30
};

// 30 variable-time divsteps on the low bits of f, g.
// Returns the new eta; writes T = (u, v, q, r) scaled by 2^30.
UF_HD int32_t divsteps30_var(int32_t eta, uint32_t f0, uint32_t g0, int32_t T[4]) {
    uint32_t u = 1, v = 0, q = 0, r = 1;
    uint32_t f = f0, g = g0, w, m;
    int i = 30, limit, zeros;
    for (;;) {
        // strip trailing zeros of g (capped at the steps left)
        zeros = ctz32(g | (0xFFFFFFFFu << i));
        g >>= zeros;
        u <<= zeros;
        v <<= zeros;
        eta -= zeros;
        i -= zeros;
        if (i == 0) break;
        // g is odd here
        if (eta < 0) {
            uint32_t tmp;
            eta = -eta;
            tmp = f; f = g; g = (uint32_t)(-(int32_t)tmp);
            tmp = u; u = q; q = (uint32_t)(-(int32_t)tmp);
            tmp = v; v = r; r = (uint32_t)(-(int32_t)tmp);
        }
        // up to min(eta+1, i, 6) steps of g <- (g + w f)/2 with no swap in between
        limit = (eta + 1) > i ? i : (eta + 1);
        m = (0xFFFFFFFFu >> (32 - limit)) & 63u;
        // w = -g / f mod 2^6; f*(f*f - 2) = -f^-1 mod 64 for odd f
        w = (f * g * (f * f - 2u)) & m;
        g += f * w;
        q += u * w;
        r += v * w;
    }
    T[0] = (int32_t)u; T[1] = (int32_t)v; T[2] = (int32_t)q; T[3] = (int32_t)r;
    return eta;
}

// [f, g] <- T [f, g] / 2^30, 9 signed 30-bit limbs each.
UF_HD void update_fg30(int32_t f[9], int32_t g[9], const int32_t T[4]) {
    const int64_t u = T[0], v = T[1], q = T[2], r = T[3];
    int64_t cf = u * f[0] + v * g[0];
    int64_t cg = q * f[0] + r * g[0];
    cf >>= 30;
    cg >>= 30;
    UF_UNROLL
    for (int i = 1; i < 9; ++i) {
        cf += u * f[i] + v * g[i];
        cg += q * f[i] + r * g[i];
        f[i - 1] = (int32_t)(cf & 0x3FFFFFFF);
        g[i - 1] = (int32_t)(cg & 0x3FFFFFFF);
        cf >>= 30;
        cg >>= 30;
    }
    f[8] = (int32_t)cf;
    g[8] = (int32_t)cg;
}

// [d, e] <- (T [d, e] + [md, me] M) / 2^30, keeping d, e in (-2M, M).
UF_HD void update_de30(int32_t d[9], int32_t e[9], const int32_t T[4], const ModInfo& mi) {
    const int32_t u = T[0], v = T[1], q = T[2], r = T[3];
    const int32_t sd = d[8] >> 31, se = e[8] >> 31;    // -1 when negative
    // pre-add M multiples for negative inputs, so the result stays in range
    int32_t md = (u & sd) + (v & se);
    int32_t me = (q & sd) + (r & se);
    int64_t cd = (int64_t)u * d[0] + (int64_t)v * e[0];
    int64_t ce = (int64_t)q * d[0] + (int64_t)r * e[0];
    // choose md, me so the low 30 bits of the numerators vanish
    md -= (int32_t)((mi.minv30 * (uint32_t)cd + (uint32_t)md) & 0x3FFFFFFFu);
    me -= (int32_t)((mi.minv30 * (uint32_t)ce + (uint32_t)me) & 0x3FFFFFFFu);
    cd += (int64_t)mi.m30[0] * md;
    ce += (int64_t)mi.m30[0] * me;
    cd >>= 30;
    ce >>= 30;
    UF_UNROLL
    for (int i = 1; i < 9; ++i) {
        cd += (int64_t)u * d[i] + (int64_t)v * e[i] + (int64_t)mi.m30[i] * md;
        ce += (int64_t)q * d[i] + (int64_t)r * e[i] + (int64_t)mi.m30[i] * me;
        d[i - 1] = (int32_t)(cd & 0x3FFFFFFF);
        e[i - 1] = (int32_t)(ce & 0x3FFFFFFF);
        cd >>= 30;
        ce >>= 30;
    }
    d[8] = (int32_t)cd;
    e[8] = (int32_t)ce;
}

UF_HD void to_s30(int32_t o[9], const uint32_t v[8]) {
    // 256 bits -> 9 limbs of 30 bits (top limb 16 bits)
    UF_UNROLL
    for (int i = 0; i < 9; ++i) {
        const int bit = 30 * i, li = bit >> 5, off = bit & 31;
        uint64_t w = v[li];
        if (li + 1 < 8) w |= (uint64_t)v[li + 1] << 32;
        o[i] = (int32_t)((w >> off) & 0x3FFFFFFFu);
    }
}

// Signed 30-bit limbs (value in (-2M, 2M), sign in the top limb) -> [0, M).
UF_HD void from_s30_mod(uint32_t out[8], const int32_t in[9], bool negate, const ModInfo& mi) {
    int32_t a[9];
    UF_UNROLL
    for (int i = 0; i < 9; ++i) a[i] = in[i];
    // carry-normalise into limbs in [0, 2^30) with a signed top limb
    {
        int64_t c = 0;
        UF_UNROLL
        for (int i = 0; i < 8; ++i) {
            c += a[i];
            a[i] = (int32_t)(c & 0x3FFFFFFF);
            c >>= 30;
        }
        a[8] = (int32_t)(c + a[8]);
    }
    if (negate) {
        int64_t c = 0;
        UF_UNROLL
        for (int i = 0; i < 8; ++i) {
            c -= a[i];
            a[i] = (int32_t)(c & 0x3FFFFFFF);
            c >>= 30;
        }
        a[8] = (int32_t)(c - a[8]);
    }
    // bring into [0, M): add M while negative, subtract M while >= M
    for (int iter = 0; iter < 4 && a[8] < 0; ++iter) {
        int64_t c = 0;
        UF_UNROLL
        for (int i = 0; i < 8; ++i) {
            c += (int64_t)a[i] + mi.m30[i];
            a[i] = (int32_t)(c & 0x3FFFFFFF);
            c >>= 30;
        }
        a[8] = (int32_t)(c + a[8] + mi.m30[8]);
    }
    // now 0 <= a < 2M: subtract M while the result stays non-negative
    for (int iter = 0; iter < 3; ++iter) {
        int32_t b[9];
        int64_t c = 0;
        UF_UNROLL
        for (int i = 0; i < 8; ++i) {
            c += (int64_t)a[i] - mi.m30[i];
            b[i] = (int32_t)(c & 0x3FFFFFFF);
            c >>= 30;
        }
        b[8] = (int32_t)(c + a[8] - mi.m30[8]);
        if (b[8] < 0) break;
        UF_UNROLL
        for (int i = 0; i < 9; ++i) a[i] = b[i];
    }
    // to 8x32 (a < M < 2^256, so nothing is lost)
    uint32_t o[8];
    UF_UNROLL
    for (int i = 0; i < 8; ++i) o[i] = 0;
    UF_UNROLL
    for (int i = 0; i < 9; ++i) {
        const int bit = 30 * i, li = bit >> 5, off = bit & 31;
        const uint64_t w = (uint64_t)(uint32_t)a[i] << off;
        o[li] |= lo32(w);
        if (li + 1 < 8) o[li + 1] |= hi32(w);
    }
    UF_UNROLL
    for (int i = 0; i < 8; ++i) out[i] = o[i];
}

// out = x^-1 mod M for 0 < x < M (x = 0 gives 0).
UF_COLD void modinv_var(uint32_t out[8], const uint32_t x[8], const ModInfo& mi) {
    int32_t f[9], g[9], d[9], e[9], T[4];
    UF_UNROLL
    for (int i = 0; i < 9; ++i) { f[i] = mi.m30[i]; d[i] = 0; e[i] = 0; }
    e[0] = 1;
    to_s30(g, x);
    int32_t eta = -1;
    // at most 20 batches are needed for 256-bit inputs; the cap bounds the loop
    for (int it = 0; it < 25; ++it) {
        eta = divsteps30_var(eta, (uint32_t)f[0], (uint32_t)g[0], T);
        update_de30(d, e, T, mi);
        update_fg30(f, g, T);
        uint32_t nz = 0;
        UF_UNROLL
        for (int i = 0; i < 9; ++i) nz |= (uint32_t)g[i];
        if (nz == 0) break;
    }
    // f = +-1: the sign of f decides the sign of the result
    from_s30_mod(out, d, f[8] < 0, mi);
}

}  // namespace uf
