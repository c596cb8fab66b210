// Points on y^2 = x^3 + 7 in Jacobian coordinates (x = X/Z^2, y = Y/Z^3).
//
// Role in the reference: jacobian_double_unchecked (src/cuda/include/secp256k1.cuh:1610),
// jacobian_add_mixed[_unchecked] (:1647, :1730), point_from_compressed (:4462),
// lift_x (src/cuda/include/schnorr.cuh:95).  Formulas are the standard a = 0
// ones from the Explicit-Formulas Database: dbl-2009-l (2M + 5S) and
// madd-2007-bl (7M + 4S).  The mixed add handles every exceptional case
// (infinite accumulator, P + P, P + (-P)) so verdicts are exact for
// adversarial inputs, not only for random ones.
#pragma once
#include "common.cuh"
#include "fe.cuh"
#include "fn.cuh"

namespace uf {

struct Aff { Fe x, y; };
struct Jac { Fe X, Y, Z; bool inf; };

UF_HD void jac_set_inf(Jac& a) {
    fe_set_u32(a.X, 0); fe_set_u32(a.Y, 1); fe_set_u32(a.Z, 0);
    a.inf = true;
}

UF_HD void jac_from_aff(Jac& a, const Fe& x, const Fe& y) {
    a.X = x; a.Y = y; fe_set_u32(a.Z, 1); a.inf = false;
}

// dbl-2009-l.  Y = 0 cannot occur on secp256k1 (no 2-torsion).
UF_HD Jac jac_dbl_c(Jac a) {
    if (a.inf) return a;
    Fe A, B, C, D, E, t;
    fe_mul(t, a.Y, a.Z);
    fe_dbl(a.Z, t);             // Z3 = 2 Y Z
    fe_sqr(A, a.X);             // A = X^2
    fe_sqr(B, a.Y);             // B = Y^2
    fe_sqr(C, B);               // C = B^2
    fe_add(t, a.X, B);
    fe_sqr(t, t);
    fe_sub(t, t, A);
    fe_sub(t, t, C);
    fe_dbl(D, t);               // D = 2((X+B)^2 - A - C)
    fe_dbl(E, A);
    fe_add(E, E, A);            // E = 3A
    fe_sqr(t, E);               // F = E^2
    fe_sub(t, t, D);
    fe_sub(a.X, t, D);          // X3 = F - 2D
    fe_sub(t, D, a.X);
    fe_mul(a.Y, E, t);
    fe_mul_pow2<3>(C, C);
    fe_sub(a.Y, a.Y, C);        // Y3 = E (D - X3) - 8C
    return a;
}

UF_POINT_FN Jac jac_dbl_v(Jac a) { return jac_dbl_c(a); }

// n >= 1 doublings in one out-of-line call (a window's doublings).
UF_POINT_FN Jac jac_dbl_n_v(Jac a, int n) {
    UF_NOUNROLL
    for (int i = 0; i < n; ++i) a = jac_dbl_c(a);
    return a;
}

UF_HD void jac_dbl(Jac& a) { a = jac_dbl_v(a); }
UF_HD void jac_dbl_n(Jac& a, int n) { a = jac_dbl_n_v(a, n); }

// a += (x2, y2) affine (madd-2007-bl), exact in all cases.
UF_POINT_FN Jac jac_add_aff_v(Jac a, Fe x2, Fe y2) {
    if (a.inf) { jac_from_aff(a, x2, y2); return a; }
    Fe Z1Z1, U2, S2, H, r, t;
    fe_sqr(Z1Z1, a.Z);
    fe_mul(U2, x2, Z1Z1);
    fe_mul(t, a.Z, Z1Z1);
    fe_mul(S2, y2, t);
    fe_sub(H, U2, a.X);
    fe_sub(r, S2, a.Y);
    if (fe_is_zero(H)) {
        if (fe_is_zero(r)) jac_dbl(a);      // same point
        else a.inf = true;                  // opposite points
        return a;
    }
    Fe HH, I, J, V;
    fe_sqr(HH, H);
    fe_mul_pow2<2>(I, HH);      // I = 4 HH
    fe_mul(J, H, I);            // J = H I
    fe_dbl(r, r);               // r = 2 (S2 - Y1)
    fe_mul(V, a.X, I);          // V = X1 I
    // Z3 = (Z1 + H)^2 - Z1Z1 - HH
    fe_add(t, a.Z, H);
    fe_sqr(t, t);
    fe_sub(t, t, Z1Z1);
    fe_sub(a.Z, t, HH);
    // X3 = r^2 - J - 2V
    fe_sqr(t, r);
    fe_sub(t, t, J);
    fe_sub(t, t, V);
    fe_sub(a.X, t, V);
    // Y3 = r (V - X3) - 2 Y1 J
    fe_sub(t, V, a.X);
    fe_mul(t, r, t);
    fe_mul(J, a.Y, J);
    fe_dbl(J, J);
    fe_sub(a.Y, t, J);
    return a;
}

UF_HD void jac_add_aff(Jac& a, const Fe& x2, const Fe& y2) { a = jac_add_aff_v(a, x2, y2); }

// General Jacobian + Jacobian (used off the hot path: table set-up, tests).
UF_HDI void jac_add(Jac& a, const Jac& b) {
    if (b.inf) return;
    if (a.inf) { a = b; return; }
    Fe Z1Z1, Z2Z2, U1, U2, S1, S2, H, R, t;
    fe_sqr(Z1Z1, a.Z);
    fe_sqr(Z2Z2, b.Z);
    fe_mul(U1, a.X, Z2Z2);
    fe_mul(U2, b.X, Z1Z1);
    fe_mul(t, a.Y, b.Z);
    fe_mul(S1, t, Z2Z2);
    fe_mul(t, b.Y, a.Z);
    fe_mul(S2, t, Z1Z1);
    fe_sub(H, U2, U1);
    fe_sub(R, S2, S1);
    if (fe_is_zero(H)) {
        if (fe_is_zero(R)) jac_dbl(a);
        else a.inf = true;
        return;
    }
    Fe HH, HHH, V;
    fe_sqr(HH, H);
    fe_mul(HHH, H, HH);
    fe_mul(V, U1, HH);
    fe_sqr(t, R);
    fe_sub(t, t, HHH);
    fe_sub(t, t, V);
    fe_sub(a.X, t, V);
    fe_sub(t, V, a.X);
    fe_mul(t, R, t);
    fe_mul(S1, S1, HHH);
    fe_sub(a.Y, t, S1);
    fe_mul(t, a.Z, b.Z);
    fe_mul(a.Z, t, H);
}

UF_HDI void fe_inv(Fe& r, const Fe& a) {
    ModInfo mi;
    modinfo_p(mi);
    Fe c = a;
    fe_normalize(c);
    modinv_var(r.v, c.v, mi);
}

// Jacobian -> affine (canonical coordinates); false for infinity.
UF_HDI bool jac_to_aff(Aff& o, const Jac& a) {
    if (a.inf) return false;
    Fe zi, zi2, zi3;
    fe_inv(zi, a.Z);
    fe_sqr(zi2, zi);
    fe_mul(zi3, zi2, zi);
    fe_mul(o.x, a.X, zi2);
    fe_mul(o.y, a.Y, zi3);
    fe_normalize(o.x);
    fe_normalize(o.y);
    return true;
}

// y^2 = x^3 + 7 for a canonical x; picks the root with parity `odd`.
// (SEC1 decompression, src/cpu/src/ecdsa.cpp:891-906; BIP-340 lift_x with
// odd = false, src/cpu/src/schnorr.cpp:50-117.)
UF_HDI bool lift_x_parity(Fe& y, const Fe& x, bool odd) {
    Fe y2, s;
    fe_sqr(y2, x);
    fe_mul(y2, y2, x);
    Fe seven;
    fe_set_u32(seven, 7);
    fe_add(y2, y2, seven);
    if (!fe_sqrt(s, y2)) return false;
    fe_normalize(s);
    if ((bool)(s.v[0] & 1) != odd) {
        fe_neg(s, s);
        fe_normalize(s);
    }
    y = s;
    return true;
}

UF_HD void fe_beta(Fe& b) {
    b.v[0] = 0x719501EEu; b.v[1] = 0xC1396C28u; b.v[2] = 0x12F58995u; b.v[3] = 0x9CF04975u;
    b.v[4] = 0xAC3434E9u; b.v[5] = 0x6E64479Eu; b.v[6] = 0x657C0710u; b.v[7] = 0x7AE96A2Bu;
}

UF_HD void gen_point(Aff& g) {
    g.x.v[0] = 0x16F81798u; g.x.v[1] = 0x59F2815Bu; g.x.v[2] = 0x2DCE28D9u; g.x.v[3] = 0x029BFCDBu;
    g.x.v[4] = 0xCE870B07u; g.x.v[5] = 0x55A06295u; g.x.v[6] = 0xF9DCBBACu; g.x.v[7] = 0x79BE667Eu;
    g.y.v[0] = 0xFB10D4B8u; g.y.v[1] = 0x9C47D08Fu; g.y.v[2] = 0xA6855419u; g.y.v[3] = 0xFD17B448u;
    g.y.v[4] = 0x0E1108A8u; g.y.v[5] = 0x5DA4FBFCu; g.y.v[6] = 0x26A3C465u; g.y.v[7] = 0x483ADA77u;
}

}  // namespace uf
