// R = a*G + b*P: the double-scalar multiplication at the centre of verify.
//
// Role in the reference: shamir_double_mul_glv (src/cuda/include/secp256k1.cuh:3575-3801,
// a bit-by-bit 4-stream Strauss with a per-signature joint table) and the CPU's
// Point::dual_scalar_mul_gen_point (src/cpu/src/point.cpp:4079).  Re-designed for
// SIMT on sm_100a:
//
//  * both scalars are GLV-split, giving four 128-bit streams: a1*G, a2*(lambda G),
//    b1*P, b2*(lambda P) with lambda(x, y) = (beta x, y);
//  * every stream uses FIXED-position signed (Booth) windows recoded on the fly,
//    so all 32 lanes of a warp add at the same loop positions (a wNAF's
//    data-dependent positions would make the warp add at almost every bit);
//  * P streams: 4-bit windows, table of 1P..8P (affine, one field inversion per
//    signature through a batch-to-affine), lambda P via one beta multiplication;
//  * G streams: UF_GWIN-bit windows (20: every fifth P window), tables of the 2^(UF_GWIN-1) multiples
//    of G and of lambda G computed once per context and read through L1 / L2;
//  * 33 P windows x 4 bits = 132 >= 129 bits, so 128 doublings in total.
#pragma once
#include "common.cuh"
#include "fe.cuh"
#include "fn.cuh"
#include "point.cuh"
#include "pubcache.cuh"

namespace uf {

// P window bits: 4 by default; the window-width variants of the verify kernel
// are compiled with 3 or 5 (UF_PWIN), and with other G windows (UF_GWIN).
#ifndef UF_PWIN
#define UF_PWIN 4
#endif
constexpr int kWP = UF_PWIN;                  // P window bits
constexpr int kNWP = (129 + kWP - 1) / kWP;   // P windows: 33 for 4 bits (132 >= 129)
constexpr int kWG = UF_GWIN;                  // G window bits (a multiple of kWP)
constexpr int kNWG = (129 + kWG - 1) / kWG;   // G windows: 7 for 20 bits (one per five P windows)
constexpr int kGEvery = kWG / kWP;            // P windows per G window
static_assert(kWG % kWP == 0 && kNWG * kGEvery >= kNWP, "G windows must align with P windows");
static_assert(kWG <= 30, "G Booth digits (up to 2^(kWG-1)) are stored as int32_t");
typedef int32_t GDigit;   // a G-stream Booth digit, |d| <= 2^(kWG-1)
constexpr int kPTab = 1 << (kWP - 1);   // 1P..8P for 4-bit windows
constexpr int kGTab = 1 << (kWG - 1); // 1G..2^19 G for 20-bit windows (and the same for lambda G)

// Signed fixed-window (Booth) digits of a magnitude k < 2^129:
// d_i = b_{wi-1} + sum_{t<w-1} b_{wi+t} 2^t - b_{wi+w-1} 2^(w-1), d_i in [-2^(w-1), 2^(w-1)],
// sum_i d_i 2^(wi) = k.
template <int W, int NW, typename T>
UF_HD void booth_recode(T* out, const uint32_t k[4]) {
    const uint32_t kk[6] = {k[0], k[1], k[2], k[3], 0u, 0u};
    const uint32_t mask = (1u << (W + 1)) - 1u;
    UF_UNROLL
    for (int i = 0; i < NW; ++i) {
        const int pos = W * i - 1;
        uint32_t raw;
        if (pos < 0) {
            raw = (kk[0] << 1) & mask;
        } else {
            const int li = pos >> 5, off = pos & 31;
            const uint64_t v = ((uint64_t)kk[li + 1] << 32) | kk[li];
            raw = (uint32_t)(v >> off) & mask;
        }
        out[i] = (T)((int)(raw & 1u) + (int)((raw >> 1) & ((1u << (W - 1)) - 1u)) - (int)((raw >> W) << (W - 1)));
    }
}

// Table of (k+1)*P for k = 0..7, affine, in two halves around its one field
// inversion, so that a block of signatures can share that inversion
// (Montgomery's trick across threads, grpinv.cuh).  _pre stores 1P..8P with
// their Jacobian X, Y in `tab` (1P affine), the Z of 2P..8P in zs and their
// running products in cs; cs[kPTab - 2] is the product of all of them.  _post
// turns the entries affine from `inv`, the inverse of that product.  Tab must
// provide store(k, Fe x, Fe y) / load(k, Fe& x, Fe& y).
template <class Tab>
UF_HDI void build_ptable_pre(Tab& tab, const Fe& px, const Fe& py, Fe zs[kPTab - 1], Fe cs[kPTab - 1]) {
    tab.store(0, px, py);
    UF_NOUNROLL
    for (int k = 2; k <= kPTab; ++k) {
        Jac t;
        t.inf = false;
        if ((k & 1) == 0) {
            if (k == 2) {
                jac_from_aff(t, px, py);
            } else {
                tab.load(k / 2 - 1, t.X, t.Y);
                t.Z = zs[k / 2 - 2];
            }
            jac_dbl(t);
        } else {
            tab.load(k - 2, t.X, t.Y);
            t.Z = zs[k - 3];
            jac_add_aff(t, px, py);
        }
        tab.store(k - 1, t.X, t.Y);
        zs[k - 2] = t.Z;
        if (k == 2) cs[0] = t.Z;
        else fe_mul(cs[k - 2], cs[k - 3], t.Z);
    }
}

template <class Tab>
UF_HDI void build_ptable_post(Tab& tab, const Fe zs[kPTab - 1], const Fe cs[kPTab - 1], Fe inv) {
    UF_NOUNROLL
    for (int k = kPTab; k >= 2; --k) {
        Fe zi, zi2, X, Y;
        if (k > 2) {
            fe_mul(zi, inv, cs[k - 3]);
            fe_mul(inv, inv, zs[k - 2]);
        } else {
            zi = inv;
        }
        fe_sqr(zi2, zi);
        tab.load(k - 1, X, Y);
        fe_mul(X, X, zi2);
        fe_mul(zi2, zi2, zi);
        fe_mul(Y, Y, zi2);
        tab.store(k - 1, X, Y);
    }
}

// The whole table with its own inversion.
template <class Tab>
UF_HDI void build_ptable(Tab& tab, const Fe& px, const Fe& py) {
    Fe zs[kPTab - 1], cs[kPTab - 1];
    build_ptable_pre(tab, px, py, zs, cs);
    Fe inv;
    fe_inv(inv, cs[kPTab - 2]);
    build_ptable_post(tab, zs, cs, inv);
}

template <class Tab>
UF_HD void add_ptab(Jac& R, const Tab& tab, int d, bool sneg, bool lam, const Fe& beta) {
    if (d == 0) return;
    const bool neg = (d < 0) != sneg;
    const int idx = (d < 0 ? -d : d) - 1;
    Fe x, y;
    tab.load(idx, x, y);
    if (lam) fe_mul(x, x, beta);
    if (neg) fe_neg(y, y);
    jac_add_aff(R, x, y);
}

template <class GT>
UF_HD void add_gtab(Jac& R, const GT& gt, int d, bool sneg, int lam) {
    if (d == 0) return;
    const bool neg = (d < 0) != sneg;
    const int idx = (d < 0 ? -d : d) - 1 + lam * kGTab;
    Fe x, y;
    gt.load(idx, x, y);
    if (neg) fe_neg(y, y);
    jac_add_aff(R, x, y);
}

// Booth digits of the four GLV streams of R = a*G + b*P, for kernels that
// split the computation into phases (kernels_verify_grp.cu).
struct DualDigits {
    int8_t dp1[kNWP], dp2[kNWP];
    GDigit dg1[kNWG], dg2[kNWG];
    bool np1, np2, ng1, ng2;
};

UF_HDI void dual_recode(DualDigits& d, const Sc& a, const Sc& b) {
    GlvSplit sa, sb;
    glv_split(sa, a);
    glv_split(sb, b);
    booth_recode<kWP, kNWP>(d.dp1, sb.k1);
    booth_recode<kWP, kNWP>(d.dp2, sb.k2);
    booth_recode<kWG, kNWG>(d.dg1, sa.k1);
    booth_recode<kWG, kNWG>(d.dg2, sa.k2);
    d.np1 = sb.neg1;
    d.np2 = sb.neg2;
    d.ng1 = sa.neg1;
    d.ng2 = sa.neg2;
}

// The main loop over recoded digits: 128 doublings, the P-table and G-table additions.
template <class Tab, class GT>
UF_HDI void dual_loop(Jac& R, const DualDigits& d, const Tab& tab, const GT& gt) {
    Fe beta;
    fe_beta(beta);
    jac_set_inf(R);
    UF_NOUNROLL
    for (int i = kNWP - 1; i >= 0; --i) {
        if (i != kNWP - 1) jac_dbl_n(R, kWP);
        add_ptab(R, tab, d.dp1[i], d.np1, false, beta);
        add_ptab(R, tab, d.dp2[i], d.np2, true, beta);
        if (i % kGEvery == 0) {
            add_gtab(R, gt, d.dg1[i / kGEvery], d.ng1, 0);
            add_gtab(R, gt, d.dg2[i / kGEvery], d.ng2, 1);
        }
    }
}

// R = a*G + b*P for P = (px, py) on the curve (not infinity).  With
// have_tab the caller already filled `tab` (a resident key) and px, py are not
// read; otherwise the table is built here, after the digit recoding (the order
// that keeps the kernel at 3 blocks per SM).
template <class Tab, class GT>
UF_HDI void dual_mul_c(Jac& R, const Sc& a, const Fe& px, const Fe& py, const Sc& b, Tab& tab, const GT& gt,
                       bool have_tab) {
    GlvSplit sa, sb;
    glv_split(sa, a);
    glv_split(sb, b);
    int8_t dp1[kNWP], dp2[kNWP];
    GDigit dg1[kNWG], dg2[kNWG];
    booth_recode<kWP, kNWP>(dp1, sb.k1);
    booth_recode<kWP, kNWP>(dp2, sb.k2);
    booth_recode<kWG, kNWG>(dg1, sa.k1);
    booth_recode<kWG, kNWG>(dg2, sa.k2);
    if (!have_tab) build_ptable(tab, px, py);
    Fe beta;
    fe_beta(beta);
    jac_set_inf(R);
    UF_NOUNROLL
    for (int i = kNWP - 1; i >= 0; --i) {
        if (i != kNWP - 1) jac_dbl_n(R, kWP);
        add_ptab(R, tab, dp1[i], sb.neg1, false, beta);
        add_ptab(R, tab, dp2[i], sb.neg2, true, beta);
        if (i % kGEvery == 0) {
            add_gtab(R, gt, dg1[i / kGEvery], sa.neg1, 0);
            add_gtab(R, gt, dg2[i / kGEvery], sa.neg2, 1);
        }
    }
}

// One lane's half of R = a*G + b*P when two lanes share a signature: half 0
// sums the a1*G and b1*P streams, half 1 the a2*(lambda G) and b2*(lambda P)
// streams (the GLV halves), each with the full 128 doublings, so that the two
// partial sums add up to R.  Both lanes build the same P table in their own
// shared-memory slots (the same instruction stream, so no divergence), unless
// have_tab says the caller already filled `tab`.
template <class Tab, class GT>
UF_HDI void dual_mul_half(Jac& R, const Sc& a, const Fe& px, const Fe& py, const Sc& b, Tab& tab, const GT& gt,
                          int half, bool have_tab = false) {
    GlvSplit sa, sb;
    glv_split(sa, a);
    glv_split(sb, b);
    uint32_t kp[4], kg[4];
    UF_UNROLL
    for (int i = 0; i < 4; ++i) {
        kp[i] = half ? sb.k2[i] : sb.k1[i];
        kg[i] = half ? sa.k2[i] : sa.k1[i];
    }
    const bool negp = half ? sb.neg2 : sb.neg1, negg = half ? sa.neg2 : sa.neg1;
    int8_t dp[kNWP];
    GDigit dg[kNWG];
    booth_recode<kWP, kNWP>(dp, kp);
    booth_recode<kWG, kNWG>(dg, kg);
    if (!have_tab) build_ptable(tab, px, py);
    Fe beta;
    fe_beta(beta);
    jac_set_inf(R);
    UF_NOUNROLL
    for (int i = kNWP - 1; i >= 0; --i) {
        if (i != kNWP - 1) jac_dbl_n(R, kWP);
        add_ptab(R, tab, dp[i], negp, half != 0, beta);
        if (i % kGEvery == 0) add_gtab(R, gt, dg[i / kGEvery], negg, half);
    }
}

template <class Tab, class GT>
UF_HDI void dual_mul(Jac& R, const Sc& a, const Fe& px, const Fe& py, const Sc& b, Tab& tab, const GT& gt) {
    dual_mul_c(R, a, px, py, b, tab, gt, false);
}

}  // namespace uf
