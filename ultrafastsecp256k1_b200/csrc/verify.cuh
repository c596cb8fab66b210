// Per-signature ECDSA and BIP-340 verification with the reference CPU's
// semantics (the reference GPU kernels are laxer; the CPU verify is the oracle).
//
// ECDSA (compact form), as ufsecp_ecdsa_verify (src/cpu/src/impl/ufsecp_ecdsa.cpp:244-272):
//   r, s in [1, n-1] (ECDSASignature::parse_compact_strict, src/cpu/src/ecdsa.cpp:94),
//   s <= n/2 (BIP-62 low-S, :259-262), pubkey 02/03 prefix, x < p, on the curve
//   (ecdsa_pubkey_parse, src/cpu/src/ecdsa.cpp:891-906), z = msg mod n,
//   R = (z/s) G + (r/s) Q, R != infinity, x(R) = r or x(R) = r + n when r + n < p,
//   checked projectively as r Z^2 == X (ecdsa_check_xcoord, src/cpu/src/ecdsa.cpp:764).
// BIP-340, as ufsecp_schnorr_verify (src/cpu/src/impl/ufsecp_ecdsa.cpp:992-1022):
//   r < p, 0 < s < n (SchnorrSignature::parse_strict, src/cpu/src/schnorr.cpp:355),
//   pubkey x < p and liftable (lift_x_cached, :275-301),
//   e = H_challenge(r || P.x || m) mod n, R = s G - e P, R != infinity,
//   y(R) even, x(R) == r (schnorr_verify, src/cpu/src/schnorr.cpp:542-612).
#pragma once
#include "common.cuh"
#include "fe.cuh"
#include "fn.cuh"
#include "point.cuh"
#include "sha256.cuh"
#include "ecmult.cuh"

namespace uf {

// p - n: when r < p - n, r + n is also a field element that could equal x(R).
UF_HD bool r_below_p_minus_n(const uint32_t r[8]) {
    const uint32_t pmn[8] = {0x2FC9BAEEu, 0x402DA172u, 0x50B75FC4u, 0x45512319u, 0x00000001u, 0, 0, 0};
    return lt256(r, pmn);
}

// x(R) == r or, when r + n < p, x(R) == r + n, checked projectively as
// r Z^2 == X (ecdsa_check_xcoord, src/cpu/src/ecdsa.cpp:764); false for R = inf.
UF_HDI bool ecdsa_check_x(const Jac& R, const Sc& r) {
    if (R.inf) return false;
    Fe z2, t, rf;
    fe_sqr(z2, R.Z);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) rf.v[i] = r.v[i];
    fe_mul(t, rf, z2);
    if (fe_equal(t, R.X)) return true;
    if (!r_below_p_minus_n(r.v)) return false;
    uint32_t n[8];
    sc_n(n);
    uint64_t c = 0;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        c = (uint64_t)r.v[i] + n[i] + (c >> 32);
        rf.v[i] = lo32(c);
    }
    fe_mul(t, rf, z2);
    return fe_equal(t, R.X);
}

// BIP-340's final check: R finite, y(R) even, x(R) == r (src/cpu/src/schnorr.cpp:595-610).
UF_HDI bool schnorr_check(const Jac& R, const uint32_t r[8]) {
    Aff A;
    if (!jac_to_aff(A, R)) return false;
    if (A.y.v[0] & 1u) return false;
    uint32_t diff = 0;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) diff |= A.x.v[i] ^ r[i];
    return diff == 0;
}

// ECDSA after the signature's scalars are parsed (r, s in [1, n-1]).  `cache`
// (SlotPubCache / NoPubCache, pubcache.cuh) may supply the key's table instead
// of decompressing the key and building it, or know the key to be off the
// curve.
template <class Tab, class GT, class Cache = NoPubCache>
UF_HDI bool ecdsa_verify_rs(const uint32_t msg_w[8], const uint8_t* pub33, const Sc& r, const Sc& s, Tab& tab,
                            const GT& gt, const Cache& cache = Cache()) {
    const uint8_t prefix = pub33[0];
    if (prefix != 0x02 && prefix != 0x03) return false;
    Fe qx, qy;
    be32_to_limbs(qx.v, pub33 + 1);
    if (!limbs_lt_p(qx.v)) return false;
    const int c = cache.fetch(tab);
    if (c == kKeyBad) return false;
    const bool cached = c == kKeyTable;
    if (!cached && !lift_x_parity(qy, qx, prefix == 0x03)) return false;
    Sc z, w, u1, u2;
    words_be_to_limbs(z.v, msg_w);
    sc_reduce_once(z);
    sc_inv(w, s);
    sc_mul(u1, z, w);
    sc_mul(u2, r, w);
    Jac R;
    dual_mul_c(R, u1, qx, qy, u2, tab, gt, cached);
    return ecdsa_check_x(R, r);
}

// msg_w / sig_w: the 32 / 64 input bytes as words loaded little-endian;
// compact big-endian r || s, low-S required.
template <class Tab, class GT, class Cache = NoPubCache>
UF_HDI bool ecdsa_verify_one(const uint32_t msg_w[8], const uint8_t* pub33, const uint32_t sig_w[16],
                             Tab& tab, const GT& gt, const Cache& cache = Cache()) {
    Sc r, s;
    words_be_to_limbs(r.v, sig_w);
    words_be_to_limbs(s.v, sig_w + 8);
    if (sc_is_zero(r) || !limbs_lt_n(r.v)) return false;
    if (sc_is_zero(s) || !limbs_lt_n(s.v)) return false;
    if (!sc_is_low(s.v)) return false;
    return ecdsa_verify_rs(msg_w, pub33, r, s, tab, gt, cache);
}

// The libsecp in-memory signature layout of the consensus surfaces
// (ufsecp_gpu_ecdsa_verify_opaque_rows / _lbtc_columns): r then s, each 32
// little-endian bytes, so the little-endian words ARE the limbs.  r, s in
// [1, n-1] without reduction; a high s is normalised to n - s, i.e. accepted
// (ecdsa_sig_parse_opaque with normalize, src/cpu/src/impl/ufsecp_ecdsa.cpp:128-139).
template <class Tab, class GT>
UF_HDI bool ecdsa_verify_opaque_one(const uint32_t msg_w[8], const uint8_t* pub33, const uint32_t sig_w[16],
                                    Tab& tab, const GT& gt) {
    Sc r, s;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        r.v[i] = sig_w[i];
        s.v[i] = sig_w[8 + i];
    }
    if (sc_is_zero(r) || !limbs_lt_n(r.v)) return false;
    if (sc_is_zero(s) || !limbs_lt_n(s.v)) return false;
    if (!sc_is_low(s.v)) sc_neg(s, s);
    return ecdsa_verify_rs(msg_w, pub33, r, s, tab, gt);
}

template <class Tab, class GT, class Cache = NoPubCache>
UF_HDI bool schnorr_verify_one(const uint32_t msg_w[8], const uint32_t px_w[8], const uint32_t sig_w[16],
                               Tab& tab, const GT& gt, const Cache& cache = Cache()) {
    uint32_t r[8];
    Sc s;
    words_be_to_limbs(r, sig_w);
    words_be_to_limbs(s.v, sig_w + 8);
    if (!limbs_lt_p(r)) return false;
    if (sc_is_zero(s) || !limbs_lt_n(s.v)) return false;
    Fe px, py;
    words_be_to_limbs(px.v, px_w);
    if (!limbs_lt_p(px.v)) return false;
    const int c = cache.fetch(tab);
    if (c == kKeyBad) return false;
    const bool cached = c == kKeyTable;
    if (!cached && !lift_x_parity(py, px, false)) return false;
    uint32_t rbe[8], pbe[8], mbe[8], h[8];
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        rbe[i] = bswap32(sig_w[i]);
        pbe[i] = bswap32(px_w[i]);
        mbe[i] = bswap32(msg_w[i]);
    }
    bip340_challenge(h, rbe, pbe, mbe);
    Sc e, ne;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) e.v[i] = h[7 - i];
    sc_reduce_once(e);
    sc_neg(ne, e);
    Jac R;
    dual_mul_c(R, s, px, py, ne, tab, gt, cached);
    return schnorr_check(R, r);
}

}  // namespace uf
