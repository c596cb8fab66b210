// Signers for synthetic workloads: RFC 6979 ECDSA (low-S) and BIP-340.
//
// Not on the verify path.  They exist so the benchmark and the serving tests
// can create large seeded corpora of valid signatures quickly (on the GPU,
// or on the host for small sets), with the same bytes the reference's CPU
// signers produce: ufsecp_ecdsa_sign (RFC 6979 nonce over the raw 32-byte
// message hash, src/cpu/src/ecdsa.cpp:335-429; low-S output) and
// ufsecp_schnorr_sign (BIP-340 default signing with aux_rand).  The tests
// check them byte-for-byte against the oracle's signers.
#pragma once
#include "common.cuh"
#include "fe.cuh"
#include "fn.cuh"
#include "point.cuh"
#include "sha256.cuh"
#include "ecmult.cuh"

namespace uf {

// SHA-256 of a short message (< 184 bytes) continuing from state h after
// `prefix_bytes` bytes were already compressed (0 for a plain hash).
UF_HDI void sha256_tail(uint32_t h[8], const uint8_t* msg, int len, int prefix_bytes) {
    uint8_t buf[192];
    for (int i = 0; i < len; ++i) buf[i] = msg[i];
    int total = len + 1 + 8;
    const int blocks = (total + 63) / 64;
    total = blocks * 64;
    buf[len] = 0x80;
    for (int i = len + 1; i < total; ++i) buf[i] = 0;
    const uint64_t bits = (uint64_t)(len + prefix_bytes) * 8;
    for (int i = 0; i < 8; ++i) buf[total - 1 - i] = (uint8_t)(bits >> (8 * i));
    for (int b = 0; b < blocks; ++b) {
        uint32_t w[16];
        for (int i = 0; i < 16; ++i) {
            const uint8_t* p = buf + 64 * b + 4 * i;
            w[i] = ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
        }
        sha256_compress(h, w);
    }
}

UF_HD void sha256_iv(uint32_t h[8]) {
    h[0] = 0x6a09e667u; h[1] = 0xbb67ae85u; h[2] = 0x3c6ef372u; h[3] = 0xa54ff53au;
    h[4] = 0x510e527fu; h[5] = 0x9b05688cu; h[6] = 0x1f83d9abu; h[7] = 0x5be0cd19u;
}

UF_HD void words_to_bytes(uint8_t* out, const uint32_t h[8]) {
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(h[i] >> 24); out[4 * i + 1] = (uint8_t)(h[i] >> 16);
        out[4 * i + 2] = (uint8_t)(h[i] >> 8); out[4 * i + 3] = (uint8_t)h[i];
    }
}

// HMAC-SHA256 with a 32-byte key.
UF_HDI void hmac_sha256_k32(uint8_t out[32], const uint8_t key[32], const uint8_t* msg, int len) {
    uint32_t h[8], w[16];
    uint8_t pad[64], ih[32];
    for (int i = 0; i < 64; ++i) pad[i] = (uint8_t)((i < 32 ? key[i] : 0) ^ 0x36);
    sha256_iv(h);
    for (int i = 0; i < 16; ++i)
        w[i] = ((uint32_t)pad[4 * i] << 24) | ((uint32_t)pad[4 * i + 1] << 16) | ((uint32_t)pad[4 * i + 2] << 8) | pad[4 * i + 3];
    sha256_compress(h, w);
    sha256_tail(h, msg, len, 64);
    words_to_bytes(ih, h);
    for (int i = 0; i < 64; ++i) pad[i] = (uint8_t)((i < 32 ? key[i] : 0) ^ 0x5c);
    sha256_iv(h);
    for (int i = 0; i < 16; ++i)
        w[i] = ((uint32_t)pad[4 * i] << 24) | ((uint32_t)pad[4 * i + 1] << 16) | ((uint32_t)pad[4 * i + 2] << 8) | pad[4 * i + 3];
    sha256_compress(h, w);
    sha256_tail(h, ih, 32, 64);
    words_to_bytes(out, h);
}

// Tagged hash from a precomputed midstate (state after SHA256(tag)||SHA256(tag)).
UF_HDI void tagged_from_mid(uint8_t out[32], const uint32_t mid[8], const uint8_t* msg, int len) {
    uint32_t h[8];
    for (int i = 0; i < 8; ++i) h[i] = mid[i];
    sha256_tail(h, msg, len, 64);
    words_to_bytes(out, h);
}

UF_HD void mid_aux(uint32_t m[8]) {
    m[0] = 0x24dd3219u; m[1] = 0x4eba7e70u; m[2] = 0xca0fabb9u; m[3] = 0x0fa3166du;
    m[4] = 0x3afbe4b1u; m[5] = 0x4c44df97u; m[6] = 0x4aac2739u; m[7] = 0x249e850au;
}
UF_HD void mid_nonce(uint32_t m[8]) {
    m[0] = 0x46615b35u; m[1] = 0xf4bfbff7u; m[2] = 0x9f8dc671u; m[3] = 0x83627ab3u;
    m[4] = 0x60217180u; m[5] = 0x57358661u; m[6] = 0x21a29e54u; m[7] = 0x68b07b4cu;
}
UF_HD void mid_challenge(uint32_t m[8]) {
    m[0] = 0x9cecba11u; m[1] = 0x23925381u; m[2] = 0x11679112u; m[3] = 0xd1627e0fu;
    m[4] = 0x97c87550u; m[5] = 0x003cc765u; m[6] = 0x90f61164u; m[7] = 0x33e9b66au;
}

// k*G through the generator tables: GLV split, two UF_GWIN-bit Booth streams.
template <class GT>
UF_HDI void gen_mul(Jac& R, const Sc& k, const GT& gt) {
    GlvSplit s;
    glv_split(s, k);
    GDigit d1[kNWG], d2[kNWG];
    booth_recode<kWG, kNWG>(d1, s.k1);
    booth_recode<kWG, kNWG>(d2, s.k2);
    jac_set_inf(R);
    UF_NOUNROLL
    for (int i = kNWG - 1; i >= 0; --i) {
        if (i != kNWG - 1) jac_dbl_n(R, kWG);
        add_gtab(R, gt, d1[i], s.neg1, 0);
        add_gtab(R, gt, d2[i], s.neg2, 1);
    }
}

UF_HD bool sc_from_be_strict_nonzero(Sc& r, const uint8_t* b) {
    be32_to_limbs(r.v, b);
    return !sc_is_zero(r) && limbs_lt_n(r.v);
}

// RFC 6979 nonce, HMAC-SHA256, h1 = the raw message hash (as the reference).
UF_HDI void rfc6979_nonce(Sc& k, const uint8_t x[32], const uint8_t msg[32]) {
    uint8_t V[32], K[32], buf[97];
    for (int i = 0; i < 32; ++i) { V[i] = 1; K[i] = 0; }
    for (int i = 0; i < 32; ++i) { buf[i] = V[i]; buf[33 + i] = x[i]; buf[65 + i] = msg[i]; }
    buf[32] = 0;
    hmac_sha256_k32(K, K, buf, 97);
    hmac_sha256_k32(V, K, V, 32);
    for (int i = 0; i < 32; ++i) buf[i] = V[i];
    buf[32] = 1;
    hmac_sha256_k32(K, K, buf, 97);
    hmac_sha256_k32(V, K, V, 32);
    for (int it = 0; it < 64; ++it) {
        hmac_sha256_k32(V, K, V, 32);
        if (sc_from_be_strict_nonzero(k, V)) return;
        uint8_t b33[33];
        for (int i = 0; i < 32; ++i) b33[i] = V[i];
        b33[32] = 0;
        hmac_sha256_k32(K, K, b33, 33);
        hmac_sha256_k32(V, K, V, 32);
    }
}

// Returns false for an invalid key.  pub33 / sig64 as the reference's ABI.
template <class GT>
UF_HDI bool ecdsa_sign_one(uint8_t pub33[33], uint8_t sig64[64], const uint8_t msg[32], const uint8_t sk[32],
                           const GT& gt) {
    Sc d, k, z, r, s, ki, t;
    if (!sc_from_be_strict_nonzero(d, sk)) return false;
    Jac P;
    Aff A;
    gen_mul(P, d, gt);
    jac_to_aff(A, P);
    pub33[0] = (uint8_t)(0x02 | (A.y.v[0] & 1u));
    limbs_to_be32(pub33 + 1, A.x.v);
    rfc6979_nonce(k, sk, msg);
    gen_mul(P, k, gt);
    jac_to_aff(A, P);
    for (int i = 0; i < 8; ++i) r.v[i] = A.x.v[i];
    sc_reduce_once(r);
    if (sc_is_zero(r)) return false;
    be32_to_limbs(z.v, msg);
    sc_reduce_once(z);
    sc_inv(ki, k);
    sc_mul(t, r, d);
    sc_add(t, t, z);
    sc_mul(s, ki, t);
    if (sc_is_zero(s)) return false;
    if (!sc_is_low(s.v)) sc_neg(s, s);
    limbs_to_be32(sig64, r.v);
    limbs_to_be32(sig64 + 32, s.v);
    return true;
}

template <class GT>
UF_HDI bool schnorr_sign_one(uint8_t xonly32[32], uint8_t sig64[64], const uint8_t msg[32], const uint8_t sk[32],
                             const uint8_t aux[32], const GT& gt) {
    Sc d, k, e, t, s;
    if (!sc_from_be_strict_nonzero(d, sk)) return false;
    Jac P;
    Aff A;
    gen_mul(P, d, gt);
    jac_to_aff(A, P);
    if (A.y.v[0] & 1u) sc_neg(d, d);
    uint8_t px[32], db[32], ah[32], buf[96], h[32];
    uint32_t mid[8];
    limbs_to_be32(px, A.x.v);
    limbs_to_be32(db, d.v);
    mid_aux(mid);
    tagged_from_mid(ah, mid, aux, 32);
    for (int i = 0; i < 32; ++i) { buf[i] = db[i] ^ ah[i]; buf[32 + i] = px[i]; buf[64 + i] = msg[i]; }
    mid_nonce(mid);
    tagged_from_mid(h, mid, buf, 96);
    be32_to_limbs(k.v, h);
    sc_reduce_once(k);
    if (sc_is_zero(k)) return false;
    gen_mul(P, k, gt);
    jac_to_aff(A, P);
    if (A.y.v[0] & 1u) sc_neg(k, k);
    uint8_t rx[32];
    limbs_to_be32(rx, A.x.v);
    for (int i = 0; i < 32; ++i) { buf[i] = rx[i]; buf[32 + i] = px[i]; buf[64 + i] = msg[i]; }
    mid_challenge(mid);
    tagged_from_mid(h, mid, buf, 96);
    be32_to_limbs(e.v, h);
    sc_reduce_once(e);
    sc_mul(t, e, d);
    sc_add(s, k, t);
    for (int i = 0; i < 32; ++i) { sig64[i] = rx[i]; xonly32[i] = px[i]; }
    limbs_to_be32(sig64 + 32, s.v);
    return true;
}

}  // namespace uf
