/*
 * secp_oracle.c -- CPU ORACLE for batch ECDSA / BIP-340 signature verification.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * verify path of ultrafastsecp256k1_b200.  Only tests/, the smoke check in
 * __graft_entry__.py and the cpu_baseline leg of bench.py may load it.  The
 * product library never links, loads or falls back to it.
 *
 * It is a plain-C restatement (simple, canonical, not fast) of the
 * reference's CPU verify semantics, UltrafastSecp256k1 v4.5.0:
 *
 *   ECDSA  ufsecp_ecdsa_verify          src/cpu/src/impl/ufsecp_ecdsa.cpp:244-272
 *          strict compact parse         src/cpu/src/ecdsa.cpp:94-102
 *          low-S rule (BIP-62)          src/cpu/src/impl/ufsecp_ecdsa.cpp:259-262,
 *                                       src/cpu/src/ecdsa.cpp:114-124
 *          pubkey parse (33 B)          src/cpu/src/ecdsa.cpp:891-906
 *          verify equation              src/cpu/src/ecdsa.cpp:929-951
 *          x-coordinate check (+r+n)    src/cpu/src/ecdsa.cpp:764-848
 *   BIP340 ufsecp_schnorr_verify        src/cpu/src/impl/ufsecp_ecdsa.cpp:992-1022
 *          strict parse r<p, 0<s<n      src/cpu/src/schnorr.cpp:355-371
 *          lift_x (x<p, even y)         src/cpu/src/schnorr.cpp:50-117, :275-301
 *          challenge hash               src/cpu/src/schnorr.cpp:190-199
 *          verify equation / checks     src/cpu/src/schnorr.cpp:542-612
 *   Signers used to make test corpora:
 *          RFC 6979 nonce               src/cpu/src/ecdsa.cpp:335-429
 *          ECDSA sign (low-S)           src/cpu/src/ecdsa.cpp:640-700, src/cpu/src/ct_sign.cpp:40-75
 *          BIP-340 sign                 src/cpu/src/schnorr.cpp:420-530 (BIP-340 "Default Signing")
 *
 * Parity of this restatement is pinned against the reference library itself
 * (compiled from the reference sources into oracle/_ref/ by oracle/Makefile)
 * and against the BIP-340 / Wycheproof vectors committed in tests/golden/.
 *
 * Representation: 256-bit integers as 4 x uint64 little-endian limbs; every
 * field / scalar value is kept fully reduced (canonical).  Points are
 * Jacobian with an explicit infinity flag and complete addition.
 */
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <pthread.h>
#include <unistd.h>

typedef unsigned __int128 u128;
typedef struct { uint64_t d[4]; } u256;

static const u256 FP = {{0xFFFFFFFEFFFFFC2FULL, 0xFFFFFFFFFFFFFFFFULL,
                         0xFFFFFFFFFFFFFFFFULL, 0xFFFFFFFFFFFFFFFFULL}};
static const u256 FN = {{0xBFD25E8CD0364141ULL, 0xBAAEDCE6AF48A03BULL,
                         0xFFFFFFFFFFFFFFFEULL, 0xFFFFFFFFFFFFFFFFULL}};
static const u256 HALF_N = {{0xDFE92F46681B20A0ULL, 0x5D576E7357A4501DULL,
                             0xFFFFFFFFFFFFFFFFULL, 0x7FFFFFFFFFFFFFFFULL}};
static const u256 GX = {{0x59F2815B16F81798ULL, 0x029BFCDB2DCE28D9ULL,
                         0x55A06295CE870B07ULL, 0x79BE667EF9DCBBACULL}};
static const u256 GY = {{0x9C47D08FFB10D4B8ULL, 0xFD17B448A6855419ULL,
                         0x5DA4FBFC0E1108A8ULL, 0x483ADA7726A3C465ULL}};

/* ---------------------------------------------------------------- u256 -- */

static int u256_cmp(const u256 *a, const u256 *b) {
    for (int i = 3; i >= 0; --i) {
        if (a->d[i] < b->d[i]) return -1;
        if (a->d[i] > b->d[i]) return 1;
    }
    return 0;
}
static int u256_is_zero(const u256 *a) { return (a->d[0] | a->d[1] | a->d[2] | a->d[3]) == 0; }
static uint64_t u256_add(u256 *r, const u256 *a, const u256 *b) {
    u128 c = 0;
    for (int i = 0; i < 4; ++i) { c += (u128)a->d[i] + b->d[i]; r->d[i] = (uint64_t)c; c >>= 64; }
    return (uint64_t)c;
}
static uint64_t u256_sub(u256 *r, const u256 *a, const u256 *b) {
    uint64_t br = 0;
    for (int i = 0; i < 4; ++i) {
        uint64_t ai = a->d[i], bi = b->d[i];
        uint64_t t = ai - bi - br;
        br = (ai < bi) || (ai == bi && br) ? 1 : 0;
        r->d[i] = t;
    }
    return br;
}
static void u256_from_be(u256 *r, const uint8_t b[32]) {
    for (int i = 0; i < 4; ++i) {
        uint64_t v = 0;
        for (int j = 0; j < 8; ++j) v = (v << 8) | b[(3 - i) * 8 + j];
        r->d[i] = v;
    }
}
static void u256_to_be(uint8_t b[32], const u256 *a) {
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 8; ++j) b[(3 - i) * 8 + j] = (uint8_t)(a->d[i] >> (56 - 8 * j));
}
static void mul_4x4(uint64_t t[8], const u256 *a, const u256 *b) {
    memset(t, 0, 8 * sizeof(uint64_t));
    for (int i = 0; i < 4; ++i) {
        u128 c = 0;
        for (int j = 0; j < 4; ++j) {
            c += (u128)a->d[i] * b->d[j] + t[i + j];
            t[i + j] = (uint64_t)c;
            c >>= 64;
        }
        t[i + 4] = (uint64_t)c;
    }
}

/* ------------------------------------------------- field mod p (canonical) -- */
/* p = 2^256 - 2^32 - 977; 2^256 = K (mod p), K = 0x1000003D1.
 * Reference: src/cpu/src/field.cpp (4x64 mul + K-fold reduction). */

static void fe_norm(u256 *a) { if (u256_cmp(a, &FP) >= 0) u256_sub(a, a, &FP); }
static void fe_add(u256 *r, const u256 *a, const u256 *b) {
    uint64_t c = u256_add(r, a, b);
    if (c || u256_cmp(r, &FP) >= 0) u256_sub(r, r, &FP);
}
static void fe_sub(u256 *r, const u256 *a, const u256 *b) {
    if (u256_sub(r, a, b)) u256_add(r, r, &FP);
}
static void fe_neg(u256 *r, const u256 *a) {
    u256 z = {{0, 0, 0, 0}};
    fe_sub(r, &z, a);
}
static void fe_mul(u256 *r, const u256 *a, const u256 *b) {
    uint64_t t[8];
    mul_4x4(t, a, b);
    const uint64_t K = 0x1000003D1ULL;
    /* fold t[4..7] * K into t[0..3] */
    uint64_t s[5];
    u128 c = 0;
    for (int i = 0; i < 4; ++i) { c += (u128)t[4 + i] * K + t[i]; s[i] = (uint64_t)c; c >>= 64; }
    s[4] = (uint64_t)c;
    /* fold s[4] * K */
    c = (u128)s[4] * K + s[0]; s[0] = (uint64_t)c; c >>= 64;
    for (int i = 1; i < 4; ++i) { c += s[i]; s[i] = (uint64_t)c; c >>= 64; }
    if (c) { /* wrapped past 2^256 again: add K once more */
        c = (u128)s[0] + K; s[0] = (uint64_t)c; c >>= 64;
        for (int i = 1; i < 4; ++i) { c += s[i]; s[i] = (uint64_t)c; c >>= 64; }
    }
    memcpy(r->d, s, 32);
    fe_norm(r);
}
static void fe_sqr(u256 *r, const u256 *a) { fe_mul(r, a, a); }
static void fe_pow(u256 *r, const u256 *a, const u256 *e) {
    u256 acc = {{1, 0, 0, 0}}, base = *a;
    for (int i = 255; i >= 0; --i) {
        fe_sqr(&acc, &acc);
        if ((e->d[i >> 6] >> (i & 63)) & 1) fe_mul(&acc, &acc, &base);
    }
    *r = acc;
}
static void fe_inv(u256 *r, const u256 *a) {
    u256 e = FP; e.d[0] -= 2;              /* p - 2 */
    fe_pow(r, a, &e);
}
/* sqrt via a^((p+1)/4); returns 1 iff the result squares back to a. */
static int fe_sqrt(u256 *r, const u256 *a) {
    u256 e = {{0xFFFFFFFFBFFFFF0CULL, 0xFFFFFFFFFFFFFFFFULL,
               0xFFFFFFFFFFFFFFFFULL, 0x3FFFFFFFFFFFFFFFULL}};
    u256 y, chk;
    fe_pow(&y, a, &e);
    fe_sqr(&chk, &y);
    *r = y;
    return u256_cmp(&chk, a) == 0;
}

/* ------------------------------------------------ scalar mod n (canonical) -- */
/* Reference: src/cpu/src/scalar.cpp (Scalar::from_bytes reduces mod n,
 * parse_bytes_strict[_nonzero] rejects >= n [and 0]). */

static void sc_reduce_once(u256 *a) { if (u256_cmp(a, &FN) >= 0) u256_sub(a, a, &FN); }
static void sc_add(u256 *r, const u256 *a, const u256 *b) {
    uint64_t c = u256_add(r, a, b);
    if (c || u256_cmp(r, &FN) >= 0) u256_sub(r, r, &FN);
}
static void sc_neg(u256 *r, const u256 *a) {
    if (u256_is_zero(a)) { *r = *a; return; }
    u256_sub(r, &FN, a);
}
/* 512-bit -> mod n by folding with C = 2^256 - n (129 bits). */
static void sc_reduce512(u256 *r, const uint64_t t_in[8]) {
    static const uint64_t C[3] = {0x402DA1732FC9BEBFULL, 0x4551231950B75FC4ULL, 0x1ULL};
    uint64_t t[8];
    memcpy(t, t_in, sizeof t);
    for (int round = 0; round < 4; ++round) {
        if ((t[4] | t[5] | t[6] | t[7]) == 0) break;
        uint64_t hi[4] = {t[4], t[5], t[6], t[7]};
        uint64_t acc[8] = {t[0], t[1], t[2], t[3], 0, 0, 0, 0};
        for (int i = 0; i < 4; ++i) {
            u128 c = 0;
            for (int j = 0; j < 3; ++j) {
                c += (u128)hi[i] * C[j] + acc[i + j];
                acc[i + j] = (uint64_t)c;
                c >>= 64;
            }
            for (int k = i + 3; k < 8 && c; ++k) { c += acc[k]; acc[k] = (uint64_t)c; c >>= 64; }
        }
        memcpy(t, acc, sizeof t);
    }
    u256 v = {{t[0], t[1], t[2], t[3]}};
    sc_reduce_once(&v);
    sc_reduce_once(&v);
    *r = v;
}
static void sc_mul(u256 *r, const u256 *a, const u256 *b) {
    uint64_t t[8];
    mul_4x4(t, a, b);
    sc_reduce512(r, t);
}
static void sc_inv(u256 *r, const u256 *a) {
    u256 e = FN; e.d[0] -= 2;              /* n - 2 */
    u256 acc = {{1, 0, 0, 0}}, base = *a;
    for (int i = 255; i >= 0; --i) {
        sc_mul(&acc, &acc, &acc);
        if ((e.d[i >> 6] >> (i & 63)) & 1) sc_mul(&acc, &acc, &base);
    }
    *r = acc;
}
static void sc_from_be_reduce(u256 *r, const uint8_t b[32]) {
    u256_from_be(r, b);
    sc_reduce_once(r);
}

/* ------------------------------------------------------------- points -- */

typedef struct { u256 x, y, z; int inf; } gej;   /* Jacobian, x = X/Z^2, y = Y/Z^3 */

static void gej_set_inf(gej *r) { memset(r, 0, sizeof *r); r->inf = 1; }
static void gej_set_affine(gej *r, const u256 *x, const u256 *y) {
    r->x = *x; r->y = *y; memset(&r->z, 0, sizeof r->z); r->z.d[0] = 1; r->inf = 0;
}
static void gej_double(gej *r, const gej *a) {
    if (a->inf || u256_is_zero(&a->y)) { gej_set_inf(r); return; }
    u256 A, B, C, D, E, F, t, X3, Y3, Z3;
    fe_sqr(&A, &a->x);                       /* A = X^2 */
    fe_sqr(&B, &a->y);                       /* B = Y^2 */
    fe_sqr(&C, &B);                          /* C = B^2 */
    fe_add(&t, &a->x, &B); fe_sqr(&t, &t);   /* (X+B)^2 */
    fe_sub(&t, &t, &A); fe_sub(&t, &t, &C);
    fe_add(&D, &t, &t);                      /* D = 2((X+B)^2 - A - C) */
    fe_add(&E, &A, &A); fe_add(&E, &E, &A);  /* E = 3A */
    fe_sqr(&F, &E);                          /* F = E^2 */
    fe_sub(&X3, &F, &D); fe_sub(&X3, &X3, &D);
    fe_sub(&t, &D, &X3); fe_mul(&Y3, &E, &t);
    u256 C8; fe_add(&C8, &C, &C); fe_add(&C8, &C8, &C8); fe_add(&C8, &C8, &C8);
    fe_sub(&Y3, &Y3, &C8);
    fe_mul(&Z3, &a->y, &a->z); fe_add(&Z3, &Z3, &Z3);
    r->x = X3; r->y = Y3; r->z = Z3; r->inf = 0;
}
/* complete Jacobian + Jacobian addition */
static void gej_add(gej *r, const gej *a, const gej *b) {
    if (a->inf) { *r = *b; return; }
    if (b->inf) { *r = *a; return; }
    u256 Z1Z1, Z2Z2, U1, U2, S1, S2, H, R, t;
    fe_sqr(&Z1Z1, &a->z); fe_sqr(&Z2Z2, &b->z);
    fe_mul(&U1, &a->x, &Z2Z2); fe_mul(&U2, &b->x, &Z1Z1);
    fe_mul(&S1, &a->y, &b->z); fe_mul(&S1, &S1, &Z2Z2);
    fe_mul(&S2, &b->y, &a->z); fe_mul(&S2, &S2, &Z1Z1);
    fe_sub(&H, &U2, &U1); fe_sub(&R, &S2, &S1);
    if (u256_is_zero(&H)) {
        if (u256_is_zero(&R)) { gej_double(r, a); return; }
        gej_set_inf(r); return;
    }
    u256 HH, HHH, V, X3, Y3, Z3;
    fe_sqr(&HH, &H); fe_mul(&HHH, &H, &HH); fe_mul(&V, &U1, &HH);
    fe_sqr(&X3, &R); fe_sub(&X3, &X3, &HHH); fe_sub(&X3, &X3, &V); fe_sub(&X3, &X3, &V);
    fe_sub(&t, &V, &X3); fe_mul(&Y3, &R, &t);
    fe_mul(&t, &S1, &HHH); fe_sub(&Y3, &Y3, &t);
    fe_mul(&Z3, &a->z, &b->z); fe_mul(&Z3, &Z3, &H);
    r->x = X3; r->y = Y3; r->z = Z3; r->inf = 0;
}
static int gej_to_affine(u256 *x, u256 *y, const gej *a) {
    if (a->inf) return 0;
    u256 zi, zi2, zi3;
    fe_inv(&zi, &a->z); fe_sqr(&zi2, &zi); fe_mul(&zi3, &zi2, &zi);
    fe_mul(x, &a->x, &zi2); fe_mul(y, &a->y, &zi3);
    return 1;
}
/* k*A with 4-bit fixed windows (k < 2^256, any value). */
static void gej_mul(gej *r, const gej *A, const u256 *k) {
    gej tab[16];
    gej_set_inf(&tab[0]);
    tab[1] = *A;
    for (int i = 2; i < 16; ++i) gej_add(&tab[i], &tab[i - 1], A);
    gej acc; gej_set_inf(&acc);
    for (int w = 63; w >= 0; --w) {
        for (int j = 0; j < 4; ++j) gej_double(&acc, &acc);
        unsigned d = (unsigned)(k->d[w >> 4] >> ((w & 15) * 4)) & 15u;
        if (d) gej_add(&acc, &acc, &tab[d]);
    }
    *r = acc;
}
/* u1*G + u2*Q (the reference computes this with a 4-stream GLV Strauss,
 * src/cpu/src/point.cpp:4079; the value is what matters here). */
static void dual_mul(gej *r, const u256 *u1, const u256 *u2, const gej *Q) {
    gej G, a, b;
    gej_set_affine(&G, &GX, &GY);
    gej_mul(&a, &G, u1);
    gej_mul(&b, Q, u2);
    gej_add(r, &a, &b);
}

/* ----------------------------------------------------------- SHA-256 -- */

typedef struct { uint32_t h[8]; uint8_t buf[64]; uint64_t len; } sha256_ctx;
static const uint32_t SHA_K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
    0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
    0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
    0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
    0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
    0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
#define ROR(x, n) (((x) >> (n)) | ((x) << (32 - (n))))
static void sha256_block(uint32_t h[8], const uint8_t p[64]) {
    uint32_t w[64];
    for (int i = 0; i < 16; ++i)
        w[i] = ((uint32_t)p[4 * i] << 24) | ((uint32_t)p[4 * i + 1] << 16) | ((uint32_t)p[4 * i + 2] << 8) | p[4 * i + 3];
    for (int i = 16; i < 64; ++i) {
        uint32_t s0 = ROR(w[i - 15], 7) ^ ROR(w[i - 15], 18) ^ (w[i - 15] >> 3);
        uint32_t s1 = ROR(w[i - 2], 17) ^ ROR(w[i - 2], 19) ^ (w[i - 2] >> 10);
        w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; ++i) {
        uint32_t S1 = ROR(e, 6) ^ ROR(e, 11) ^ ROR(e, 25);
        uint32_t ch = (e & f) ^ (~e & g);
        uint32_t t1 = hh + S1 + ch + SHA_K[i] + w[i];
        uint32_t S0 = ROR(a, 2) ^ ROR(a, 13) ^ ROR(a, 22);
        uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        uint32_t t2 = S0 + mj;
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}
static void sha256_init(sha256_ctx *c) {
    static const uint32_t iv[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                                   0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    memcpy(c->h, iv, sizeof iv); c->len = 0;
}
static void sha256_update(sha256_ctx *c, const uint8_t *p, size_t n) {
    while (n) {
        size_t off = (size_t)(c->len & 63), take = 64 - off;
        if (take > n) take = n;
        memcpy(c->buf + off, p, take);
        c->len += take; p += take; n -= take;
        if ((c->len & 63) == 0) sha256_block(c->h, c->buf);
    }
}
static void sha256_final(sha256_ctx *c, uint8_t out[32]) {
    uint64_t bits = c->len * 8;
    uint8_t pad = 0x80, z = 0;
    sha256_update(c, &pad, 1);
    while ((c->len & 63) != 56) sha256_update(c, &z, 1);
    uint8_t lb[8];
    for (int i = 0; i < 8; ++i) lb[i] = (uint8_t)(bits >> (56 - 8 * i));
    sha256_update(c, lb, 8);
    for (int i = 0; i < 8; ++i) {
        out[4 * i] = (uint8_t)(c->h[i] >> 24); out[4 * i + 1] = (uint8_t)(c->h[i] >> 16);
        out[4 * i + 2] = (uint8_t)(c->h[i] >> 8); out[4 * i + 3] = (uint8_t)c->h[i];
    }
}
void oracle_sha256(const uint8_t *p, size_t n, uint8_t out[32]) {
    sha256_ctx c; sha256_init(&c); sha256_update(&c, p, n); sha256_final(&c, out);
}
/* BIP-340 tagged hash: SHA256(SHA256(tag) || SHA256(tag) || data) */
static void tagged_hash(const char *tag, const uint8_t *data, size_t n, uint8_t out[32]) {
    uint8_t th[32];
    oracle_sha256((const uint8_t *)tag, strlen(tag), th);
    sha256_ctx c; sha256_init(&c);
    sha256_update(&c, th, 32); sha256_update(&c, th, 32); sha256_update(&c, data, n);
    sha256_final(&c, out);
}
static void hmac_sha256(const uint8_t key[32], const uint8_t *msg, size_t n, uint8_t out[32]) {
    uint8_t k[64], ih[32];
    memset(k, 0, 64); memcpy(k, key, 32);
    uint8_t ipad[64], opad[64];
    for (int i = 0; i < 64; ++i) { ipad[i] = k[i] ^ 0x36; opad[i] = k[i] ^ 0x5c; }
    sha256_ctx c;
    sha256_init(&c); sha256_update(&c, ipad, 64); sha256_update(&c, msg, n); sha256_final(&c, ih);
    sha256_init(&c); sha256_update(&c, opad, 64); sha256_update(&c, ih, 32); sha256_final(&c, out);
}

/* ------------------------------------------------------- key handling -- */

/* 33-byte SEC1 compressed pubkey -> point (src/cpu/src/ecdsa.cpp:891-906):
 * prefix 02/03, x < p strictly, y = sqrt(x^3+7) must exist, pick parity. */
static int pubkey33_parse(gej *P, const uint8_t pk[33]) {
    if (pk[0] != 0x02 && pk[0] != 0x03) return 0;
    u256 x, y, y2, seven = {{7, 0, 0, 0}};
    u256_from_be(&x, pk + 1);
    if (u256_cmp(&x, &FP) >= 0) return 0;
    fe_sqr(&y2, &x); fe_mul(&y2, &y2, &x); fe_add(&y2, &y2, &seven);
    if (!fe_sqrt(&y, &y2)) return 0;
    if ((int)(y.d[0] & 1) != (pk[0] == 0x03)) fe_neg(&y, &y);
    gej_set_affine(P, &x, &y);
    return 1;
}
/* BIP-340 lift_x (src/cpu/src/schnorr.cpp:50-117, x < p check :290-291). */
static int lift_x(gej *P, const uint8_t x32[32]) {
    u256 x, y, y2, seven = {{7, 0, 0, 0}};
    u256_from_be(&x, x32);
    if (u256_cmp(&x, &FP) >= 0) return 0;
    fe_sqr(&y2, &x); fe_mul(&y2, &y2, &x); fe_add(&y2, &y2, &seven);
    if (!fe_sqrt(&y, &y2)) return 0;
    if (y.d[0] & 1) fe_neg(&y, &y);
    gej_set_affine(P, &x, &y);
    return 1;
}

/* ------------------------------------------------------------ verify -- */

/* Returns 1 = valid, 0 = invalid (ufsecp_ecdsa_verify == UFSECP_OK). */
int oracle_ecdsa_verify(const uint8_t msg32[32], const uint8_t pub33[33], const uint8_t sig64[64]) {
    u256 r, s, z, w, u1, u2;
    u256_from_be(&r, sig64);
    u256_from_be(&s, sig64 + 32);
    /* strict: r, s in [1, n-1] */
    if (u256_is_zero(&r) || u256_cmp(&r, &FN) >= 0) return 0;
    if (u256_is_zero(&s) || u256_cmp(&s, &FN) >= 0) return 0;
    /* BIP-62 low-S: s <= n/2 */
    if (u256_cmp(&s, &HALF_N) > 0) return 0;
    gej Q;
    if (!pubkey33_parse(&Q, pub33)) return 0;
    sc_from_be_reduce(&z, msg32);
    sc_inv(&w, &s);
    sc_mul(&u1, &z, &w);
    sc_mul(&u2, &r, &w);
    gej R;
    dual_mul(&R, &u1, &u2, &Q);
    u256 x, y;
    if (!gej_to_affine(&x, &y, &R)) return 0;
    /* x-coordinate check: x == r, or x == r + n when r + n < p
     * (src/cpu/src/ecdsa.cpp:764-848); equivalently x mod n == r. */
    sc_reduce_once(&x);
    return u256_cmp(&x, &r) == 0;
}

/* Opaque libsecp-layout ECDSA signature (r then s, each 32 little-endian
 * bytes) as ufsecp_ecdsa_verify_opaque_rows reads it
 * (src/cpu/src/impl/ufsecp_ecdsa.cpp:105-117, :128-139, :180-189, :412-452):
 * r, s in [1, n-1] without reduction, s normalised to low-S (high-S accepted),
 * then the compact verify. */
int oracle_ecdsa_verify_opaque(const uint8_t msg32[32], const uint8_t pub33[33], const uint8_t opaque64[64]) {
    uint8_t be[64];
    for (int i = 0; i < 32; ++i) { be[i] = opaque64[31 - i]; be[32 + i] = opaque64[63 - i]; }
    u256 r, sv;
    u256_from_be(&r, be);
    u256_from_be(&sv, be + 32);
    if (u256_is_zero(&r) || u256_cmp(&r, &FN) >= 0) return 0;
    if (u256_is_zero(&sv) || u256_cmp(&sv, &FN) >= 0) return 0;
    if (u256_cmp(&sv, &HALF_N) > 0) {
        u256 t;
        u256_sub(&t, &FN, &sv);
        u256_to_be(be + 32, &t);
    }
    return oracle_ecdsa_verify(msg32, pub33, be);
}

/* Returns 1 = valid, 0 = invalid (ufsecp_schnorr_verify == UFSECP_OK). */
int oracle_schnorr_verify(const uint8_t msg32[32], const uint8_t xonly32[32], const uint8_t sig64[64]) {
    u256 r, s, e, ne;
    u256_from_be(&r, sig64);
    u256_from_be(&s, sig64 + 32);
    if (u256_cmp(&r, &FP) >= 0) return 0;                       /* r < p */
    if (u256_is_zero(&s) || u256_cmp(&s, &FN) >= 0) return 0;  /* 0 < s < n */
    gej P;
    if (!lift_x(&P, xonly32)) return 0;
    uint8_t buf[96], h[32];
    memcpy(buf, sig64, 32); memcpy(buf + 32, xonly32, 32); memcpy(buf + 64, msg32, 32);
    tagged_hash("BIP0340/challenge", buf, 96, h);
    sc_from_be_reduce(&e, h);
    sc_neg(&ne, &e);
    gej R;
    dual_mul(&R, &s, &ne, &P);
    u256 x, y;
    if (!gej_to_affine(&x, &y, &R)) return 0;                   /* R = infinity */
    if (y.d[0] & 1) return 0;                                   /* odd y */
    return u256_cmp(&x, &r) == 0;
}

/* ------------------------------------------------------------ signing -- */

static int sc_parse_strict_nonzero(u256 *r, const uint8_t b[32]) {
    u256_from_be(r, b);
    return !u256_is_zero(r) && u256_cmp(r, &FN) < 0;
}
static void gen_mul(gej *r, const u256 *k) {
    gej G; gej_set_affine(&G, &GX, &GY);
    gej_mul(r, &G, k);
}

/* Compressed pubkey of sk (ufsecp_pubkey_create). Returns 0 on bad key. */
int oracle_pubkey_create(const uint8_t sk32[32], uint8_t pub33[33]) {
    u256 d; gej P; u256 x, y;
    if (!sc_parse_strict_nonzero(&d, sk32)) return 0;
    gen_mul(&P, &d);
    gej_to_affine(&x, &y, &P);
    pub33[0] = (uint8_t)(0x02 | (y.d[0] & 1));
    u256_to_be(pub33 + 1, &x);
    return 1;
}
int oracle_pubkey_xonly(const uint8_t sk32[32], uint8_t x32[32]) {
    uint8_t pub[33];
    if (!oracle_pubkey_create(sk32, pub)) return 0;
    memcpy(x32, pub + 1, 32);
    return 1;
}

/* RFC 6979 nonce exactly as the reference derives it
 * (src/cpu/src/ecdsa.cpp:335-429: h1 = the raw 32-byte message hash). */
static void rfc6979_nonce(u256 *k, const u256 *d, const uint8_t msg32[32]) {
    uint8_t V[32], K[32], x[32], buf[97];
    memset(V, 0x01, 32); memset(K, 0x00, 32);
    u256_to_be(x, d);
    memcpy(buf, V, 32); buf[32] = 0x00; memcpy(buf + 33, x, 32); memcpy(buf + 65, msg32, 32);
    hmac_sha256(K, buf, 97, K);
    hmac_sha256(K, V, 32, V);
    memcpy(buf, V, 32); buf[32] = 0x01; memcpy(buf + 33, x, 32); memcpy(buf + 65, msg32, 32);
    hmac_sha256(K, buf, 97, K);
    hmac_sha256(K, V, 32, V);
    for (;;) {
        hmac_sha256(K, V, 32, V);
        if (sc_parse_strict_nonzero(k, V)) return;
        uint8_t b33[33]; memcpy(b33, V, 32); b33[32] = 0;
        hmac_sha256(K, b33, 33, K);
        hmac_sha256(K, V, 32, V);
    }
}

/* ECDSA sign (ufsecp_ecdsa_sign): RFC 6979 nonce, low-S normalised compact r||s. */
int oracle_ecdsa_sign(const uint8_t msg32[32], const uint8_t sk32[32], uint8_t sig64[64]) {
    u256 d, k, z, r, s, ki, t;
    if (!sc_parse_strict_nonzero(&d, sk32)) return 0;
    rfc6979_nonce(&k, &d, msg32);
    gej R; u256 x, y;
    gen_mul(&R, &k);
    gej_to_affine(&x, &y, &R);
    r = x; sc_reduce_once(&r);
    if (u256_is_zero(&r)) return 0;
    sc_from_be_reduce(&z, msg32);
    sc_inv(&ki, &k);
    sc_mul(&t, &r, &d);
    sc_add(&t, &t, &z);
    sc_mul(&s, &ki, &t);
    if (u256_is_zero(&s)) return 0;
    if (u256_cmp(&s, &HALF_N) > 0) sc_neg(&s, &s);
    u256_to_be(sig64, &r);
    u256_to_be(sig64 + 32, &s);
    return 1;
}

/* BIP-340 sign with aux_rand (ufsecp_schnorr_sign). */
int oracle_schnorr_sign(const uint8_t msg32[32], const uint8_t sk32[32], const uint8_t aux32[32],
                        uint8_t sig64[64]) {
    u256 d, k, e, s, t;
    if (!sc_parse_strict_nonzero(&d, sk32)) return 0;
    gej P; u256 px, py;
    gen_mul(&P, &d);
    gej_to_affine(&px, &py, &P);
    if (py.d[0] & 1) sc_neg(&d, &d);
    uint8_t pxb[32], db[32], ah[32], tb[32], buf[96], h[32];
    u256_to_be(pxb, &px);
    u256_to_be(db, &d);
    tagged_hash("BIP0340/aux", aux32, 32, ah);
    for (int i = 0; i < 32; ++i) tb[i] = db[i] ^ ah[i];
    memcpy(buf, tb, 32); memcpy(buf + 32, pxb, 32); memcpy(buf + 64, msg32, 32);
    tagged_hash("BIP0340/nonce", buf, 96, h);
    sc_from_be_reduce(&k, h);
    if (u256_is_zero(&k)) return 0;
    gej R; u256 rx, ry;
    gen_mul(&R, &k);
    gej_to_affine(&rx, &ry, &R);
    if (ry.d[0] & 1) sc_neg(&k, &k);
    uint8_t rxb[32];
    u256_to_be(rxb, &rx);
    memcpy(buf, rxb, 32); memcpy(buf + 32, pxb, 32); memcpy(buf + 64, msg32, 32);
    tagged_hash("BIP0340/challenge", buf, 96, h);
    sc_from_be_reduce(&e, h);
    sc_mul(&t, &e, &d);
    sc_add(&s, &k, &t);
    memcpy(sig64, rxb, 32);
    u256_to_be(sig64 + 32, &s);
    return 1;
}

/* ------------------------------------------------------- batch helpers -- */

/* Minimal static-partition parallel-for over pthreads (nthreads <= 0: all cores). */
typedef void (*item_fn)(void *ctx, long i);
typedef struct { item_fn fn; void *ctx; long begin, end; } range_job;
static void *range_worker(void *arg) {
    range_job *j = (range_job *)arg;
    for (long i = j->begin; i < j->end; ++i) j->fn(j->ctx, i);
    return NULL;
}
static int g_threads = 0;
void oracle_set_threads(int n) { g_threads = n; }
static void parallel_for(long n, item_fn fn, void *ctx) {
    long t = g_threads > 0 ? g_threads : sysconf(_SC_NPROCESSORS_ONLN);
    if (t < 1) t = 1;
    if (t > 256) t = 256;
    if (t > n) t = n > 0 ? n : 1;
    pthread_t th[256];
    range_job jobs[256];
    for (long k = 0; k < t; ++k) {
        jobs[k].fn = fn; jobs[k].ctx = ctx;
        jobs[k].begin = n * k / t; jobs[k].end = n * (k + 1) / t;
    }
    for (long k = 1; k < t; ++k) pthread_create(&th[k], NULL, range_worker, &jobs[k]);
    range_worker(&jobs[0]);
    for (long k = 1; k < t; ++k) pthread_join(th[k], NULL);
}

typedef struct { const uint8_t *msgs, *pubs, *sigs, *sks, *auxs; uint8_t *out, *pubs_out, *sigs_out; } batch_ctx;
static void ecdsa_verify_item(void *c, long i) {
    batch_ctx *b = (batch_ctx *)c;
    b->out[i] = (uint8_t)oracle_ecdsa_verify(b->msgs + 32 * i, b->pubs + 33 * i, b->sigs + 64 * i);
}
static void schnorr_verify_item(void *c, long i) {
    batch_ctx *b = (batch_ctx *)c;
    b->out[i] = (uint8_t)oracle_schnorr_verify(b->msgs + 32 * i, b->pubs + 32 * i, b->sigs + 64 * i);
}
static void ecdsa_sign_item(void *c, long i) {
    batch_ctx *b = (batch_ctx *)c;
    int a = oracle_pubkey_create(b->sks + 32 * i, b->pubs_out + 33 * i);
    int s = oracle_ecdsa_sign(b->msgs + 32 * i, b->sks + 32 * i, b->sigs_out + 64 * i);
    b->out[i] = (uint8_t)(a && s);
}
static void schnorr_sign_item(void *c, long i) {
    batch_ctx *b = (batch_ctx *)c;
    int a = oracle_pubkey_xonly(b->sks + 32 * i, b->pubs_out + 32 * i);
    int s = oracle_schnorr_sign(b->msgs + 32 * i, b->sks + 32 * i, b->auxs + 32 * i, b->sigs_out + 64 * i);
    b->out[i] = (uint8_t)(a && s);
}

void oracle_ecdsa_verify_batch(const uint8_t *msgs, const uint8_t *pubs, const uint8_t *sigs,
                               size_t n, uint8_t *out) {
    batch_ctx b = {msgs, pubs, sigs, NULL, NULL, out, NULL, NULL};
    parallel_for((long)n, ecdsa_verify_item, &b);
}
void oracle_schnorr_verify_batch(const uint8_t *msgs, const uint8_t *pubs, const uint8_t *sigs,
                                 size_t n, uint8_t *out) {
    batch_ctx b = {msgs, pubs, sigs, NULL, NULL, out, NULL, NULL};
    parallel_for((long)n, schnorr_verify_item, &b);
}
/* Per-item batch operations next to verify (the reference GPU's libbitcoin
 * bridge ops, src/gpu/src/gpu_backend_cuda.cu:748-803):
 * x-only key valid = x < p and lift_x succeeds; compressed key valid = prefix
 * 02/03, x < p, on the curve; BIP-341 commitment valid = lift_x(internal) +
 * (tweak mod n) G is finite with x == tweaked_x and y parity == parity. */
int oracle_xonly_validate(const uint8_t x32[32]) { gej P; return lift_x(&P, x32); }
int oracle_pubkey_validate(const uint8_t pub33[33]) { gej P; return pubkey33_parse(&P, pub33); }
int oracle_commitment_verify(const uint8_t ix[32], const uint8_t tw[32], const uint8_t tx[32], uint8_t parity) {
    gej P, T, Q;
    if (!lift_x(&P, ix)) return 0;
    u256 t, x, y, want;
    u256_from_be(&t, tw);
    sc_reduce_once(&t);
    gen_mul(&T, &t);
    gej_add(&Q, &T, &P);
    if (!gej_to_affine(&x, &y, &Q)) return 0;
    u256_from_be(&want, tx);
    return u256_cmp(&x, &want) == 0 && (int)(y.d[0] & 1) == (parity ? 1 : 0);
}
void oracle_ops_batch(int op, const uint8_t *a, const uint8_t *b, const uint8_t *c, const uint8_t *d, size_t n,
                      uint8_t *out) {
    for (size_t i = 0; i < n; ++i) {
        if (op == 0) out[i] = (uint8_t)oracle_xonly_validate(a + 32 * i);
        else if (op == 1) out[i] = (uint8_t)oracle_pubkey_validate(a + 33 * i);
        else out[i] = (uint8_t)oracle_commitment_verify(a + 32 * i, b + 32 * i, c + 32 * i, d[i]);
    }
}

/* sum k_i P_i as ufsecp_multi_scalar_mul (src/cpu/src/impl/ufsecp_taproot.cpp:957-991):
 * returns 0 and the compressed sum, 5 for a scalar >= n, 3 for an invalid
 * point (first bad item in order, scalar before point), 7 for infinity. */
int oracle_msm(const uint8_t *scalars, const uint8_t *points, size_t n, uint8_t out33[33]) {
    memset(out33, 0, 33);
    gej acc, P, T;
    gej_set_inf(&acc);
    for (size_t i = 0; i < n; ++i) {
        u256 k;
        u256_from_be(&k, scalars + 32 * i);
        if (u256_cmp(&k, &FN) >= 0) return 5;
        if (!pubkey33_parse(&P, points + 33 * i)) return 3;
    }
    for (size_t i = 0; i < n; ++i) {
        u256 k;
        u256_from_be(&k, scalars + 32 * i);
        pubkey33_parse(&P, points + 33 * i);
        gej_mul(&T, &P, &k);
        gej_add(&acc, &acc, &T);
    }
    u256 x, y;
    if (!gej_to_affine(&x, &y, &acc)) return 7;
    out33[0] = (uint8_t)(0x02 | (y.d[0] & 1));
    u256_to_be(out33 + 1, &x);
    return 0;
}

/* Opaque ECDSA rows [msg 32 | pubkey 33 | opaque sig 64 | tail], `stride` bytes apart. */
typedef struct { const uint8_t *rows; size_t stride; uint8_t *out; } rows_ctx;
static void ecdsa_opaque_item(void *c, long i) {
    rows_ctx *b = (rows_ctx *)c;
    const uint8_t *row = b->rows + (size_t)i * b->stride;
    b->out[i] = (uint8_t)oracle_ecdsa_verify_opaque(row, row + 32, row + 65);
}
void oracle_ecdsa_verify_opaque_rows(const uint8_t *rows, size_t stride, size_t n, uint8_t *out) {
    rows_ctx b = {rows, stride, out};
    parallel_for((long)n, ecdsa_opaque_item, &b);
}
/* Signs n items; ok[i] = 1 on success. */
void oracle_ecdsa_sign_batch(const uint8_t *msgs, const uint8_t *sks, size_t n,
                             uint8_t *pubs33, uint8_t *sigs, uint8_t *ok) {
    batch_ctx b = {msgs, NULL, NULL, sks, NULL, ok, pubs33, sigs};
    parallel_for((long)n, ecdsa_sign_item, &b);
}
void oracle_schnorr_sign_batch(const uint8_t *msgs, const uint8_t *sks, const uint8_t *auxs, size_t n,
                               uint8_t *xonly32, uint8_t *sigs, uint8_t *ok) {
    batch_ctx b = {msgs, NULL, NULL, sks, auxs, ok, xonly32, sigs};
    parallel_for((long)n, schnorr_sign_item, &b);
}

/* Arithmetic probes used by the tests to pin device building blocks. */
void oracle_fe_mul(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]) {
    u256 x, y, r; u256_from_be(&x, a); u256_from_be(&y, b);
    fe_norm(&x); fe_norm(&y); fe_mul(&r, &x, &y); u256_to_be(out, &r);
}
void oracle_fe_inv(const uint8_t a[32], uint8_t out[32]) {
    u256 x, r; u256_from_be(&x, a); fe_norm(&x); fe_inv(&r, &x); u256_to_be(out, &r);
}
void oracle_sc_inv(const uint8_t a[32], uint8_t out[32]) {
    u256 x, r; u256_from_be(&x, a); sc_reduce_once(&x); sc_inv(&r, &x); u256_to_be(out, &r);
}
void oracle_sc_mul(const uint8_t a[32], const uint8_t b[32], uint8_t out[32]) {
    u256 x, y, r; u256_from_be(&x, a); u256_from_be(&y, b);
    sc_reduce_once(&x); sc_reduce_once(&y); sc_mul(&r, &x, &y); u256_to_be(out, &r);
}
/* k*G affine (x, y) big-endian; returns 0 for k = 0 mod n. */
int oracle_gen_mul(const uint8_t k32[32], uint8_t x32[32], uint8_t y32[32]) {
    u256 k; gej R; u256 x, y;
    sc_from_be_reduce(&k, k32);
    gen_mul(&R, &k);
    if (!gej_to_affine(&x, &y, &R)) return 0;
    u256_to_be(x32, &x); u256_to_be(y32, &y);
    return 1;
}
