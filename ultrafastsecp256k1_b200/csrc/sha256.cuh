// SHA-256 compression (FIPS 180-4) and the BIP-340 challenge hash on device.
//
// Role in the reference: sha256_compress (src/cuda/include/ecdsa.cuh:57),
// tagged_hash_fast + BIP340_MIDSTATES (src/cuda/include/schnorr.cuh:55-82),
// CPU schnorr_challenge_scalar (src/cpu/src/schnorr.cpp:190-199) with
// g_challenge_midstate (src/cpu/include/secp256k1/tagged_hash.hpp:61).
//
// e = SHA256(SHA256(tag) || SHA256(tag) || R.x || P.x || m) mod n with
// tag = "BIP0340/challenge".  The first 64-byte block is constant, so the
// state after it (the midstate below, computed for this file) is the starting
// point; two compressions remain: (R.x || P.x) and (m || padding || 1280).
#pragma once
#include "common.cuh"

namespace uf {

UF_HD uint32_t rotr32(uint32_t x, int n) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_r(x, x, n);
#else
    return (x >> n) | (x << (32 - n));
#endif
}

#if defined(__CUDA_ARCH__)
__device__ __constant__ uint32_t UF_SHA_K[64] = {
#else
static const uint32_t UF_SHA_K[64] = {
#endif
    0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u, 0x923f82a4u, 0xab1c5ed5u,
    0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u, 0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u,
    0xe49b69c1u, 0xefbe4786u, 0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
    0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u, 0x06ca6351u, 0x14292967u,
    0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u, 0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u,
    0xa2bfe8a1u, 0xa81a664bu, 0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
    0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au, 0x5b9cca4fu, 0x682e6ff3u,
    0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u, 0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};

// One compression: h <- h + F(h, w); w = 16 big-endian message words.
UF_HD void sha256_compress(uint32_t h[8], const uint32_t win[16]) {
    uint32_t w[16];
    UF_UNROLL
    for (int i = 0; i < 16; ++i) w[i] = win[i];
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    UF_UNROLL
    for (int i = 0; i < 64; ++i) {
        uint32_t wi;
        if (i < 16) {
            wi = w[i];
        } else {
            const uint32_t w15 = w[(i - 15) & 15], w2 = w[(i - 2) & 15];
            const uint32_t s0 = rotr32(w15, 7) ^ rotr32(w15, 18) ^ (w15 >> 3);
            const uint32_t s1 = rotr32(w2, 17) ^ rotr32(w2, 19) ^ (w2 >> 10);
            wi = w[i & 15] + s0 + w[(i - 7) & 15] + s1;
            w[i & 15] = wi;
        }
        const uint32_t S1 = rotr32(e, 6) ^ rotr32(e, 11) ^ rotr32(e, 25);
        const uint32_t ch = (e & f) ^ (~e & g);
        const uint32_t t1 = hh + S1 + ch + UF_SHA_K[i] + wi;
        const uint32_t S0 = rotr32(a, 2) ^ rotr32(a, 13) ^ rotr32(a, 22);
        const uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        const uint32_t t2 = S0 + mj;
        hh = g; g = f; f = e; e = d + t1; d = c; c = b; b = a; a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
}

// BIP-340 challenge digest; inputs are the 32-byte big-endian strings as
// 8 big-endian words each.  Output: 8 big-endian digest words.
UF_HD void bip340_challenge(uint32_t out[8], const uint32_t rx_be[8], const uint32_t px_be[8],
                            const uint32_t m_be[8]) {
    uint32_t h[8] = {0x9cecba11u, 0x23925381u, 0x11679112u, 0xd1627e0fu,
                     0x97c87550u, 0x003cc765u, 0x90f61164u, 0x33e9b66au};
    uint32_t w[16];
    UF_UNROLL
    for (int i = 0; i < 8; ++i) { w[i] = rx_be[i]; w[8 + i] = px_be[i]; }
    sha256_compress(h, w);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) w[i] = m_be[i];
    w[8] = 0x80000000u;
    UF_UNROLL
    for (int i = 9; i < 15; ++i) w[i] = 0;
    w[15] = 1280;   // (64 + 96) bytes * 8
    sha256_compress(h, w);
    UF_UNROLL
    for (int i = 0; i < 8; ++i) out[i] = h[i];
}

}  // namespace uf
