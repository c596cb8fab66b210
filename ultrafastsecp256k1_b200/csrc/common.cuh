// Shared helpers for the sm_100a verify path.
//
// Every arithmetic header in this directory is written as portable C++ with
// __host__ __device__ entry points.  The CUDA library compiles them for
// sm_100a; the test suite also compiles them with g++ into a host-side unit
// test harness (tests/native/), which is how the math is checked against the
// oracle without a GPU.  The shipped library never runs them on the host.
#pragma once
#include <stdint.h>

// Window width (bits) of the generator streams, library-wide: the per-context
// G / lambda G tables hold 2^(UF_GWIN-1) multiples each.  20-bit windows (one
// per five 4-bit P windows, 2 x 2^19 entries, 64 MB, served from the 126 MB
// L2): 14 table additions per verify, against 18 for 16-bit windows (4 MB),
// 22 for 12-bit ones (256 KB) and 34 for 8-bit ones (16 KB).
#ifndef UF_GWIN
#define UF_GWIN 20
#endif

#if defined(__CUDACC__)
#define UF_HD __host__ __device__ __forceinline__
#define UF_HDI __host__ __device__ inline
#else
#define UF_HD static inline
#define UF_HDI static inline
#endif

// Code-size control.  The verify kernel is long straight-line integer code;
// when every field operation is inlined into every point operation the hot
// loop no longer fits the instruction cache.  UF_FIELD_FN / UF_POINT_FN mark
// the field multiply/square and the point double/add as out-of-line
// subroutines in device code when the translation unit asks for it
// (UF_NOINLINE_FIELD / UF_NOINLINE_POINT); UF_COLD marks large routines that
// run once or twice per signature (inversion, square root) out of line always.
#if defined(__CUDACC__)
#define UF_NOINL __host__ __device__ __noinline__
#define UF_COLD static UF_NOINL
#if defined(UF_NOINLINE_FIELD)
#define UF_FIELD_FN static UF_NOINL
#else
#define UF_FIELD_FN UF_HD
#endif
#if defined(UF_NOINLINE_POINT)
#define UF_POINT_FN static UF_NOINL
#else
#define UF_POINT_FN UF_HD
#endif
#else
#define UF_COLD static inline
#define UF_FIELD_FN static inline
#define UF_POINT_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define UF_UNROLL _Pragma("unroll")
#define UF_NOUNROLL _Pragma("unroll 1")
#else
#define UF_UNROLL
#define UF_NOUNROLL
#endif

namespace uf {

UF_HD uint32_t lo32(uint64_t x) { return (uint32_t)x; }
UF_HD uint32_t hi32(uint64_t x) { return (uint32_t)(x >> 32); }

// number of trailing zero bits, x != 0
UF_HD int ctz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __ffs((int)x) - 1;
#else
    return __builtin_ctz(x);
#endif
}

UF_HD uint32_t bswap32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __byte_perm(x, 0, 0x0123);
#else
    return __builtin_bswap32(x);
#endif
}

// 32 big-endian bytes -> 8 little-endian 32-bit limbs.
UF_HD void be32_to_limbs(uint32_t v[8], const uint8_t* b) {
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        const uint8_t* p = b + 4 * (7 - i);
        v[i] = ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3];
    }
}

// Same, from 8 words loaded little-endian from a 4-byte aligned buffer.
UF_HD void words_be_to_limbs(uint32_t v[8], const uint32_t w[8]) {
    UF_UNROLL
    for (int i = 0; i < 8; ++i) v[i] = bswap32(w[7 - i]);
}

UF_HD void limbs_to_be32(uint8_t* b, const uint32_t v[8]) {
    UF_UNROLL
    for (int i = 0; i < 8; ++i) {
        uint8_t* p = b + 4 * (7 - i);
        p[0] = (uint8_t)(v[i] >> 24); p[1] = (uint8_t)(v[i] >> 16);
        p[2] = (uint8_t)(v[i] >> 8);  p[3] = (uint8_t)v[i];
    }
}

// a < b for 8-limb little-endian integers
UF_HD bool lt256(const uint32_t a[8], const uint32_t b[8]) {
    UF_UNROLL
    for (int i = 7; i >= 0; --i) {
        if (a[i] != b[i]) return a[i] < b[i];
    }
    return false;
}

UF_HD bool is_zero256(const uint32_t a[8]) {
    uint32_t acc = 0;
    UF_UNROLL
    for (int i = 0; i < 8; ++i) acc |= a[i];
    return acc == 0;
}

}  // namespace uf
