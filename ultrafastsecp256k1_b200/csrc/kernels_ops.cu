// Per-item batch operations next to the verify path (the reference's
// libbitcoin-bridge batch ops, src/gpu/src/gpu_backend_cuda.cu:748-803 behind
// ufsecp_gpu_xonly_validate / _pubkey_validate / _commitment_verify /
// _tagged_hash / _tagged_hash_var, include/ufsecp/ufsecp_gpu.h:408-507),
// re-built on this library's field, point and SHA-256 code.  One item per
// thread, grid-stride.
#include "kernels.h"
#include "dev_tables.cuh"
#include "sign.cuh"

namespace uf {

namespace {

// x (big-endian bytes) < p and lift_x succeeds with the given parity.
__device__ __forceinline__ bool lift_bytes(const uint8_t* x32, bool odd, Fe& x, Fe& y) {
    be32_to_limbs(x.v, x32);
    if (!limbs_lt_p(x.v)) return false;
    return lift_x_parity(y, x, odd);
}

__global__ void __launch_bounds__(128)
k_xonly_validate(const uint8_t* __restrict__ keys, uint32_t n, uint8_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Fe x, y;
        out[i] = lift_bytes(keys + 32ull * i, false, x, y) ? 1 : 0;
    }
}

__global__ void __launch_bounds__(128)
k_pubkey_validate(const uint8_t* __restrict__ pubs, uint32_t n, uint8_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint8_t* p = pubs + 33ull * i;
        Fe x, y;
        out[i] = ((p[0] == 0x02 || p[0] == 0x03) && lift_bytes(p + 1, p[0] == 0x03, x, y)) ? 1 : 0;
    }
}

// BIP-341 tweak check: Q = lift_x(internal) + t G (t = tweak mod n); valid when
// Q is finite, x(Q) == tweaked_x and y(Q) has the claimed parity.
__global__ void __launch_bounds__(128)
k_commitment_verify(const uint8_t* __restrict__ ix, const uint8_t* __restrict__ tw,
                    const uint8_t* __restrict__ tx, const uint8_t* __restrict__ par, uint32_t n,
                    const uint4* __restrict__ gt, uint8_t* __restrict__ out) {
    const GlobalGT G{gt};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Fe px, py;
        if (!lift_bytes(ix + 32ull * i, false, px, py)) {
            out[i] = 0;
            continue;
        }
        Sc t;
        be32_to_limbs(t.v, tw + 32ull * i);
        sc_reduce_once(t);
        Jac Q;
        gen_mul(Q, t, G);
        jac_add_aff(Q, px, py);
        Aff q;
        if (!jac_to_aff(q, Q)) {
            out[i] = 0;
            continue;
        }
        uint32_t want[8];
        be32_to_limbs(want, tx + 32ull * i);
        bool ok = ((q.y.v[0] & 1u) != 0) == (par[i] != 0);
        for (int k = 0; k < 8; ++k) ok = ok && q.x.v[k] == want[k];
        out[i] = ok ? 1 : 0;
    }
}

// SHA-256 continuing from `mid` after 64 prefix bytes, over len bytes of msg
// (byte loads: rows need not be aligned).  Big-endian digest bytes to out.
__device__ void sha256_from_mid(const uint32_t mid[8], const uint8_t* msg, uint32_t len, uint8_t* out) {
    uint32_t h[8];
    for (int k = 0; k < 8; ++k) h[k] = mid[k];
    uint32_t w[16];
    uint32_t off = 0;
    for (; off + 64 <= len; off += 64) {
        for (int k = 0; k < 16; ++k) {
            const uint8_t* p = msg + off + 4 * k;
            w[k] = ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
        }
        sha256_compress(h, w);
    }
    // tail: remaining bytes, 0x80, zeros, 64-bit bit length of prefix + message
    const uint32_t rem = len - off;
    const uint64_t bits = (uint64_t)(len + 64) * 8;
    const int blocks = rem + 9 <= 64 ? 1 : 2;
    for (int b = 0; b < blocks; ++b) {
        for (int k = 0; k < 16; ++k) {
            uint32_t v = 0;
            for (int j = 0; j < 4; ++j) {
                const uint32_t pos = 64u * b + 4u * k + j;
                uint32_t byte;
                if (pos < rem) byte = msg[off + pos];
                else if (pos == rem) byte = 0x80;
                else if (pos >= 64u * blocks - 8) byte = (uint32_t)(bits >> (8 * (64u * blocks - 1 - pos))) & 0xFF;
                else byte = 0;
                v = (v << 8) | byte;
            }
            w[k] = v;
        }
        sha256_compress(h, w);
    }
    for (int k = 0; k < 8; ++k) {
        out[4 * k] = (uint8_t)(h[k] >> 24);
        out[4 * k + 1] = (uint8_t)(h[k] >> 16);
        out[4 * k + 2] = (uint8_t)(h[k] >> 8);
        out[4 * k + 3] = (uint8_t)h[k];
    }
}

struct Mid {
    uint32_t h[8];
};

// lens == nullptr: every message is fixed_len bytes.
__global__ void __launch_bounds__(128)
k_tagged_hash(Mid mid, const uint8_t* __restrict__ msgs, const uint32_t* __restrict__ lens, uint32_t fixed_len,
              uint32_t stride, uint32_t n, uint8_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t len = lens ? lens[i] : fixed_len;
        sha256_from_mid(mid.h, msgs + (uint64_t)stride * i, len, out + 32ull * i);
    }
}

// Field arithmetic exactly as the verify kernels compile it (this file is
// built with their flags: PTX carry chains, out-of-line multiply): per item
// a | b (any 256-bit values, i.e. weakly reduced) -> a*b, a^2, a+b, a-b, 4a,
// 8a, each normalized, big-endian.
__global__ void __launch_bounds__(128)
k_field_diag(const uint8_t* __restrict__ in, uint32_t n, uint8_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Fe a, b, r;
        be32_to_limbs(a.v, in + 64ull * i);
        be32_to_limbs(b.v, in + 64ull * i + 32);
        uint8_t* o = out + 192ull * i;
        fe_mul(r, a, b);
        fe_normalize(r);
        limbs_to_be32(o, r.v);
        fe_sqr(r, a);
        fe_normalize(r);
        limbs_to_be32(o + 32, r.v);
        fe_add(r, a, b);
        fe_normalize(r);
        limbs_to_be32(o + 64, r.v);
        fe_sub(r, a, b);
        fe_normalize(r);
        limbs_to_be32(o + 96, r.v);
        fe_mul_pow2<2>(r, a);
        fe_normalize(r);
        limbs_to_be32(o + 128, r.v);
        fe_mul_pow2<3>(r, a);
        fe_normalize(r);
        limbs_to_be32(o + 160, r.v);
    }
}

inline int grid_ops(uint32_t n, int sms) {
    const int need = (int)((n + 127) / 128);
    return need < sms * 8 ? need : sms * 8;
}

}  // namespace

cudaError_t launch_xonly_validate(const uint8_t* keys, uint32_t n, uint8_t* out, int sms, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_xonly_validate<<<grid_ops(n, sms), 128, 0, s>>>(keys, n, out);
    return cudaGetLastError();
}

cudaError_t launch_pubkey_validate(const uint8_t* pubs, uint32_t n, uint8_t* out, int sms, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_pubkey_validate<<<grid_ops(n, sms), 128, 0, s>>>(pubs, n, out);
    return cudaGetLastError();
}

cudaError_t launch_commitment_verify(const uint8_t* ix, const uint8_t* tw, const uint8_t* tx, const uint8_t* par,
                                     uint32_t n, const void* d_gtab, uint8_t* out, int sms, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_commitment_verify<<<grid_ops(n, sms), 128, 0, s>>>(ix, tw, tx, par, n, (const uint4*)d_gtab, out);
    return cudaGetLastError();
}

cudaError_t launch_field_diag(const uint8_t* in, uint32_t n, uint8_t* out, int sms, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    k_field_diag<<<grid_ops(n, sms), 128, 0, s>>>(in, n, out);
    return cudaGetLastError();
}

cudaError_t launch_tagged_hash(const uint8_t tag_hash[32], const uint8_t* msgs, const uint32_t* lens,
                               uint32_t fixed_len, uint32_t stride, uint32_t n, uint8_t* out, int sms,
                               cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    // midstate after the constant first block SHA256(tag) || SHA256(tag)
    Mid mid;
    sha256_iv(mid.h);
    uint32_t w[16];
    for (int k = 0; k < 8; ++k) {
        const uint8_t* p = tag_hash + 4 * k;
        w[k] = w[k + 8] = ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
    }
    sha256_compress(mid.h, w);
    k_tagged_hash<<<grid_ops(n, sms), 128, 0, s>>>(mid, msgs, lens, fixed_len, stride, n, out);
    return cudaGetLastError();
}

}  // namespace uf
