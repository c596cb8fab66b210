// Support kernels of the verify path: generator-table set-up, the arithmetic
// probes used by the tests, and the IMAD issue-rate probe.  The verify kernels
// themselves are in kernels_verify.cu.
#include "kernels.h"
#include "verify.cuh"
#include "dev_tables.cuh"

namespace uf {

// ---------------------------------------------------------------- G tables --
// entry t < half: (t+1)*G ; t >= half: (t-half+1)*lambda*G = (beta x, y),
// half = 2^(w-1) for w-bit windows
__global__ void k_gtable_init(uint4* out, int half) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * half) return;
    const int m = (t & (half - 1)) + 1;
    Aff G;
    gen_point(G);
    Jac acc;
    jac_set_inf(acc);
    for (int b = 31 - __clz(m); b >= 0; --b) {     // left-to-right double and add
        jac_dbl(acc);
        if ((m >> b) & 1) jac_add_aff(acc, G.x, G.y);
    }
    Aff A;
    jac_to_aff(A, acc);
    if (t >= half) {
        Fe beta;
        fe_beta(beta);
        fe_mul(A.x, A.x, beta);
        fe_normalize(A.x);
    }
    uint4* q = out + 4 * t;
    q[0] = make_uint4(A.x.v[0], A.x.v[1], A.x.v[2], A.x.v[3]);
    q[1] = make_uint4(A.x.v[4], A.x.v[5], A.x.v[6], A.x.v[7]);
    q[2] = make_uint4(A.y.v[0], A.y.v[1], A.y.v[2], A.y.v[3]);
    q[3] = make_uint4(A.y.v[4], A.y.v[5], A.y.v[6], A.y.v[7]);
}

cudaError_t launch_gtable_init_w(void* d_gtab, int wbits, cudaStream_t s) {
    const int half = 1 << (wbits - 1);
    k_gtable_init<<<(2 * half + 255) / 256, 256, 0, s>>>(reinterpret_cast<uint4*>(d_gtab), half);
    return cudaGetLastError();
}

cudaError_t launch_gtable_init(void* d_gtab, cudaStream_t s) { return launch_gtable_init_w(d_gtab, UF_GWIN, s); }

// ---------------------------------------------------------- diagnostics --
// op: 1 fe_mul(64->32) 2 fe_sqr(32->32) 3 fe_inv(32->32) 4 fe_sqrt(32->33)
//     5 sc_mul(64->32) 6 sc_inv(32->32) 7 glv(32->34) 8 gen_mul(32->64)
//     9 dual_mul(96->65) 10 challenge(96->32)
__device__ __forceinline__ void diag_io(uint32_t op, int& in_sz, int& out_sz) {
    switch (op) {
        case 1: in_sz = 64; out_sz = 32; break;
        case 2: case 3: case 6: in_sz = 32; out_sz = 32; break;
        case 4: in_sz = 32; out_sz = 33; break;
        case 5: in_sz = 64; out_sz = 32; break;
        case 7: in_sz = 32; out_sz = 34; break;
        case 8: in_sz = 32; out_sz = 64; break;
        case 9: in_sz = 96; out_sz = 65; break;
        case 10: in_sz = 96; out_sz = 32; break;
        default: in_sz = 0; out_sz = 0; break;
    }
}

__global__ void __launch_bounds__(kVerifyThreads)
k_diag(uint32_t op, const uint8_t* __restrict__ in, uint32_t n, uint8_t* __restrict__ out, const uint4* __restrict__ gt) {
    extern __shared__ uint4 smem_tab[];
    const SmemTab tab{smem_tab + threadIdx.x, blockDim.x};
    const GlobalGT g{gt};
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int isz, osz;
    diag_io(op, isz, osz);
    const uint8_t* a = in + (size_t)isz * i;
    uint8_t* o = out + (size_t)osz * i;
    Fe x, y, r;
    Sc sx, sy, sr;
    switch (op) {
        case 1: be32_to_limbs(x.v, a); be32_to_limbs(y.v, a + 32); fe_mul(r, x, y); fe_normalize(r); limbs_to_be32(o, r.v); break;
        case 2: be32_to_limbs(x.v, a); fe_sqr(r, x); fe_normalize(r); limbs_to_be32(o, r.v); break;
        case 3: be32_to_limbs(x.v, a); fe_inv(r, x); fe_normalize(r); limbs_to_be32(o, r.v); break;
        case 4: {
            be32_to_limbs(x.v, a);
            const bool ok = fe_sqrt(r, x);
            fe_normalize(r);
            o[0] = ok;
            limbs_to_be32(o + 1, r.v);
            break;
        }
        case 5: be32_to_limbs(sx.v, a); be32_to_limbs(sy.v, a + 32); sc_mul(sr, sx, sy); limbs_to_be32(o, sr.v); break;
        case 6: be32_to_limbs(sx.v, a); sc_inv(sr, sx); limbs_to_be32(o, sr.v); break;
        case 7: {
            be32_to_limbs(sx.v, a);
            GlvSplit gs;
            glv_split(gs, sx);
            uint32_t t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            uint8_t buf[32];
            for (int k = 0; k < 4; ++k) t[k] = gs.k1[k];
            limbs_to_be32(buf, t);
            for (int k = 0; k < 16; ++k) o[k] = buf[16 + k];
            for (int k = 0; k < 4; ++k) t[k] = gs.k2[k];
            limbs_to_be32(buf, t);
            for (int k = 0; k < 16; ++k) o[16 + k] = buf[16 + k];
            o[32] = gs.neg1;
            o[33] = gs.neg2;
            break;
        }
        case 8: case 9: {
            Sc sa, sb;
            Aff P;
            if (op == 8) {
                be32_to_limbs(sa.v, a);
                sc_reduce_once(sa);
                for (int k = 0; k < 8; ++k) sb.v[k] = 0;
                gen_point(P);
            } else {
                be32_to_limbs(sa.v, a);
                be32_to_limbs(P.x.v, a + 32);
                be32_to_limbs(sb.v, a + 64);
                sc_reduce_once(sa);
                sc_reduce_once(sb);
                if (!lift_x_parity(P.y, P.x, false)) { o[0] = 2; break; }
            }
            Jac R;
            dual_mul(R, sa, P.x, P.y, sb, tab, g);
            Aff A;
            const bool fin = jac_to_aff(A, R);
            if (op == 8) {
                if (!fin) { for (int k = 0; k < 64; ++k) o[k] = 0; break; }
                limbs_to_be32(o, A.x.v);
                limbs_to_be32(o + 32, A.y.v);
            } else {
                o[0] = fin;
                if (!fin) { for (int k = 1; k < 65; ++k) o[k] = 0; break; }
                limbs_to_be32(o + 1, A.x.v);
                limbs_to_be32(o + 33, A.y.v);
            }
            break;
        }
        case 10: {
            uint32_t rw[8], pw[8], mw[8], h[8];
            for (int k = 0; k < 8; ++k) {
                rw[k] = ((uint32_t)a[4 * k] << 24) | ((uint32_t)a[4 * k + 1] << 16) | ((uint32_t)a[4 * k + 2] << 8) | a[4 * k + 3];
                pw[k] = ((uint32_t)a[32 + 4 * k] << 24) | ((uint32_t)a[33 + 4 * k] << 16) | ((uint32_t)a[34 + 4 * k] << 8) | a[35 + 4 * k];
                mw[k] = ((uint32_t)a[64 + 4 * k] << 24) | ((uint32_t)a[65 + 4 * k] << 16) | ((uint32_t)a[66 + 4 * k] << 8) | a[67 + 4 * k];
            }
            bip340_challenge(h, rw, pw, mw);
            for (int k = 0; k < 8; ++k) {
                o[4 * k] = (uint8_t)(h[k] >> 24); o[4 * k + 1] = (uint8_t)(h[k] >> 16);
                o[4 * k + 2] = (uint8_t)(h[k] >> 8); o[4 * k + 3] = (uint8_t)h[k];
            }
            break;
        }
        default: break;
    }
}

cudaError_t launch_diag(uint32_t op, const uint8_t* in, uint32_t n, uint8_t* out, const void* d_gtab,
                        cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t smem = kVerifyThreads * kVerifySmemPerThread;
    cudaError_t e = cudaFuncSetAttribute(k_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_diag<<<(n + kVerifyThreads - 1) / kVerifyThreads, kVerifyThreads, smem, s>>>(
        op, in, n, out, reinterpret_cast<const uint4*>(d_gtab));
    return cudaGetLastError();
}

// ----------------------------------------------------- IMAD issue probe --
__global__ void k_imad_peak(uint32_t* sink, int iters) {
    uint32_t a[16];
    const uint32_t m = 0x9E3779B9u ^ threadIdx.x;
    const uint32_t c = 0x7F4A7C15u + blockIdx.x;
#pragma unroll
    for (int j = 0; j < 16; ++j) a[j] = threadIdx.x * 16u + j;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int j = 0; j < 16; ++j) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[j]) : "r"(m), "r"(c));
    }
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) acc ^= a[j];
    if (acc == 0x12345678u) sink[blockIdx.x] = acc;   // practically never: keeps the loop alive
}

cudaError_t launch_imad_peak(uint32_t* d_sink, int blocks, int threads, int iters, cudaStream_t s) {
    k_imad_peak<<<blocks, threads, 0, s>>>(d_sink, iters);
    return cudaGetLastError();
}

}  // namespace uf
