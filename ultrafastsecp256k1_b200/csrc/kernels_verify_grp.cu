// Per-signature verify kernels with block-wide batch inversion.
//
// The plain kernels (kernels_verify.cu) invert per thread: each BIP-340
// signature inverts its 1P..8P table's Z product and its result's Z, each
// ECDSA signature its table product and s.  Here those inversions are shared
// by the G threads of a block (grpinv.cuh: one inversion per block and site
// instead of one per warp).  The verdicts are those of ecdsa_verify_one /
// ecdsa_verify_opaque_one / schnorr_verify_one (verify.cuh) with the same
// checks in the same order; the computation is split into phases around the
// block-wide inversions, and every thread of the block takes every phase
// (a thread whose item failed a check, or has no item, carries the value one
// through the inversions).  The grid-stride loop advances whole blocks, so
// every thread reaches every barrier.  Compiled with the code generation of
// variant 4 (out-of-line field and point operations, PTX carry chains).
#include "kernels.h"
#include "verify.cuh"
#include "dev_tables.cuh"
#include "grpinv.cuh"

namespace uf {
namespace {

// kKind: 0 ECDSA (compact r || s, low-S), 1 BIP-340, 2 ECDSA (opaque
// little-endian r, s; high-S normalised).  G threads per block = the group.
template <int kKind, int G>
__global__ void __launch_bounds__(G, 384 / G)
k_verify_grp(const uint8_t* __restrict__ msgs, const uint8_t* __restrict__ pubs, const uint8_t* __restrict__ sigs,
             uint32_t n, const uint4* __restrict__ gt, uint8_t* __restrict__ out, int collect) {
    extern __shared__ uint4 smem[];
    const SmemTab tab{smem + threadIdx.x, G};
    uint32_t* gsh = reinterpret_cast<uint32_t*>(smem + (size_t)G * 4 * kPTab);
    const GlobalGT g{gt};
    for (uint32_t base = blockIdx.x * G; base < n; base += gridDim.x * G) {
        const uint32_t i = base + threadIdx.x;
        bool ok = i < n;
        uint32_t mw[8], sw[16];
        Fe px, py;
        Sc r, s;
        if (ok) {
            load_words8(mw, msgs + 32ull * i);
            load_words8(sw, sigs + 64ull * i);
            load_words8(sw + 8, sigs + 64ull * i + 32);
        }
        DualDigits d;
        if (kKind == 1) {
            // ---- BIP-340: parse, lift_x, challenge (schnorr_verify_one) ----
            uint32_t pw[8];
            if (ok) {
                load_words8(pw, pubs + 32ull * i);
                words_be_to_limbs(r.v, sw);
                words_be_to_limbs(s.v, sw + 8);
                ok = limbs_lt_p(r.v) && !sc_is_zero(s) && limbs_lt_n(s.v);
            }
            if (ok) {
                words_be_to_limbs(px.v, pw);
                ok = limbs_lt_p(px.v) && lift_x_parity(py, px, false);
            }
            if (ok) {
                uint32_t rbe[8], pbe[8], mbe[8], h[8];
                UF_UNROLL
                for (int k = 0; k < 8; ++k) {
                    rbe[k] = bswap32(sw[k]);
                    pbe[k] = bswap32(pw[k]);
                    mbe[k] = bswap32(mw[k]);
                }
                bip340_challenge(h, rbe, pbe, mbe);
                Sc e, ne;
                UF_UNROLL
                for (int k = 0; k < 8; ++k) e.v[k] = h[7 - k];
                sc_reduce_once(e);
                sc_neg(ne, e);
                dual_recode(d, s, ne);
            }
        } else {
            // ---- ECDSA: parse, key, then w = s^-1 shared by the block ----
            if (ok) {
                if (kKind == 0) {
                    words_be_to_limbs(r.v, sw);
                    words_be_to_limbs(s.v, sw + 8);
                } else {
                    UF_UNROLL
                    for (int k = 0; k < 8; ++k) {
                        r.v[k] = sw[k];
                        s.v[k] = sw[8 + k];
                    }
                }
                ok = !sc_is_zero(r) && limbs_lt_n(r.v) && !sc_is_zero(s) && limbs_lt_n(s.v);
                if (ok) {
                    if (kKind == 0) ok = sc_is_low(s.v);
                    else if (!sc_is_low(s.v)) sc_neg(s, s);
                }
            }
            if (ok) {
                const uint8_t* pub = pubs + 33ull * i;
                const uint8_t prefix = pub[0];
                ok = prefix == 0x02 || prefix == 0x03;
                if (ok) {
                    be32_to_limbs(px.v, pub + 1);
                    ok = limbs_lt_p(px.v) && lift_x_parity(py, px, prefix == 0x03);
                }
            }
            Sc w = s;
            if (!ok) grp_one(w);
            ok = group_invert<GrpScalarOps, G>(w, gsh) && ok;
            if (ok) {
                Sc z, u1, u2;
                words_be_to_limbs(z.v, mw);
                sc_reduce_once(z);
                sc_mul(u1, z, w);
                sc_mul(u2, r, w);
                dual_recode(d, u1, u2);
            }
        }
        // ---- the P table, its inversion shared by the block ----
        Fe zs[kPTab - 1], cs[kPTab - 1], inv;
        grp_one(inv);
        if (ok) {
            build_ptable_pre(tab, px, py, zs, cs);
            inv = cs[kPTab - 2];
        }
        ok = group_invert<GrpFieldOps, G>(inv, gsh) && ok;
        if (ok) build_ptable_post(tab, zs, cs, inv);
        Jac R;
        jac_set_inf(R);
        if (ok) dual_loop(R, d, tab, g);
        if (kKind == 1) {
            // ---- BIP-340 final check: R finite, y even, x == r; Z^-1 shared ----
            const bool fin = ok && !R.inf;
            Fe zi = R.Z;
            if (!fin) grp_one(zi);
            ok = group_invert<GrpFieldOps, G>(zi, gsh) && fin;
            if (ok) {
                Fe zi2, zi3, ax, ay;
                fe_sqr(zi2, zi);
                fe_mul(zi3, zi2, zi);
                fe_mul(ax, R.X, zi2);
                fe_mul(ay, R.Y, zi3);
                fe_normalize(ax);
                fe_normalize(ay);
                uint32_t diff = 0;
                UF_UNROLL
                for (int k = 0; k < 8; ++k) diff |= ax.v[k] ^ r.v[k];
                ok = (ay.v[0] & 1u) == 0 && diff == 0;
            }
        } else {
            ok = ok && ecdsa_check_x(R, r);
        }
        if (i < n) {
            if (collect) {
                if (ok) out[i] = 0;
            } else {
                out[i] = ok ? 1 : 0;
            }
        }
    }
}

template <int G>
constexpr size_t grp_smem() {
    return (size_t)G * kPTab * 64 + 32 * (size_t)G;   // tables + the group scratch
}

template <int G>
cudaError_t launch_g(int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs, uint32_t n,
                     const uint4* gt, uint8_t* out, int collect, int grid, cudaStream_t s) {
    const int need = (int)((n + G - 1) / G);
    if (grid <= 0 || grid > need) grid = need;
    const size_t smem = grp_smem<G>();
    if (kind == 0) k_verify_grp<0, G><<<grid, G, smem, s>>>(msgs, pubs, sigs, n, gt, out, collect);
    else if (kind == 2) k_verify_grp<2, G><<<grid, G, smem, s>>>(msgs, pubs, sigs, n, gt, out, collect);
    else k_verify_grp<1, G><<<grid, G, smem, s>>>(msgs, pubs, sigs, n, gt, out, collect);
    return cudaGetLastError();
}

template <int G>
int occupancy_g(int kind) {
    const size_t smem = grp_smem<G>();
    int blocks = 0;
    auto f0 = k_verify_grp<0, G>;
    auto f1 = k_verify_grp<1, G>;
    auto f2 = k_verify_grp<2, G>;
    cudaFuncSetAttribute(f0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(f1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(f2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kind == 1 ? f1 : f0, G, smem);
    return blocks;
}

}  // namespace

cudaError_t launch_verify_grp(int group, int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs,
                              uint32_t n, const void* d_gtab, uint8_t* out, int collect, int grid, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint4* gt = reinterpret_cast<const uint4*>(d_gtab);
    if (group == 64) return launch_g<64>(kind, msgs, pubs, sigs, n, gt, out, collect, grid, s);
    if (group == 128) return launch_g<128>(kind, msgs, pubs, sigs, n, gt, out, collect, grid, s);
    return cudaErrorInvalidValue;
}

int verify_grp_occupancy(int group, int kind) {
    if (group == 64) return occupancy_g<64>(kind);
    if (group == 128) return occupancy_g<128>(kind);
    return 0;
}

}  // namespace uf
