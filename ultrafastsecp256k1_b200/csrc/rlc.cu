// RLC batch verification: device kernels and the host round loop (rlc.h).
//
// Memory per call of n items: items 192 B (three affine points), magnitudes
// 48 B, t_i = a_i s_i 32 B, parse flag 1 B.  Per round of S segments with
// c-bit windows (W = ceil(129 / c) windows, B = 2^(c-1) buckets per window):
// one 4-byte entry per non-zero digit (at most (3 len + 2) W per segment),
// counters and offsets over the K = S W B bucket keys, a Jacobian sum (112 B)
// per bucket and per chunk of chunk() entries, two per bucket sub-range and one
// per window.
#include "rlc.h"

#include <string.h>

#include <algorithm>

#include <cub/device/device_scan.cuh>

#include "dev_tables.cuh"
#include "kernels.h"
#include "keytable.h"
#include "sign.cuh"
#include "grpinv.cuh"
#include "verify.cuh"
#include "nvtx.h"
#include "rlc_dev.cuh"
#include "rlc_serial.h"

namespace uf {

namespace {

using namespace rlcdev;

struct RlcItem {
    uint4 pt[3][4];     // affine R, +-P, +-lambda P (x then y, 8 words each)
};

struct RlcSeed {
    uint8_t b[32];
};

// Running sums of a window's B buckets are split into S sub-ranges of B / S
// buckets (one thread each) and the S partial results are combined by one
// thread; S = 2^floor((c - 1) / 2) balances the two serial chains.
inline int sub_ranges(int c) { return 1 << ((c - 1) / 2); }

// Signed digit of window w (c bits) of a magnitude m + hi 2^128 < 2^160 (the
// recoding of booth_recode in ecmult.cuh with a run-time window width).
__device__ __forceinline__ int booth_digit(const uint4 m, uint32_t hi, int w, int c) {
    const uint32_t k[6] = {m.x, m.y, m.z, m.w, hi, 0u};
    const int pos = c * w - 1;
    const uint32_t mask = (1u << (c + 1)) - 1u;
    uint32_t raw;
    if (pos < 0) {
        raw = (k[0] << 1) & mask;
    } else {
        const int li = pos >> 5, off = pos & 31;
        const uint64_t v = ((uint64_t)k[li + 1] << 32) | k[li];
        raw = (uint32_t)(v >> off) & mask;
    }
    return (int)(raw & 1u) + (int)((raw >> 1) & ((1u << (c - 1)) - 1u)) - (int)((raw >> c) << (c - 1));
}

// Point pidx of the round: 3 per item, then G / lambda G per segment.
__device__ __forceinline__ void load_point(uint32_t pidx, const RlcItem* __restrict__ items, uint32_t n3,
                                           const uint4* __restrict__ gt, Fe& x, Fe& y) {
    if (pidx < n3) {
        load_aff(items[pidx / 3u].pt[pidx % 3u], x, y);
    } else {
        const GlobalGT G{gt};
        G.load(((pidx - n3) & 1u) ? kGTab : 0, x, y);
    }
}

// ---------------------------------------------------------------- prep --
// Per item: strict parse (r < p, 0 < s < n, x(P) < p), lift_x of P and R,
// challenge e, weight a, the three points with their 128-bit magnitudes (GLV
// signs folded into y) and t = a s mod n.  Items that fail to parse get zero
// magnitudes and t = 0, so they drop out of the equation; their verdict is 0.
__global__ void __launch_bounds__(128)
k_rlc_prep(const uint8_t* __restrict__ msgs, const uint8_t* __restrict__ xs, const uint8_t* __restrict__ sigs,
           uint32_t n, RlcSeed seed, RlcItem* __restrict__ items, uint4* __restrict__ mags,
           uint32_t* __restrict__ tsc, uint8_t* __restrict__ okb, uint8_t* __restrict__ out,
           const PubCacheSlot* __restrict__ keys, uint32_t key_mask, unsigned long long* __restrict__ key_hits) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned live = __activemask();       // the warp's threads with an item
    uint32_t mw[8], pw[8], sw[16];
    load_words8(mw, msgs + 32ull * i);
    load_words8(pw, xs + 32ull * i);
    load_words8(sw, sigs + 64ull * i);
    load_words8(sw + 8, sigs + 64ull * i + 32);
    uint32_t r[8];
    Sc s;
    Fe px, py, rx, ry;
    words_be_to_limbs(r, sw);
    words_be_to_limbs(s.v, sw + 8);
    words_be_to_limbs(px.v, pw);
    bool ok = limbs_lt_p(r) && !sc_is_zero(s) && limbs_lt_n(s.v) && limbs_lt_p(px.v);
    // a key resident in the context's key table (left by earlier mixed-job
    // calls) gives its y without the square root; a key known to be off the
    // curve fails as lift_x would
    bool lifted = false;
    if (ok && keys) {
        const uint32_t idx = key_lookup(keys, key_mask, px, false);
        if (idx != kNoSlot) {
            const PubCacheSlot& ks = keys[idx];
            if (slot_state(ks) == kSlotBad) {
                ok = false;
            } else {
                Fe kx;
                load_aff(ks.tab, kx, py);     // entry 0 of the table: the key's point
            }
            lifted = true;
        }
    }
    if (keys) {
        const unsigned hits = __ballot_sync(live, lifted);
        if (hits && (threadIdx.x & 31u) == (uint32_t)(__ffs(live) - 1)) atomicAdd(key_hits, (unsigned long long)__popc(hits));
    }
    if (ok && !lifted) ok = lift_x_parity(py, px, false);
    if (ok) {
        for (int k = 0; k < 8; ++k) rx.v[k] = r[k];
        ok = lift_x_parity(ry, rx, false);
    }
    okb[i] = ok ? 1 : 0;
    out[i] = ok ? 1 : 0;
    if (!ok) {
        const uint4 z = make_uint4(0, 0, 0, 0);
        mags[3ull * i] = z;
        mags[3ull * i + 1] = z;
        mags[3ull * i + 2] = z;
        for (int k = 0; k < 8; ++k) tsc[8ull * i + k] = 0;
        return;
    }
    // the challenge takes the byte strings as big-endian words
    uint32_t rbe[8], pbe[8], mbe[8], h[8];
    for (int k = 0; k < 8; ++k) { rbe[k] = bswap32(sw[k]); pbe[k] = bswap32(pw[k]); mbe[k] = bswap32(mw[k]); }
    bip340_challenge(h, rbe, pbe, mbe);
    Sc e;
    for (int k = 0; k < 8; ++k) e.v[k] = h[7 - k];
    sc_reduce_once(e);
    // a = SHA-256(seed || le32 i), first 16 bytes as a big-endian integer
    uint8_t buf[36];
    for (int k = 0; k < 32; ++k) buf[k] = seed.b[k];
    for (int k = 0; k < 4; ++k) buf[32 + k] = (uint8_t)(i >> (8 * k));
    uint32_t ah[8];
    sha256_iv(ah);
    sha256_tail(ah, buf, 36, 0);
    Sc a;
    a.v[0] = ah[3]; a.v[1] = ah[2]; a.v[2] = ah[1]; a.v[3] = ah[0];
    for (int k = 4; k < 8; ++k) a.v[k] = 0;
    if ((a.v[0] | a.v[1] | a.v[2] | a.v[3]) == 0) a.v[0] = 1;
    Sc ae, t;
    sc_mul(ae, a, e);
    sc_mul(t, a, s);
    GlvSplit g;
    glv_split(g, ae);
    Fe beta, yn, lx;
    fe_beta(beta);
    store_aff(items[i].pt[0], rx, ry);
    yn = py;
    if (g.neg1) { fe_neg(yn, py); fe_normalize(yn); }
    store_aff(items[i].pt[1], px, yn);
    yn = py;
    if (g.neg2) { fe_neg(yn, py); fe_normalize(yn); }
    fe_mul(lx, px, beta);
    fe_normalize(lx);
    store_aff(items[i].pt[2], lx, yn);
    mags[3ull * i] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
    mags[3ull * i + 1] = make_uint4(g.k1[0], g.k1[1], g.k1[2], g.k1[3]);
    mags[3ull * i + 2] = make_uint4(g.k2[0], g.k2[1], g.k2[2], g.k2[3]);
    for (int k = 0; k < 8; ++k) tsc[8ull * i + k] = t.v[k];
}

// largest k < n with a[k] <= t (a non-decreasing, a[0] = 0 <= t)
__device__ __forceinline__ uint32_t upper_index(const uint32_t* __restrict__ a, uint32_t n, uint32_t t) {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(a + mid) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Per segment: sum of t_i and count of unparsed items; then the magnitudes of
// the two generator points from the GLV split of -sum t_i.
// With `scaled` (the locate round) item i of a segment starting at i0 enters
// with the weight j = i - i0 + 1: the sum is of j t_i.
__global__ void __launch_bounds__(256)
k_rlc_tsum(RoundGeo g, const uint32_t* __restrict__ tsc, const uint8_t* __restrict__ okb,
           uint4* __restrict__ segmag, uint8_t* __restrict__ segneg, uint32_t* __restrict__ segbad, int scaled) {
    __shared__ uint32_t red[8][256];
    __shared__ uint32_t bad;
    const uint32_t s = blockIdx.x, tid = threadIdx.x;
    if (tid == 0) bad = 0;
    __syncthreads();
    const uint32_t i0 = g.seg[2 * s], len = g.seg[2 * s + 1];
    Sc acc;
    for (int k = 0; k < 8; ++k) acc.v[k] = 0;
    uint32_t nbad = 0;
    for (uint32_t i = i0 + tid; i < i0 + len; i += blockDim.x) {
        Sc t;
        const uint4* q = reinterpret_cast<const uint4*>(tsc + 8ull * i);
        const uint4 lo = q[0], hi = q[1];
        t.v[0] = lo.x; t.v[1] = lo.y; t.v[2] = lo.z; t.v[3] = lo.w;
        t.v[4] = hi.x; t.v[5] = hi.y; t.v[6] = hi.z; t.v[7] = hi.w;
        if (scaled) {
            Sc jj;
            jj.v[0] = i - i0 + 1;
            for (int k = 1; k < 8; ++k) jj.v[k] = 0;
            sc_mul(t, t, jj);
        }
        sc_add(acc, acc, t);
        nbad += okb[i] ? 0u : 1u;
    }
    if (nbad) atomicAdd(&bad, nbad);
    for (int k = 0; k < 8; ++k) red[k][tid] = acc.v[k];
    __syncthreads();
    for (uint32_t st = blockDim.x / 2; st > 0; st >>= 1) {
        if (tid < st) {
            Sc a, b;
            for (int k = 0; k < 8; ++k) { a.v[k] = red[k][tid]; b.v[k] = red[k][tid + st]; }
            sc_add(a, a, b);
            for (int k = 0; k < 8; ++k) red[k][tid] = a.v[k];
        }
        __syncthreads();
    }
    if (tid == 0) {
        Sc sum;
        for (int k = 0; k < 8; ++k) sum.v[k] = red[k][0];
        sc_neg(sum, sum);
        GlvSplit gs;
        glv_split(gs, sum);
        segmag[2 * s] = make_uint4(gs.k1[0], gs.k1[1], gs.k1[2], gs.k1[3]);
        segmag[2 * s + 1] = make_uint4(gs.k2[0], gs.k2[1], gs.k2[2], gs.k2[3]);
        segneg[2 * s] = gs.neg1 ? 1 : 0;
        segneg[2 * s + 1] = gs.neg2 ? 1 : 0;
        segbad[s] = bad;
    }
}

// One thread per point of the round: its segment (one search), magnitude and
// sign are read once and all W of its c-bit digits go to their buckets.
// pass 0 counts entries per (segment, window, |digit|) key (key = (segment W
// + window) B + |digit| - 1) and keeps each entry's rank, pass 1 writes entry
// = point index | sign << 31 at the key's scanned offset + rank (order within
// a bucket is arbitrary: bucket sums do not depend on it).
__global__ void __launch_bounds__(256)
k_rlc_digits(RoundGeo g, const uint4* __restrict__ mags, const uint32_t* __restrict__ mags_hi,
             const uint4* __restrict__ segmag, const uint8_t* __restrict__ segneg, uint32_t total,
             uint32_t* __restrict__ counts, uint32_t* __restrict__ ranks, const uint32_t* __restrict__ offsets,
             uint32_t* __restrict__ entries, int pass) {
    const uint32_t W = (uint32_t)g.W;
    const uint32_t npts = total / W;
    const uint32_t tp = blockIdx.x * blockDim.x + threadIdx.x;     // point of the round
    if (tp >= npts) return;
    const uint32_t s = upper_index(g.pwf, g.n_seg, tp * W);
    const uint32_t p = tp - g.pwf[s] / W;
    const uint32_t len = g.seg[2 * s + 1];
    uint32_t pidx, mhi = 0;
    uint4 m;
    bool neg = false;
    if (p < 3u * len) {
        pidx = 3u * g.seg[2 * s] + p;
        m = mags[pidx];
        if (mags_hi) {
            // locate round: bits 128.. of the magnitude, bit 31 = the point enters negated
            mhi = mags_hi[pidx];
            neg = (mhi >> 31) != 0;
            mhi &= 0x7FFFFFFFu;
        }
    } else {
        const uint32_t j = 2u * s + (p - 3u * len);
        pidx = g.n3 + j;
        m = segmag[j];
        neg = segneg[j] != 0;
    }
    const uint32_t key0 = s * W * (uint32_t)g.B;
    for (uint32_t w = 0; w < W; ++w) {
        const int d = booth_digit(m, mhi, (int)w, g.c);
        if (d == 0) continue;
        const uint32_t key = key0 + w * (uint32_t)g.B + (uint32_t)((d < 0 ? -d : d) - 1);
        // the count pass's atomic returns the entry's rank in its bucket; the
        // scatter pass writes it there, with no atomic of its own
        if (pass == 0) ranks[(size_t)w * npts + tp] = atomicAdd(&counts[key], 1u);
        else entries[offsets[key] + ranks[(size_t)w * npts + tp]] = pidx | (((d < 0) != neg) ? 0x80000000u : 0u);
    }
}

// chunks per key, for the chunk scan; nch[K] = 0
__global__ void k_rlc_nchunks(const uint32_t* __restrict__ counts, uint32_t K, uint32_t chunk,
                              uint32_t* __restrict__ nch) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) nch[k] = (counts[k] + chunk - 1) / chunk;
    else if (k == K) nch[k] = 0;
}

// One thread per chunk of at most `chunk` entries of one bucket.  A bucket
// with a single chunk is written straight to its bucket slot.
__global__ void __launch_bounds__(128)
k_rlc_chunks(const uint32_t* __restrict__ coff, uint32_t K, uint32_t chunk, const uint32_t* __restrict__ offsets,
             const uint32_t* __restrict__ entries, const RlcItem* __restrict__ items, uint32_t n3,
             const uint4* __restrict__ gt, uint4* __restrict__ partials, uint4* __restrict__ buckets) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= coff[K]) return;
    const uint32_t key = upper_index(coff, K, t);
    const uint32_t j = t - coff[key];
    const uint32_t e0 = offsets[key] + j * chunk;
    const uint32_t e1 = min(e0 + chunk, offsets[key + 1]);
    Jac acc;
    jac_set_inf(acc);
    for (uint32_t e = e0; e < e1; ++e) {
        const uint32_t v = entries[e];
        Fe x, y;
        load_point(v & 0x7FFFFFFFu, items, n3, gt, x, y);
        if (v >> 31) fe_neg(y, y);
        jac_add_aff(acc, x, y);
    }
    if (coff[key + 1] - coff[key] == 1) store_jac(buckets + kJacQ * (uint64_t)key, acc);
    else store_jac(partials + kJacQ * (uint64_t)t, acc);
}

// ------------------------------------------------- batch-affine chunk sums --
// The same chunks summed in affine coordinates.  Each chunk is reduced by a
// pairwise tree (level 1 adds entries 2p and 2p + 1, each later level the
// results of the level before); an affine addition needs one inversion, and
// every inversion of a level is shared by the whole grid (Montgomery's trick,
// one safegcd per level and piece of chunks):
//
//   forward (k_aff_fwd): per thread, the denominators of its pairs multiplied
//     up (suffix products kept in `suf`), the thread's product into `tp`;
//   the threads' products are inverted together (k_binv_*: serial products of
//     16 values per thread, a block-level product tree over 512 threads,
//     repeated down to one inversion);
//   backward (k_aff_bwd): from the thread's inverse, its pairs from the first
//     up: 1 / den of pair q = inverse x suf[q + 1], the affine sum, written to
//     the chunk's slot p.
//
// An affine addition with the shared inversion costs about 5 multiplies and
// 1 squaring against 7 and 4 for a mixed Jacobian addition, the product tree
// adds about 4 multiplies per thread and level, and the chunks' results
// are affine, so the bucket merge uses mixed additions too.  Level l gives each
// thread 2^(l-1) consecutive chunks, so a thread has up to C / 2 pairs at every
// level.
//
// Addition cases of A + B (affine, each possibly infinity) and the
// denominator each needs inverted (never zero: y = 0 has no point on this
// curve).
enum : int { kPairGen = 0, kPairDbl = 1, kPairInf = 2, kPairA = 3, kPairB = 4 };

__device__ __forceinline__ int pair_den(const Fe& xa, const Fe& ya, bool ia, const Fe& xb, const Fe& yb, bool ib,
                                        Fe& den) {
    if (ia || ib) {
        fe_set_u32(den, 1);
        return ia ? kPairB : kPairA;
    }
    fe_sub(den, xb, xa);
    if (!fe_is_zero(den)) return kPairGen;
    Fe t;
    fe_sub(t, yb, ya);
    if (fe_is_zero(t)) {            // A == B: tangent slope 3 x^2 / 2 y
        fe_add(den, ya, ya);
        return kPairDbl;
    }
    fe_set_u32(den, 1);             // A == -B
    return kPairInf;
}

// A <- A + B given inv = 1 / den of pair_den.
__device__ __forceinline__ void pair_sum(int kase, Fe& xa, Fe& ya, bool& ia, const Fe& xb, const Fe& yb, bool ib,
                                         const Fe& inv) {
    if (kase == kPairA) return;
    if (kase == kPairB) {
        xa = xb;
        ya = yb;
        ia = ib;
        return;
    }
    if (kase == kPairInf) {
        ia = true;
        return;
    }
    Fe lam, t, x3;
    if (kase == kPairGen) {
        fe_sub(t, yb, ya);
    } else {
        fe_sqr(t, xa);
        fe_mul_small(t, t, 3u);
    }
    fe_mul(lam, t, inv);
    fe_sqr(x3, lam);
    fe_sub(x3, x3, xa);
    fe_sub(x3, x3, xb);             // xb == xa when doubling
    fe_sub(t, xa, x3);
    fe_mul(t, lam, t);
    fe_sub(ya, t, ya);
    xa = x3;
}

__device__ __forceinline__ void ld_fe(const uint4* q, Fe& a) {
    const uint4 u = q[0], v = q[1];
    a.v[0] = u.x; a.v[1] = u.y; a.v[2] = u.z; a.v[3] = u.w;
    a.v[4] = v.x; a.v[5] = v.y; a.v[6] = v.z; a.v[7] = v.w;
}

__device__ __forceinline__ void st_fe(uint4* q, const Fe& a) {
    q[0] = make_uint4(a.v[0], a.v[1], a.v[2], a.v[3]);
    q[1] = make_uint4(a.v[4], a.v[5], a.v[6], a.v[7]);
}

// Warp-level exclusive prefix and suffix products of the lanes' values:
// returns the product of the other 31 lanes' values; *all = the warp's product.
__device__ __forceinline__ Fe warp_others(const Fe& x, Fe* all) {
    const int lane = (int)(threadIdx.x & 31u);
    Fe incl = x, suf = x;
    UF_UNROLL
    for (int d = 1; d < 32; d <<= 1) {
        const Fe a = grp_shfl_up(incl, d);
        if (lane >= d) fe_mul(incl, incl, a);
        const Fe b = grp_shfl_down(suf, d);
        if (lane + d < 32) fe_mul(suf, suf, b);
    }
    Fe ex = grp_shfl_up(incl, 1), sx = grp_shfl_down(suf, 1);
    if (lane == 0) fe_set_u32(ex, 1);
    if (lane == 31) fe_set_u32(sx, 1);
    *all = grp_shfl(incl, 31);
    Fe o;
    fe_mul(o, ex, sx);
    return o;
}

// ---- grid-wide batch inversion of n values (2 uint4 each) in place ----
constexpr int kBinvQ = 16;                         // values per thread, serial
constexpr int kBinvBlock = 512;                    // threads per block
constexpr uint32_t kBinvTop = (uint32_t)kBinvQ * kBinvBlock;   // sizes up to this: one block

// Serial prefix products of thread j's values [Q j, Q j + Q) into w; returns
// their product (one past n: 1).
__device__ __forceinline__ Fe binv_serial(const uint4* __restrict__ v, uint4* __restrict__ w, uint32_t n,
                                          uint32_t j) {
    const uint32_t i0 = j * kBinvQ;
    Fe acc, x;
    fe_set_u32(acc, 1);
    for (int k = 0; k < kBinvQ; ++k) {
        if (i0 + k >= n) break;
        ld_fe(v + 2ull * (i0 + k), x);
        if (k == 0) acc = x;
        else fe_mul(acc, acc, x);
        st_fe(w + 2ull * (i0 + k), acc);
    }
    return acc;
}

// Block-level product tree (every thread of the block calls it): returns the
// product of the block's other threads' values; *all = the block's product.
__device__ __forceinline__ Fe binv_block(const Fe& x, Fe* all, uint32_t (*wsh)[8]) {
    const uint32_t lane = threadIdx.x & 31u, wi = threadIdx.x >> 5, nw = blockDim.x >> 5;
    Fe wall;
    Fe oth = warp_others(x, &wall);
    if (lane == 0)
        for (int k = 0; k < 8; ++k) wsh[wi][k] = wall.v[k];
    __syncthreads();
    if (wi == 0) {
        Fe wv, ball;
        if (lane < nw) {
            for (int k = 0; k < 8; ++k) wv.v[k] = wsh[lane][k];
        } else {
            fe_set_u32(wv, 1);
        }
        const Fe wo = warp_others(wv, &ball);       // product of the other warps' products
        __syncwarp();
        if (lane < nw)
            for (int k = 0; k < 8; ++k) wsh[lane][k] = wo.v[k];
        if (lane == 0)
            for (int k = 0; k < 8; ++k) wsh[31][k] = ball.v[k];   // lane 31's slot is read back below
        // (nw <= 16: slot 31 holds no warp's value)
    }
    __syncthreads();
    Fe wo;
    for (int k = 0; k < 8; ++k) {
        wo.v[k] = wsh[wi][k];
        all->v[k] = wsh[31][k];
    }
    __syncthreads();
    fe_mul(oth, oth, wo);
    return oth;
}

// Inverses of thread j's values, in place, from t = 1 / (their product).
__device__ __forceinline__ void binv_unwind(uint4* __restrict__ v, const uint4* __restrict__ w, uint32_t n,
                                            uint32_t j, Fe t) {
    const uint32_t i0 = j * kBinvQ;
    if (i0 >= n) return;
    Fe x, r;
    const int cnt = (int)min((uint32_t)kBinvQ, n - i0);
    for (int k = cnt - 1; k >= 0; --k) {
        ld_fe(v + 2ull * (i0 + k), x);
        if (k > 0) {
            ld_fe(w + 2ull * (i0 + k - 1), r);
            fe_mul(r, t, r);
        } else {
            r = t;
        }
        fe_mul(t, t, x);
        st_fe(v + 2ull * (i0 + k), r);
    }
}

// Block b's product into u[b]; o[j] = product of the block's other values.
__global__ void __launch_bounds__(kBinvBlock)
k_binv_up(const uint4* __restrict__ v, uint4* __restrict__ w, uint4* __restrict__ o, uint4* __restrict__ u,
          uint32_t n) {
    __shared__ uint32_t wsh[32][8];
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const Fe acc = binv_serial(v, w, n, j);
    Fe all;
    const Fe oth = binv_block(acc, &all, wsh);
    st_fe(o + 2ull * j, oth);
    if (threadIdx.x == 0) st_fe(u + 2ull * blockIdx.x, all);
}

// With uinv[b] = 1 / (block b's product): thread j's inverses.
__global__ void __launch_bounds__(kBinvBlock)
k_binv_down(uint4* __restrict__ v, const uint4* __restrict__ w, const uint4* __restrict__ o,
            const uint4* __restrict__ uinv, uint32_t n) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j * kBinvQ >= n) return;
    Fe t, x;
    ld_fe(uinv + 2ull * blockIdx.x, t);
    ld_fe(o + 2ull * j, x);
    fe_mul(t, t, x);
    binv_unwind(v, w, n, j, t);
}

// n <= kBinvTop values: one block; the block's product is inverted once (by
// warp 0, every lane on the same value).
__global__ void __launch_bounds__(kBinvBlock) k_binv_top(uint4* __restrict__ v, uint4* __restrict__ w, uint32_t n) {
    __shared__ uint32_t wsh[32][8];
    __shared__ uint32_t ish[8];
    const uint32_t j = threadIdx.x;
    const Fe acc = binv_serial(v, w, n, j);
    Fe all;
    Fe t = binv_block(acc, &all, wsh);
    if (threadIdx.x < 32) {
        Fe inv;
        fe_inv(inv, all);
        if (threadIdx.x == 0)
            for (int k = 0; k < 8; ++k) ish[k] = inv.v[k];
    }
    __syncthreads();
    Fe inv;
    for (int k = 0; k < 8; ++k) inv.v[k] = ish[k];
    fe_mul(t, t, inv);
    binv_unwind(v, w, n, j, t);
}

// ---- the chunk trees ----
struct AffArgs {
    const uint32_t* coff;       // chunk offsets per bucket key (K + 1)
    uint32_t K, chunk;
    const uint32_t* offsets;    // entry offsets per bucket key
    const uint32_t* entries;
    const RlcItem* items;
    uint32_t n3;
    const uint4* gt;
    uint32_t t0, tn;            // this piece: chunks t0 .. t0 + tn - 1 (those below coff[K] exist)
    uint4* pts;                 // slot s of piece chunk c, quad q: pts[(4 s + q) tn + c]
    uint32_t* ckey;             // per piece chunk: bucket key
    uint32_t* ce0;              // first entry
    uint8_t* cm0;               // entries (0: no chunk)
    uint32_t* cinf;             // bit s: slot s holds infinity
    uint4* suf;                 // per thread of a level: up to C / 2 suffix products, [q][thread]
    uint4* tp;                  // per thread of a level: product of its denominators (inverted in place
                                // between the passes)
    uint4* partials;
    uint4* buckets;
};

// x (and with `full` y) of entry e.
__device__ __forceinline__ void aff_entry(const AffArgs& a, uint32_t e, Fe& x, Fe& y, bool full) {
    const uint32_t v = a.entries[e];
    const uint32_t pidx = v & 0x7FFFFFFFu;
    const uint4* q;
    if (pidx < a.n3) {
        q = a.items[pidx / 3u].pt[pidx % 3u];
    } else {
        q = a.gt + 4 * (((pidx - a.n3) & 1u) ? kGTab : 0);
    }
    ld_fe(q, x);
    if (full) {
        ld_fe(q + 2, y);
        if (v >> 31) fe_neg(y, y);
    }
}

__device__ __forceinline__ void aff_slot_get(const AffArgs& a, uint32_t c, int s, Fe& x, Fe& y, bool full) {
    const uint4* q = a.pts + (size_t)(4 * s) * a.tn + c;
    const uint4 q0 = q[0], q1 = q[a.tn];
    x.v[0] = q0.x; x.v[1] = q0.y; x.v[2] = q0.z; x.v[3] = q0.w;
    x.v[4] = q1.x; x.v[5] = q1.y; x.v[6] = q1.z; x.v[7] = q1.w;
    if (full) {
        const uint4 q2 = q[2 * (size_t)a.tn], q3 = q[3 * (size_t)a.tn];
        y.v[0] = q2.x; y.v[1] = q2.y; y.v[2] = q2.z; y.v[3] = q2.w;
        y.v[4] = q3.x; y.v[5] = q3.y; y.v[6] = q3.z; y.v[7] = q3.w;
    }
}

__device__ __forceinline__ void aff_slot_put(const AffArgs& a, uint32_t c, int s, const Fe& x, const Fe& y) {
    uint4* q = a.pts + (size_t)(4 * s) * a.tn + c;
    q[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    q[a.tn] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
    q[2 * (size_t)a.tn] = make_uint4(y.v[0], y.v[1], y.v[2], y.v[3]);
    q[3 * (size_t)a.tn] = make_uint4(y.v[4], y.v[5], y.v[6], y.v[7]);
}

// Pair p of piece chunk c at `level` (1: entries e0 + 2p, + 1; else slots 2p,
// 2p + 1).  With `full` the two points are loaded whole; without, only the x
// coordinates, and the y coordinates only when the x coordinates are equal
// (the forward pass needs just the denominator).
__device__ __forceinline__ int aff_pair(const AffArgs& a, int level, uint32_t c, uint32_t e0, uint32_t inf, int p,
                                        bool full, Fe& xa, Fe& ya, bool& ia, Fe& xb, Fe& yb, bool& ib, Fe& den) {
    if (level == 1) {
        ia = ib = false;
    } else {
        ia = (inf >> (2 * p)) & 1u;
        ib = (inf >> (2 * p + 1)) & 1u;
    }
    if (level == 1) {
        aff_entry(a, e0 + 2 * p, xa, ya, full);
        aff_entry(a, e0 + 2 * p + 1, xb, yb, full);
    } else {
        aff_slot_get(a, c, 2 * p, xa, ya, full);
        aff_slot_get(a, c, 2 * p + 1, xb, yb, full);
    }
    if (!full && !ia && !ib) {
        fe_sub(den, xb, xa);
        if (!fe_is_zero(den)) return kPairGen;
        if (level == 1) {
            aff_entry(a, e0 + 2 * p, xa, ya, true);
            aff_entry(a, e0 + 2 * p + 1, xb, yb, true);
        } else {
            aff_slot_get(a, c, 2 * p, xa, ya, true);
            aff_slot_get(a, c, 2 * p + 1, xb, yb, true);
        }
    }
    return pair_den(xa, ya, ia, xb, yb, ib, den);
}

// Points of a chunk of m0 entries at `level`: ceil(m0 / 2^(level-1)).
__device__ __forceinline__ uint32_t aff_count(uint32_t m0, int level) {
    return (m0 + (1u << (level - 1)) - 1u) >> (level - 1);
}

// One thread per bucket key: the key, first entry and entry count of each of
// its chunks that falls in the piece.
__global__ void __launch_bounds__(256) k_aff_keys(AffArgs a) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.K) return;
    const uint32_t c0 = max(a.coff[k], a.t0), c1 = min(a.coff[k + 1], a.t0 + a.tn);
    const uint32_t o0 = a.offsets[k], o1 = a.offsets[k + 1];
    for (uint32_t t = c0; t < c1; ++t) {
        const uint32_t e0 = o0 + (t - a.coff[k]) * a.chunk;
        a.ckey[t - a.t0] = k;
        a.ce0[t - a.t0] = e0;
        a.cm0[t - a.t0] = (uint8_t)(min(e0 + a.chunk, o1) - e0);
    }
}

// Forward pass of `level` (128 threads per block; thread u of `threads` has
// the piece chunks u, u + threads, ..., fewer than 2^(level-1) of them, so
// that neighbouring threads touch neighbouring chunks).
__global__ void __launch_bounds__(128)
k_aff_fwd(AffArgs a, int level, uint32_t threads) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t span = 1u << (level - 1);
    Fe acc;
    fe_set_u32(acc, 1);
    if (u < threads) {
        uint32_t np_all = 0;
        for (uint32_t k = 0; k < span; ++k) {
            const uint32_t c = u + k * threads;
            if (c >= a.tn) break;
            np_all += aff_count(a.cm0[c], level) / 2u;
        }
        uint32_t q = np_all;
        for (uint32_t k = span; k-- > 0;) {
            const uint32_t c = u + k * threads;
            if (c >= a.tn) continue;
            const uint32_t m0 = a.cm0[c];
            if (m0 < 2) continue;
            const int np = (int)(aff_count(m0, level) / 2u);
            const uint32_t e0 = level == 1 ? a.ce0[c] : 0u;
            const uint32_t inf = level == 1 ? 0u : a.cinf[c];
            for (int p = np - 1; p >= 0; --p) {
                Fe xa, ya, xb, yb, den;
                bool ia, ib;
                aff_pair(a, level, c, e0, inf, p, false, xa, ya, ia, xb, yb, ib, den);
                if (q == np_all) acc = den;
                else fe_mul(acc, acc, den);
                --q;
                st_fe(a.suf + 2 * ((size_t)q * threads + u), acc);
            }
        }
    }
    if (u < threads) st_fe(a.tp + 2ull * u, acc);
}

// Backward pass of `level`: the sums, the odd points moved, and after the last
// level each chunk's point written to its bucket (a bucket of one chunk) or
// to its partial, Jacobian with Z = 1.
__global__ void __launch_bounds__(128)
k_aff_bwd(AffArgs a, int level, uint32_t threads, int last) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= threads) return;
    const uint32_t span = 1u << (level - 1);
    Fe inv;
    ld_fe(a.tp + 2ull * u, inv);
    uint32_t np_all = 0;
    for (uint32_t k = 0; k < span; ++k) {
        const uint32_t c = u + k * threads;
        if (c >= a.tn) break;
        np_all += aff_count(a.cm0[c], level) / 2u;
    }
    uint32_t q = 0;
    for (uint32_t k = 0; k < span; ++k) {
        const uint32_t c = u + k * threads;
        if (c >= a.tn) break;
        const uint32_t m0 = a.cm0[c];
        if (m0 == 0) continue;
        const uint32_t m = aff_count(m0, level);
        const int np = (int)(m / 2u);
        const uint32_t e0 = level == 1 ? a.ce0[c] : 0u;
        const uint32_t inf = level == 1 ? 0u : a.cinf[c];
        uint32_t ninf = 0;
        for (int p = 0; p < np; ++p) {
            Fe xa, ya, xb, yb, den, ip;
            bool ia, ib;
            const int kase = aff_pair(a, level, c, e0, inf, p, true, xa, ya, ia, xb, yb, ib, den);
            if (q + 1 < np_all) {
                ld_fe(a.suf + 2 * ((size_t)(q + 1) * threads + u), ip);
                fe_mul(ip, inv, ip);
            } else {
                ip = inv;
            }
            fe_mul(inv, inv, den);
            ++q;
            pair_sum(kase, xa, ya, ia, xb, yb, ib, ip);
            aff_slot_put(a, c, p, xa, ya);
            ninf |= (ia ? 1u : 0u) << p;
        }
        if (m & 1u) {
            Fe x, y;
            if (level == 1) {
                aff_entry(a, e0 + m - 1, x, y, true);
                aff_slot_put(a, c, np, x, y);
            } else {
                ninf |= ((inf >> (m - 1)) & 1u) << np;
                if (np > 0) {
                    aff_slot_get(a, c, (int)m - 1, x, y, true);
                    aff_slot_put(a, c, np, x, y);
                }
            }
        }
        a.cinf[c] = ninf;
        if (last) {
            Jac r;
            aff_slot_get(a, c, 0, r.X, r.Y, true);
            fe_set_u32(r.Z, 1);
            r.inf = (ninf & 1u) != 0;
            const uint32_t key = a.ckey[c];
            if (a.coff[key + 1] - a.coff[key] == 1) store_jac(a.buckets + kJacQ * (uint64_t)key, r);
            else store_jac(a.partials + kJacQ * (uint64_t)(a.t0 + c), r);
        }
    }
}

// ---------------------------------------------------------------- locate --
// A failing segment S (its sum T = sum a_i D_i != infinity, D_i the defect of
// item i: R_i + e_i P_i - s_i G, infinity for a valid item) with exactly one
// invalid item j has T = a_j D_j.  The locate round computes, with the same
// MSM, T' = sum (i - i0 + 1) a_i D_i, which is then (j - i0 + 1) T, and a
// baby-step giant-step search over the multiples 1 .. len of T recovers j.
// With two or more invalid items T' is no such multiple (but for a 2^-128
// event over the weights), nothing is found and the segment is bisected.  The
// candidate is verified by the plain kernel, so a verdict never rests on the
// search.

// Per item of the listed segments, the locate round's magnitudes for the
// weight j a with j = i - i0 + 1: R's magnitude a times j (up to 128 + 16
// bits: four words in lmags, the fifth in lmags_hi), and for the two P
// points the GLV halves of j (a e) mod n, re-split so that they stay below
// 2^128 (the check round's halves times j would need up to 16 more bits, and
// so more windows of entries).  The stored points are P1 = s1 P and
// P2 = s2 lambda P (signs folded into y), so a e = k1 + s lambda k2 with
// s = s1 s2 (read off the two stored y coordinates), and for a new split
// K = j a e = t1 k1' + t2 lambda k2' the terms are t1 k1' P1 + (t2 s) k2' P2;
// bit 31 of lmags_hi marks a term whose point enters negated.
__global__ void __launch_bounds__(256)
k_rlc_scale(const uint32_t* __restrict__ seg, const uint4* __restrict__ mags, const RlcItem* __restrict__ items,
            uint4* __restrict__ lmags, uint32_t* __restrict__ lmags_hi) {
    const Sc LAM = {{0x1B23BD72u, 0xDF02967Cu, 0x20816678u, 0x122E22EAu,
                     0x8812645Au, 0xA5261C02u, 0xC05C30E0u, 0x5363AD4Cu}};
    const uint32_t s = blockIdx.x;
    const uint32_t i0 = seg[2 * s], len = seg[2 * s + 1];
    // blockIdx.y: which blockDim.x items of the segment
    for (uint32_t k = blockIdx.y * blockDim.x + threadIdx.x; k < len; k += gridDim.y * blockDim.x) {
        const uint64_t i = (uint64_t)i0 + k;
        const uint32_t j = k + 1u;
        const uint4 m = mags[3 * i];
        uint64_t c = (uint64_t)m.x * j;
        uint4 r;
        r.x = (uint32_t)c;
        c = (uint64_t)m.y * j + (c >> 32);
        r.y = (uint32_t)c;
        c = (uint64_t)m.z * j + (c >> 32);
        r.z = (uint32_t)c;
        c = (uint64_t)m.w * j + (c >> 32);
        r.w = (uint32_t)c;
        lmags[3 * i] = r;
        lmags_hi[3 * i] = (uint32_t)(c >> 32);
        const uint4 a1 = mags[3 * i + 1], a2 = mags[3 * i + 2];
        Sc k1 = {{a1.x, a1.y, a1.z, a1.w, 0, 0, 0, 0}}, k2 = {{a2.x, a2.y, a2.z, a2.w, 0, 0, 0, 0}};
        // s = +1 when the stored P1 and P2 have the same y
        const uint4* y1 = items[i].pt[1] + 2;
        const uint4* y2 = items[i].pt[2] + 2;
        const uint4 u0 = y1[0], u1 = y1[1], v0 = y2[0], v1 = y2[1];
        const bool flip = ((u0.x ^ v0.x) | (u0.y ^ v0.y) | (u0.z ^ v0.z) | (u0.w ^ v0.w) | (u1.x ^ v1.x) |
                           (u1.y ^ v1.y) | (u1.z ^ v1.z) | (u1.w ^ v1.w)) != 0;
        Sc t, K, jj = {{j, 0, 0, 0, 0, 0, 0, 0}};
        sc_mul(t, k2, LAM);
        if (flip) sc_neg(t, t);
        sc_add(K, k1, t);
        sc_mul(K, K, jj);
        GlvSplit g;
        glv_split(g, K);
        lmags[3 * i + 1] = make_uint4(g.k1[0], g.k1[1], g.k1[2], g.k1[3]);
        lmags[3 * i + 2] = make_uint4(g.k2[0], g.k2[1], g.k2[2], g.k2[3]);
        lmags_hi[3 * i + 1] = g.neg1 ? 0x80000000u : 0u;
        lmags_hi[3 * i + 2] = (g.neg2 != flip) ? 0x80000000u : 0u;
    }
}

// P = k T for a small k >= 0 (double and add from the top bit).
__device__ __forceinline__ void jac_small_mul(Jac& P, const Jac& T, uint32_t k) {
    jac_set_inf(P);
    for (int b = 31; b >= 0; --b) {
        if (!P.inf) jac_dbl(P);
        if ((k >> b) & 1u) jac_add(P, T);
    }
}

// One block per segment to locate: T = tsave[s] (the segment's sum of the
// check round), T' = tpr[s] (the locate round's).  With m = ceil(sqrt(len + 1))
// (blockDim.x >= m), thread t computes the baby step t T and the giant step
// T' - t m T, both affine; a giant step equal to baby step i gives
// T' = (t m + i) T.  found[s] = that j in [1, len], or 0.
__global__ void __launch_bounds__(256)
k_rlc_locate(const uint4* __restrict__ tsave, const uint4* __restrict__ tpr, const uint32_t* __restrict__ seg,
             uint32_t* __restrict__ found) {
    __shared__ uint32_t bx[8][256], by[8][256];
    __shared__ uint8_t binf[256];
    const uint32_t s = blockIdx.x, t = threadIdx.x;
    const uint32_t len = seg[2 * s + 1];
    uint32_t m = 1;
    while (m * m < len + 1) ++m;
    if (t == 0) found[s] = 0;
    Jac T, Tp;
    load_jac(tsave + kJacQ * (uint64_t)s, T);
    load_jac(tpr + kJacQ * (uint64_t)s, Tp);
    if (t < m) {
        Jac B;
        jac_small_mul(B, T, t);
        Aff a;
        const bool fin = jac_to_aff(a, B);
        binf[t] = fin ? 0 : 1;
        for (int k = 0; k < 8; ++k) {
            bx[k][t] = fin ? a.x.v[k] : 0u;
            by[k][t] = fin ? a.y.v[k] : 0u;
        }
    }
    __syncthreads();
    if (t < m) {
        Jac Q;
        jac_small_mul(Q, T, t * m);
        if (!Q.inf) {
            fe_neg(Q.Y, Q.Y);
            fe_normalize(Q.Y);
        }
        jac_add(Q, Tp);
        Aff a;
        const bool fin = jac_to_aff(a, Q);
        for (uint32_t i = 0; i < m; ++i) {
            bool eq;
            if (!fin) {
                eq = binf[i] != 0;
            } else {
                uint32_t d = binf[i];
                for (int k = 0; k < 8; ++k) d |= (bx[k][i] ^ a.x.v[k]) | (by[k][i] ^ a.y.v[k]);
                eq = d == 0;
            }
            const uint32_t j = t * m + i;
            if (eq && j >= 1 && j <= len) atomicMax(&found[s], j);
        }
    }
}

// dst[k] = src[idx[k]] for Jacobian points (7 x uint4)
__global__ void k_rlc_gather_pts(const uint32_t* __restrict__ idx, uint32_t m, const uint4* __restrict__ src,
                                 uint4* __restrict__ dst) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    for (int q = 0; q < kJacQ; ++q) dst[kJacQ * (uint64_t)k + q] = src[kJacQ * (uint64_t)idx[k] + q];
}

__global__ void k_rlc_gather(const uint32_t* __restrict__ idx, uint32_t m, const uint8_t* __restrict__ msgs,
                             const uint8_t* __restrict__ xs, const uint8_t* __restrict__ sigs, uint8_t* __restrict__ gm,
                             uint8_t* __restrict__ gx, uint8_t* __restrict__ gs) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const uint64_t i = idx[k];
    const uint4* a = reinterpret_cast<const uint4*>(msgs + 32 * i);
    const uint4* b = reinterpret_cast<const uint4*>(xs + 32 * i);
    const uint4* c = reinterpret_cast<const uint4*>(sigs + 64 * i);
    uint4* ga = reinterpret_cast<uint4*>(gm + 32ull * k);
    uint4* gb = reinterpret_cast<uint4*>(gx + 32ull * k);
    uint4* gc = reinterpret_cast<uint4*>(gs + 64ull * k);
    ga[0] = a[0]; ga[1] = a[1];
    gb[0] = b[0]; gb[1] = b[1];
    gc[0] = c[0]; gc[1] = c[1]; gc[2] = c[2]; gc[3] = c[3];
}

__global__ void k_rlc_scatter(const uint32_t* __restrict__ idx, uint32_t m, const uint8_t* __restrict__ v,
                              uint8_t* __restrict__ out) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) out[idx[k]] = v[k];
}

// Input binding of the batch seed.  The reference hashes every entry's
// r || s || x(P) || m into its batch seed before mixing in CSPRNG bytes
// (src/cpu/src/batch_verify.cpp:355-380).  Here the same 128 bytes per item
// are hashed on the device as a tree: k_rlc_leafhash gives one SHA-256 digest
// per item, k_rlc_treehash hashes groups of kTreeFan consecutive digests
// until one remains; the host then takes SHA-256(root || le32 n).
constexpr uint32_t kTreeFan = 16;

__global__ void k_rlc_leafhash(const uint8_t* __restrict__ msgs, const uint8_t* __restrict__ xs,
                               const uint8_t* __restrict__ sigs, uint32_t n, uint32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t w[16], t[8], h[8];
    sha256_iv(h);
    load_words8(t, sigs + 64ull * i);
    for (int k = 0; k < 8; ++k) w[k] = bswap32(t[k]);
    load_words8(t, sigs + 64ull * i + 32);
    for (int k = 0; k < 8; ++k) w[8 + k] = bswap32(t[k]);
    sha256_compress(h, w);
    load_words8(t, xs + 32ull * i);
    for (int k = 0; k < 8; ++k) w[k] = bswap32(t[k]);
    load_words8(t, msgs + 32ull * i);
    for (int k = 0; k < 8; ++k) w[8 + k] = bswap32(t[k]);
    sha256_compress(h, w);
    w[0] = 0x80000000u;
    for (int k = 1; k < 15; ++k) w[k] = 0;
    w[15] = 1024;   // 128 bytes
    sha256_compress(h, w);
    for (int k = 0; k < 8; ++k) out[8ull * i + k] = h[k];
}

// Node j: SHA-256 of digests [j*kTreeFan, min(n, (j+1)*kTreeFan)) concatenated.
__global__ void k_rlc_treehash(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ out) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lo = j * kTreeFan;
    if (lo >= n) return;
    const uint32_t cnt = min(kTreeFan, n - lo);
    uint32_t w[16], h[8];
    sha256_iv(h);
    uint32_t k = 0;
    for (; k + 2 <= cnt; k += 2) {
        for (int q = 0; q < 16; ++q) w[q] = in[8ull * (lo + k) + q];
        sha256_compress(h, w);
    }
    int q = 0;
    if (k < cnt) {
        for (; q < 8; ++q) w[q] = in[8ull * (lo + k) + q];
    }
    w[q++] = 0x80000000u;
    for (; q < 15; ++q) w[q] = 0;
    w[15] = cnt * 256;   // bits
    sha256_compress(h, w);
    for (int t = 0; t < 8; ++t) out[8ull * j + t] = h[t];
}

// Rows [x 32 | msg 32 | sig 64] -> three arrays, and the reference's parse
// gate: *first = min over failing rows of (row << 2 | code - 3), code 3 for
// x >= p, 4 for r >= p or s outside [1, n-1] (the x test comes first).
__global__ void k_rlc_rows(const uint8_t* __restrict__ rows, uint32_t n, uint8_t* __restrict__ gm,
                           uint8_t* __restrict__ gx, uint8_t* __restrict__ gs, uint32_t* __restrict__ first) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4* q = reinterpret_cast<const uint4*>(rows + 128ull * i);
    uint4 v[8];
    for (int k = 0; k < 8; ++k) v[k] = q[k];
    uint4* a = reinterpret_cast<uint4*>(gx + 32ull * i);
    uint4* b = reinterpret_cast<uint4*>(gm + 32ull * i);
    uint4* c = reinterpret_cast<uint4*>(gs + 64ull * i);
    a[0] = v[0]; a[1] = v[1];
    b[0] = v[2]; b[1] = v[3];
    c[0] = v[4]; c[1] = v[5]; c[2] = v[6]; c[3] = v[7];
    const uint8_t* row = rows + 128ull * i;
    uint32_t w[8], lim[8];
    be32_to_limbs(w, row);
    uint32_t code = 0;
    if (!limbs_lt_p(w)) {
        code = 3;
    } else {
        be32_to_limbs(w, row + 64);
        be32_to_limbs(lim, row + 96);
        if (!limbs_lt_p(w) || is_zero256(lim) || !limbs_lt_n(lim)) code = 4;
    }
    if (code) atomicMin(first, (i << 2) | (code - 3));
}

// MSM input: scalar k (32 bytes big-endian, k < n) and compressed point P per
// item.  Item i becomes the points P and lambda P with the GLV halves of k (signs
// folded into y) in the first two point slots of the RLC item layout; the third
// slot and t are zero, so the round computes sum k_i P_i with no generator term.
// *first = min over bad items of (i << 2 | 0 for k >= n, 1 for a bad point),
// the scalar tested first (ufsecp_multi_scalar_mul, src/cpu/src/impl/ufsecp_taproot.cpp:975-983).
__global__ void __launch_bounds__(128)
k_msm_prep(const uint8_t* __restrict__ scalars, const uint8_t* __restrict__ points, uint32_t n,
           RlcItem* __restrict__ items, uint4* __restrict__ mags, uint32_t* __restrict__ tsc,
           uint8_t* __restrict__ okb, uint32_t* __restrict__ first) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Sc k;
    be32_to_limbs(k.v, scalars + 32ull * i);
    const uint8_t* p = points + 33ull * i;
    Fe x, y;
    uint32_t code = 0xFFFFFFFFu;
    if (!limbs_lt_n(k.v)) {
        code = 0;
    } else {
        be32_to_limbs(x.v, p + 1);
        if ((p[0] != 0x02 && p[0] != 0x03) || !limbs_lt_p(x.v) || !lift_x_parity(y, x, p[0] == 0x03)) code = 1;
    }
    okb[i] = 1;
    for (int j = 0; j < 8; ++j) tsc[8ull * i + j] = 0;
    const uint4 z = make_uint4(0, 0, 0, 0);
    mags[3ull * i + 2] = z;
    if (code != 0xFFFFFFFFu) {
        atomicMin(first, (i << 2) | code);
        mags[3ull * i] = z;
        mags[3ull * i + 1] = z;
        return;
    }
    GlvSplit g;
    glv_split(g, k);
    Fe beta, yn, lx;
    fe_beta(beta);
    yn = y;
    if (g.neg1) { fe_neg(yn, y); fe_normalize(yn); }
    store_aff(items[i].pt[0], x, yn);
    yn = y;
    if (g.neg2) { fe_neg(yn, y); fe_normalize(yn); }
    fe_mul(lx, x, beta);
    fe_normalize(lx);
    store_aff(items[i].pt[1], lx, yn);
    mags[3ull * i] = make_uint4(g.k1[0], g.k1[1], g.k1[2], g.k1[3]);
    mags[3ull * i + 1] = make_uint4(g.k2[0], g.k2[1], g.k2[2], g.k2[3]);
}

// Jacobian sum -> 33-byte compressed point; ok = 0 for infinity.
__global__ void k_msm_out(const uint4* __restrict__ pt, uint8_t* __restrict__ out33, uint8_t* __restrict__ ok) {
    Jac P;
    load_jac(pt, P);
    Aff a;
    if (!jac_to_aff(a, P)) {
        *ok = 0;
        for (int k = 0; k < 33; ++k) out33[k] = 0;
        return;
    }
    *ok = 1;
    out33[0] = (a.y.v[0] & 1u) ? 0x03 : 0x02;
    limbs_to_be32(out33 + 1, a.x.v);
}

inline unsigned grid_for(uint64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }


}  // namespace

int rlc_window_bits(uint32_t len) {
    // cost in mixed-addition units: one per non-zero digit, about 1.5 per
    // Jacobian addition of the bucket reduction, 0.7 per Horner doubling
    int best = 4;
    double best_cost = 1e300;
    for (int c = 4; c <= 16; ++c) {
        const int W = (129 + c - 1) / c, B = 1 << (c - 1);
        const double cost = (3.0 * len + 2.0) * W + 1.5 * 2.0 * W * B + 0.7 * (W - 1) * c;
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

RlcVerifier::~RlcVerifier() {
    for (DevBuf* b : {&items_, &mags_, &tsc_, &okb_, &segs_, &segmag_, &segneg_, &segbad_, &counts_, &offsets_,
                      &cursor_, &nch_, &coff_, &entries_, &partials_, &buckets_, &wu_, &wt_, &wins_, &segok_,
                      &scan_tmp_, &leaf_idx_, &leaf_m_, &leaf_x_, &leaf_s_, &leaf_out_, &in_m_, &in_x_, &in_s_,
                      &in_out_, &in_rows_, &gate_, &segpt_, &dig_a_, &dig_b_, &lmags_, &lmags_hi_, &tsave_,
                      &loc_idx_, &found_, &heavy_, &aff_pts_, &aff_suf_, &aff_tp_, &aff_meta_, &binv_, &keyhit_})
        b->release();
    job_host_.release();
}

int RlcVerifier::run_round(const std::vector<uint32_t>& seg, int c, cudaStream_t s, std::vector<uint8_t>& ok,
                           bool locate) {
    NvtxRange range(locate ? "RLC locate round" : "RLC round");
    if (const int rc = be_->fault_point("RLC round")) return rc;
    const uint32_t n_seg = (uint32_t)(seg.size() / 2);
    uint32_t maxlen = 0;
    for (uint32_t k = 0; k < n_seg; ++k) maxlen = std::max(maxlen, seg[2 * k + 1]);
    // a locate round's R magnitudes carry the factor j <= maxlen: 128 + bits(maxlen)
    // bits, + 1 for the signed top digit (its P halves stay below 2^128)
    int mag_bits = 129;
    if (locate)
        for (uint32_t v = maxlen; v; v >>= 1) ++mag_bits;
    const int W = (mag_bits + c - 1) / c, B = 1 << (c - 1), S = sub_ranges(c);
    std::vector<uint32_t> host(3 * (size_t)n_seg + 1);
    uint64_t total = 0;
    for (uint32_t k = 0; k < n_seg; ++k) {
        host[2 * k] = seg[2 * k];
        host[2 * k + 1] = seg[2 * k + 1];
        host[2 * n_seg + k] = (uint32_t)total;
        total += (3ull * seg[2 * k + 1] + 2) * (uint64_t)W;
        if (total >= 0x7FFFFFFFull) return be_->set_error(kErrBadInput, "RLC round too large");
    }
    host[3 * (size_t)n_seg] = (uint32_t)total;
    const uint64_t K = (uint64_t)n_seg * W * B;
    if (K >= 0x7FFFFFFFull) return be_->set_error(kErrBadInput, "RLC round too large");
    const uint32_t chunk = be_->rlc_chunk(maxlen);
    const uint64_t chunk_cap = total / chunk + K + 1;
    size_t scan_bytes = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                                  (int)(K + 1), s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC scan size");
    if ((e = segs_.ensure(host.size() * 4)) != cudaSuccess || (e = segmag_.ensure(32ull * n_seg)) != cudaSuccess ||
        (e = segneg_.ensure(2ull * n_seg)) != cudaSuccess || (e = segbad_.ensure(4ull * n_seg)) != cudaSuccess ||
        (e = counts_.ensure((K + 1) * 4)) != cudaSuccess || (e = offsets_.ensure((K + 1) * 4)) != cudaSuccess ||
        (e = cursor_.ensure(std::max<uint64_t>(total, 1) * 4)) != cudaSuccess ||
        (e = nch_.ensure((K + 1) * 4)) != cudaSuccess ||
        (e = coff_.ensure((K + 1) * 4)) != cudaSuccess ||
        (e = entries_.ensure(std::max<uint64_t>(total, 1) * 4)) != cudaSuccess ||
        (e = partials_.ensure(chunk_cap * 112)) != cudaSuccess || (e = buckets_.ensure(K * 112)) != cudaSuccess ||
        (e = wu_.ensure((uint64_t)n_seg * W * S * 112)) != cudaSuccess ||
        (e = wt_.ensure((uint64_t)n_seg * W * S * 112)) != cudaSuccess ||
        (e = wins_.ensure((uint64_t)n_seg * W * 112)) != cudaSuccess || (e = segok_.ensure(n_seg)) != cudaSuccess ||
        (e = segpt_.ensure((uint64_t)n_seg * 112)) != cudaSuccess ||
        // a heavy bucket holds more than kHeavyChunks of the at most chunk_cap chunks
        (e = heavy_.ensure((chunk_cap / (kHeavyChunks + 1) + 2) * 4)) != cudaSuccess ||
        (e = scan_tmp_.ensure(std::max<size_t>(scan_bytes, 16))) != cudaSuccess)
        return be_->cuda_error(e, "RLC round buffers");
    if (locate && ((e = lmags_.ensure(48ull * n_)) != cudaSuccess || (e = lmags_hi_.ensure(12ull * n_)) != cudaSuccess))
        return be_->cuda_error(e, "RLC locate buffers");
    uint32_t* d_seg = (uint32_t*)segs_.p;
    const RoundGeo g{d_seg, d_seg + 2 * n_seg, n_seg, 3u * n_, c, W, B, S};
    uint32_t* counts = (uint32_t*)counts_.p;
    uint32_t* offsets = (uint32_t*)offsets_.p;
    uint32_t* nch = (uint32_t*)nch_.p;
    uint32_t* coff = (uint32_t*)coff_.p;
    const uint4* mags = locate ? (const uint4*)lmags_.p : (const uint4*)mags_.p;
    const uint32_t* mags_hi = locate ? (const uint32_t*)lmags_hi_.p : nullptr;
    // `host` is pageable: the copy is staged before cudaMemcpyAsync returns
    e = cudaMemcpyAsync(d_seg, host.data(), host.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(counts, 0, (K + 1) * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(heavy_.p, 0, 4, s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC round set-up");
    if (locate)
        k_rlc_scale<<<dim3(n_seg, (maxlen + 255) / 256), 256, 0, s>>>(d_seg, (const uint4*)mags_.p,
                                                                      (const RlcItem*)items_.p, (uint4*)lmags_.p,
                                                                      (uint32_t*)lmags_hi_.p);
    k_rlc_tsum<<<n_seg, 256, 0, s>>>(g, (const uint32_t*)tsc_.p, (const uint8_t*)okb_.p, (uint4*)segmag_.p,
                                     (uint8_t*)segneg_.p, (uint32_t*)segbad_.p, locate ? 1 : 0);
    uint32_t* ranks = (uint32_t*)cursor_.p;
    k_rlc_digits<<<grid_for(total / (size_t)W, 256), 256, 0, s>>>(g, mags, mags_hi, (const uint4*)segmag_.p,
                                                                 (const uint8_t*)segneg_.p, (uint32_t)total, counts,
                                                                 ranks, nullptr, nullptr, 0);
    size_t tb = scan_tmp_.cap;
    e = cub::DeviceScan::ExclusiveSum(scan_tmp_.p, tb, counts, offsets, (int)(K + 1), s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC scan");
    k_rlc_digits<<<grid_for(total / (size_t)W, 256), 256, 0, s>>>(g, mags, mags_hi, (const uint4*)segmag_.p,
                                                                 (const uint8_t*)segneg_.p, (uint32_t)total, nullptr,
                                                                 ranks, offsets, (uint32_t*)entries_.p, 1);
    k_rlc_nchunks<<<grid_for(K + 1, 256), 256, 0, s>>>(counts, (uint32_t)K, chunk, nch);
    tb = scan_tmp_.cap;
    e = cub::DeviceScan::ExclusiveSum(scan_tmp_.p, tb, nch, coff, (int)(K + 1), s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC chunk scan");
    const bool aff = be_->rlc_affine() && chunk <= 16;
    if (aff) {
        // the exact chunk count sizes the trees' grids and pieces
        uint32_t nch = 0;
        e = cudaMemcpyAsync(&nch, coff + K, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return be_->cuda_error(e, "RLC chunk count");
        if (const int rc = affine_chunks(chunk, nch, chunk_cap, coff, (uint32_t)K, offsets, s)) return rc;
        e = launch_rlc_bucket_merge(true, coff, (uint32_t)K, (const uint4*)partials_.p, (uint4*)buckets_.p,
                                    (uint32_t*)heavy_.p, be_->sms() * 4, s);
        if (e != cudaSuccess) return be_->cuda_error(e, "RLC bucket merge");
    } else {
        k_rlc_chunks<<<grid_for(chunk_cap, 128), 128, 0, s>>>(coff, (uint32_t)K, chunk, offsets,
                                                              (const uint32_t*)entries_.p, (const RlcItem*)items_.p,
                                                              3u * n_, (const uint4*)be_->gtab(),
                                                              (uint4*)partials_.p, (uint4*)buckets_.p);
        e = launch_rlc_bucket_merge(false, coff, (uint32_t)K, (const uint4*)partials_.p, (uint4*)buckets_.p,
                                    (uint32_t*)heavy_.p, be_->sms() * 4, s);
        if (e != cudaSuccess) return be_->cuda_error(e, "RLC bucket merge");
    }
    e = launch_rlc_windows(g, (const uint4*)buckets_.p, (uint4*)wu_.p, (uint4*)wt_.p, (uint4*)wins_.p,
                           (const uint32_t*)segbad_.p, (uint8_t*)segok_.p, (uint4*)segpt_.p, s);
    if (e == cudaSuccess) e = cudaGetLastError();
    ok.resize(n_seg);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ok.data(), segok_.p, n_seg, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC round");
    return kOk;
}

// Grid-wide batch inversion of n values at v (2 uint4 each): levels of
// k_binv_up (one value per block of 8 K values) down to kBinvTop values,
// k_binv_top, then k_binv_down back up.  Scratch: for each level w (n values),
// o (one per thread), u (one per block).
static size_t binv_scratch_values(uint32_t n) {
    size_t total = 0;
    while (n > kBinvTop) {
        const uint32_t grid = (uint32_t)(((n + kBinvQ - 1) / kBinvQ + kBinvBlock - 1) / kBinvBlock);
        total += n + (size_t)grid * kBinvBlock + grid;
        n = grid;
    }
    return total + n;
}

static cudaError_t binv_launch(uint4* v, uint32_t n, uint4* scratch, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    if (n <= kBinvTop) {
        k_binv_top<<<1, kBinvBlock, 0, s>>>(v, scratch, n);
        return cudaGetLastError();
    }
    const uint32_t grid = (uint32_t)(((n + kBinvQ - 1) / kBinvQ + kBinvBlock - 1) / kBinvBlock);
    uint4* w = scratch;
    uint4* o = w + 2ull * n;
    uint4* u = o + 2ull * grid * kBinvBlock;
    uint4* rest = u + 2ull * grid;
    k_binv_up<<<grid, kBinvBlock, 0, s>>>(v, w, o, u, n);
    cudaError_t e = binv_launch(u, grid, rest, s);
    if (e != cudaSuccess) return e;
    k_binv_down<<<grid, kBinvBlock, 0, s>>>(v, w, o, u, n);
    return cudaGetLastError();
}

int RlcVerifier::affine_chunks(uint32_t chunk, uint64_t nch, uint64_t chunk_cap, const uint32_t* coff, uint32_t K,
                               const uint32_t* offsets, cudaStream_t s) {
    if (nch == 0) return kOk;
    const int C = chunk <= 8 ? 8 : 16, c2 = C / 2;
    int levels = 1;
    while ((1u << levels) < chunk) ++levels;
    // per chunk: c2 slots (64 B), c2 suffix products and one block-other product
    // (32 B), key, first entry, infinity bits (4 B each), entries (1 B)
    const uint64_t per_chunk = 64ull * c2 + 32ull * c2 + 32 + 13 + 80;
    const uint64_t piece_max = std::max<uint64_t>(kAffPieceBytes / per_chunk, 1024);
    const uint64_t piece = std::min<uint64_t>(nch, piece_max);
    // buffers sized by the round's chunk bound (fixed by the segment lengths),
    // not by this call's count, so that calls of one shape allocate once
    const uint64_t cap = std::min<uint64_t>(chunk_cap, piece_max);
    cudaError_t e;
    if ((e = aff_pts_.ensure(cap * c2 * 64)) != cudaSuccess || (e = aff_suf_.ensure(cap * c2 * 32)) != cudaSuccess ||
        (e = aff_tp_.ensure(cap * 32)) != cudaSuccess || (e = aff_meta_.ensure(cap * 13 + 64)) != cudaSuccess ||
        (e = binv_.ensure(binv_scratch_values((uint32_t)cap) * 32 + 32)) != cudaSuccess)
        return be_->cuda_error(e, "RLC affine buffers");
    AffArgs a;
    a.coff = coff;
    a.K = K;
    a.chunk = chunk;
    a.offsets = offsets;
    a.entries = (const uint32_t*)entries_.p;
    a.items = (const RlcItem*)items_.p;
    a.n3 = 3u * n_;
    a.gt = (const uint4*)be_->gtab();
    a.pts = (uint4*)aff_pts_.p;
    a.ckey = (uint32_t*)aff_meta_.p;
    a.ce0 = a.ckey + piece;
    a.cinf = a.ce0 + piece;
    a.cm0 = (uint8_t*)(a.cinf + piece);
    a.suf = (uint4*)aff_suf_.p;
    a.tp = (uint4*)aff_tp_.p;
    a.partials = (uint4*)partials_.p;
    a.buckets = (uint4*)buckets_.p;
    for (uint64_t t0 = 0; t0 < nch; t0 += piece) {
        a.t0 = (uint32_t)t0;
        a.tn = (uint32_t)std::min<uint64_t>(piece, nch - t0);
        k_aff_keys<<<grid_for(K, 256), 256, 0, s>>>(a);
        for (int level = 1; level <= levels; ++level) {
            const uint32_t threads = (uint32_t)((a.tn + (1ull << (level - 1)) - 1) >> (level - 1));
            const uint32_t blocks = (threads + 127) / 128;
            k_aff_fwd<<<blocks, 128, 0, s>>>(a, level, threads);
            if ((e = binv_launch(a.tp, threads, (uint4*)binv_.p, s)) != cudaSuccess) break;
            k_aff_bwd<<<blocks, 128, 0, s>>>(a, level, threads, level == levels ? 1 : 0);
        }
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) return be_->cuda_error(e, "RLC affine chunks");
    }
    return kOk;
}

int RlcVerifier::verify_leaves(const std::vector<uint32_t>& leaves, const uint8_t* d_msgs, const uint8_t* d_xs,
                               const uint8_t* d_sigs, uint8_t* d_out, cudaStream_t s, RlcStats* stats) {
    NvtxRange range("RLC leaves");
    std::vector<uint32_t> idx;
    for (size_t k = 0; k < leaves.size(); k += 2)
        for (uint32_t i = 0; i < leaves[k + 1]; ++i) idx.push_back(leaves[k] + i);
    return verify_indices(idx, d_msgs, d_xs, d_sigs, d_out, s, stats, nullptr);
}

int RlcVerifier::verify_indices(const std::vector<uint32_t>& idx, const uint8_t* d_msgs, const uint8_t* d_xs,
                                const uint8_t* d_sigs, uint8_t* d_out, cudaStream_t s, RlcStats* stats,
                                std::vector<uint8_t>* host_out) {
    const uint32_t m = (uint32_t)idx.size();
    if (m == 0) return kOk;
    cudaError_t e;
    if ((e = leaf_idx_.ensure(4ull * m)) != cudaSuccess || (e = leaf_m_.ensure(32ull * m)) != cudaSuccess ||
        (e = leaf_x_.ensure(32ull * m)) != cudaSuccess || (e = leaf_s_.ensure(64ull * m)) != cudaSuccess ||
        (e = leaf_out_.ensure(m)) != cudaSuccess)
        return be_->cuda_error(e, "RLC leaf buffers");
    e = cudaMemcpyAsync(leaf_idx_.p, idx.data(), 4ull * m, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC leaf indices");
    k_rlc_gather<<<grid_for(m, 256), 256, 0, s>>>((const uint32_t*)leaf_idx_.p, m, d_msgs, d_xs, d_sigs,
                                                 (uint8_t*)leaf_m_.p, (uint8_t*)leaf_x_.p, (uint8_t*)leaf_s_.p);
    if ((e = cudaGetLastError()) != cudaSuccess) return be_->cuda_error(e, "RLC gather");
    const int rc = be_->verify_device(1, (const uint8_t*)leaf_m_.p, (const uint8_t*)leaf_x_.p,
                                      (const uint8_t*)leaf_s_.p, m, (uint8_t*)leaf_out_.p, s);
    if (rc != kOk) return rc;
    k_rlc_scatter<<<grid_for(m, 256), 256, 0, s>>>((const uint32_t*)leaf_idx_.p, m, (const uint8_t*)leaf_out_.p,
                                                  d_out);
    if ((e = cudaGetLastError()) != cudaSuccess) return be_->cuda_error(e, "RLC scatter");
    if (host_out) {
        host_out->resize(m);
        if ((e = cudaMemcpyAsync(host_out->data(), leaf_out_.p, m, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
            return be_->cuda_error(e, "RLC leaf verdicts");
    }
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return be_->cuda_error(e, "RLC leaves");
    if (stats) stats->leaf_items += m;
    return kOk;
}

int RlcVerifier::locate(const std::vector<uint32_t>& round_idx, const std::vector<uint32_t>& loc,
                        const uint8_t* d_msgs, const uint8_t* d_xs, const uint8_t* d_sigs, uint8_t* d_out,
                        cudaStream_t s, RlcStats* stats, std::vector<uint8_t>& resolved) {
    NvtxRange range("RLC locate");
    const uint32_t n_loc = (uint32_t)(loc.size() / 2);
    resolved.assign(n_loc, 0);
    if (n_loc == 0) return kOk;
    cudaError_t e;
    if ((e = tsave_.ensure(112ull * n_loc)) != cudaSuccess || (e = loc_idx_.ensure(4ull * n_loc)) != cudaSuccess ||
        (e = found_.ensure(4ull * n_loc)) != cudaSuccess)
        return be_->cuda_error(e, "RLC locate buffers");
    // the check round's sums T of these segments, before the locate round overwrites them
    e = cudaMemcpyAsync(loc_idx_.p, round_idx.data(), 4ull * n_loc, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC locate indices");
    k_rlc_gather_pts<<<grid_for(n_loc, 128), 128, 0, s>>>((const uint32_t*)loc_idx_.p, n_loc,
                                                          (const uint4*)segpt_.p, (uint4*)tsave_.p);
    if ((e = cudaGetLastError()) != cudaSuccess) return be_->cuda_error(e, "RLC locate gather");
    uint32_t maxlen = 0;
    for (uint32_t k = 0; k < n_loc; ++k) maxlen = std::max(maxlen, loc[2 * k + 1]);
    std::vector<uint8_t> ok;
    int rc = run_round(loc, be_->rlc_window(maxlen), s, ok, true);
    if (rc != kOk) return rc;
    if (stats) {
        stats->rounds++;
        stats->segments += n_loc;
    }
    // one thread per baby / giant step: ceil(sqrt(len + 1)) of them, rounded
    // up to whole warps (fewer threads per block let more blocks share an SM)
    uint32_t m = 1;
    while (m * m < maxlen + 1) ++m;
    const unsigned loc_threads = std::min(256u, (m + 31u) & ~31u);
    k_rlc_locate<<<n_loc, loc_threads, 0, s>>>((const uint4*)tsave_.p, (const uint4*)segpt_.p, (const uint32_t*)segs_.p,
                                       (uint32_t*)found_.p);
    std::vector<uint32_t> found(n_loc);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(found.data(), found_.p, 4ull * n_loc, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC locate");
    // the candidates are verified one by one; only an invalid candidate resolves its segment
    std::vector<uint32_t> cand, owner;
    for (uint32_t q = 0; q < n_loc; ++q)
        if (found[q] >= 1 && found[q] <= loc[2 * q + 1]) {
            cand.push_back(loc[2 * q] + found[q] - 1);
            owner.push_back(q);
        }
    std::vector<uint8_t> verdicts;
    rc = verify_indices(cand, d_msgs, d_xs, d_sigs, d_out, s, stats, &verdicts);
    if (rc != kOk) return rc;
    for (size_t k = 0; k < cand.size(); ++k)
        if (verdicts[k] == 0) resolved[owner[k]] = 1;
    if (stats) stats->located += (uint64_t)std::count(resolved.begin(), resolved.end(), (uint8_t)1);
    return kOk;
}

int RlcVerifier::verify(const uint8_t* d_msgs, const uint8_t* d_xs, const uint8_t* d_sigs, uint32_t n,
                        uint32_t batch_size, const uint8_t seed[32], int window_bits, uint8_t* d_out,
                        uint8_t* h_batch_ok, cudaStream_t s, RlcStats* stats) {
    if (n == 0) return kOk;
    if (n > kMaxItems) return be_->set_error(kErrBadInput, "RLC: more than 2^24 items in one call");
    if (window_bits != 0 && (window_bits < 4 || window_bits > 16))
        return be_->set_error(kErrBadInput, "RLC: window_bits must be 0 or 4..16");
    if (((uintptr_t)d_msgs | (uintptr_t)d_xs | (uintptr_t)d_sigs) & 15u)
        return be_->set_error(kErrBadInput, "device inputs must be 16-byte aligned");
    if (batch_size == 0 || batch_size > n) batch_size = n;
    n_ = n;
    cudaError_t e;
    if ((e = items_.ensure((uint64_t)n * sizeof(RlcItem))) != cudaSuccess ||
        (e = mags_.ensure((uint64_t)n * 48)) != cudaSuccess || (e = tsc_.ensure((uint64_t)n * 32)) != cudaSuccess ||
        (e = okb_.ensure(n)) != cudaSuccess)
        return be_->cuda_error(e, "RLC item buffers");
    RlcSeed sd;
    memcpy(sd.b, seed, 32);
    // keys resident in the context's key table skip their square root
    const KeyTable* kt = be_->key_table();
    const bool use_keys = kt && kt->on();
    if (use_keys && ((e = keyhit_.ensure(8)) != cudaSuccess || (e = cudaMemsetAsync(keyhit_.p, 0, 8, s)) != cudaSuccess))
        return be_->cuda_error(e, "RLC key counter");
    k_rlc_prep<<<grid_for(n, 128), 128, 0, s>>>(d_msgs, d_xs, d_sigs, n, sd, (RlcItem*)items_.p, (uint4*)mags_.p,
                                                (uint32_t*)tsc_.p, (uint8_t*)okb_.p, d_out,
                                                use_keys ? kt->slots() : nullptr, use_keys ? kt->mask() : 0u,
                                                use_keys ? (unsigned long long*)keyhit_.p : nullptr);
    if ((e = cudaGetLastError()) != cudaSuccess) return be_->cuda_error(e, "RLC prep");
    if (stats && use_keys) {
        unsigned long long hits = 0;
        e = cudaMemcpyAsync(&hits, keyhit_.p, 8, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return be_->cuda_error(e, "RLC key counter");
        stats->key_hits += hits;
    }
    std::vector<uint32_t> seg, next, leaves, loc, loc_round;
    for (uint32_t b = 0; b < n; b += batch_size) {
        seg.push_back(b);
        seg.push_back(std::min(batch_size, n - b));
    }
    int round = 0;
    while (!seg.empty()) {
        uint32_t maxlen = 0;
        for (size_t k = 1; k < seg.size(); k += 2) maxlen = std::max(maxlen, seg[k]);
        const int c = window_bits > 0 ? window_bits : be_->rlc_window(maxlen);
        const int rc = run_round(seg, c, s, ok_host_);
        if (rc != kOk) return rc;
        if (stats) {
            stats->rounds++;
            stats->segments += seg.size() / 2;
            if (round == 0) stats->window_bits = c;
        }
        if (round == 0 && h_batch_ok)
            for (size_t k = 0; k < ok_host_.size(); ++k) h_batch_ok[k] = ok_host_[k] == 1 ? 1 : 0;
        size_t n_fail = 0;
        for (size_t k = 0; k < ok_host_.size(); ++k) n_fail += (ok_host_[k] & 1) ? 0 : 1;
        // dense failures (most segments of a bisection level fail): stop splitting
        const bool dense = round > 0 && n_fail >= 8 && 4 * n_fail > 3 * ok_host_.size();
        next.clear();
        loc.clear();
        loc_round.clear();
        auto split = [&](uint32_t st, uint32_t len) {
            // kFanout near-equal children
            const uint32_t parts = std::min<uint32_t>(kFanout, len);
            for (uint32_t q = 0; q < parts; ++q) {
                const uint32_t a = (uint32_t)((uint64_t)len * q / parts), b = (uint32_t)((uint64_t)len * (q + 1) / parts);
                next.push_back(st + a);
                next.push_back(b - a);
            }
        };
        for (size_t k = 0; k < ok_host_.size(); ++k) {
            if (ok_host_[k] & 1) continue;
            const uint32_t st = seg[2 * k], len = seg[2 * k + 1];
            if (dense || len <= kLeaf) {
                leaves.push_back(st);
                leaves.push_back(len);
            } else if (be_->rlc_locate() && len <= kLocateMax) {
                loc.push_back(st);
                loc.push_back(len);
                loc_round.push_back((uint32_t)k);
            } else {
                split(st, len);
            }
        }
        if (!loc.empty()) {
            // one more MSM over these segments finds a single invalid item; the
            // others (two or more invalid items) are bisected
            std::vector<uint8_t> resolved;
            const int lrc = locate(loc_round, loc, d_msgs, d_xs, d_sigs, d_out, s, stats, resolved);
            if (lrc != kOk) return lrc;
            for (size_t q = 0; q < resolved.size(); ++q)
                if (!resolved[q]) split(loc[2 * q], loc[2 * q + 1]);
        }
        seg.swap(next);
        ++round;
    }
    return verify_leaves(leaves, d_msgs, d_xs, d_sigs, d_out, s, stats);
}

int RlcVerifier::verify_host(const uint8_t* msgs, const uint8_t* xs, const uint8_t* sigs, uint32_t n,
                             uint32_t batch_size, const uint8_t seed[32], int window_bits, uint8_t* out,
                             uint8_t* h_batch_ok, RlcStats* stats) {
    if (n == 0) return kOk;
    if (n > kMaxItems) return be_->set_error(kErrBadInput, "RLC: more than 2^24 items in one call");
    const cudaStream_t s = be_->stream();
    cudaError_t e;
    if ((e = in_m_.ensure(32ull * n)) != cudaSuccess || (e = in_x_.ensure(32ull * n)) != cudaSuccess ||
        (e = in_s_.ensure(64ull * n)) != cudaSuccess || (e = in_out_.ensure(n)) != cudaSuccess)
        return be_->cuda_error(e, "RLC staging buffers");
    e = cudaMemcpyAsync(in_m_.p, msgs, 32ull * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(in_x_.p, xs, 32ull * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(in_s_.p, sigs, 64ull * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC copy in");
    const int rc = verify((const uint8_t*)in_m_.p, (const uint8_t*)in_x_.p, (const uint8_t*)in_s_.p, n, batch_size,
                          seed, window_bits, (uint8_t*)in_out_.p, h_batch_ok, s, stats);
    if (rc != kOk) return rc;
    e = cudaMemcpyAsync(out, in_out_.p, n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC copy out");
    return kOk;
}

int RlcVerifier::stage_jobs(const VerifyJob* jobs, size_t n_jobs, size_t* j, size_t* off) {
    part_.clear();
    start_.clear();
    uint64_t n = 0;
    while (*j < n_jobs && n < kMaxItems) {
        const VerifyJob& J = jobs[*j];
        if (*off >= J.count) {
            ++*j;
            *off = 0;
            continue;
        }
        const size_t take = std::min<size_t>(J.count - *off, kMaxItems - n);
        part_.push_back(VerifyJob{J.kind, take, J.msgs + 32 * *off, J.pubs + 32 * *off, J.sigs + 64 * *off,
                                  J.out + *off});
        start_.push_back(n);
        n += take;
        *off += take;
    }
    staged_ = n;
    if (n == 0) return kOk;
    cudaError_t e;
    if ((e = in_m_.ensure(32ull * n)) != cudaSuccess || (e = in_x_.ensure(32ull * n)) != cudaSuccess ||
        (e = in_s_.ensure(64ull * n)) != cudaSuccess || (e = in_out_.ensure(n)) != cudaSuccess ||
        (e = job_host_.ensure(129ull * n)) != cudaSuccess)
        return be_->cuda_error(e, "RLC job staging buffers");
    return kOk;
}

void RlcVerifier::pack_staged(size_t lo, size_t hi) {
    const uint64_t n = staged_;
    uint8_t* hm = (uint8_t*)job_host_.p;
    uint8_t* hx = hm + 32 * n;
    uint8_t* hs = hx + 32 * n;
    size_t q = std::upper_bound(start_.begin(), start_.end(), (uint64_t)lo) - start_.begin() - 1;
    for (size_t i = lo; i < hi && q < part_.size(); ++q) {
        const VerifyJob& P = part_[q];
        const size_t a0 = i - start_[q], a1 = std::min<size_t>(P.count, hi - start_[q]);
        memcpy(hm + 32 * i, P.msgs + 32 * a0, 32 * (a1 - a0));
        memcpy(hx + 32 * i, P.pubs + 32 * a0, 32 * (a1 - a0));
        memcpy(hs + 64 * i, P.sigs + 64 * a0, 64 * (a1 - a0));
        i += a1 - a0;
    }
}

int RlcVerifier::run_staged(uint32_t segment, const uint8_t rand32[32], RlcStats* stats) {
    const uint64_t n = staged_;
    if (n == 0) return kOk;
    const cudaStream_t s = be_->stream();
    uint8_t* hm = (uint8_t*)job_host_.p;
    uint8_t* hx = hm + 32 * n;
    uint8_t* hs = hx + 32 * n;
    uint8_t* ho = hs + 64 * n;
    uint8_t* dm = (uint8_t*)in_m_.p;
    uint8_t* dx = (uint8_t*)in_x_.p;
    uint8_t* ds = (uint8_t*)in_s_.p;
    cudaError_t e = cudaMemcpyAsync(dm, hm, 32 * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dx, hx, 32 * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ds, hs, 64 * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC job copy in");
    uint8_t seed[32];
    int rc = input_digest(dm, dx, ds, (uint32_t)n, s, seed);
    if (rc != kOk) return rc;
    for (int k = 0; k < 32; ++k) seed[k] ^= rand32[k];
    rc = verify(dm, dx, ds, (uint32_t)n, segment, seed, 0, (uint8_t*)in_out_.p, nullptr, s, stats);
    if (rc != kOk) return rc;
    e = cudaMemcpyAsync(ho, in_out_.p, n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC job copy out");
    for (size_t q = 0; q < part_.size(); ++q) memcpy(part_[q].out, ho + start_[q], part_[q].count);
    return kOk;
}

int RlcVerifier::input_digest(const uint8_t* d_msgs, const uint8_t* d_xs, const uint8_t* d_sigs, uint32_t n,
                              cudaStream_t s, uint8_t out[32]) {
    // two ping-pong digest arrays: n leaves, then n / kTreeFan nodes per level
    const uint64_t cap = std::max<uint64_t>(n, 1);
    cudaError_t e;
    if ((e = dig_a_.ensure(32 * cap)) != cudaSuccess || (e = dig_b_.ensure(32 * (cap / kTreeFan + 1))) != cudaSuccess)
        return be_->cuda_error(e, "RLC digest buffers");
    uint32_t* a = (uint32_t*)dig_a_.p;
    uint32_t* b = (uint32_t*)dig_b_.p;
    uint32_t root[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // n == 0: the all-zero root
    if (n) k_rlc_leafhash<<<grid_for(n, 128), 128, 0, s>>>(d_msgs, d_xs, d_sigs, n, a);
    uint32_t m = n;
    while (m > 1) {
        const uint32_t nodes = (m + kTreeFan - 1) / kTreeFan;
        k_rlc_treehash<<<grid_for(nodes, 128), 128, 0, s>>>(a, m, b);
        std::swap(a, b);
        m = nodes;
    }
    e = cudaGetLastError();
    if (e == cudaSuccess && n) e = cudaMemcpyAsync(root, a, 32, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC input digest");
    // SHA-256(root || le32 n)
    uint8_t buf[36];
    words_to_bytes(buf, root);
    for (int k = 0; k < 4; ++k) buf[32 + k] = (uint8_t)(n >> (8 * k));
    uint32_t h[8];
    sha256_iv(h);
    sha256_tail(h, buf, 36, 0);
    words_to_bytes(out, h);
    return kOk;
}

int RlcVerifier::input_digest_host(const uint8_t* msgs, const uint8_t* xs, const uint8_t* sigs, uint32_t n,
                                   uint8_t out[32]) {
    const cudaStream_t s = be_->stream();
    const uint64_t cap = std::max<uint32_t>(n, 1);
    cudaError_t e;
    if ((e = in_m_.ensure(32 * cap)) != cudaSuccess || (e = in_x_.ensure(32 * cap)) != cudaSuccess ||
        (e = in_s_.ensure(64 * cap)) != cudaSuccess)
        return be_->cuda_error(e, "RLC staging buffers");
    if (n) {
        e = cudaMemcpyAsync(in_m_.p, msgs, 32ull * n, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(in_x_.p, xs, 32ull * n, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(in_s_.p, sigs, 64ull * n, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) return be_->cuda_error(e, "RLC copy in");
    }
    return input_digest((const uint8_t*)in_m_.p, (const uint8_t*)in_x_.p, (const uint8_t*)in_s_.p, n, s, out);
}

int RlcVerifier::verify_entries(const uint8_t* rows, uint32_t n, const uint8_t rand32[32], uint8_t* h_out,
                                int* gate_code, uint32_t* gate_index, RlcStats* stats) {
    *gate_code = 0;
    *gate_index = 0;
    if (n == 0) return kOk;
    if (n > kMaxItems) return be_->set_error(kErrBadInput, "RLC: more than 2^24 items in one call");
    const cudaStream_t s = be_->stream();
    cudaError_t e;
    if ((e = in_rows_.ensure(128ull * n)) != cudaSuccess || (e = in_m_.ensure(32ull * n)) != cudaSuccess ||
        (e = in_x_.ensure(32ull * n)) != cudaSuccess || (e = in_s_.ensure(64ull * n)) != cudaSuccess ||
        (e = in_out_.ensure(n)) != cudaSuccess || (e = gate_.ensure(4)) != cudaSuccess)
        return be_->cuda_error(e, "RLC staging buffers");
    uint32_t first = 0xFFFFFFFFu;
    e = cudaMemcpyAsync(in_rows_.p, rows, 128ull * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(gate_.p, 0xFF, 4, s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC copy in");
    k_rlc_rows<<<grid_for(n, 256), 256, 0, s>>>((const uint8_t*)in_rows_.p, n, (uint8_t*)in_m_.p, (uint8_t*)in_x_.p,
                                               (uint8_t*)in_s_.p, (uint32_t*)gate_.p);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&first, gate_.p, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC row gate");
    if (first != 0xFFFFFFFFu) {
        *gate_code = 3 + (int)(first & 3u);
        *gate_index = first >> 2;
        return kOk;
    }
    // batch seed = digest of every row's r || s || x(P) || m, XOR fresh random bytes
    uint8_t seed[32];
    int rc = input_digest((const uint8_t*)in_m_.p, (const uint8_t*)in_x_.p, (const uint8_t*)in_s_.p, n, s, seed);
    if (rc != kOk) return rc;
    for (int k = 0; k < 32; ++k) seed[k] ^= rand32[k];
    rc = verify((const uint8_t*)in_m_.p, (const uint8_t*)in_x_.p, (const uint8_t*)in_s_.p, n, n, seed, 0,
                (uint8_t*)in_out_.p, nullptr, s, stats);
    if (rc != kOk) return rc;
    e = cudaMemcpyAsync(h_out, in_out_.p, n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "RLC copy out");
    return kOk;
}

int RlcVerifier::msm_host(const uint8_t* scalars32, const uint8_t* points33, uint32_t n, uint8_t out33[33],
                          int* status) {
    *status = 0;
    if (n == 0) return kOk;
    if (n > kMaxItems) return be_->set_error(kErrBadInput, "MSM: more than 2^24 points");
    const cudaStream_t s = be_->stream();
    cudaError_t e;
    if ((e = in_m_.ensure(32ull * n)) != cudaSuccess || (e = in_x_.ensure(33ull * n + 16)) != cudaSuccess ||
        (e = items_.ensure((uint64_t)n * sizeof(RlcItem))) != cudaSuccess ||
        (e = mags_.ensure((uint64_t)n * 48)) != cudaSuccess || (e = tsc_.ensure((uint64_t)n * 32)) != cudaSuccess ||
        (e = okb_.ensure(n)) != cudaSuccess || (e = gate_.ensure(64)) != cudaSuccess)
        return be_->cuda_error(e, "MSM buffers");
    uint32_t first = 0xFFFFFFFFu;
    e = cudaMemcpyAsync(in_m_.p, scalars32, 32ull * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(in_x_.p, points33, 33ull * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(gate_.p, 0xFF, 4, s);
    if (e != cudaSuccess) return be_->cuda_error(e, "MSM copy in");
    k_msm_prep<<<grid_for(n, 128), 128, 0, s>>>((const uint8_t*)in_m_.p, (const uint8_t*)in_x_.p, n,
                                                (RlcItem*)items_.p, (uint4*)mags_.p, (uint32_t*)tsc_.p,
                                                (uint8_t*)okb_.p, (uint32_t*)gate_.p);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&first, gate_.p, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "MSM parse");
    if (first != 0xFFFFFFFFu) {
        *status = (first & 3u) == 0 ? kErrBadInput : 3;   // scalar >= n / invalid point
        return kOk;
    }
    n_ = n;
    const std::vector<uint32_t> seg = {0u, n};
    const int rc = run_round(seg, be_->rlc_window(n), s, ok_host_);
    if (rc != kOk) return rc;
    uint8_t* d_out = (uint8_t*)gate_.p + 16;
    uint8_t ok = 0;
    k_msm_out<<<1, 1, 0, s>>>((const uint4*)segpt_.p, d_out, d_out + 40);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out33, d_out, 33, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&ok, d_out + 40, 1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return be_->cuda_error(e, "MSM result");
    if (!ok) *status = 7;   // the sum is the point at infinity
    return kOk;
}

}  // namespace uf
