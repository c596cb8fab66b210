// Device-side pieces shared by the RLC translation units (rlc.cu and
// rlc_serial.cu): point storage in global memory and the round geometry.
#pragma once
#include "common.cuh"
#include "fe.cuh"
#include "point.cuh"

namespace uf {
namespace rlcdev {

__device__ __forceinline__ void store_aff(uint4* q, const Fe& x, const Fe& y) {
    q[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    q[1] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
    q[2] = make_uint4(y.v[0], y.v[1], y.v[2], y.v[3]);
    q[3] = make_uint4(y.v[4], y.v[5], y.v[6], y.v[7]);
}

__device__ __forceinline__ void load_aff(const uint4* q, Fe& x, Fe& y) {
    const uint4 a = q[0], b = q[1], c = q[2], d = q[3];
    x.v[0] = a.x; x.v[1] = a.y; x.v[2] = a.z; x.v[3] = a.w;
    x.v[4] = b.x; x.v[5] = b.y; x.v[6] = b.z; x.v[7] = b.w;
    y.v[0] = c.x; y.v[1] = c.y; y.v[2] = c.z; y.v[3] = c.w;
    y.v[4] = d.x; y.v[5] = d.y; y.v[6] = d.z; y.v[7] = d.w;
}

// Jacobian point in global memory: X, Y, Z and the infinity flag (7 x uint4).
constexpr int kJacQ = 7;

__device__ __forceinline__ void store_jac(uint4* q, const Jac& P) {
    store_aff(q, P.X, P.Y);
    q[4] = make_uint4(P.Z.v[0], P.Z.v[1], P.Z.v[2], P.Z.v[3]);
    q[5] = make_uint4(P.Z.v[4], P.Z.v[5], P.Z.v[6], P.Z.v[7]);
    q[6] = make_uint4(P.inf ? 1u : 0u, 0u, 0u, 0u);
}

__device__ __forceinline__ void load_jac(const uint4* q, Jac& P) {
    load_aff(q, P.X, P.Y);
    const uint4 a = q[4], b = q[5];
    P.Z.v[0] = a.x; P.Z.v[1] = a.y; P.Z.v[2] = a.z; P.Z.v[3] = a.w;
    P.Z.v[4] = b.x; P.Z.v[5] = b.y; P.Z.v[6] = b.z; P.Z.v[7] = b.w;
    P.inf = q[6].x != 0;
}

// Round geometry in device memory: seg[2s], seg[2s+1] = first item, length of
// segment s; pwf[s] = first (point, window) index of segment s, pwf[S] = total.
struct RoundGeo {
    const uint32_t* seg;
    const uint32_t* pwf;
    uint32_t n_seg;
    uint32_t n3;             // 3 * items of the call: index of the first generator point
    int c, W, B, S;          // window bits, windows, buckets per window, sub-ranges per window
};

// A bucket of more than this many chunks is merged by a warp (k_rlc_bucket_heavy).
constexpr uint32_t kHeavyChunks = 48;

}  // namespace rlcdev
}  // namespace uf
