// Device-side table accessors shared by the kernels.
//
// SmemTab: a thread's 1P..8P table in dynamic shared memory, laid out
// [entry][quad][thread] as uint4 so that each thread owns a bank column and a
// warp's data-dependent reads never conflict.  GlobalGT: the per-context
// 1..2^(UF_GWIN-1) multiples of G and lambda*G in global memory (64 MB for
// 20-bit windows; served from L2), read through the read-only L1 path.
#pragma once
#include "fe.cuh"

namespace uf {

struct SmemTab {
    uint4* base;        // this thread's column
    uint32_t stride;    // blockDim.x
    __device__ __forceinline__ void store(int k, const Fe& x, const Fe& y) const {
        uint4* p = base + (uint32_t)(k * 4) * stride;
        p[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
        p[stride] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
        p[2 * stride] = make_uint4(y.v[0], y.v[1], y.v[2], y.v[3]);
        p[3 * stride] = make_uint4(y.v[4], y.v[5], y.v[6], y.v[7]);
    }
    __device__ __forceinline__ void load(int k, Fe& x, Fe& y) const {
        const uint4* p = base + (uint32_t)(k * 4) * stride;
        uint4 a = p[0], b = p[stride], c = p[2 * stride], d = p[3 * stride];
        x.v[0] = a.x; x.v[1] = a.y; x.v[2] = a.z; x.v[3] = a.w;
        x.v[4] = b.x; x.v[5] = b.y; x.v[6] = b.z; x.v[7] = b.w;
        y.v[0] = c.x; y.v[1] = c.y; y.v[2] = c.z; y.v[3] = c.w;
        y.v[4] = d.x; y.v[5] = d.y; y.v[6] = d.z; y.v[7] = d.w;
    }
};

// 1P in registers, 2P..8P in shared memory: 448 bytes per thread instead of
// 512, so four 128-thread blocks fit an SM's shared memory.
struct SmemTab7 {
    uint4* base;        // this thread's column
    uint32_t stride;    // blockDim.x
    Fe x0, y0;
    __device__ __forceinline__ void store(int k, const Fe& x, const Fe& y) {
        if (k == 0) {
            x0 = x;
            y0 = y;
            return;
        }
        uint4* p = base + (uint32_t)((k - 1) * 4) * stride;
        p[0] = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
        p[stride] = make_uint4(x.v[4], x.v[5], x.v[6], x.v[7]);
        p[2 * stride] = make_uint4(y.v[0], y.v[1], y.v[2], y.v[3]);
        p[3 * stride] = make_uint4(y.v[4], y.v[5], y.v[6], y.v[7]);
    }
    __device__ __forceinline__ void load(int k, Fe& x, Fe& y) const {
        if (k == 0) {
            x = x0;
            y = y0;
            return;
        }
        const uint4* p = base + (uint32_t)((k - 1) * 4) * stride;
        uint4 a = p[0], b = p[stride], c = p[2 * stride], d = p[3 * stride];
        x.v[0] = a.x; x.v[1] = a.y; x.v[2] = a.z; x.v[3] = a.w;
        x.v[4] = b.x; x.v[5] = b.y; x.v[6] = b.z; x.v[7] = b.w;
        y.v[0] = c.x; y.v[1] = c.y; y.v[2] = c.z; y.v[3] = c.w;
        y.v[4] = d.x; y.v[5] = d.y; y.v[6] = d.z; y.v[7] = d.w;
    }
};

struct GlobalGT {
    const uint4* __restrict__ p;
    __device__ __forceinline__ void load(int k, Fe& x, Fe& y) const {
        const uint4* q = p + 4 * k;
        uint4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2), d = __ldg(q + 3);
        x.v[0] = a.x; x.v[1] = a.y; x.v[2] = a.z; x.v[3] = a.w;
        x.v[4] = b.x; x.v[5] = b.y; x.v[6] = b.z; x.v[7] = b.w;
        y.v[0] = c.x; y.v[1] = c.y; y.v[2] = c.z; y.v[3] = c.w;
        y.v[4] = d.x; y.v[5] = d.y; y.v[6] = d.z; y.v[7] = d.w;
    }
};

__device__ __forceinline__ void load_words8(uint32_t w[8], const uint8_t* p) {
    const uint4* q = reinterpret_cast<const uint4*>(p);
    uint4 a = __ldg(q), b = __ldg(q + 1);
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
}

}  // namespace uf
