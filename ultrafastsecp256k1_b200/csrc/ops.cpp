// Host side of the per-item batch operations (kernels_ops.cu): one staging
// upload of every input array, one launch, one download, on the context's
// stream; synchronous like the reference's calls
// (src/gpu/src/gpu_backend_cuda.cu:1580-1740).
#include <cuda_runtime.h>
#include <string.h>

#include <initializer_list>
#include <utility>

#include "backend.h"
#include "kernels.h"

namespace uf {

namespace {

struct In {
    const void* p;
    size_t bytes;
};

size_t a256(size_t v) { return (v + 255) & ~size_t{255}; }

}  // namespace

// Uploads `ins` into ops_in_ (each 256-byte aligned), runs launch(device
// pointers, out) and downloads out_bytes into `out`.
template <class F>
static int run_op(Backend& be, DevBuf& in_buf, DevBuf& out_buf, std::initializer_list<In> ins, size_t out_bytes,
                  uint8_t* out, F&& launch) {
    cudaError_t e = cudaSetDevice(be.device());
    if (e != cudaSuccess) return be.cuda_error(e, "cudaSetDevice");
    size_t total = 0;
    for (const In& x : ins) total += a256(x.bytes);
    if ((e = in_buf.ensure(total + 256)) != cudaSuccess) return be.cuda_error(e, "cudaMalloc(op inputs)");
    if ((e = out_buf.ensure(out_bytes + 256)) != cudaSuccess) return be.cuda_error(e, "cudaMalloc(op outputs)");
    const uint8_t* dev[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t off = 0;
    int k = 0;
    const cudaStream_t s = be.stream();
    for (const In& x : ins) {
        uint8_t* d = (uint8_t*)in_buf.p + off;
        if ((e = cudaMemcpyAsync(d, x.p, x.bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return be.cuda_error(e, "host->device copy");
        dev[k++] = d;
        off += a256(x.bytes);
    }
    if ((e = launch(dev, (uint8_t*)out_buf.p, s)) != cudaSuccess) return be.cuda_error(e, "op launch");
    if ((e = cudaMemcpyAsync(out, out_buf.p, out_bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
        return be.cuda_error(e, "device->host copy");
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return be.cuda_error(e, "op");
    be.clear_error();
    return kOk;
}

int Backend::xonly_validate(const uint8_t* keys32, size_t n, uint8_t* out) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    return run_op(*this, ops_in_, out_, {{keys32, 32 * n}}, n, out, [&](const uint8_t** d, uint8_t* o, cudaStream_t s) {
        return launch_xonly_validate(d[0], (uint32_t)n, o, sms_, s);
    });
}

int Backend::pubkey_validate(const uint8_t* pubs33, size_t n, uint8_t* out) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    return run_op(*this, ops_in_, out_, {{pubs33, 33 * n}}, n, out, [&](const uint8_t** d, uint8_t* o, cudaStream_t s) {
        return launch_pubkey_validate(d[0], (uint32_t)n, o, sms_, s);
    });
}

int Backend::commitment_verify(const uint8_t* ix, const uint8_t* tw, const uint8_t* tx, const uint8_t* par, size_t n,
                               uint8_t* out) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    return run_op(*this, ops_in_, out_, {{ix, 32 * n}, {tw, 32 * n}, {tx, 32 * n}, {par, n}}, n, out,
                  [&](const uint8_t** d, uint8_t* o, cudaStream_t s) {
                      return launch_commitment_verify(d[0], d[1], d[2], d[3], (uint32_t)n, d_gtab_, o, sms_, s);
                  });
}

int Backend::tagged_hash(const uint8_t* tag_hash32, const uint8_t* msgs, const uint32_t* lens, size_t fixed_len,
                         size_t stride, size_t n, uint8_t* out32) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    if (lens) {
        for (size_t i = 0; i < n; ++i)
            if (lens[i] == 0 || lens[i] > stride)
                return set_error(kErrBadInput, "message length outside 1..stride");
        return run_op(*this, ops_in_, out_, {{msgs, stride * n}, {lens, 4 * n}}, 32 * n, out32,
                      [&](const uint8_t** d, uint8_t* o, cudaStream_t s) {
                          return launch_tagged_hash(tag_hash32, d[0], (const uint32_t*)d[1], 0, (uint32_t)stride,
                                                    (uint32_t)n, o, sms_, s);
                      });
    }
    return run_op(*this, ops_in_, out_, {{msgs, fixed_len * n}}, 32 * n, out32,
                  [&](const uint8_t** d, uint8_t* o, cudaStream_t s) {
                      return launch_tagged_hash(tag_hash32, d[0], nullptr, (uint32_t)fixed_len, (uint32_t)fixed_len,
                                                (uint32_t)n, o, sms_, s);
                  });
}

}  // namespace uf
