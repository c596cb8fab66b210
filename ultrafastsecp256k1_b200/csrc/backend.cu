// CUDA backend implementation (see backend.h).
#include "backend.h"

#include <algorithm>
#include <string.h>

#include "kernels.h"

namespace uf {

namespace {
// Items per host->device chunk: bounds device memory at ~130 B x 2^22 = 0.5 GB.
constexpr size_t kChunk = size_t{1} << 22;
}  // namespace

cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    release();
    size_t want = std::max(bytes, cap * 2);
    want = (want + 255) & ~size_t{255};
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        p = nullptr;
        cap = 0;
        (void)cudaGetLastError();
        return e;
    }
    cap = want;
    return cudaSuccess;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

Backend::~Backend() {
    if (dev_ >= 0) {
        cudaSetDevice(dev_);
        if (stream_) cudaStreamSynchronize(stream_);
        msgs_.release();
        pubs_.release();
        sigs_.release();
        out_.release();
        scratch_.release();
        if (d_gtab_) cudaFree(d_gtab_);
        if (stream_) cudaStreamDestroy(stream_);
    }
}

int Backend::set_error(int code, const char* what) {
    last_err_ = code;
    last_msg_ = what ? what : "";
    return code;
}

int Backend::cuda_error(cudaError_t e, const char* what) {
    int code = kErrGpuBackend;
    if (e == cudaErrorMemoryAllocation) code = kErrGpuMemory;
    else if (e == cudaErrorLaunchFailure || e == cudaErrorLaunchOutOfResources || e == cudaErrorInvalidConfiguration ||
             e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDeviceFunction)
        code = kErrGpuLaunch;
    else if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice) code = kErrGpuDevice;
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    (void)cudaGetLastError();
    return set_error(code, msg.c_str());
}

int Backend::init(int device_index) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        return set_error(kErrGpuUnavailable, "no CUDA device");
    }
    if (device_index < 0 || device_index >= count) return set_error(kErrGpuDevice, "device index out of range");
    dev_ = device_index;
    if ((e = cudaSetDevice(dev_)) != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, dev_)) != cudaSuccess) return cuda_error(e, "cudaGetDeviceProperties");
    if (prop.major < 10) return set_error(kErrGpuDevice, "this build targets sm_100a (B200)");
    sms_ = prop.multiProcessorCount;
    if ((e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_error(e, "cudaStreamCreate");
    if ((e = cudaMalloc(&d_gtab_, kGTableBytes)) != cudaSuccess) return cuda_error(e, "cudaMalloc(gtab)");
    if ((e = launch_gtable_init(d_gtab_, stream_)) != cudaSuccess) return cuda_error(e, "gtable init launch");
    if ((e = cudaStreamSynchronize(stream_)) != cudaSuccess) return cuda_error(e, "gtable init");
    grid_ecdsa_ = std::max(1, verify_blocks_per_sm(0)) * sms_;
    grid_schnorr_ = std::max(1, verify_blocks_per_sm(1)) * sms_;
    (void)cudaGetLastError();
    ready_ = true;
    clear_error();
    return kOk;
}

int Backend::verify_device(int kind, const uint8_t* d_msgs, const uint8_t* d_pubs, const uint8_t* d_sigs,
                           size_t count, uint8_t* d_out, cudaStream_t stream) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    if (count == 0) return kOk;
    if (count > 0xFFFFFFFFu) return set_error(kErrBadInput, "count too large");
    if (((uintptr_t)d_msgs | (uintptr_t)d_sigs | (kind == 1 ? (uintptr_t)d_pubs : 0)) & 15u)
        return set_error(kErrBadInput, "device inputs must be 16-byte aligned");
    cudaError_t e = cudaSetDevice(dev_);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    cudaStream_t s = stream ? stream : stream_;
    e = kind == 0 ? launch_ecdsa_verify(d_msgs, d_pubs, d_sigs, (uint32_t)count, d_gtab_, d_out, 0, grid_ecdsa_, s)
                  : launch_schnorr_verify(d_msgs, d_pubs, d_sigs, (uint32_t)count, d_gtab_, d_out, 0, grid_schnorr_, s);
    if (e != cudaSuccess) return cuda_error(e, "verify launch");
    clear_error();
    return kOk;
}

int Backend::verify_host(int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs, size_t count,
                         uint8_t* out, bool collect) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    if (count == 0) return kOk;
    cudaError_t e = cudaSetDevice(dev_);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    const size_t pub_sz = kind == 0 ? 33 : 32;
    const size_t chunk = std::min(count, kChunk);
    if ((e = msgs_.ensure(chunk * 32)) != cudaSuccess) return cuda_error(e, "cudaMalloc(msgs)");
    if ((e = pubs_.ensure(chunk * pub_sz)) != cudaSuccess) return cuda_error(e, "cudaMalloc(pubs)");
    if ((e = sigs_.ensure(chunk * 64)) != cudaSuccess) return cuda_error(e, "cudaMalloc(sigs)");
    if ((e = out_.ensure(chunk)) != cudaSuccess) return cuda_error(e, "cudaMalloc(out)");
    uint8_t* dm = (uint8_t*)msgs_.p;
    uint8_t* dp = (uint8_t*)pubs_.p;
    uint8_t* ds = (uint8_t*)sigs_.p;
    uint8_t* dout = (uint8_t*)out_.p;
    for (size_t off = 0; off < count; off += chunk) {
        const size_t m = std::min(chunk, count - off);
        if ((e = cudaMemcpyAsync(dm, msgs + off * 32, m * 32, cudaMemcpyHostToDevice, stream_)) != cudaSuccess ||
            (e = cudaMemcpyAsync(dp, pubs + off * pub_sz, m * pub_sz, cudaMemcpyHostToDevice, stream_)) != cudaSuccess ||
            (e = cudaMemcpyAsync(ds, sigs + off * 64, m * 64, cudaMemcpyHostToDevice, stream_)) != cudaSuccess)
            return cuda_error(e, "host->device copy");
        if (collect && (e = cudaMemcpyAsync(dout, out + off, m, cudaMemcpyHostToDevice, stream_)) != cudaSuccess)
            return cuda_error(e, "host->device copy");
        e = kind == 0 ? launch_ecdsa_verify(dm, dp, ds, (uint32_t)m, d_gtab_, dout, collect, grid_ecdsa_, stream_)
                      : launch_schnorr_verify(dm, dp, ds, (uint32_t)m, d_gtab_, dout, collect, grid_schnorr_, stream_);
        if (e != cudaSuccess) return cuda_error(e, "verify launch");
        if ((e = cudaMemcpyAsync(out + off, dout, m, cudaMemcpyDeviceToHost, stream_)) != cudaSuccess)
            return cuda_error(e, "device->host copy");
    }
    if ((e = cudaStreamSynchronize(stream_)) != cudaSuccess) return cuda_error(e, "verify");
    clear_error();
    return kOk;
}

int Backend::sign_device(int kind, const uint8_t* d_msgs, const uint8_t* d_sks, const uint8_t* d_auxs, size_t count,
                         uint8_t* d_pubs, uint8_t* d_sigs, uint8_t* d_ok, cudaStream_t stream) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    if (count == 0) return kOk;
    if (count > 0xFFFFFFFFu) return set_error(kErrBadInput, "count too large");
    cudaError_t e = cudaSetDevice(dev_);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    e = launch_sign(kind, d_msgs, d_sks, d_auxs, (uint32_t)count, d_gtab_, d_pubs, d_sigs, d_ok, sms_ * 16,
                    stream ? stream : stream_);
    if (e != cudaSuccess) return cuda_error(e, "sign launch");
    clear_error();
    return kOk;
}

int Backend::diag(uint32_t op, const uint8_t* in, size_t n, uint8_t* out, size_t in_sz, size_t out_sz) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    if (n == 0) return kOk;
    cudaError_t e = cudaSetDevice(dev_);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    if ((e = msgs_.ensure(n * in_sz + 16)) != cudaSuccess) return cuda_error(e, "cudaMalloc");
    if ((e = out_.ensure(n * out_sz + 16)) != cudaSuccess) return cuda_error(e, "cudaMalloc");
    if ((e = cudaMemcpyAsync(msgs_.p, in, n * in_sz, cudaMemcpyHostToDevice, stream_)) != cudaSuccess)
        return cuda_error(e, "copy");
    if ((e = launch_diag(op, (const uint8_t*)msgs_.p, (uint32_t)n, (uint8_t*)out_.p, d_gtab_, stream_)) != cudaSuccess)
        return cuda_error(e, "diag launch");
    if ((e = cudaMemcpyAsync(out, out_.p, n * out_sz, cudaMemcpyDeviceToHost, stream_)) != cudaSuccess)
        return cuda_error(e, "copy");
    if ((e = cudaStreamSynchronize(stream_)) != cudaSuccess) return cuda_error(e, "diag");
    clear_error();
    return kOk;
}

int Backend::imad_peak(double* ops_per_s) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    cudaError_t e = cudaSetDevice(dev_);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    if ((e = scratch_.ensure(4096 * sizeof(uint32_t))) != cudaSuccess) return cuda_error(e, "cudaMalloc");
    const int threads = 256, blocks = sms_ * 8, iters = 4096;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(a, stream_);
        e = launch_imad_peak((uint32_t*)scratch_.p, blocks, threads, iters, stream_);
        cudaEventRecord(b, stream_);
        if (e != cudaSuccess) break;
        if ((e = cudaEventSynchronize(b)) != cudaSuccess) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0) best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return cuda_error(e, "imad probe");
    *ops_per_s = (double)blocks * threads * iters * 16.0 / (best * 1e-3);
    clear_error();
    return kOk;
}

int Backend::probe(int op, int blocks, int threads, int iters, float* ms) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    cudaError_t e = cudaSetDevice(dev_);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    if ((e = scratch_.ensure(4096 * sizeof(uint32_t))) != cudaSuccess) return cuda_error(e, "cudaMalloc");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    e = launch_probe(op, blocks, threads, 1, (uint32_t*)scratch_.p, stream_);   // warm-up
    if (e == cudaSuccess) {
        cudaEventRecord(a, stream_);
        e = launch_probe(op, blocks, threads, iters, (uint32_t*)scratch_.p, stream_);
        cudaEventRecord(b, stream_);
    }
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    if (e == cudaSuccess) cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return cuda_error(e, "probe");
    clear_error();
    return kOk;
}

}  // namespace uf
