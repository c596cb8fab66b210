// Allocation-free entry point: mixed ECDSA / BIP-340 verification of
// device-resident batches with the work-queue kernel's scratch held in a
// file-scope device array instead of memory the library allocates.
//
// Who needs it: callers that cannot call cudaMalloc -- a host application
// whose GPU memory is owned by another allocator or framework, code running
// under a fixed device-memory budget, or integrations that forbid the
// verifier from allocating behind their back.  They pass inputs and outputs
// they already own (device-accessible pointers); this path allocates nothing.
//
// The scratch is kNoAllocScratchBytes (49,408 bytes) of static device memory:
// the queue head and a table of at most kNoAllocJobLimit job descriptors.  Every GPU that loads
// the library holds it until the process exits.  All calls share it and it
// keeps the last call's contents: the queue head is cleared on every call, and
// calls whose work overlaps on the GPU (different streams, or different host
// threads on one device) race on it and must be serialised by the caller.
//
// In host code `g_noalloc_scratch` is only a host-side stand-in for the symbol,
// not a device address; its device address is looked up once per device with
// cudaGetSymbolAddress (with that device current) on the first call on that
// device, so that first call should come before any stream capture.  The
// descriptor table is copied from a per-thread host staging array (pageable
// memory the library owns, not an allocation per call); cudaMemcpyAsync has
// staged those bytes when it returns, so the array is free for the next call
// on the thread without waiting for the stream.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>

#include "kernels.h"
#include "verify.cuh"
#include "dev_tables.cuh"

namespace uf {

struct NoAllocJob {
    const uint8_t* msgs;
    const uint8_t* pubs;
    const uint8_t* sigs;
    uint8_t* out;
    uint32_t kind;
    uint32_t count;
    uint32_t first;     // index of the job's first item in the concatenated item space
    uint32_t pad;
};

static_assert(sizeof(NoAllocJob) == kNoAllocJobBytes, "descriptor layout");
constexpr size_t kNoAllocHeader = kNoAllocHeaderBytes;   // queue head, job count, total items

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

__global__ void __launch_bounds__(kVerifyThreads)
k_verify_jobs_noalloc(uint8_t* scratch, const uint4* __restrict__ gt) {
    extern __shared__ uint4 smem_tab[];
    const SmemTab tab{smem_tab + threadIdx.x, blockDim.x};
    const GlobalGT g{gt};
    unsigned int* head = reinterpret_cast<unsigned int*>(scratch);
    const uint32_t n_jobs = reinterpret_cast<const uint32_t*>(scratch)[1];
    const uint32_t total = reinterpret_cast<const uint32_t*>(scratch)[2];
    const NoAllocJob* jobs = reinterpret_cast<const NoAllocJob*>(scratch + kNoAllocHeader);
    const uint32_t lane = threadIdx.x & 31u;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(head, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= total) break;
        const uint32_t i = base + lane;
        if (i >= total) continue;
        // job holding item i: last job with first <= i
        uint32_t lo = 0, hi = n_jobs - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (jobs[mid].first <= i) lo = mid;
            else hi = mid - 1;
        }
        const NoAllocJob J = jobs[lo];
        const uint32_t k = i - J.first;
        uint32_t mw[8], sw[16];
        load_words8(mw, J.msgs + 32ull * k);
        load_words8(sw, J.sigs + 64ull * k);
        load_words8(sw + 8, J.sigs + 64ull * k + 32);
        bool ok;
        if (J.kind == 0) {
            ok = ecdsa_verify_one(mw, J.pubs + 33ull * k, sw, tab, g);
        } else {
            uint32_t pw[8];
            load_words8(pw, J.pubs + 32ull * k);
            ok = schnorr_verify_one(mw, pw, sw, tab, g);
        }
        J.out[k] = ok ? 1 : 0;
    }
}

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {};   // device address of the scratch, per device ordinal
int g_noalloc_grid[64] = {};
}  // namespace

// Host part of the entry point.  `jobs` is the caller's host array of
// descriptors whose buffers are device-accessible; returns a cudaError_t, or
// cudaErrorInvalidValue (with *limit_hit set) when a limit is exceeded.
cudaError_t verify_jobs_noalloc(int device, const ufsecp_gpu_ext_job_t* jobs, size_t n_jobs, const void* d_gtab,
                                cudaStream_t s, int* limit_hit) {
    *limit_hit = 0;
    if (n_jobs > kNoAllocJobLimit) {
        *limit_hit = 1;
        return cudaErrorInvalidValue;
    }
    uint64_t total = 0;
    for (size_t j = 0; j < n_jobs; ++j) total += jobs[j].count;
    if (total > 0xFFFFFFE0ull) {
        *limit_hit = 2;
        return cudaErrorInvalidValue;
    }
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    void* addr;
    int grid;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[device]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return e;
            const size_t smem = kVerifyThreads * kVerifySmemPerThread;
            e = cudaFuncSetAttribute(k_verify_jobs_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            int blocks = 0, sms = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_verify_jobs_noalloc, kVerifyThreads, smem);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
            g_noalloc_grid[device] = (blocks > 0 ? blocks : 1) * (sms > 0 ? sms : 1);
            g_noalloc_addr[device] = p;
        }
        addr = g_noalloc_addr[device];
        grid = g_noalloc_grid[device];
    }
    if (total == 0) return cudaSuccess;
    // header + descriptor table, built straight into this thread's staging
    // array and copied in one piece
    alignas(16) static thread_local uint8_t staged[kNoAllocScratchBytes];
    memset(staged, 0, kNoAllocHeader);
    uint32_t* hdr = reinterpret_cast<uint32_t*>(staged);
    hdr[0] = 0;                        // queue head starts at zero on every call
    hdr[1] = (uint32_t)n_jobs;
    hdr[2] = (uint32_t)total;
    NoAllocJob* tab = reinterpret_cast<NoAllocJob*>(staged + kNoAllocHeader);
    uint32_t first = 0;
    for (size_t j = 0; j < n_jobs; ++j) {
        const ufsecp_gpu_ext_job_t& J = jobs[j];
        tab[j] = NoAllocJob{J.msg_hashes32, J.pubkeys, J.sigs64, J.out_results, J.kind, (uint32_t)J.count, first, 0};
        first += (uint32_t)J.count;
    }
    const size_t bytes = kNoAllocHeader + n_jobs * sizeof(NoAllocJob);
    cudaError_t e = cudaMemcpyAsync(addr, staged, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const int need = (int)((total + kVerifyThreads - 1) / kVerifyThreads);
        const int g = grid < need ? grid : need;
        const size_t smem = kVerifyThreads * kVerifySmemPerThread;
        k_verify_jobs_noalloc<<<g, kVerifyThreads, smem, s>>>(reinterpret_cast<uint8_t*>(addr),
                                                              reinterpret_cast<const uint4*>(d_gtab));
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        // fail closed: no verdict byte of this call may read as valid
        for (size_t j = 0; j < n_jobs; ++j)
            if (jobs[j].count && jobs[j].out_results) (void)cudaMemsetAsync(jobs[j].out_results, 0, jobs[j].count, s);
    }
    return e;
}

}  // namespace uf
