// CUDA backend of the C ABI: one device, its stream, the generator tables and
// grow-only staging buffers.
//
// Role in the reference: CudaBackend (src/gpu/src/gpu_backend_cuda.cu:833;
// ecdsa_verify_batch :972, schnorr_verify_batch :1085) behind the GpuBackend
// interface (src/gpu/include/gpu_backend.hpp:79-607).  Differences by design:
// device buffers are kept and grown instead of cudaMalloc/cudaFree per call,
// every launch goes to the context's own stream, and the kernels are the
// sm_100a ones of kernels.cu.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <algorithm>
#include <atomic>
#include <map>
#include <functional>
#include <memory>
#include <string>

namespace uf {

// ABI error codes (same values as ufsecp_error.h / ufsecp_gpu.h).
enum : int {
    kOk = 0, kErrNullArg = 1, kErrBadInput = 5, kErrInternal = 9, kErrCancelled = 13,
    kErrGpuUnavailable = 100, kErrGpuDevice = 101, kErrGpuLaunch = 102, kErrGpuMemory = 103,
    kErrGpuUnsupported = 104, kErrGpuBackend = 105, kErrGpuQueue = 106,
};

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

// Pinned (page-locked) host buffer, grow-only.
struct HostBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

struct VerifyJob;
class BatchSlot;
class RlcVerifier;
class PackPool;
class KeyTable;

class Backend {
public:
    Backend();
    ~Backend();
    Backend(const Backend&) = delete;
    Backend& operator=(const Backend&) = delete;

    int init(int device_index);
    bool ready() const { return ready_; }
    int last_error() const { return last_err_; }
    const char* last_error_msg() const { return last_msg_.c_str(); }
    int device() const { return dev_; }
    cudaStream_t stream() const { return stream_; }
    const void* gtab() const { return d_gtab_; }
    int sms() const { return sms_; }

    // Host buffers in, host verdicts out; synchronous (the reference contract).
    // kind 0 ECDSA (compact big-endian r || s, low-S), 1 BIP-340, 2 ECDSA with the
    // opaque little-endian signature layout (high-S accepted).
    int verify_host(int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs, size_t count,
                    uint8_t* out, bool collect);
    // The same with byte strides between consecutive items of each field (rows).
    int verify_host_strided(int kind, const uint8_t* msgs, size_t m_stride, const uint8_t* pubs, size_t p_stride,
                            const uint8_t* sigs, size_t s_stride, size_t count, uint8_t* out, bool collect);
    // Device buffers in / out, asynchronous on `stream` (nullptr = context stream).
    int verify_device(int kind, const uint8_t* d_msgs, const uint8_t* d_pubs, const uint8_t* d_sigs, size_t count,
                      uint8_t* d_out, cudaStream_t stream);
    // Batch signing (workload generator), device buffers, asynchronous.
    int sign_device(int kind, const uint8_t* d_msgs, const uint8_t* d_sks, const uint8_t* d_auxs, size_t count,
                    uint8_t* d_pubs, uint8_t* d_sigs, uint8_t* d_ok, cudaStream_t stream);
    // Mixed ECDSA / BIP-340 jobs (host buffers) in one persistent-queue launch;
    // synchronous.  Keys go through the context's resident key table when it
    // is on (set_key_table).  Kind 2 jobs (BIP-340 by RLC) are verified after
    // the others by the RLC verifier, all in one batch of `rlc_segment`-item
    // segments (0 = kRlcJobSegment), its weights seeded by the items' digest
    // XOR rand32.
    int verify_jobs(const VerifyJob* jobs, size_t n_jobs, uint32_t rlc_segment = 0,
                    const uint8_t* rand32 = nullptr);
    static constexpr uint32_t kRlcJobSegment = 16384;
    // Resident key table of verify_jobs: 0 = off, 8..24 = an empty table of
    // 2^log2 slots (the current table emptied in place when it has that size,
    // else a new one made on the next verify_jobs call).  The default is the
    // tuning file's key_table_log2, else UFSECP_B200_KEY_TABLE, else 18.
    int set_key_table(uint32_t log2);
    uint32_t key_table_log2() const { return key_log2_; }
    // The table itself once made (null before the first mixed-job call).
    const KeyTable* key_table() const { return keys_.get(); }
    // lookups, hits since the table was made; slots (0 = off / not made yet)
    int key_table_stats(uint64_t* lookups, uint64_t* hits, uint64_t* slots);
    // RLC batch verifier of BIP-340 signatures (created on first use).
    RlcVerifier& rlc();
    // Pippenger window bits for an RLC segment of `len` items: the tuned value
    // of the nearest tuned batch size (tuning file lines "rlc_window_<n> <c>"),
    // else the cost model.
    int rlc_window(uint32_t len) const;
    // Bucket points summed by one RLC chunk thread for segments of `len`
    // items: the fixed override if set, else the value of the nearest tuned
    // batch size (tuning file lines "rlc_chunk_<n> <points>"), else 16.
    uint32_t rlc_chunk(uint32_t len) const;
    // 2..256 fixes the chunk for every segment length; 0 restores the tuned values.
    int set_rlc_chunk(uint32_t chunk);
    // Whether a failing RLC segment first gets a locate round (one more MSM
    // that finds a single invalid item) before it is bisected.  On by default;
    // the tuning file's rlc_locate or UFSECP_B200_RLC_LOCATE may turn it off.
    bool rlc_locate() const { return rlc_locate_; }
    void set_rlc_locate(bool on) { rlc_locate_ = on; }
    // Whether RLC bucket chunks (of at most 16 points) are summed by affine
    // pairwise trees with grid-shared inversions (k_aff_fwd / k_aff_bwd)
    // instead of mixed Jacobian additions (k_rlc_chunks).  On by default; the
    // tuning file's rlc_affine or UFSECP_B200_RLC_AFFINE may turn it off.
    bool rlc_affine() const { return rlc_affine_; }
    void set_rlc_affine(bool on) { rlc_affine_ = on; }
    int queue_grid() const { return queue_grid_; }
    int queue_pair_grid() const { return queue_pair_grid_; }
    // Mixed-job launches of at most this many items (both kinds together) run
    // the two-lane queue kernels: the smaller of the kinds' two-lane limits.
    uint32_t queue_pair_items() const { return std::min(pair_items_[0], pair_items_[1]); }
    // Per-item batch operations (ops.cpp): host buffers, synchronous.
    int xonly_validate(const uint8_t* keys32, size_t n, uint8_t* out);
    int pubkey_validate(const uint8_t* pubs33, size_t n, uint8_t* out);
    int commitment_verify(const uint8_t* internal_x, const uint8_t* tweak, const uint8_t* tweaked_x,
                          const uint8_t* parity, size_t n, uint8_t* out);
    // lens == nullptr: fixed_len bytes per message, else lens[i] (each <= stride).
    int tagged_hash(const uint8_t* tag_hash32, const uint8_t* msgs, const uint32_t* lens, size_t fixed_len,
                    size_t stride, size_t n, uint8_t* out32);
    int diag(uint32_t op, const uint8_t* in, size_t n, uint8_t* out, size_t in_sz, size_t out_sz);
    int imad_peak(double* ops_per_s);
    int probe(int op, int blocks, int threads, int iters, float* ms);

    // Kernel variant per signature kind (0 ECDSA, 1 BIP-340) and its grid.
    int variant(int kind) const { return variant_[kind & 1]; }
    int small_variant(int kind) const { return small_variant_[kind & 1]; }
    uint32_t small_items(int kind) const { return small_items_[kind & 1]; }
    int set_variant(int kind, int v);
    int set_small_variant(int kind, int v, uint32_t items);   // v = -1: none
    int set_lanes(int kind, int lanes, uint32_t items);       // lanes 2 for calls of <= items, 1: never
    // Inversion group per kind: 1 = every signature inverts alone (the
    // variant kernels), 64 / 128 = the block-wide batch-inversion kernels with
    // that many threads per block share each inversion.  Applies to the main
    // launches (not the two-lane or small-launch paths).  set_variant resets
    // it to 1.
    int set_inversion_group(int kind, int group);
    int inversion_group(int kind) const { return inv_group_[kind & 1]; }
    uint32_t pair_items(int kind) const { return pair_items_[kind & 1]; }
    int verify_grid(int kind) const { return grid_[variant_[kind & 1]][kind & 1]; }
    int blocks_per_sm(int kind, int v) const { return sms_ ? grid_[v][kind & 1] / sms_ : 0; }

    int set_error(int code, const char* what);
    int cuda_error(cudaError_t e, const char* what);

    // Host-side fault injection, for the fail-closed tests: once armed, the
    // (after + 1)-th fault point this context crosses fails as kind says --
    // 1: a CUDA call returned cudaErrorMemoryAllocation, 2: a launch returned
    // cudaErrorLaunchFailure, 3: std::bad_alloc is thrown -- and the injector
    // disarms itself; kind 0 disarms.  Fault points: each chunk launch of the
    // host-buffer verify, each device-buffer verify call, each mixed-job /
    // served launch (BatchSlot::enqueue) and each RLC round.  Nothing reaches
    // the device: the failing call is not made.
    void arm_fault(uint32_t after, int kind) {
        fault_after_.store((long long)after);
        fault_kind_.store(kind);
    }
    int fault_point(const char* where);
    void clear_error() { last_err_ = kOk; last_msg_ = "OK"; }

private:
    bool ready_ = false;
    int dev_ = -1;
    int sms_ = 0;
    std::string dev_name_;
    int grid_[12][2] = {};       // [variant][kind] resident-grid size
    void* gtab_w_[32] = {};      // generator tables of other window widths (window variants), by bits
    const void* gtab_for(int v) const;
    int ensure_variant_tables(int v);
    int variant_[2] = {4, 4};    // chosen variant per kind (4: out-of-line field / point ops, PTX chains)
    // Verify calls of at most small_items_[kind] items (latency-bound: a few
    // warps per SM) use small_variant_[kind] instead, when the tuning names
    // one; an explicit set_variant / environment override clears it.
    int small_variant_[2] = {-1, -1};
    uint32_t small_items_[2] = {0, 0};
    // Calls of at most pair_items_[kind] items (kinds 0 and 1) run two lanes
    // per signature (kernels_pair.cu); 0 = never.  Also cleared by an explicit
    // variant choice.
    uint32_t pair_items_[2] = {0, 0};
    int inv_group_[2] = {1, 1};
    int grp_grid_[2][2] = {};    // [64, 128][kind] resident-grid size of the batch-inversion kernels
    // call_items: the size of the whole call this launch belongs to; the
    // small-launch variant is used only when the whole call is small (the
    // chunks of a large call run beside one another at full occupancy).
    cudaError_t launch_verify(int kind, const uint8_t* m, const uint8_t* p, const uint8_t* s, uint32_t n,
                              uint8_t* out, int collect, cudaStream_t st, size_t call_items);
    void load_tuning();
    cudaStream_t stream_ = nullptr;
    void* d_gtab_ = nullptr;
    DevBuf msgs_, pubs_, sigs_, out_, scratch_, ops_in_;
    // host-buffer calls: kPipeSlots pinned staging slots, each with its own
    // stream, so that the CPU packs chunk k + 2 while the device verifies
    // chunks k and k + 1 (the next launch is always queued behind the running
    // ones, and their last partial waves overlap)
    static constexpr int kPipeSlots = 3;
    HostBuf pstage_[kPipeSlots];
    DevBuf dstage_[kPipeSlots];
    cudaStream_t pstream_[kPipeSlots] = {};
    cudaEvent_t pev_[kPipeSlots] = {};
    // threads that copy one chunk into its staging slot (the caller and
    // pack_threads_ - 1 helpers; by core count, or UFSECP_B200_PACK_THREADS),
    // made on first use
    int pack_threads_ = 1;
    std::unique_ptr<PackPool> pack_pool_;
    // large device-buffer calls: second stream with fork / join events
    cudaStream_t dstream_ = nullptr;
    cudaEvent_t dfork_ = nullptr, djoin_ = nullptr;
    int queue_grid_ = 0;
    int queue_pair_grid_ = 0;
    std::unique_ptr<BatchSlot> batch_[2];   // slots of the synchronous mixed-batch call (two for large calls)
    std::unique_ptr<KeyTable> keys_;        // resident key table of verify_jobs (made on first use)
    int verify_queue_jobs(const VerifyJob* jobs, size_t n_jobs);   // kinds 0 and 1

public:
    // fn(lo, hi) over [0, n) split between the staging-copy threads (the
    // caller included) when n is large enough to pay for them.
    void parallel_copy(size_t n, const std::function<void(size_t, size_t)>& fn);

private:
    uint32_t key_log2_ = 18;
    std::unique_ptr<RlcVerifier> rlc_;
    std::map<uint32_t, int> rlc_window_;   // tuned window bits per RLC batch size
    std::map<uint32_t, uint32_t> rlc_chunk_;  // tuned bucket points per chunk thread per RLC batch size
    uint32_t rlc_chunk_fixed_ = 0;            // set_rlc_chunk / UFSECP_B200_RLC_CHUNK override, 0 = tuned
    bool rlc_locate_ = true;
    bool rlc_affine_ = true;
    int last_err_ = kOk;
    std::string last_msg_ = "OK";
    std::atomic<long long> fault_after_{-1};
    std::atomic<int> fault_kind_{0};
};

}  // namespace uf
