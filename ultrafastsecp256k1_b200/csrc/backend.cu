// CUDA backend implementation (see backend.h).
#include "backend.h"

#include <dlfcn.h>

#include <algorithm>
#include <new>
#include <thread>
#include <vector>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "batch.h"
#include "keytable.h"
#include "kernels.h"
#include "pack_pool.h"
#include "rlc.h"
#include "nvtx.h"

namespace uf {

namespace {
// Items per host->device chunk: bounds device memory at ~130 B x 2^22 = 0.5 GB.
constexpr size_t kPipeChunk = size_t{1} << 17;   // items per staging slot of a host-buffer call
constexpr size_t kPipeFirst = size_t{1} << 14;   // items in a host-buffer call's first chunk
constexpr size_t kJobsPipeItems = size_t{1} << 16;   // most items per sub-call of a large mixed-job call
constexpr size_t kPackSplitItems = size_t{1} << 13;  // chunks at least this large are packed by the pool
constexpr size_t kDeviceChunk = size_t{1} << 17; // items per launch of a large device-buffer call

const verify_launcher kLaunchers[kVerifyVariants] = {launch_verify_v0, launch_verify_v1, launch_verify_v2,
                                                     launch_verify_v3, launch_verify_v4, launch_verify_v5,
                                                     launch_verify_v6, launch_verify_v7, launch_verify_v8,
                                                     launch_verify_v9, launch_verify_v10, launch_verify_v11};
const verify_occupancy_fn kOccupancy[kVerifyVariants] = {verify_occupancy_v0, verify_occupancy_v1,
                                                         verify_occupancy_v2, verify_occupancy_v3,
                                                         verify_occupancy_v4, verify_occupancy_v5,
                                                         verify_occupancy_v6, verify_occupancy_v7,
                                                         verify_occupancy_v8, verify_occupancy_v9,
                                                         verify_occupancy_v10, verify_occupancy_v11};

int env_int(const char* name, int dflt) {
    const char* v = getenv(name);
    return (v && *v) ? atoi(v) : dflt;
}
}  // namespace

cudaError_t Backend::launch_verify(int kind, const uint8_t* m, const uint8_t* p, const uint8_t* s, uint32_t n,
                                   uint8_t* out, int collect, cudaStream_t st, size_t call_items) {
    const int k = kind & 1;
    if (kind != 2 && call_items <= pair_items_[k])
        return launch_verify_pair(kind, m, p, s, n, d_gtab_, out, collect, st);
    const bool small = small_variant_[k] >= 0 && call_items <= small_items_[k];
    if (!small && inv_group_[k] > 1) {
        const int gi = inv_group_[k] == 64 ? 0 : 1;
        return launch_verify_grp(inv_group_[k], kind, m, p, s, n, d_gtab_, out, collect, grp_grid_[gi][k], st);
    }
    const int v = small ? small_variant_[k] : variant_[k];
    return kLaunchers[v](kind, m, p, s, n, gtab_for(v), out, collect, grid_[v][k], st);
}

const void* Backend::gtab_for(int v) const {
    const int w = kVariantGWin[v];
    return w == UF_GWIN ? d_gtab_ : gtab_w_[w];
}

int Backend::ensure_variant_tables(int v) {
    const int w = kVariantGWin[v];
    if (w == UF_GWIN || gtab_w_[w]) return kOk;
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, (size_t)64 << w);
    if (e == cudaSuccess) e = launch_gtable_init_w(p, w, stream_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
    if (e != cudaSuccess) {
        if (p) cudaFree(p);
        return cuda_error(e, "generator tables of a window variant");
    }
    gtab_w_[w] = p;
    return kOk;
}

int Backend::set_inversion_group(int kind, int group) {
    if (kind < 0 || kind > 1 || (group != 1 && group != 64 && group != 128))
        return set_error(kErrBadInput, "inversion group must be 1, 64 or 128");
    inv_group_[kind] = group;
    clear_error();
    return kOk;
}

int Backend::set_variant(int kind, int v) {
    if (kind < 0 || kind > 1 || v < 0 || v >= kVerifyVariants) return set_error(kErrBadInput, "bad variant");
    if (const int rc = ensure_variant_tables(v)) return rc;
    variant_[kind] = v;
    small_variant_[kind] = -1;   // an explicit choice applies to every launch size
    pair_items_[kind] = 0;
    inv_group_[kind] = 1;
    clear_error();
    return kOk;
}

int Backend::set_lanes(int kind, int lanes, uint32_t items) {
    if (kind < 0 || kind > 1 || lanes < 1 || lanes > 2) return set_error(kErrBadInput, "bad lanes");
    pair_items_[kind] = lanes == 2 ? items : 0;
    clear_error();
    return kOk;
}

int Backend::set_small_variant(int kind, int v, uint32_t items) {
    if (kind < 0 || kind > 1 || v < -1 || v >= kVerifyVariants) return set_error(kErrBadInput, "bad variant");
    if (v >= 0)
        if (const int rc = ensure_variant_tables(v)) return rc;
    small_variant_[kind] = v;
    small_items_[kind] = v >= 0 ? items : 0;
    clear_error();
    return kOk;
}

// Per-device tuning: a file of "key value" lines (ecdsa_variant,
// schnorr_variant, their small-launch counterparts ecdsa_small_variant /
// ecdsa_small_items and schnorr_small_variant / schnorr_small_items, the
// two-lane limits ecdsa_pair_items / schnorr_pair_items, and
// rlc_window_<batch>) written by ultrafastsecp256k1_b200.autotune.  It is the
// file named by UFSECP_B200_TUNING, else tuning/<device name>_<SMs>sm.txt
// beside the library's lib/ directory.  UFSECP_B200_VARIANT_ECDSA / _SCHNORR
// override a kind's variant for every launch size.
void Backend::load_tuning() {
    std::string path_s;
    const char* env = getenv("UFSECP_B200_TUNING");
    if (env && *env) {
        path_s = env;
    } else {
        Dl_info info;
        if (dladdr((void*)&launch_verify_v0, &info) && info.dli_fname) {
            std::string lib = info.dli_fname;
            const size_t slash = lib.rfind('/');
            const std::string dir = slash == std::string::npos ? std::string(".") : lib.substr(0, slash);
            std::string name;
            bool sep = false;
            for (const char* c = dev_name_.c_str(); *c; ++c) {
                const bool alnum = (*c >= 'a' && *c <= 'z') || (*c >= 'A' && *c <= 'Z') || (*c >= '0' && *c <= '9');
                if (alnum) {
                    if (sep && !name.empty()) name += '_';
                    name += *c;
                    sep = false;
                } else {
                    sep = true;
                }
            }
            path_s = dir + "/../tuning/" + name + "_" + std::to_string(sms_) + "sm.txt";
        }
    }
    const char* path = path_s.c_str();
    if (*path) {
        FILE* f = fopen(path, "r");
        if (f) {
            char key[64];
            int val;
            while (fscanf(f, "%63s %d", key, &val) == 2) {
                if (!strcmp(key, "ecdsa_variant") && val >= 0 && val < kVerifyVariants) variant_[0] = val;
                if (!strcmp(key, "schnorr_variant") && val >= 0 && val < kVerifyVariants) variant_[1] = val;
                if (!strcmp(key, "ecdsa_small_variant") && val >= 0 && val < kVerifyVariants) small_variant_[0] = val;
                if (!strcmp(key, "schnorr_small_variant") && val >= 0 && val < kVerifyVariants)
                    small_variant_[1] = val;
                if (!strcmp(key, "ecdsa_small_items") && val > 0) small_items_[0] = (uint32_t)val;
                if (!strcmp(key, "schnorr_small_items") && val > 0) small_items_[1] = (uint32_t)val;
                if (!strcmp(key, "ecdsa_pair_items") && val >= 0) pair_items_[0] = (uint32_t)val;
                if (!strcmp(key, "schnorr_pair_items") && val >= 0) pair_items_[1] = (uint32_t)val;
                unsigned size = 0;
                if (sscanf(key, "rlc_window_%u", &size) == 1 && size > 0 && val >= 4 && val <= 16)
                    rlc_window_[size] = val;
                if (sscanf(key, "rlc_chunk_%u", &size) == 1 && size > 0 && val >= 2 && val <= 256)
                    rlc_chunk_[size] = (uint32_t)val;
                if (!strcmp(key, "key_table_log2") && (val == 0 || (val >= 8 && val <= 24)))
                    key_log2_ = (uint32_t)val;
                if (!strcmp(key, "rlc_locate") && (val == 0 || val == 1)) rlc_locate_ = val != 0;
                if (!strcmp(key, "rlc_affine") && (val == 0 || val == 1)) rlc_affine_ = val != 0;
                if (!strcmp(key, "ecdsa_inv_group") && (val == 1 || val == 64 || val == 128)) inv_group_[0] = val;
                if (!strcmp(key, "schnorr_inv_group") && (val == 1 || val == 64 || val == 128)) inv_group_[1] = val;
            }
            fclose(f);
        }
    }
    // staging copies: 4 threads on hosts of 8+ cores (one core's memcpy rate is
    // near what the device consumes at full speed), 2 on 4+ cores
    const unsigned hw = std::thread::hardware_concurrency();
    pack_threads_ = hw >= 8 ? 4 : (hw >= 4 ? 2 : 1);
    const int kt = env_int("UFSECP_B200_KEY_TABLE", -1);
    if (kt == 0 || (kt >= 8 && kt <= 24)) key_log2_ = (uint32_t)kt;
    const int pt = env_int("UFSECP_B200_PACK_THREADS", 0);
    if (pt >= 1 && pt <= 16) pack_threads_ = pt;
    const int lo_env = env_int("UFSECP_B200_RLC_LOCATE", -1);
    if (lo_env == 0 || lo_env == 1) rlc_locate_ = lo_env != 0;
    const int af_env = env_int("UFSECP_B200_RLC_AFFINE", -1);
    if (af_env == 0 || af_env == 1) rlc_affine_ = af_env != 0;
    const int rc_env = env_int("UFSECP_B200_RLC_CHUNK", 0);
    if (rc_env >= 2 && rc_env <= 256) rlc_chunk_fixed_ = (uint32_t)rc_env;
    const int ve = env_int("UFSECP_B200_VARIANT_ECDSA", -1), vs = env_int("UFSECP_B200_VARIANT_SCHNORR", -1);
    if (ve >= 0 && ve < kVerifyVariants) {
        variant_[0] = ve;
        small_variant_[0] = -1;
        pair_items_[0] = 0;
        inv_group_[0] = 1;
    }
    if (vs >= 0 && vs < kVerifyVariants) {
        variant_[1] = vs;
        small_variant_[1] = -1;
        pair_items_[1] = 0;
        inv_group_[1] = 1;
    }
    const int ig = env_int("UFSECP_B200_INV_GROUP", 0);
    if (ig == 1 || ig == 64 || ig == 128) inv_group_[0] = inv_group_[1] = ig;
}

cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    // grow by at least half the current size, so that slowly rising requests
    // do not reallocate on every call
    size_t want = std::max(bytes, cap + cap / 2);
    want = (want + 255) & ~size_t{255};
    release();
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

Backend::Backend() = default;

int Backend::rlc_window(uint32_t len) const {
    // the tuned batch size nearest in log scale, else the cost model
    if (rlc_window_.empty() || len == 0) return rlc_window_bits(len);
    int best = 0;
    double dist = 1e300;
    for (const auto& kv : rlc_window_) {
        const double d = fabs(log2((double)kv.first) - log2((double)len));
        if (d < dist) {
            dist = d;
            best = kv.second;
        }
    }
    return best;
}

uint32_t Backend::rlc_chunk(uint32_t len) const {
    // a fixed override, else the tuned batch size nearest in log scale
    if (rlc_chunk_fixed_) return rlc_chunk_fixed_;
    if (rlc_chunk_.empty() || len == 0) return RlcVerifier::kChunk;
    uint32_t best = RlcVerifier::kChunk;
    double dist = 1e300;
    for (const auto& kv : rlc_chunk_) {
        const double d = fabs(log2((double)kv.first) - log2((double)len));
        if (d < dist) {
            dist = d;
            best = kv.second;
        }
    }
    return best;
}

int Backend::set_rlc_chunk(uint32_t chunk) {
    if (chunk != 0 && (chunk < 2 || chunk > 256)) return set_error(kErrBadInput, "RLC chunk must be 0 or 2..256");
    rlc_chunk_fixed_ = chunk;
    return kOk;
}

RlcVerifier& Backend::rlc() {
    if (!rlc_) rlc_.reset(new RlcVerifier(this));
    return *rlc_;
}

Backend::~Backend() {
    batch_[0].reset();
    batch_[1].reset();
    keys_.reset();
    if (dev_ >= 0) cudaSetDevice(dev_);
    rlc_.reset();
    if (dev_ >= 0) {
        cudaSetDevice(dev_);
        if (stream_) cudaStreamSynchronize(stream_);
        msgs_.release();
        pubs_.release();
        sigs_.release();
        out_.release();
        ops_in_.release();
        scratch_.release();
        if (dstream_) {
            cudaStreamSynchronize(dstream_);
            cudaEventDestroy(dfork_);
            cudaEventDestroy(djoin_);
            cudaStreamDestroy(dstream_);
        }
        for (int j = 0; j < kPipeSlots; ++j) {
            if (pstream_[j]) cudaStreamSynchronize(pstream_[j]);
            pstage_[j].release();
            dstage_[j].release();
            if (pev_[j]) cudaEventDestroy(pev_[j]);
            if (pstream_[j]) cudaStreamDestroy(pstream_[j]);
        }
        if (d_gtab_) cudaFree(d_gtab_);
        for (void*& t : gtab_w_)
            if (t) cudaFree(t);
        if (stream_) cudaStreamDestroy(stream_);
    }
}

int Backend::fault_point(const char* where) {
    if (fault_kind_.load(std::memory_order_relaxed) == 0) return kOk;
    if (fault_after_.fetch_sub(1) != 0) return kOk;
    const int kind = fault_kind_.exchange(0);
    if (kind == 3) throw std::bad_alloc();
    if (kind == 1) return cuda_error(cudaErrorMemoryAllocation, where);
    if (kind == 2) return cuda_error(cudaErrorLaunchFailure, where);
    return kOk;
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
    dev_name_ = prop.name;
    if ((e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_error(e, "cudaStreamCreate");
    if ((e = cudaMalloc(&d_gtab_, kGTableBytes)) != cudaSuccess) return cuda_error(e, "cudaMalloc(gtab)");
    if ((e = launch_gtable_init(d_gtab_, stream_)) != cudaSuccess) return cuda_error(e, "gtable init launch");
    if ((e = cudaStreamSynchronize(stream_)) != cudaSuccess) return cuda_error(e, "gtable init");
    for (int v = 0; v < kVerifyVariants; ++v)
        for (int k = 0; k < 2; ++k) grid_[v][k] = std::max(1, kOccupancy[v](k)) * sms_;
    queue_grid_ = std::max(1, verify_queue_occupancy()) * sms_;
    for (int gi = 0; gi < 2; ++gi)
        for (int k = 0; k < 2; ++k) grp_grid_[gi][k] = std::max(1, verify_grp_occupancy(gi ? 128 : 64, k)) * sms_;
    queue_pair_grid_ = std::max(1, verify_pair_occupancy()) * sms_;   // also the two-lane kernels' shared-memory opt-in
    load_tuning();
    // generator tables of the window widths the chosen variants use; a variant
    // whose tables cannot be made falls back to variant 4
    for (int k = 0; k < 2; ++k) {
        if (ensure_variant_tables(variant_[k]) != kOk) variant_[k] = 4;
        if (small_variant_[k] >= 0 && ensure_variant_tables(small_variant_[k]) != kOk) small_variant_[k] = -1;
    }
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
    if (count < 2 * kDeviceChunk) {
        e = launch_verify(kind, d_msgs, d_pubs, d_sigs, (uint32_t)count, d_out, 0, s, count);
        if (e != cudaSuccess) return cuda_error(e, "verify launch");
        clear_error();
        return kOk;
    }
    // Large calls: chunks of kDeviceChunk alternate between the caller's stream
    // and a second stream forked from it and joined back, so that one chunk's
    // tail (its last, partly filled wave of signatures) overlaps the next
    // chunk's start.  Completion is still ordered on the caller's stream.
    if (!dstream_) {
        if ((e = cudaStreamCreateWithFlags(&dstream_, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&dfork_, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&djoin_, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_error(e, "device-call streams");
    }
    if ((e = cudaEventRecord(dfork_, s)) != cudaSuccess || (e = cudaStreamWaitEvent(dstream_, dfork_, 0)) != cudaSuccess)
        return cuda_error(e, "fork");
    const size_t pub_sz = kind == 1 ? 32 : 33;
    if (const int rc = fault_point("verify launch")) return rc;
    size_t k = 0;
    for (size_t off = 0; off < count; off += kDeviceChunk, ++k) {
        const size_t m = std::min(kDeviceChunk, count - off);
        e = launch_verify(kind, d_msgs + 32 * off, d_pubs + pub_sz * off, d_sigs + 64 * off, (uint32_t)m, d_out + off,
                          0, (k & 1) ? dstream_ : s, count);
        if (e != cudaSuccess) return cuda_error(e, "verify launch");
    }
    if ((e = cudaEventRecord(djoin_, dstream_)) != cudaSuccess || (e = cudaStreamWaitEvent(s, djoin_, 0)) != cudaSuccess)
        return cuda_error(e, "join");
    clear_error();
    return kOk;
}

int Backend::verify_host(int kind, const uint8_t* msgs, const uint8_t* pubs, const uint8_t* sigs, size_t count,
                         uint8_t* out, bool collect) {
    return verify_host_strided(kind, msgs, 32, pubs, kind == 1 ? 32 : 33, sigs, 64, count, out, collect);
}

int Backend::verify_host_strided(int kind, const uint8_t* msgs, size_t m_stride, const uint8_t* pubs,
                                 size_t p_stride, const uint8_t* sigs, size_t s_stride, size_t count, uint8_t* out,
                                 bool collect) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    if (count == 0) return kOk;
    NvtxRange range("ufsecp verify (host buffers)");
    cudaError_t e = cudaSetDevice(dev_);
    if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
    if (!pstream_[0]) {
        for (int j = 0; j < kPipeSlots && e == cudaSuccess; ++j) {
            e = cudaStreamCreateWithFlags(&pstream_[j], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pev_[j], cudaEventDisableTiming);
        }
        if (e != cudaSuccess) return cuda_error(e, "pipeline streams");
    }
    // Chunks of up to kPipeChunk items rotate through kPipeSlots pinned
    // staging slots: the CPU packs chunk k + 2 (and unpacks chunk k - 1's
    // verdicts) while the device copies in and verifies chunks k and k + 1.  Per chunk the slot is
    // laid out msgs | keys | sigs (16-byte aligned) | verdicts, copied in and
    // out with one transfer each way.
    const size_t pub_sz = kind == 1 ? 32 : 33;
    const size_t sub = std::min(count, kPipeChunk);
    auto a16 = [](size_t v) { return (v + 15) & ~size_t{15}; };
    const size_t slot_bytes = a16(sub * (32 + pub_sz)) + sub * 64 + sub + 16;
    const int slots = count > kPipeFirst ? kPipeSlots : 1;   // chunks of the ramp below use every slot
    for (int j = 0; j < slots; ++j) {
        if ((e = pstage_[j].ensure(slot_bytes)) != cudaSuccess) return cuda_error(e, "cudaHostAlloc(staging)");
        if ((e = dstage_[j].ensure(slot_bytes)) != cudaSuccess) return cuda_error(e, "cudaMalloc(staging)");
    }
    size_t pend_off[kPipeSlots] = {}, pend_n[kPipeSlots] = {}, pend_out[kPipeSlots] = {};
    auto drain = [&](int j) -> cudaError_t {
        if (!pend_n[j]) return cudaSuccess;
        const cudaError_t r = cudaEventSynchronize(pev_[j]);
        if (r == cudaSuccess) memcpy(out + pend_off[j], (const uint8_t*)pstage_[j].p + pend_out[j], pend_n[j]);
        pend_n[j] = 0;
        return r;
    };
    // Chunk sizes ramp up from kPipeFirst, doubling to kPipeChunk: the
    // pipeline's fill (packing and copying the first chunk while the device
    // is idle) costs a small chunk, and the device fills up while the CPU
    // packs the next, larger ones.
    // every early return waits for the slots' streams first, so that no copy
    // of this call is still in flight when the next call packs a slot
    auto fail = [&](int rc) {
        for (int q = 0; q < kPipeSlots; ++q)
            if (pstream_[q]) (void)cudaStreamSynchronize(pstream_[q]);
        (void)cudaGetLastError();
        return rc;
    };
    size_t k = 0, m = 0;
    for (size_t off = 0; off < count; off += m, ++k) {
        const int j = (int)(k % kPipeSlots);
        if ((e = drain(j)) != cudaSuccess) return fail(cuda_error(e, "verify"));
        if (const int rc = fault_point("verify launch")) return fail(rc);
        m = std::min(std::min(sub, kPipeFirst << std::min<size_t>(k, 20)), count - off);
        const size_t o_p = m * 32, o_s = a16(o_p + m * pub_sz), o_o = o_s + m * 64;
        uint8_t* h = (uint8_t*)pstage_[j].p;
        uint8_t* d = (uint8_t*)dstage_[j].p;
        // items [lo, hi) of this chunk into the slot
        auto pack = [&](size_t lo, size_t hi) {
            auto one = [&](uint8_t* dst, const uint8_t* src, size_t width, size_t stride) {
                if (stride == width) {
                    memcpy(dst + lo * width, src + (off + lo) * width, (hi - lo) * width);
                } else {
                    for (size_t i = lo; i < hi; ++i) memcpy(dst + i * width, src + (off + i) * stride, width);
                }
            };
            one(h, msgs, 32, m_stride);
            one(h + o_p, pubs, pub_sz, p_stride);
            one(h + o_s, sigs, 64, s_stride);
        };
        NvtxRange pack_range("pack chunk");
        if (pack_threads_ > 1 && m >= kPackSplitItems) {
            if (!pack_pool_) pack_pool_.reset(new PackPool(pack_threads_));
            const int parts = pack_pool_->threads();
            pack_pool_->run(parts, [&](int p) { pack(m * p / parts, m * (p + 1) / parts); });
        } else {
            pack(0, m);
        }
        if (collect) memcpy(h + o_o, out + off, m);
        const size_t in_bytes = o_o + (collect ? m : 0);
        if ((e = cudaMemcpyAsync(d, h, in_bytes, cudaMemcpyHostToDevice, pstream_[j])) != cudaSuccess)
            return fail(cuda_error(e, "host->device copy"));
        e = launch_verify(kind, d, d + o_p, d + o_s, (uint32_t)m, d + o_o, collect, pstream_[j], count);
        if (e != cudaSuccess) return fail(cuda_error(e, "verify launch"));
        if ((e = cudaMemcpyAsync(h + o_o, d + o_o, m, cudaMemcpyDeviceToHost, pstream_[j])) != cudaSuccess)
            return fail(cuda_error(e, "device->host copy"));
        if ((e = cudaEventRecord(pev_[j], pstream_[j])) != cudaSuccess) return fail(cuda_error(e, "event record"));
        pend_off[j] = off;
        pend_n[j] = m;
        pend_out[j] = o_o;
    }
    for (int j = 0; j < kPipeSlots; ++j)
        if ((e = drain(j)) != cudaSuccess) return fail(cuda_error(e, "verify"));
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

int Backend::set_key_table(uint32_t log2) {
    if (log2 != 0 && (log2 < KeyTable::kMinLog2 || log2 > KeyTable::kMaxLog2))
        return set_error(kErrBadInput, "key table: log2 slots must be 0 or 8..24");
    if (keys_ && keys_->on() && log2 == key_log2_) {
        // same size: empty the table in place (the batch slots and their graphs stay)
        cudaError_t e = keys_->clear(stream_);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
        if (e != cudaSuccess) return cuda_error(e, "key table clear");
        clear_error();
        return kOk;
    }
    // the batch slots' captured graphs hold the old table's pointers
    batch_[0].reset();
    batch_[1].reset();
    keys_.reset();
    key_log2_ = log2;
    clear_error();
    return kOk;
}

int Backend::key_table_stats(uint64_t* lookups, uint64_t* hits, uint64_t* slots) {
    *lookups = *hits = *slots = 0;
    if (!keys_ || !keys_->on()) return kOk;
    *slots = keys_->slot_count();
    const cudaError_t e = keys_->read_counters(lookups, hits);
    if (e != cudaSuccess) return cuda_error(e, "key table counters");
    return kOk;
}

int Backend::verify_jobs(const VerifyJob* jobs, size_t n_jobs, uint32_t rlc_segment, const uint8_t* rand32) {
    if (!ready_) return set_error(kErrGpuDevice, "context not ready");
    size_t n_rlc = 0;
    for (size_t j = 0; j < n_jobs; ++j) n_rlc += (jobs[j].kind == 2 && jobs[j].count) ? 1 : 0;
    if (n_rlc == 0) return verify_queue_jobs(jobs, n_jobs);
    std::vector<VerifyJob> queue, rlc_jobs;
    queue.reserve(n_jobs - n_rlc);
    rlc_jobs.reserve(n_rlc);
    for (size_t j = 0; j < n_jobs; ++j) {
        if (jobs[j].kind == 2) {
            if (jobs[j].count) rlc_jobs.push_back(jobs[j]);
        } else {
            queue.push_back(jobs[j]);
        }
    }
    uint8_t zero[32] = {0};
    const uint8_t* r32 = rand32 ? rand32 : zero;
    const uint32_t seg = rlc_segment ? rlc_segment : kRlcJobSegment;
    RlcVerifier& R = rlc();
    int rc = kOk;
    size_t j = 0, off = 0;
    if (!queue.empty()) {
        // the first RLC pass's items are copied into pinned staging by helper
        // threads while the kind 0 / 1 jobs run (their packing and device time)
        if ((rc = R.stage_jobs(rlc_jobs.data(), rlc_jobs.size(), &j, &off)) != kOk) return rc;
        const size_t n = R.staged();
        const int helpers = std::max(1, pack_threads_ - 1);
        std::vector<std::thread> th;
        // joined on every way out, an exception from the queue part included
        struct JoinAll {
            std::vector<std::thread>& v;
            ~JoinAll() {
                for (std::thread& x : v)
                    if (x.joinable()) x.join();
            }
        } join_all{th};
        for (int t = 0; t < helpers; ++t)
            th.emplace_back([&R, n, t, helpers]() { R.pack_staged(n * t / helpers, n * (t + 1) / helpers); });
        rc = verify_queue_jobs(queue.data(), queue.size());
        for (std::thread& x : th) x.join();
        if (rc != kOk) return rc;
        if ((rc = R.run_staged(seg, r32, nullptr)) != kOk) return rc;
    }
    // the rest (all of it without kind 0 / 1 jobs), kMaxItems items per pass
    while (j < rlc_jobs.size()) {
        if ((rc = R.stage_jobs(rlc_jobs.data(), rlc_jobs.size(), &j, &off)) != kOk) return rc;
        if (R.staged() == 0) break;
        parallel_copy(R.staged(), [&R](size_t lo, size_t hi) { R.pack_staged(lo, hi); });
        if ((rc = R.run_staged(seg, r32, nullptr)) != kOk) return rc;
    }
    clear_error();
    return kOk;
}

void Backend::parallel_copy(size_t n, const std::function<void(size_t, size_t)>& fn) {
    if (pack_threads_ > 1 && n >= kPackSplitItems) {
        if (!pack_pool_) pack_pool_.reset(new PackPool(pack_threads_));
        const int parts = pack_pool_->threads();
        pack_pool_->run(parts, [&](int p) { fn(n * p / parts, n * (p + 1) / parts); });
    } else {
        fn(0, n);
    }
}

int Backend::verify_queue_jobs(const VerifyJob* jobs, size_t n_jobs) {
    NvtxRange range("ufsecp verify_jobs");
    if (key_log2_ && !keys_) {
        auto kt = std::make_unique<KeyTable>();
        const int rc = kt->create(this, key_log2_);
        if (rc != kOk) return rc;
        keys_ = std::move(kt);
    }
    for (int q = 0; q < 2; ++q) {
        if (!batch_[q]) {
            auto slot = std::make_unique<BatchSlot>();
            const int rc = slot->init(this);
            if (rc != kOk) return rc;
            if (keys_) slot->set_cache(keys_->slots(), keys_->mask(), keys_->counters());
            batch_[q] = std::move(slot);
        }
        if (q == 0) {
            size_t total = 0;
            for (size_t j = 0; j < n_jobs; ++j) total += jobs[j].count;
            if (total <= kJobsPipeItems) {
                int rc = batch_[0]->enqueue(jobs, n_jobs);
                if (rc == kOk) rc = batch_[0]->finish(jobs, n_jobs);
                if (rc == kOk) clear_error();
                return rc;
            }
        }
    }
    // A large call: sub-calls of at most kJobsPipeItems items (jobs cut at the
    // boundaries; verdicts are per item) alternate between the two slots, so
    // the CPU packs sub-call k + 1 while the device verifies sub-call k.  The
    // jobs are taken ECDSA first, then BIP-340 (each in call order): a
    // sub-call holding one kind runs one queue kernel over the whole device,
    // where interleaved kinds split every sub-call between two kernels, each
    // with its own tail (4000 mixed jobs: 65 -> 54 ms).  Verdicts go through
    // each job's own output pointer, so the order is free.
    std::vector<size_t> order;
    order.reserve(n_jobs);
    for (int kind = 0; kind < 2; ++kind)
        for (size_t i = 0; i < n_jobs; ++i)
            if ((jobs[i].kind == 0) == (kind == 0)) order.push_back(i);
    std::vector<VerifyJob> part[2];
    bool pending[2] = {false, false};
    int rc = kOk;
    size_t j = 0, off = 0;
    for (int k = 0; j < n_jobs && rc == kOk; ++k) {
        const int q = k & 1;
        if (pending[q]) {
            pending[q] = false;
            if ((rc = batch_[q]->finish(part[q].data(), part[q].size())) != kOk) break;
        }
        part[q].clear();
        // the first sub-calls ramp up from kPipeFirst items, so the device
        // starts while the CPU packs the next one, to one wave of the queue
        // kernel's resident grid (56,832 items on a 148-SM B200): a sub-call
        // of 65,536 items was 1.15 waves and ran its tail alone (mixed jobs in
        // one call 28.8 -> 30.0 M sigs/s, one BIP-340 job 32.2 -> 33.7 M)
        const size_t wave = std::max<size_t>(kPipeFirst, std::min(kJobsPipeItems, (size_t)queue_grid_ * kVerifyThreads));
        const size_t cap = std::min(wave, kPipeFirst << std::min(k, 8));
        size_t n = 0;
        while (j < n_jobs && n < cap) {
            const VerifyJob& J = jobs[order[j]];
            if (off >= J.count) {
                ++j;
                off = 0;
                continue;
            }
            const size_t take = std::min(J.count - off, cap - n);
            VerifyJob P = J;
            P.count = take;
            P.msgs = J.msgs + 32 * off;
            P.pubs = J.pubs + (J.kind == 0 ? 33 : 32) * off;
            P.sigs = J.sigs + 64 * off;
            P.out = J.out + off;
            part[q].push_back(P);
            n += take;
            off += take;
        }
        if (part[q].empty()) break;
        if ((rc = batch_[q]->enqueue(part[q].data(), part[q].size())) == kOk) pending[q] = true;
    }
    for (int q = 0; q < 2; ++q) {
        if (!pending[q]) continue;
        const int r = batch_[q]->finish(part[q].data(), part[q].size());
        if (rc == kOk) rc = r;
    }
    if (rc == kOk) clear_error();
    return rc;
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
    e = op == 11 ? launch_field_diag((const uint8_t*)msgs_.p, (uint32_t)n, (uint8_t*)out_.p, sms_, stream_)
                 : launch_diag(op, (const uint8_t*)msgs_.p, (uint32_t)n, (uint8_t*)out_.p, d_gtab_, stream_);
    if (e != cudaSuccess) return cuda_error(e, "diag launch");
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
    // the probe copy built like the BIP-340 verify kernel's current variant
    static const probe_launcher kProbes[kVerifyVariants] = {launch_probe_v0, launch_probe_v1, launch_probe_v2,
                                                            launch_probe_v3, launch_probe_v4, launch_probe_v5,
                                                            launch_probe_v6, launch_probe_v7, launch_probe_v8};
    const probe_launcher launch_probe = kProbes[variant_[1]];
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
