// BIP-340 batch verification by random linear combination (RLC) on the GPU,
// with bisection down to per-signature verdicts.
//
// Role in the reference: the CPU batch verify schnorr_batch_verify_impl
// (src/cpu/src/batch_verify.cpp:324-424: strict parse, lift_x of R and P,
// challenge e, weights a_i = SHA-256(batch_seed || le32 i) (batch_weight :272),
// one multi-scalar multiplication checked against infinity, Pippenger in
// src/cpu/src/pippenger.cpp:73) behind ufsecp_schnorr_batch_verify and
// ufsecp_schnorr_batch_identify_invalid (src/cpu/src/impl/ufsecp_taproot.cpp:703,
// :849), which re-verifies every item one by one when the batch fails.  Here:
//
//  * item i gets the weight a_i = first 16 bytes of SHA-256(seed || le32 i)
//    (never 0) and the batch equation
//        sum_i a_i R_i + sum_i (a_i e_i) P_i - (sum_i a_i s_i) G == infinity
//    is ONE Pippenger multi-scalar multiplication over 3 points per item
//    (R_i with a_i; P_i and lambda P_i with the two GLV halves of a_i e_i) plus
//    2 points per segment (G and lambda G with the GLV halves of
//    -sum a_i s_i), every scalar below 2^128;
//  * signed c-bit windows: a counting sort places every (point, window) with a
//    non-zero digit into bucket (segment, window, |digit|); each bucket is
//    summed in chunks of a tuned number of points (16 by default), each
//    window reduced by running sums over sub-ranges of buckets, windows
//    combined by Horner's rule;
//  * a failing segment is split into kFanout near-equal children, all checked
//    again in the next round (the per-item data is computed once; eight-way
//    splits need half the rounds of halving and less MSM work in total: about
//    2.1x the batch instead of 3x for one invalid item); segments of at most kLeaf items, or all
//    failing segments once most of a round fails, are verified per signature by
//    the plain kernel.  Verdicts equal the per-signature verify item by item
//    (a false accept needs a 2^-128 event per failing segment).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "backend.h"
#include "batch.h"

namespace uf {

struct RlcStats {
    uint64_t rounds = 0;          // MSM rounds (the first check and each bisection level)
    uint64_t segments = 0;        // segments checked by MSM, all rounds
    uint64_t leaf_items = 0;      // items verified one by one (bisection leaves and locate candidates)
    int window_bits = 0;          // window of the first round
    uint64_t located = 0;         // failing segments resolved by a locate round
    uint64_t key_hits = 0;        // items whose key came from the context's key table
};

class RlcVerifier {
public:
    static constexpr uint32_t kLeaf = 32;      // segments this small are verified per signature
    static constexpr uint32_t kChunk = 16;     // default bucket points summed by one thread
    static constexpr uint32_t kFanout = 8;     // children of a failing segment
    static constexpr uint32_t kLocateMax = 65535;   // longest segment a locate round searches
    static constexpr uint32_t kMaxItems = 1u << 24;
    // device bytes the affine chunk trees use per piece of a round's chunks
    static constexpr uint64_t kAffPieceBytes = 4ull << 30;

    explicit RlcVerifier(Backend* be) : be_(be) {}

    ~RlcVerifier();

    // Device-resident BIP-340 items (32-byte messages, 32-byte x-only keys,
    // 64-byte signatures, 16-byte aligned); batch_size items per batch, the
    // last batch ragged (0 = one batch).  window_bits 0 = chosen by segment
    // length, else 4..16.  Writes d_out[i] = 1 / 0 and, if h_batch_ok is not
    // null, one byte per batch: 1 when every item of the batch is valid.
    // Synchronous on `s`.
    int verify(const uint8_t* d_msgs, const uint8_t* d_xs, const uint8_t* d_sigs, uint32_t n, uint32_t batch_size,
               const uint8_t seed[32], int window_bits, uint8_t* d_out, uint8_t* h_batch_ok, cudaStream_t s,
               RlcStats* stats);

    // Host buffers: copies the items in, runs verify() and copies the verdicts
    // back on the backend's stream.
    int verify_host(const uint8_t* msgs, const uint8_t* xs, const uint8_t* sigs, uint32_t n, uint32_t batch_size,
                    const uint8_t seed[32], int window_bits, uint8_t* out, uint8_t* h_batch_ok, RlcStats* stats);

    // Host-buffer BIP-340 jobs (kind 2 of verify_jobs) as one RLC batch of
    // segment-length segments, in three steps so that the host copies can
    // overlap other device work: stage_jobs takes the jobs from (*j, *off) on,
    // up to kMaxItems items (advancing *j, *off; a job may be split between
    // passes), and sizes the buffers; pack_staged copies staged items [lo, hi)
    // into pinned staging (host memory only: any thread, ranges split between
    // threads); run_staged verifies them (weights seeded by input_digest() of
    // the pass XOR rand32) and writes each job's verdicts.  Synchronous.
    int stage_jobs(const VerifyJob* jobs, size_t n_jobs, size_t* j, size_t* off);
    uint64_t staged() const { return staged_; }
    void pack_staged(size_t lo, size_t hi);
    int run_staged(uint32_t segment, const uint8_t rand32[32], RlcStats* stats);

    // Rows of the reference batch API, [x(P) 32 | message 32 | signature 64]
    // (ufsecp_schnorr_batch_verify, src/cpu/src/impl/ufsecp_taproot.cpp:703).
    // Rows are gated in index order as the reference does: the first row with
    // x(P) >= p sets *gate_code = 3 (BAD_PUBKEY), one with r >= p or s outside
    // [1, n-1] sets 4 (BAD_SIG), and *gate_index to that row; then nothing is
    // verified.  Otherwise *gate_code = 0 and h_out[i] = 1 / 0 per row, all rows
    // in one RLC batch whose seed binds the inputs as the reference's does
    // (src/cpu/src/batch_verify.cpp:355-380): input_digest() of the rows XOR
    // the 32 random bytes rand32.
    int verify_entries(const uint8_t* entries, uint32_t n, const uint8_t rand32[32], uint8_t* h_out, int* gate_code,
                       uint32_t* gate_index, RlcStats* stats);

    // SHA-256 tree digest of n device-resident items: one digest of
    // r || s || x(P) || m per item, then 16-way tree levels, then
    // SHA-256(root || le32 n).  Synchronous on `s`.
    int input_digest(const uint8_t* d_msgs, const uint8_t* d_xs, const uint8_t* d_sigs, uint32_t n, cudaStream_t s,
                     uint8_t out[32]);
    // The same over host buffers (copied in on the backend's stream).
    int input_digest_host(const uint8_t* msgs, const uint8_t* xs, const uint8_t* sigs, uint32_t n, uint8_t out[32]);

    // Multi-scalar multiplication sum k_i P_i over host arrays (32-byte
    // big-endian scalars, 33-byte compressed points) with the same Pippenger
    // rounds (ufsecp_gpu_msm).  *status: 0 and out33 = the compressed sum; 5
    // (BAD_INPUT) for a scalar >= n, 3 (BAD_PUBKEY) for an invalid point (the
    // first bad item in index order decides, scalar before point); 7 (ARITH)
    // when the sum is infinity.
    int msm_host(const uint8_t* scalars32, const uint8_t* points33, uint32_t n, uint8_t out33[33], int* status);

private:
    // One MSM check of every segment (start, length pairs); ok[k] bit 0 = the
    // equation holds, bit 1 = the segment holds an item that failed to parse.
    // locate: the round of the locate step (magnitudes and the G scalar
    // weighted by j = i - start + 1 within each segment).
    int run_round(const std::vector<uint32_t>& seg, int c, cudaStream_t s, std::vector<uint8_t>& ok,
                  bool locate = false);
    // The round's bucket chunks (at most 16 points each) summed by affine
    // pairwise trees with grid-shared inversions (k_aff_fwd / k_aff_bwd):
    // results into partials_ / buckets_ as affine points (Z = 1).
    int affine_chunks(uint32_t chunk, uint64_t nch, uint64_t chunk_cap, const uint32_t* coff, uint32_t K,
                      const uint32_t* offsets, cudaStream_t s);
    int verify_leaves(const std::vector<uint32_t>& leaves, const uint8_t* d_msgs, const uint8_t* d_xs,
                      const uint8_t* d_sigs, uint8_t* d_out, cudaStream_t s, RlcStats* stats);
    // Plain verify of the listed items; verdicts into d_out (and host_out).
    int verify_indices(const std::vector<uint32_t>& idx, const uint8_t* d_msgs, const uint8_t* d_xs,
                       const uint8_t* d_sigs, uint8_t* d_out, cudaStream_t s, RlcStats* stats,
                       std::vector<uint8_t>* host_out);
    // The locate step for the failing segments `loc` (start, length pairs;
    // round_idx: their positions in the check round just run, whose sums are
    // in segpt_): resolved[q] = 1 when segment q's single invalid item was
    // found and verified invalid (its verdict written, the rest stay valid).
    int locate(const std::vector<uint32_t>& round_idx, const std::vector<uint32_t>& loc, const uint8_t* d_msgs,
               const uint8_t* d_xs, const uint8_t* d_sigs, uint8_t* d_out, cudaStream_t s, RlcStats* stats,
               std::vector<uint8_t>& resolved);

    Backend* be_;
    uint32_t n_ = 0;
    // per item
    DevBuf items_, mags_, tsc_, okb_;
    // per round
    // cursor_: each entry's rank in its bucket (k_rlc_digits)
    DevBuf segs_, segmag_, segneg_, segbad_, counts_, offsets_, cursor_, nch_, coff_, entries_, partials_,
        buckets_, wu_, wt_, wins_, segok_, scan_tmp_;
    // leaves
    DevBuf leaf_idx_, leaf_m_, leaf_x_, leaf_s_, leaf_out_;
    // host-buffer calls
    DevBuf in_m_, in_x_, in_s_, in_out_, in_rows_, gate_;
    DevBuf segpt_;       // each segment's final sum (Jacobian, 112 B)
    DevBuf dig_a_, dig_b_;   // input digest tree levels
    DevBuf lmags_, lmags_hi_, tsave_, loc_idx_, found_;   // locate step
    DevBuf heavy_;       // count and keys of the buckets with many chunks (k_rlc_bucket_heavy)
    DevBuf aff_pts_, aff_suf_, aff_tp_, aff_meta_, binv_;   // affine chunk trees
    HostBuf job_host_;   // pinned staging of the staged jobs
    DevBuf keyhit_;      // key-table hits of the prep pass
    std::vector<VerifyJob> part_;   // the staged job pieces, and their first items
    std::vector<uint64_t> start_;
    uint64_t staged_ = 0;
    std::vector<uint8_t> ok_host_;
};

// Window bits that minimise the modelled point-addition count for a segment
// of `len` items.
int rlc_window_bits(uint32_t len);

}  // namespace uf
