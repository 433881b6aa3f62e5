// Launch parameters of the HNSW search kernel (shared by host and device).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace hnswgpu {

#ifndef HNSWGPU_WPB
#define HNSWGPU_WPB 1
#endif
#ifndef HNSWGPU_MINB
#define HNSWGPU_MINB 16
#endif
// Low-precision beams use less shared memory per warp (fp8: ~11 KB), so more
// warps fit; 20 resident CTAs (<= 102 registers) measured 8 % faster for the
// fp8 beam on the 1M x 128 workload than 16 (the float32 beam, whose shared
// memory allows ~16 warps, is better served by 16 and 128 registers).
#ifndef HNSWGPU_MINB_LOWP
#define HNSWGPU_MINB_LOWP 20
#endif
constexpr int kWarpsPerBlock = HNSWGPU_WPB;  // independent query warps per CTA
// Early-termination network: kTermFeatures -> kTermHidden -> kTermHidden -> 1.
constexpr int kTermFeatures = 16;
constexpr int kTermHidden = 64;
// Packed float32 parameters, in this order:
//   mu[16], inv_sigma[16] (feature standardisation),
//   W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3[1].
constexpr int kTermOffMu = 0;
constexpr int kTermOffInvSigma = kTermOffMu + kTermFeatures;
constexpr int kTermOffW1 = kTermOffInvSigma + kTermFeatures;
constexpr int kTermOffB1 = kTermOffW1 + kTermHidden * kTermFeatures;
constexpr int kTermOffW2 = kTermOffB1 + kTermHidden;
constexpr int kTermOffB2 = kTermOffW2 + kTermHidden * kTermHidden;
constexpr int kTermOffW3 = kTermOffB2 + kTermHidden;
constexpr int kTermOffB3 = kTermOffW3 + kTermHidden;
constexpr int kTermParams = kTermOffB3 + 1;
// Inference form (device): both layers run on the tensor cores (mma.sync
// m16n8k16, fp16 operands, fp32 accumulation), weights pre-arranged in the B
// fragments each lane reads.  With g = lane / 4 and t = lane % 4, tile v of a
// layer covers units 8v .. 8v + 7 and lane (g, t) accumulates units 8v + 2t
// and 8v + 2t + 1 of every tile.  In order:
//   float mu[16], inv_sigma[16], b3, pad[3]                    (kTermPackedHead floats)
//   float2 b1f[4][8], b2f[4][8]: (b[8v + 2t], b[8v + 2t + 1]) at [t][v]
//   half2 w3f[4][8]:             (w3[8v + 2t], w3[8v + 2t + 1]) at [t][v]
//   half2 W1f[32][8][2]:         (W1[8v + g][2t + 8h], W1[8v + g][2t + 8h + 1])
//                                at [lane][v][h]
//   half2 W2f[32][4][8][2]:      (W2[8v + g][16s + 2t + 8h],
//                                 W2[8v + g][16s + 2t + 8h + 1]) at [lane][s][v][h]
static_assert(kTermFeatures == 16, "layer 1 is one m16n8k16 k-step: 16 features");
constexpr int kTermPackedHead = 2 * kTermFeatures + 4;
constexpr int kTermPackedFloats = kTermPackedHead + 2 * 4 * 8 * 2;
constexpr int kTermPackedHalf2 = 4 * 8 + 32 * 8 * 2 + 32 * 4 * 8 * 2;
constexpr size_t kTermPackedBytes = (size_t)kTermPackedFloats * 4 + (size_t)kTermPackedHalf2 * 4;
// Convert the float32 parameter vector (kTermParams) into the inference form.
void pack_term_model(const float* params, unsigned char* out);
// Training side (term_train.cu), host pointers, current device:
// mean loss and its gradient over n samples;
cudaError_t term_loss_grad(const float* params, const float* feats, const float* labels, uint64_t n,
                           float pos_weight, float* out_loss, float* out_grad);
// Adam over shuffled mini-batches, params updated in place;
cudaError_t term_train(const float* feats, const float* labels, uint64_t n, float* params, uint32_t epochs,
                       uint32_t batch, float lr, float pos_weight, float weight_decay, uint64_t seed,
                       float* out_epoch_loss);
// logits of the search's in-warp inference (fp16 weights) for n feature rows.
cudaError_t term_logits(const float* params, const float* feats, uint64_t n, float* out);
constexpr int kMinBlocks = HNSWGPU_MINB;     // launch bound: resident CTAs per SM
constexpr uint32_t HNSWGPU_STATUS_TIMEOUT_BIT = 0x1u;
constexpr uint32_t HNSWGPU_STATUS_OVERFLOW_BIT = 0x2u;
constexpr uint32_t kTieBit = 0x80000000u;  // per-query, never reported: the run met a steering tie

struct SearchParams {
    // index (device pointers)
    const float* vecs;            // count x row_floats, rows zero-padded
    const uint32_t* links0;       // count x maxM0 ids, unused slots = 0xffffffff
    const uint32_t* upper_off;    // per node: first upper-level row, or 0xffffffff
    const uint32_t* upper_links;  // rows of (maxM + 1) u32: [count][ids]
    const uint64_t* labels;       // count
    const uint32_t* deleted_bits; // bitmap over internal ids (null: none deleted)
    const uint8_t* allow;         // filter mask over internal ids (null: no filter)
    uint32_t count, dim, row_floats, row_bytes;
    uint32_t maxM, maxM0, ep;
    int32_t maxlevel;
    // query batch
    const float* queries;
    uint32_t nq, q_stride, k, ef;
    uint32_t bare, normalize;
    uint32_t max_expansions;      // safety bound on level-0 expansions per query
    uint32_t fast16;              // dim % 16 == 0: 4-lanes-per-row distance path
    uint32_t links_unique;        // no level-0 list repeats an id (checked at load)
    uint32_t exact;               // replay the reference's heaps (tie order exact)
    // epsilon search (searchStopConditionClosest with EpsilonSearchStopCondition;
    // tie-exact general loop only): k = ef = max_num_candidates
    uint32_t eps_mode;            // 1: stop once a candidate lies beyond eps with eps_min items held
    float eps;                    // epsilon (a distance, squared for L2)
    uint32_t eps_min;             // min_num_candidates
    uint32_t pool_cap;            // ef (canonical) or ef + 32 (tie-exact)
    uint32_t cand_cap;            // tie-exact: candidate heap entries in shared memory
    uint32_t cand_spill_cap;      // tie-exact: further entries per warp in cand_spill
    uint32_t cand_spill_warps;    // warps that cand_spill has room for
    uint64_t* cand_spill;         // tie-exact: global tail of each warp's candidate heap
    // outputs
    uint64_t* out_labels;
    float* out_dists;
    int32_t* out_counts;
    uint32_t* trace;
    uint32_t* work_counter;       // zero at launch; reset to zero by the last block
    uint32_t* done_counter;       // blocks finished (same slot discipline)
    uint32_t* status;
    // tie-exact mode in two passes: the id-order beam lists the queries whose
    // run met a distance tie that can steer the reference's heaps, then the
    // heap replay runs on those queries only
    uint32_t* tie_list;           // first pass: flagged query indices (null: no listing)
    uint32_t* tie_count;          // first pass: entries appended to tie_list (zero at launch)
    const uint32_t* qlist;        // second pass: query indices to run (null: 0 .. nq - 1)
    const uint32_t* qcount;       // second pass: device word holding the entries of qlist
    unsigned long long* phase_cycles;  // 10 counters, profiling builds only (may be null)
    // learned early termination (mode 1 = record checkpoints, 2 = stop early)
    uint32_t term_mode;
    uint32_t term_period;        // expansions between checkpoints (T)
    uint32_t term_max_ckpt;      // checkpoint rows per query (trace mode)
    float* ckpt_feat;            // trace: nq x max_ckpt x kTermFeatures
    uint32_t* ckpt_ids;          // trace: nq x max_ckpt x ckpt_width ids of the first beam entries
    float* ckpt_dists;           // trace (optional): their float32 distances, recomputed from the rows
    uint32_t ckpt_width;
    uint32_t* ckpt_count;        // trace: checkpoints written per query
    const float* term_model;     // learned: packed network (see term_model_layout)
    float term_logit;            // learned: stop when the network's logit exceeds this
    // low-precision traversal (prec 1 = bf16, 2 = fp8 e4m3 + per-row scale)
    uint32_t prec;
    const unsigned char* tvecs;  // traversal rows, tstride bytes apart
    uint32_t trow_bytes;         // bytes copied per traversal row (16-multiple)
    uint32_t tstage_bytes;       // staging stride of a traversal row
    uint32_t tslots;             // traversal rows per staging batch
    uint32_t rerank;             // best candidates re-ranked with fp32 distances
    uint32_t rr_slots;           // fp32 rows per re-rank staging batch
    // lean fp8 beam (hnsw_lean.cu): id tie order, no filter or deletions;
    // `lean_w` link rows expanded per iteration (64 link slots per pass)
    uint32_t lean, lean_w;
    uint32_t off_q8, off_cid, off_lacc, lean_stage;
    // per-warp shared memory layout
    uint32_t stage_slots, stage_stride, extra_cap, log2_vis;
    uint32_t off_query, off_stage, off_pool, off_extra, off_vis, off_top, off_cand, off_acc, off_ev, warp_smem;
};

// Scratch of hnswgpu_search_noalloc: words [0] work counter, [1] finished-CTA
// counter, [2] status bits; 64 words = 256 bytes.
constexpr int kNoallocScratchWords = 64;
constexpr int kMaxDevices = 64;
// Device address of the fixed scratch on `device`, which must be current.
cudaError_t noalloc_scratch_address(int device, uint32_t** out);

// Bounded-wait self-test: one warp waits (at most `limit` tries) on an
// mbarrier phase that never completes and ORs HNSWGPU_STATUS_TIMEOUT_BIT into
// *status (device memory).
cudaError_t launch_wait_timeout_selftest(uint32_t limit, uint32_t* status, cudaStream_t stream);

// Fills the off_* fields and warp_smem from the sizes; returns warp_smem.
size_t warp_smem_layout(SearchParams& p);
// The lean fp8 beam's per-warp layout (called by warp_smem_layout when p.lean).
size_t lean_smem_layout(SearchParams& p);
// Whether the lean fp8 beam can run these parameters: fp8 copy, id tie order,
// no filter / deletions / checkpoint listing, maxM0 <= 64, fp8 data bytes per
// row a multiple of 32 and either <= 128 or a multiple of 128.
bool lean_eligible(const SearchParams& p);
cudaError_t launch_hnsw_lean(const SearchParams& p, int space, int num_sms, cudaStream_t stream, int* blocks_out);
constexpr int kLeanWarpsPerBlock = 2;
// learned-stop lean kernels: four query warps share one copy of the packed
// network in shared memory
constexpr int kLeanWarpsPerBlockLearned = 4;
constexpr size_t kLeanModelSmem = (kTermPackedBytes + 127) & ~(size_t)127;

// Low-precision traversal copies (quantize.cu).  Row layouts:
//   bf16: dim x bf16, zero padded to a 16-byte multiple;
//   fp8 : dim x e4m3 (value / scale, scale = max|x| / 448), zero padded to a
//         16-byte multiple, then 16 bytes holding the float scale and the
//         float squared norm of the dequantized row.
uint32_t traversal_row_bytes(uint32_t prec, uint32_t dim);
cudaError_t launch_quantize_rows(const float* src, uint32_t count, uint32_t dim, uint32_t src_stride, uint32_t prec,
                                 unsigned char* dst, cudaStream_t stream);
cudaError_t launch_hnsw_search(const SearchParams& p, int space, int num_sms, cudaStream_t stream, int* blocks_out);

}  // namespace hnswgpu
