// Lean fp8 beam for batched HNSW k-NN search on B200 (sm_100a).
//
// Serves HierarchicalNSW::searchKnn (hnswlib/hnswalg.h:1269-1323: upper-layer
// greedy descent, then the level-0 beam of searchBaseLayerST,
// hnswlib/hnswalg.h:308-440) over the per-row-scaled e4m3 copy of the
// vectors, for batches without deletions or a filter, in the id tie order;
// the best candidates are then re-ranked with exact float32 distances in the
// reference's summation order, so every returned distance is the reference's.
//
// Compared with the general pipelined beam (hnsw_search.cu) it spends far
// fewer instructions per expansion:
//   * per-lane gathers: each lane copies its quarter of four candidate rows
//     into its own shared-memory stage slots with cp.async (no registers
//     held while the copies fly, no warp-wide barrier: a lane reads back only
//     what it copied), then reads them as mma fragments;
//   * distances on the tensor cores: mma.sync m16n8k32 e4m3 x e4m3 -> f32.
//     The query is split into two e4m3 vectors q ~ s_hi * hi + s_lo * lo
//     (the second holds the rounding residual of the first), placed in the
//     even and odd columns of B, so the two products of one row land in the
//     lane that owns that candidate: no shuffles.  L2 = |q|^2 - 2 q.x + |x|^2
//     with |x|^2 of the dequantized row stored beside its scale;
//   * several link rows per iteration: the `lean_w` best unexpanded pool
//     entries (2 when maxM0 <= 32, else 1) are expanded together, 64 link
//     slots, two per lane.  maxM0 = 64 (M = 32 graphs) runs one row per
//     iteration in the same code;
//   * acceptance by the beam's bound (pool not full, or closer than its
//     worst entry), then one sorted merge of the accepted keys;
//   * optional learned stop: a checkpoint every term_period expansions (at
//     states where the top-k has been stable for a period and no waiting
//     candidate is closer than the k-th result) runs the termination network
//     on the tensor cores from a per-CTA shared-memory copy.
//
// Exactness is not the goal of this beam (its distances are approximate and
// several rows are expanded at once); the returned distances are exact
// float32 distances of the returned labels, and recall is measured against
// the exact top-k.
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_common.cuh"
#include "hnsw_search.h"
#include "launch_cache.h"
#include "term_mlp.cuh"

// launch bound, resident 2-warp CTAs per SM.  On the 1M x 128 workload a
// bound of 10 (96 registers, 20 query warps) was 9 % faster than 8 (128
// registers); 11 and 12 were slower.  With a bound of 9 the compiler still
// allocates 96 registers (10 CTAs reside) but schedules the loop differently,
// 2 % faster than the bound of 10 (same-box A/B)
#ifndef HNSWGPU_MINB_LEAN
#define HNSWGPU_MINB_LEAN 9
#endif

// Where the learned-stop kernels read the packed network: 1 = one copy in
// shared memory per 4-warp CTA (residency 16 warps per SM), 0 = through the
// read-only cache from 2-warp CTAs (the fixed-ef residency).
#ifndef HNSWGPU_LEAN_MODEL_SMEM
#define HNSWGPU_LEAN_MODEL_SMEM 1
#endif

namespace hnswgpu {

// Optional self-checks (compile with -DHNSWGPU_BOUNDS_CHECK; the shipped
// library is built without them): each global and shared-memory index of the
// lean beam is checked against its buffer; the first violation is recorded in
// g_lean_dbg (code, two values, block) and the access is skipped.
#ifdef HNSWGPU_BOUNDS_CHECK
__device__ unsigned long long g_lean_dbg[8];
__device__ __forceinline__ bool lean_ok(bool cond, unsigned code, unsigned long long a, unsigned long long b) {
    if (cond) return true;
    if (atomicCAS(&g_lean_dbg[0], 0ull, (unsigned long long)code) == 0ull) {
        g_lean_dbg[1] = a;
        g_lean_dbg[2] = b;
        g_lean_dbg[3] = blockIdx.x;
    }
    return false;
}
#define LCHK(cond, code, a, b) lean_ok((cond), (code), (unsigned long long)(a), (unsigned long long)(b))
cudaError_t read_lean_debug_record(unsigned long long* out) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_lean_dbg, sizeof(unsigned long long) * 8);
    if (e != cudaSuccess) return e;
    unsigned long long z[8] = {0};
    return cudaMemcpyToSymbol(g_lean_dbg, z, sizeof(z));
}
#else
#define LCHK(cond, code, a, b) true
#endif

namespace {

struct LeanSmem {
    float* q;            // float32 query (row_floats), normalised for cosine
    unsigned char* q8;   // e4m3 query: [hi: D bytes][lo: D bytes]
    uint32_t* cid;       // fresh ids of one iteration, compacted (64)
    uint64_t* lacc;      // accepted keys of one iteration, compacted (64)
    uint64_t* pool;      // sorted (distance key, id | EXP_BIT), at most ef
    uint32_t* vis;       // direct-mapped visited cache; re-rank scratch after the beam
    unsigned char* stage;  // 32 row slots (lean_stage bytes apart): one distance pass's gathered rows
    float2* tails;       // 32 (scale, squared norm) of the pass's candidates
    const float* model;  // learned stop: the CTA's copy of the packed network
};

struct LeanQuery {
    float qn;            // |q|^2 (L2)
    float s_hi, s_lo;    // scales of the two e4m3 parts of the query
};

struct LeanCounters {
    uint32_t upper_hops, upper_dists, l0_exp, l0_dists;
};

// Optional per-phase cycle accounting (compile with -DHNSWGPU_PHASE_TIMING;
// the shipped library is built without it).  Phases: 0 query setup, 1
// upper-layer descent, 2 candidate selection, 3 link rows + visited cache +
// compaction, 4 distance passes, 5 acceptance, 6 merge, 7 checkpoint, 8
// re-rank + output.
#ifdef HNSWGPU_PHASE_TIMING
struct LeanClock {
    long long last = 0;
    long long acc[9] = {0};
    __device__ void start() { last = clock64(); }
    __device__ void mark(int i) {
        const long long t = clock64();
        acc[i] += t - last;
        last = t;
    }
};
#define LPT(i) lc.mark(i)
#else
struct LeanClock {
    __device__ void start() {}
};
#define LPT(i)
#endif

__device__ __forceinline__ void mma_e4m3(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k32.row.col.f32.e4m3.e4m3.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Per-lane asynchronous copies global -> shared (no registers held while
// they are in flight); each lane later reads back only what it copied, so
// waiting for its own copies is enough.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Byte layout of one 128-byte block of a row (or of the whole row when it is
// shorter) over the four lanes t of a quad: lane t reads load units of U
// bytes (U = 16 when NS is even, else 8) at offsets (4 j + t) U, j = 0, 1, ...
// so that one warp load instruction covers contiguous bytes of each row; mma
// step st takes the lane's bytes [8 st, 8 st + 8).  Rows and the query use
// the same layout, so the k-permutation cancels in the dot product.
template <int NS>
__device__ __forceinline__ int lane_step_offset(int st, int t) {
    return NS % 2 == 0 ? ((st >> 1) * 4 + t) * 16 + (st & 1) * 8 : (st * 4 + t) * 8;
}

// Copy this lane's quarter of a row block (its load units) into its stage
// slot, same offsets.
template <int NS>
__device__ __forceinline__ void stage_quarter(uint32_t slot, const unsigned char* row, int t) {
    if (NS % 2 == 0) {
#pragma unroll
        for (int j = 0; j < NS / 2; j++) cp_async16(slot + (j * 4 + t) * 16, row + (j * 4 + t) * 16);
    } else {
#pragma unroll
        for (int j = 0; j < NS; j++) cp_async8(slot + (j * 4 + t) * 8, row + (j * 4 + t) * 8);
    }
}

// Read the quarter back (zero for an empty row) as the mma A operand bytes.
template <int NS>
__device__ __forceinline__ void read_quarter(const unsigned char* slot, int t, bool valid, uint32_t (&r)[2 * NS]) {
    if (!valid) {
#pragma unroll
        for (int i = 0; i < 2 * NS; i++) r[i] = 0u;
        return;
    }
    if (NS % 2 == 0) {
#pragma unroll
        for (int j = 0; j < NS / 2; j++) {
            const uint4 v = *reinterpret_cast<const uint4*>(slot + (j * 4 + t) * 16);
            r[4 * j] = v.x;
            r[4 * j + 1] = v.y;
            r[4 * j + 2] = v.z;
            r[4 * j + 3] = v.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < NS; j++) {
            const uint2 v = *reinterpret_cast<const uint2*>(slot + (j * 4 + t) * 8);
            r[2 * j] = v.x;
            r[2 * j + 1] = v.y;
        }
    }
}

// B fragments of one 128-byte block (or the whole short row) of the query:
// lanes of even quads hold the hi part, odd quads the lo part.
template <int NS>
__device__ __forceinline__ void load_bfrag(const LeanSmem& s, uint32_t D, int blk, int lane, uint32_t (&b)[2 * NS]) {
    const int g = lane >> 2, t = lane & 3;
    const unsigned char* src = s.q8 + (g & 1) * D + blk * 128;
#pragma unroll
    for (int st = 0; st < NS; st++) {
        const uint2 v = *reinterpret_cast<const uint2*>(src + lane_step_offset<NS>(st, t));
        b[2 * st] = v.x;
        b[2 * st + 1] = v.y;
    }
}

// Approximate distances of the candidates cid[base .. base + 32) (those
// below nnew): lane L returns the distance of candidate base + L and its id.
// Quad g owns candidates base + 4g .. base + 4g + 3; in the two m16n8k32
// tiles of the pass, tile 0 holds candidate base + 4g in row g and base + 4g
// + 2 in row g + 8, tile 1 holds base + 4g + 1 and base + 4g + 3.  With the
// hi / lo query in the even / odd columns of B, lane (g, t) receives both
// products of candidate base + 4g + t in its accumulator pair (c0, c1) or
// (c2, c3).  Each lane gathers its quarter of the quad's four rows (and the
// scale / norm tail of its own candidate) into its stage slots with
// asynchronous copies, then reads them back tile by tile.
template <int SPACE, int NS, bool MULTI>
__device__ __forceinline__ float lean_pass(const SearchParams& p, const LeanSmem& s, const LeanQuery& lq, int base,
                                           int nnew, int lane, uint32_t& my_id) {
    const int g = lane >> 2, t = lane & 3;
    const uint4 ids4 = *reinterpret_cast<const uint4*>(s.cid + base + 4 * g);
    const uint32_t ids[4] = {ids4.x, ids4.y, ids4.z, ids4.w};
    const uint32_t D = p.trow_bytes - 16;
    const uint32_t SS = p.lean_stage;  // stage slot stride (bytes)
    bool valid[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        valid[r] = base + 4 * g + r < nnew && LCHK(base + 4 * g + r < 64, 199, base, nnew);
        if (valid[r] && !LCHK(ids[r] < p.count, 200, ids[r], p.count)) valid[r] = false;
    }
    my_id = t == 0 ? ids[0] : t == 1 ? ids[1] : t == 2 ? ids[2] : ids[3];
    const bool mine = base + lane < nnew && LCHK(my_id < p.count, 201, my_id, base + lane);
    const uint32_t stage = smem_u32(s.stage);
    float c0[4] = {0.f, 0.f, 0.f, 0.f}, c1[4] = {0.f, 0.f, 0.f, 0.f};
    float2 tail = make_float2(0.f, 0.f);
    const int nblk = MULTI ? (int)(D >> 7) : 1;
    for (int blk = 0; blk < nblk; blk++) {
#pragma unroll
        for (int r = 0; r < 4; r++)
            if (valid[r])
                stage_quarter<NS>(stage + (uint32_t)(4 * g + r) * SS,
                                  p.tvecs + (size_t)ids[r] * p.trow_bytes + blk * 128, t);
        if (blk == 0 && mine)
            cp_async8(smem_u32(s.tails + lane), p.tvecs + (size_t)my_id * p.trow_bytes + D);
        cp_async_wait_all();
        __syncwarp();  // mma.sync needs the whole warp converged
        // tile 0: rows (g, g + 8) = candidates 4g, 4g + 2; tile 1: 4g + 1, 4g + 3.
        // One load unit at a time (both tiles), so that few fragments are live.
        const unsigned char* qsrc = s.q8 + (g & 1) * D + blk * 128;
        const unsigned char* r0 = s.stage + (4 * g) * SS;
        if (NS % 2 == 0) {
#pragma unroll
            for (int u = 0; u < NS / 2; u++) {
                const int off = (u * 4 + t) * 16;
                const uint4 bq = *reinterpret_cast<const uint4*>(qsrc + off);
#pragma unroll
                for (int tile = 0; tile < 2; tile++) {
                    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
                    const uint4 x0 = valid[tile] ? *reinterpret_cast<const uint4*>(r0 + tile * SS + off) : z;
                    const uint4 x1 = valid[tile + 2] ? *reinterpret_cast<const uint4*>(r0 + (tile + 2) * SS + off) : z;
                    float (&c)[4] = tile == 0 ? c0 : c1;
                    mma_e4m3(c, x0.x, x1.x, x0.y, x1.y, bq.x, bq.y);  // step 2u
                    mma_e4m3(c, x0.z, x1.z, x0.w, x1.w, bq.z, bq.w);  // step 2u + 1
                }
            }
        } else {
#pragma unroll
            for (int st = 0; st < NS; st++) {
                const int off = (st * 4 + t) * 8;
                const uint2 bq = *reinterpret_cast<const uint2*>(qsrc + off);
#pragma unroll
                for (int tile = 0; tile < 2; tile++) {
                    const uint2 z = make_uint2(0u, 0u);
                    const uint2 x0 = valid[tile] ? *reinterpret_cast<const uint2*>(r0 + tile * SS + off) : z;
                    const uint2 x1 = valid[tile + 2] ? *reinterpret_cast<const uint2*>(r0 + (tile + 2) * SS + off) : z;
                    float (&c)[4] = tile == 0 ? c0 : c1;
                    mma_e4m3(c, x0.x, x1.x, x0.y, x1.y, bq.x, bq.y);
                }
            }
        }
        if (blk == 0 && mine) tail = s.tails[lane];
        if (MULTI) __syncwarp();
    }
    const float hi = t == 0 ? c0[0] : t == 1 ? c1[0] : t == 2 ? c0[2] : c1[2];
    const float lo = t == 0 ? c0[1] : t == 1 ? c1[1] : t == 2 ? c0[3] : c1[3];
    // explicit rounding: every call site must give a node the same key (the
    // pool recognises a node evaluated again by its exact key)
    const float dot = __fmul_rn(tail.x, __fmaf_rn(lq.s_hi, hi, __fmul_rn(lq.s_lo, lo)));
    if (SPACE == 0) return __fmaf_rn(-2.0f, dot, __fadd_rn(lq.qn, tail.y));
    return __fsub_rn(1.0f, dot);
}

// Count of entries of the sorted array a[0, n) whose key (flag masked) is < key.
__device__ __forceinline__ int lower_bound_masked(const uint64_t* a, int n, uint64_t key) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((a[mid] & KEY_MASK) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Insert the distinct keys of the lanes in `amask` (not present in the pool;
// `pos` = lower_bound_masked of the lane's key) into the sorted pool, keeping
// at most cap entries.  `klist[i]` is lane i's key (in shared memory: one
// broadcast load per key instead of two shuffles).  Returns the smallest insertion index; `top` is set
// when a key lands within the first kq entries.
__device__ __forceinline__ int lean_merge(uint64_t* pool, int& size, int cap, unsigned amask, uint64_t key, int pos,
                                         int lane, int kq, bool& top, const uint64_t* klist) {
    const int na = __popc(amask);
    const bool mine = (amask >> lane) & 1u;
    int rank = 0;
    for (unsigned m = amask; m; m &= m - 1) {
        const uint64_t k2 = klist[__ffs(m) - 1];
        rank += k2 < key;
    }
    const int mpos = (int)__reduce_min_sync(FULL, mine ? (unsigned)pos : 0x7fffffffu);
    if (size > mpos) {
        // move the entries [mpos, size) right, last chunk first
        const int nmove = size - mpos;
        for (int b = mpos + ((nmove - 1) & ~31); b >= mpos; b -= 32) {
            const int i = b + lane;
            const bool have = i < size;
            const uint64_t e = have ? pool[i] : 0ull;
            const uint64_t em = e & KEY_MASK;
            int sh = 0;
            for (unsigned m = amask; m; m &= m - 1) sh += klist[__ffs(m) - 1] < em;
            __syncwarp();
            if (have && i + sh < cap && LCHK(i + sh >= 0, 231, i, sh)) pool[i + sh] = e;
            __syncwarp();
        }
    }
    const int np = pos + rank;
    if (mine && np < cap && LCHK(np >= 0 && pos <= size, 232, np, pos)) pool[np] = key;
    __syncwarp();
    top = __any_sync(FULL, mine && np < kq);
    size = min(size + na, cap);
    return mpos;
}

// Link slots of an iteration: slot j = lane (id0) and lane + 32 (id1) is
// entry j % maxM0 of the level-0 row of candidate j / maxM0 (c0, c1), for
// the sel candidates taken; INVALID_ID elsewhere.
__device__ __forceinline__ void lean_links(const SearchParams& p, int maxM0, int sel, uint32_t c0, uint32_t c1,
                                           int lane, uint32_t& id0, uint32_t& id1) {
    id0 = INVALID_ID;
    id1 = INVALID_ID;
    const int j0 = lane, ci0 = j0 >= maxM0 ? 1 : 0;
    if (ci0 < sel && LCHK((ci0 ? c1 : c0) < p.count, 210, ci0 ? c1 : c0, sel) &&
        LCHK(j0 - ci0 * maxM0 < maxM0, 211, j0, ci0))
        id0 = __ldg(p.links0 + (size_t)(ci0 ? c1 : c0) * maxM0 + (j0 - ci0 * maxM0));
    const int j1 = lane + 32, ci1 = j1 >= maxM0 ? (j1 >= 2 * maxM0 ? 2 : 1) : 0;
    if (ci1 < sel && LCHK((ci1 ? c1 : c0) < p.count, 212, ci1 ? c1 : c0, sel) &&
        LCHK(j1 - ci1 * maxM0 < maxM0 && j1 - ci1 * maxM0 >= 0, 213, j1, ci1))
        id1 = __ldg(p.links0 + (size_t)(ci1 ? c1 : c0) * maxM0 + (j1 - ci1 * maxM0));
}

struct LeanTerm {
    uint32_t last_change = 0;  // expansions when the top-k last changed
    uint32_t nchange = 0;      // expansions (iterations) that changed the top-k
    uint32_t nckpt = 0;        // checkpoints taken
    uint32_t next = 0;         // expansion count of the next checkpoint
    uint32_t prev_e = 0, prev_d = 0;  // expansions and distance evaluations at the previous checkpoint
};

__device__ __forceinline__ TermInputs lean_term_inputs(const SearchParams& p, float e, float d1, float dk, float dn,
                                                       float d_entry, float qn, uint32_t dists, const LeanTerm& ts) {
    TermInputs in;
    in.e = e;
    in.d1 = d1;
    in.dk = dk;
    in.dn = dn;
    in.d_entry = d_entry;
    in.qn = qn;
    in.since_change = e - (float)ts.last_change;
    in.inv_period = 1.0f / (float)p.term_period;
    in.nchange = (float)ts.nchange;
    in.eval_rate = (float)(dists - ts.prev_d) / fmaxf(e - (float)ts.prev_e, 1.0f);
    return in;
}

// Trace mode: the ids of the first ckpt_width beam entries of a checkpoint
// row, and (when asked for) their float32 distances.
template <int SPACE>
__device__ __forceinline__ void lean_record_ids(const SearchParams& p, const LeanSmem& s, int lane, size_t row,
                                                int psize) {
    const int w = (int)p.ckpt_width;
    for (int i = lane; i < w; i += 32) p.ckpt_ids[row * w + i] = i < psize ? kid(s.pool[i]) : INVALID_ID;
    if (p.ckpt_dists) {
        float* out = p.ckpt_dists + row * w;
        for (int i = psize + lane; i < w; i += 32) out[i] = __int_as_float(0x7f800000);
        trace_dists<SPACE>(p, s.q, s.pool, min(w, psize), lane, out);
    }
}

// Checkpoint of the learned termination (trace mode 1 records it, mode 2
// asks the network whether to stop), with the general beam's features.
template <int SPACE, int TERM>
__device__ __forceinline__ bool lean_checkpoint(const SearchParams& p, const LeanSmem& s, int lane, uint32_t qi,
                                                uint32_t e, uint32_t dists, int psize, uint32_t next_dk,
                                                float d_entry, float qn, LeanTerm& ts) {
    if (psize == 0) return false;
    const int kq = (int)p.k;
    const int kk = min(kq, psize);
    float fe[kTermFeatures];
    const TermInputs in = lean_term_inputs(p, (float)e, funkey(khi(s.pool[0])), funkey(khi(s.pool[kk - 1])),
                                           funkey(next_dk), d_entry, qn, dists, ts);
    term_features(in, s.pool, psize, (int)p.ef, lane, fe);
    ts.prev_e = e;
    ts.prev_d = dists;
    if (TERM == 1) {
        if (ts.nckpt + 1 < p.term_max_ckpt) {
            const size_t row = (size_t)qi * p.term_max_ckpt + ts.nckpt;
            if (lane < kTermFeatures) p.ckpt_feat[row * kTermFeatures + lane] = fe[lane];
            lean_record_ids<SPACE>(p, s, lane, row, psize);
        }
        ts.nckpt++;
        return false;
    }
    if (HNSWGPU_LEAN_MODEL_SMEM) return term_logit<true>(s.model, fe, lane) > p.term_logit;
    return term_logit<false>(p.term_model, fe, lane) > p.term_logit;
}

template <int SPACE>
__device__ __forceinline__ void lean_final_row(const SearchParams& p, const LeanSmem& s, int lane, uint32_t qi,
                                               uint32_t e, uint32_t dists, int psize, float d_entry, float qn,
                                               const LeanTerm& ts) {
    if (p.term_max_ckpt == 0) {
        if (lane == 0) p.ckpt_count[qi] = 0;
        return;
    }
    const int kq = (int)p.k;
    const uint32_t r = min(ts.nckpt, p.term_max_ckpt - 1);
    const size_t row = (size_t)qi * p.term_max_ckpt + r;
    const int kk = min(kq, psize);
    const float d1 = kk > 0 ? funkey(khi(s.pool[0])) : 0.f;
    const float dk = kk > 0 ? funkey(khi(s.pool[kk - 1])) : 0.f;
    float fe[kTermFeatures];
    if (psize > 0) {
        term_features(lean_term_inputs(p, (float)e, d1, dk, dk, d_entry, qn, dists, ts), s.pool, psize, (int)p.ef,
                      lane, fe);
    } else {
        for (int i = 0; i < kTermFeatures; i++) fe[i] = 0.f;
    }
    if (lane < kTermFeatures) p.ckpt_feat[row * kTermFeatures + lane] = fe[lane];
    lean_record_ids<SPACE>(p, s, lane, row, psize);
    if (lane == 0) p.ckpt_count[qi] = r + 1;
}

// Exact float32 re-rank of the best R pool entries: 8 rows per pass, 4 lanes
// per row, each lane keeping 4 of the reference's 16 AVX-512 accumulators
// (group4_reduce restates the reference's reduction order), rows loaded
// straight from global memory.  The pool is then re-sorted by the exact
// (distance, id) keys.
template <int SPACE>
__device__ void lean_rerank(const SearchParams& p, const LeanSmem& s, int lane, int& psize) {
    const int R = min(psize, (int)p.rerank);
    const int a = lane & 3;
    const int n16 = (int)(p.dim >> 4);
    const float4* q4 = reinterpret_cast<const float4*>(s.q);
    for (int b = 0; b < R; b += 8) {
        const int v = b + (lane >> 2);
        const bool valid = v < R;
        uint32_t id = kid(s.pool[valid ? v : b]);
        if (!LCHK(id < p.count && R <= (int)p.ef, 250, id, R)) id = 0;
        const float4* x4 = reinterpret_cast<const float4*>(p.vecs + (size_t)id * p.row_floats);
        float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
        for (int cb = 0; cb < n16; cb += 4) {
            float4 xv[4];
#pragma unroll
            for (int c = 0; c < 4; c++)
                if (cb + c < n16) xv[c] = __ldg(x4 + 4 * (cb + c) + a);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                if (cb + c < n16) {
                    const float4 qv = q4[4 * (cb + c) + a];
                    if (SPACE == 0) {
                        const float t0 = __fsub_rn(qv.x, xv[c].x), t1 = __fsub_rn(qv.y, xv[c].y),
                                    t2 = __fsub_rn(qv.z, xv[c].z), t3 = __fsub_rn(qv.w, xv[c].w);
                        c0 = __fmaf_rn(t0, t0, c0);
                        c1 = __fmaf_rn(t1, t1, c1);
                        c2 = __fmaf_rn(t2, t2, c2);
                        c3 = __fmaf_rn(t3, t3, c3);
                    } else {
                        c0 = __fmaf_rn(qv.x, xv[c].x, c0);
                        c1 = __fmaf_rn(qv.y, xv[c].y, c1);
                        c2 = __fmaf_rn(qv.z, xv[c].z, c2);
                        c3 = __fmaf_rn(qv.w, xv[c].w, c3);
                    }
                }
            }
        }
        const float r = group4_reduce<SPACE>(c0, c1, c2, c3);
        if (a == 0 && valid) s.pool[v] = mkkey(r, id);
        __syncwarp();
    }
    // rank by counting into the idle visited cache (equal keys by position,
    // so every slot is written), then copy back
    uint64_t* tmp = reinterpret_cast<uint64_t*>(s.vis);
    for (int r = lane; r < R; r += 32) {
        const uint64_t kr = s.pool[r];
        int rank = 0;
        for (int t = 0; t < R; t++) rank += s.pool[t] < kr || (s.pool[t] == kr && t < r);
        if (LCHK((size_t)(rank + 1) * 8 <= ((size_t)4 << p.log2_vis), 252, rank, R)) tmp[rank] = kr;
    }
    __syncwarp();
    for (int r = lane; r < R; r += 32) s.pool[r] = tmp[r];
    __syncwarp();
    psize = R;
}

template <int SPACE, int TERM, int NS, bool MULTI>
__device__ void lean_search(const SearchParams& p, const LeanSmem& s, uint32_t qi, int lane, LeanCounters& ct,
                            LeanClock& lc) {
    lc.start();
    const int dim = (int)p.dim;
    const uint32_t D = p.trow_bytes - 16;
    // ---- query row (normalised for the cosine space)
    const float* qg = p.queries + (size_t)qi * p.q_stride;
    for (int i = lane; i < (int)p.row_floats; i += 32) s.q[i] = i < dim ? qg[i] : 0.f;
    __syncwarp();
    if (p.normalize) {
        float sc = 0.f;
        if (lane == 0) sc = norm_scale(s.q, dim);
        sc = __shfl_sync(FULL, sc, 0);
        __syncwarp();
        for (int i = lane; i < dim; i += 32) s.q[i] = __fmul_rn(s.q[i], sc);
        __syncwarp();
    }
    // ---- e4m3 hi / lo parts of the query and |q|^2
    LeanQuery lq;
    {
        float amax = 0.f, qn = 0.f;
        for (int i = lane; i < dim; i += 32) {
            const float v = s.q[i];
            amax = fmaxf(amax, fabsf(v));
            qn = fmaf(v, v, qn);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            amax = fmaxf(amax, __shfl_xor_sync(FULL, amax, o));
            qn += __shfl_xor_sync(FULL, qn, o);
        }
        lq.qn = qn;
        lq.s_hi = amax > 0.f ? amax / 448.0f : 1.0f;
        const float inv_hi = 1.0f / lq.s_hi;
        float rmax = 0.f;
        for (int i = 2 * lane; i < (int)D; i += 64) {
            const float2 v = make_float2(i < dim ? s.q[i] : 0.f, i + 1 < dim ? s.q[i + 1] : 0.f);
            const __nv_fp8x2_storage_t h = __nv_cvt_float2_to_fp8x2(make_float2(v.x * inv_hi, v.y * inv_hi),
                                                                    __NV_SATFINITE, __NV_E4M3);
            *reinterpret_cast<__nv_fp8x2_storage_t*>(s.q8 + i) = h;
            const float2 hb = __half22float2(__half2(__nv_cvt_fp8x2_to_halfraw2(h, __NV_E4M3)));
            rmax = fmaxf(rmax, fmaxf(fabsf(fmaf(-lq.s_hi, hb.x, v.x)), fabsf(fmaf(-lq.s_hi, hb.y, v.y))));
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(FULL, rmax, o));
        lq.s_lo = rmax > 0.f ? rmax / 448.0f : 1.0f;
        const float inv_lo = 1.0f / lq.s_lo;
        __syncwarp();
        for (int i = 2 * lane; i < (int)D; i += 64) {
            const float2 v = make_float2(i < dim ? s.q[i] : 0.f, i + 1 < dim ? s.q[i + 1] : 0.f);
            const __nv_fp8x2_storage_t h = *reinterpret_cast<const __nv_fp8x2_storage_t*>(s.q8 + i);
            const float2 hb = __half22float2(__half2(__nv_cvt_fp8x2_to_halfraw2(h, __NV_E4M3)));
            const float2 r = make_float2(fmaf(-lq.s_hi, hb.x, v.x) * inv_lo, fmaf(-lq.s_hi, hb.y, v.y) * inv_lo);
            *reinterpret_cast<__nv_fp8x2_storage_t*>(s.q8 + D + i) =
                __nv_cvt_float2_to_fp8x2(r, __NV_SATFINITE, __NV_E4M3);
        }
    }
    const uint32_t nvis = 1u << p.log2_vis;
    for (uint32_t i = lane; i < nvis; i += 32) s.vis[i] = INVALID_ID;
    __syncwarp();
    LPT(0);

    // ---- upper-layer greedy descent (hnswalg.h:1274-1302) on the fp8 rows
    uint32_t cur = p.ep, unused;
    if (lane == 0) s.cid[0] = cur;
    __syncwarp();
    float curd = __shfl_sync(FULL, lean_pass<SPACE, NS, MULTI>(p, s, lq, 0, 1, lane, unused), 0);
    __syncwarp();
    ct.upper_dists += 1;
    const uint32_t up_stride = p.maxM + 1;
    // the upper-layer offset of the current node; each pass loads its
    // candidates' offsets beside their rows, so the next hop's is known
    uint32_t cur_off = LCHK(cur < p.count, 272, cur, 0) ? __ldg(p.upper_off + cur) : 0xffffffffu;
    for (int level = p.maxlevel; level > 0; level--) {
        while (true) {
            if (!LCHK(cur < p.count && cur_off != 0xffffffffu, 270, cur, level)) break;
            const uint32_t* row = p.upper_links + (size_t)(cur_off + (uint32_t)(level - 1)) * up_stride;
            const int cnt = LCHK((__ldg(row) & 0xffffu) <= p.maxM, 271, __ldg(row), cur) ? (int)(__ldg(row) & 0xffffu) : 0;
            ct.upper_hops += 1;
            ct.upper_dists += cnt;
            float best = curd;
            uint32_t best_id = INVALID_ID, best_off = 0xffffffffu;
            for (int c0 = 0; c0 < cnt; c0 += 64) {
                const int n = min(64, cnt - c0);
                const uint32_t ida = lane < n ? __ldg(row + 1 + c0 + lane) : INVALID_ID;
                const uint32_t idb = lane + 32 < n ? __ldg(row + 1 + c0 + lane + 32) : INVALID_ID;
                if (lane < n) s.cid[lane] = ida;
                if (lane + 32 < n) s.cid[lane + 32] = idb;
                const uint32_t offa = ida < p.count ? __ldg(p.upper_off + ida) : 0xffffffffu;
                const uint32_t offb = idb < p.count ? __ldg(p.upper_off + idb) : 0xffffffffu;
                __syncwarp();
                uint32_t i0, i1 = INVALID_ID;
                float d0 = lean_pass<SPACE, NS, MULTI>(p, s, lq, 0, n, lane, i0);
                float d1 = __int_as_float(0x7f800000);
                if (n > 32) d1 = lean_pass<SPACE, NS, MULTI>(p, s, lq, 32, n, lane, i1);
                if (lane >= n) d0 = __int_as_float(0x7f800000);
                if (lane + 32 >= n) d1 = __int_as_float(0x7f800000);
                float m = fminf(d0, d1);
#pragma unroll
                for (int o = 16; o; o >>= 1) m = fminf(m, __shfl_xor_sync(FULL, m, o));
                if (m < best) {
                    // the first neighbour in list order with that distance
                    const unsigned h0 = __ballot_sync(FULL, d0 == m), h1 = __ballot_sync(FULL, d1 == m);
                    const int src = h0 ? __ffs(h0) - 1 : __ffs(h1) - 1;
                    best = m;
                    best_id = __shfl_sync(FULL, h0 ? i0 : i1, src);
                    best_off = __shfl_sync(FULL, h0 ? offa : offb, src);
                }
                __syncwarp();
            }
            if (best_id == INVALID_ID) break;
            cur = best_id;
            curd = best;
            cur_off = best_off;
        }
    }

    LPT(1);
    // ---- level-0 beam
    const int ef = (int)p.ef;
    const int kq = (int)p.k;
    const int W = (int)p.lean_w;
    const int maxM0 = (int)p.maxM0;
    int psize = 1, hint = 0;
    if (lane == 0) {
        s.pool[0] = mkkey(curd, cur);
        s.vis[vis_slot(cur, p.log2_vis)] = cur;
    }
    __syncwarp();
    const float d_entry = curd;
    LeanTerm ts;
    ts.next = TERM ? p.term_period : 0u;
    while (true) {
        // ---- the (up to) W best unexpanded pool entries
        uint32_t cand0 = INVALID_ID, cand1 = INVALID_ID, next_dk = 0xffffffffu;
        int sel = 0;
        for (int b = hint; b < psize && sel < W; b += 32) {
            const int i = b + lane;
            const uint64_t e = i < psize ? s.pool[i] : 0ull;
            const bool u = i < psize && !((uint32_t)e & EXP_BIT);
            const unsigned m = __ballot_sync(FULL, u);
            if (!m) {
                if (sel == 0) hint = min(b + 32, psize);
                continue;
            }
            const int take = min(__popc(m), W - sel);
            if (u && __popc(m & lanemask_lt()) < take && LCHK(i < ef && psize <= ef, 230, i, psize))
                s.pool[i] = e | EXP_BIT;
            const int src0 = __ffs(m) - 1;
            const uint32_t id0s = __shfl_sync(FULL, kid(e), src0);
            const uint32_t dk0 = __shfl_sync(FULL, khi(e), src0);
            const int src1 = take > 1 ? __ffs(m & (m - 1)) - 1 : src0;
            const uint32_t id1s = __shfl_sync(FULL, kid(e), src1);
            if (sel == 0) {
                cand0 = id0s;
                next_dk = dk0;
                hint = b + src0;
                if (take > 1) cand1 = id1s;
            } else {
                cand1 = id0s;
            }
            sel += take;
        }
        __syncwarp();
        LPT(2);
        if (sel == 0) break;
        // ---- link slots j = lane and lane + 32 (row j / maxM0, entry j % maxM0),
        // loaded before a checkpoint so that the network runs in their shadow
        uint32_t id0, id1;
        lean_links(p, maxM0, sel, cand0, cand1, lane, id0, id1);
        // a checkpoint falls due every term_period expansions; it is taken
        // (trace mode records it, learned mode consults the network) at the
        // first iteration from then on where the top-k has not changed for a
        // period and no unexpanded candidate is closer than the current k-th
        // result, the only states in which stopping can keep the top-k
        if (TERM && ct.l0_exp >= ts.next && ct.l0_exp - ts.last_change >= p.term_period && psize >= kq &&
            next_dk > khi(s.pool[kq - 1])) {
            const bool stop =
                lean_checkpoint<SPACE, TERM>(p, s, lane, qi, ct.l0_exp, ct.l0_dists, psize, next_dk, d_entry, lq.qn, ts);
            while (ts.next <= ct.l0_exp) ts.next += p.term_period;
            if (stop) break;
        }
        LPT(7);
        if (ct.l0_exp >= p.max_expansions) break;
        ct.l0_exp += (uint32_t)sel;

        bool f0 = id0 != INVALID_ID, f1 = id1 != INVALID_ID;
        if (!p.links_unique) {
            const unsigned p0 = __match_any_sync(FULL, id0), p1 = __match_any_sync(FULL, id1);
            f0 = f0 && __ffs(p0) - 1 == lane;
            f1 = f1 && __ffs(p1) - 1 == lane;
        }
        // visited cache, first slot set then the second, so that a node that
        // both rows link is evaluated once (the merge drops any duplicate a
        // cache collision lets through)
        const uint32_t sl0 = f0 ? vis_slot(id0, p.log2_vis) : 0u;
        if (f0 && s.vis[sl0] == id0) f0 = false;
        __syncwarp();
        if (f0) s.vis[sl0] = id0;
        __syncwarp();
        const uint32_t sl1 = f1 ? vis_slot(id1, p.log2_vis) : 0u;
        if (f1 && s.vis[sl1] == id1) f1 = false;
        __syncwarp();
        if (f1) s.vis[sl1] = id1;
        const unsigned m0 = __ballot_sync(FULL, f0), m1 = __ballot_sync(FULL, f1);
        const int n0 = __popc(m0);
        const int nnew = n0 + __popc(m1);
        if (f0 && LCHK(id0 < p.count, 214, id0, lane)) s.cid[__popc(m0 & lanemask_lt())] = id0;
        if (f1 && LCHK(id1 < p.count, 215, id1, lane)) s.cid[n0 + __popc(m1 & lanemask_lt())] = id1;
        __syncwarp();
        LPT(3);

        bool accA = false, accB = false;
        uint64_t kA = ~0ull, kB = ~0ull;
        if (nnew > 0) {
            ct.l0_dists += (uint32_t)nnew;
            // ---- distances (lane L: candidates L and L + 32)
            uint32_t cidA, cidB = INVALID_ID;
            const float dA = lean_pass<SPACE, NS, MULTI>(p, s, lq, 0, nnew, lane, cidA);
            float dB = 0.f;
            if (nnew > 32) dB = lean_pass<SPACE, NS, MULTI>(p, s, lq, 32, nnew, lane, cidB);
            LPT(4);
            // ---- acceptance by the beam's bound
            const bool full = psize == ef;
            const uint32_t lbk = full ? khi(s.pool[psize - 1]) : 0xffffffffu;
            const uint32_t dkA = fkey(dA), dkB = fkey(dB);
            accA = lane < nnew && (!full || dkA < lbk);
            accB = lane + 32 < nnew && (!full || dkB < lbk);
            if (accA) kA = ((uint64_t)dkA << 32) | cidA;
            if (accB) kB = ((uint64_t)dkB << 32) | cidB;
        }
        const unsigned am0 = __ballot_sync(FULL, accA), am1 = __ballot_sync(FULL, accB);
        const int na0 = __popc(am0);
        const int na = na0 + __popc(am1);
        LPT(5);
        if (na == 0) continue;
        if (accA) s.lacc[__popc(am0 & lanemask_lt())] = kA;
        if (accB) s.lacc[na0 + __popc(am1 & lanemask_lt())] = kB;
        __syncwarp();
        // ---- merge into the pool (at most 32 keys per round)
        bool top = false;
        for (int b0 = 0; b0 < na; b0 += 32) {
            const int nr = min(32, na - b0);
            const bool have = lane < nr;
            const uint64_t key = have ? s.lacc[b0 + lane] : ~0ull;
            int pos = 0;
            bool keep = have;
            if (have) {
                pos = lower_bound_masked(s.pool, psize, key);
                if (pos < psize && (s.pool[pos] & KEY_MASK) == key) keep = false;  // already in the pool
            }
            const unsigned hm = __ballot_sync(FULL, keep);
            if (keep) {
                const unsigned peers = __match_any_sync(hm, key);
                keep = __ffs(peers) - 1 == lane;  // one copy of a key evaluated twice
            }
            const unsigned amask = __ballot_sync(FULL, keep);
            if (!amask) continue;
            bool t2 = false;
            hint = min(hint, lean_merge(s.pool, psize, ef, amask, key, pos, lane, kq, t2, s.lacc + b0));
            top |= t2;
        }
        if (TERM && top) {
            ts.last_change = ct.l0_exp;
            ts.nchange++;
        }
        LPT(6);
    }
    if (TERM == 1) lean_final_row<SPACE>(p, s, lane, qi, ct.l0_exp, ct.l0_dists, psize, d_entry, lq.qn, ts);

    // ---- exact re-rank, then the k best ordered by (distance, label)
    lean_rerank<SPACE>(p, s, lane, psize);
    const int kk = min(kq, psize);
    uint64_t* olab = p.out_labels + (size_t)qi * kq;
    float* odist = p.out_dists + (size_t)qi * kq;
    for (int r = lane; r < kk; r += 32) {
        uint64_t e = s.pool[r];
        if (!LCHK(kid(e) < p.count, 260, kid(e), r)) e = 0;
        const uint32_t dk = khi(e);
        const uint64_t lab = p.labels[kid(e)];
        int st = r;
        while (st > 0 && khi(s.pool[st - 1]) == dk) st--;
        int below = 0;
        for (int t = st; t < kk && khi(s.pool[t]) == dk; t++) {
            const uint64_t lt = LCHK(kid(s.pool[t]) < p.count, 261, kid(s.pool[t]), t) ? p.labels[kid(s.pool[t])] : 0;
            if (t != r && (lt < lab || (lt == lab && t < r))) below++;
        }
        if (LCHK(st + below < kk, 262, st + below, kk)) {
            olab[st + below] = lab;
            odist[st + below] = funkey(dk);
        }
    }
    for (int r = kk + lane; r < kq; r += 32) {
        olab[r] = ~0ull;
        odist[r] = __int_as_float(0x7f800000);
    }
    if (lane == 0) p.out_counts[qi] = kk;
    LPT(8);
}

// Query warps per CTA of each kernel form.
template <int TERM>
struct LeanCta {
    static constexpr bool kSmemModel = TERM == 2 && HNSWGPU_LEAN_MODEL_SMEM;
    static constexpr int kWarps = kSmemModel ? kLeanWarpsPerBlockLearned : kLeanWarpsPerBlock;
    static constexpr size_t kModel = kSmemModel ? kLeanModelSmem : 0;
    // learned stop in shared memory: the network copy limits residency to four CTAs (16 warps)
    static constexpr int kMinBlocks = kSmemModel ? 4 : HNSWGPU_MINB_LEAN;
};

template <int SPACE, int TERM, int NS, bool MULTI>
__global__ void __launch_bounds__(LeanCta<TERM>::kWarps * 32, LeanCta<TERM>::kMinBlocks)
    hnsw_lean_kernel(SearchParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (LeanCta<TERM>::kSmemModel) {
        const uint4* src = reinterpret_cast<const uint4*>(p.term_model);
        uint4* dst = reinterpret_cast<uint4*>(smem);
        for (uint32_t i = threadIdx.x; i < (uint32_t)(kTermPackedBytes / 16); i += blockDim.x) dst[i] = __ldg(src + i);
        __syncthreads();
    }
    unsigned char* base = smem + LeanCta<TERM>::kModel + (size_t)warp * p.warp_smem;
    LeanSmem s;
    s.q = reinterpret_cast<float*>(base + p.off_query);
    s.q8 = base + p.off_q8;
    s.cid = reinterpret_cast<uint32_t*>(base + p.off_cid);
    s.lacc = reinterpret_cast<uint64_t*>(base + p.off_lacc);
    s.pool = reinterpret_cast<uint64_t*>(base + p.off_pool);
    s.vis = reinterpret_cast<uint32_t*>(base + p.off_vis);
    s.stage = base + p.off_stage;
    s.tails = reinterpret_cast<float2*>(base + p.off_lacc + 64 * 8);
    s.model = reinterpret_cast<const float*>(smem);
    LeanClock lc;
    if (!LCHK(p.off_vis + ((size_t)4 << p.log2_vis) <= p.warp_smem && p.off_pool + (size_t)8 * p.ef <= p.off_vis,
              280, p.off_vis, p.warp_smem))
        return;
    while (true) {
        uint32_t qi = 0;
        if (lane == 0) {
            qi = atomicAdd(p.work_counter, 1u);
            if (qi >= p.nq) qi = 0xffffffffu;
        }
        qi = __shfl_sync(FULL, qi, 0);
        if (qi >= p.nq) break;
        LeanCounters ct = {0, 0, 0, 0};
        lean_search<SPACE, TERM, NS, MULTI>(p, s, qi, lane, ct, lc);
        if (p.trace && lane == 0) {
            uint32_t* t = p.trace + (size_t)qi * 4;
            t[0] = ct.upper_hops;
            t[1] = ct.upper_dists;
            t[2] = ct.l0_exp;
            t[3] = ct.l0_dists;
        }
    }
#ifdef HNSWGPU_PHASE_TIMING
    if (lane == 0 && p.phase_cycles)
        for (int i = 0; i < 9; i++) atomicAdd(p.phase_cycles + i, (unsigned long long)lc.acc[i]);
#endif
    // the last block to finish re-arms this launch's counters
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(p.done_counter, 1u) == gridDim.x - 1) {
            *p.work_counter = 0;
            *p.done_counter = 0;
            __threadfence();
        }
    }
}

template <int SPACE, int TERM, int NS, bool MULTI>
cudaError_t launch_lean_t(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    static LaunchCache cache;  // per device: opt-in shared memory and occupancy
    const void* fn = (const void*)hnsw_lean_kernel<SPACE, TERM, NS, MULTI>;
    constexpr int wpb = LeanCta<TERM>::kWarps;
    const size_t smem = LeanCta<TERM>::kModel + (size_t)p.warp_smem * wpb;
    int occ_per_sm = 0;
    cudaError_t e = cache.blocks_per_sm(fn, wpb * 32, smem, &occ_per_sm);
    if (e != cudaSuccess) return e;
    if (occ_per_sm < 1) return cudaErrorInvalidConfiguration;
    const uint64_t need = (p.nq + wpb - 1) / wpb;
    uint64_t blocks = (uint64_t)occ_per_sm * (uint64_t)num_sms;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    if (blocks_out) *blocks_out = (int)blocks;
    hnsw_lean_kernel<SPACE, TERM, NS, MULTI><<<(unsigned)blocks, wpb * 32, smem, stream>>>(p);
    return cudaGetLastError();
}

template <int SPACE, int TERM>
cudaError_t launch_lean_d(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    switch (p.trow_bytes - 16) {
        case 32: return launch_lean_t<SPACE, TERM, 1, false>(p, num_sms, stream, blocks_out);
        case 64: return launch_lean_t<SPACE, TERM, 2, false>(p, num_sms, stream, blocks_out);
        case 96: return launch_lean_t<SPACE, TERM, 3, false>(p, num_sms, stream, blocks_out);
        case 128: return launch_lean_t<SPACE, TERM, 4, false>(p, num_sms, stream, blocks_out);
        default: return launch_lean_t<SPACE, TERM, 4, true>(p, num_sms, stream, blocks_out);
    }
}

template <int SPACE>
cudaError_t launch_lean_s(const SearchParams& p, int num_sms, cudaStream_t stream, int* blocks_out) {
    if (p.term_mode == 1) return launch_lean_d<SPACE, 1>(p, num_sms, stream, blocks_out);
    if (p.term_mode == 2) return launch_lean_d<SPACE, 2>(p, num_sms, stream, blocks_out);
    return launch_lean_d<SPACE, 0>(p, num_sms, stream, blocks_out);
}

}  // namespace

bool lean_eligible(const SearchParams& p) {
    if (p.prec != 2 || !p.bare || p.exact || p.tie_list || p.eps_mode || !p.fast16) return false;
    if (p.maxM0 == 0 || p.maxM0 > 64) return false;
    const uint32_t D = p.trow_bytes - 16;
    return D % 32 == 0 && (D <= 128 || D % 128 == 0);
}

size_t lean_smem_layout(SearchParams& p) {
    const uint32_t D = p.trow_bytes - 16;
    size_t off = 0;
    p.off_query = (uint32_t)off;
    off += ((size_t)p.row_floats * 4 + 15) & ~(size_t)15;
    p.off_q8 = (uint32_t)off;
    off += ((size_t)2 * D + 15) & ~(size_t)15;
    p.off_cid = (uint32_t)off;
    off += 64 * 4;
    p.off_lacc = (uint32_t)off;
    off += 64 * 8 + 32 * 8;  // accepted keys, then the pass's 32 row tails
    // stage slots: one 128-byte block (or the whole shorter row) plus 16 bytes
    // of padding, so that the two quads of a quarter-warp read disjoint banks
    p.lean_stage = std::min<uint32_t>(D, 128u) + 16u;
    p.off_stage = (uint32_t)off;
    off += (size_t)32 * p.lean_stage;
    p.off_pool = (uint32_t)off;
    off += (size_t)p.ef * 8;
    off = (off + 15) & ~(size_t)15;
    // the visited cache doubles as the re-rank's sort buffer (ef keys)
    while (((size_t)4 << p.log2_vis) < (size_t)8 * p.ef) p.log2_vis++;
    p.off_vis = (uint32_t)off;
    off += (size_t)4 << p.log2_vis;
    off = (off + 127) & ~(size_t)127;
    p.warp_smem = (uint32_t)off;
    return off;
}

cudaError_t launch_hnsw_lean(const SearchParams& p, int space, int num_sms, cudaStream_t stream, int* blocks_out) {
    return space == 0 ? launch_lean_s<0>(p, num_sms, stream, blocks_out)
                      : launch_lean_s<1>(p, num_sms, stream, blocks_out);
}

}  // namespace hnswgpu
