// Tensor-core brute force (sm_100a): low-precision scores on tcgen05, fused
// candidate filtering, exact float32 re-rank.  Replaces, for the BF16 / FP8
// precisions of a BruteforceSearch index, the linear scan of
// hnswlib/bruteforce.h:106-125 (whose exact form is bf_search.cu).
//
// A query's exact top-k is found in three steps:
// 1. threshold: scores of every query against a strided sample of the rows
//    (the same kernel, MODE 1) give each query the 16th-best approximate
//    distance of the sample, tau_q; the sample size is chosen so that about
//    5 x R rows of the whole set are expected below tau_q (R = over-fetch);
// 2. scores: S = Q . X^T over all rows (MODE 0), 128 queries x 256 rows per
//    tile, accumulated in TMEM by tcgen05.mma (kind::f16 for bf16,
//    kind::f8f6f4 for e4m3 with per-row scales); the epilogue turns each
//    score into an approximate distance (IP: -s, L2: |x|^2 - 2 s) and
//    appends (distance, row) to the query's candidate list when it is at
//    most tau_q -- nothing of S is written to memory;
// 3. select + re-rank (one CTA per query): the R smallest approximate
//    distances are kept, their float32 rows re-scored with the reference's
//    distance function (same summation order), and the k best by
//    (distance, label) returned, as BruteforceSearch orders them.
// A query whose list overflowed, or which found fewer than R candidates
// below a sampled threshold, is answered by the exact kernel instead.
//
// The GEMM is warp-specialised: warp 0 issues TMA loads (128-byte swizzled
// K-major tiles, 4-stage ring), one thread of warp 1 issues the MMAs
// (M=128, N=256, cta_group::1) and owns the TMEM allocation (two 256-column
// accumulators, so the epilogue of one tile overlaps the MMAs of the next),
// warps 2-5 drain TMEM (each warp its 32-lane quarter).  Every wait is
// bounded; on a timeout the kernel raises a status bit and stops.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>

#include "bf_tc.h"
#include "device_common.cuh"
#include "hnsw_search.h"

namespace hnswgpu {
namespace {

constexpr int kStages = 4;
constexpr int kTileM = 128;                    // queries per tile
constexpr int kTileN = 256;                    // rows per tile
constexpr int kKBytes = 128;                   // bytes of K per stage (one swizzle atom)
constexpr int kABytes = kTileM * kKBytes;      // 16 KB
constexpr int kBBytes = kTileN * kKBytes;      // 32 KB
constexpr int kStageBytes = kABytes + kBBytes;
// warp 0: TMA producer; warp 1: MMA issuer; warps 2-9: epilogue, two warps
// per TMEM lane quarter (each reads half of a tile's columns), so that every
// scheduler has two epilogue warps to interleave
constexpr int kEpiWarps = 8;
constexpr int kThreads = (2 + kEpiWarps) * 32;
constexpr int kTopT = 16;                      // sample rank of the threshold
constexpr int kStageC = 4;                     // candidates staged per epilogue thread and tile
// Resident query tile (fp8, K <= 768 bytes): the work item's A tiles stay in
// shared memory for all its row tiles (one L2 read instead of one per row
// tile) and only the B tiles stream, through a 3-stage ring; the two layouts
// take the same bytes (6 x 16 KB + 3 x 32 KB = 4 x 48 KB).
constexpr int kResAKb = 6;
constexpr int kStagesB = 3;
static_assert(kResAKb * kABytes + kStagesB * kBBytes == kStages * kStageBytes, "resident layout");

#ifdef HNSWGPU_TC_TIMING
// Opt-in role timing of the scores pass (not in the shipped library): per
// CTA, cycles of [producer wait-empty, producer total, MMA wait-full, MMA
// wait-tmem, MMA total, epilogue wait-tfull, epilogue busy, epilogue total].
__device__ unsigned long long g_tc_timing[256][10];
#define TCT_ADD(i, v) atomicAdd(&g_tc_timing[blockIdx.x & 255][i], (unsigned long long)(v))
#else
#define TCT_ADD(i, v)
#endif

struct TcSmem {
    float2 hinfo[2][kTileN];  // per-row helpers of the tiles in the two accumulators
    uint64_t cst[2][128][2][kStageC];  // candidates of the current / previous tile per epilogue thread
    uint64_t full[kStages], empty[kStages], tfull[2], tempty[2], done;
    uint64_t afull, aempty;  // resident query tile loaded / no longer read by the MMAs
    uint32_t tmem, error;
};
constexpr size_t kSmemBytes = 1024 + (size_t)kStages * kStageBytes + sizeof(TcSmem);

// Bounded pipeline wait without a suspend-time hint: the tile pipeline waits
// ~26 times per tile, and a suspended thread's late wake-up cost more than
// the spin (measured).  The bound (2^26 polls, seconds) only ends a wait
// that can no longer complete.
__device__ __forceinline__ bool tc_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < (1u << 26); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// UMMA shared-memory descriptor of a K-major tile with 128-byte swizzle:
// 8-row core groups 1024 bytes apart, version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

template <int PREC>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    if (PREC == 1) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
            "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
            "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
    }
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 64 consecutive fp32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float* v) {
    uint32_t r[64];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; i++) v[i] = __uint_as_float(r[i]);
}

// One accumulator column of this thread's TMEM lane (whole warp).
__device__ __forceinline__ float tmem_ld1(uint32_t taddr) {
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    return __uint_as_float(r);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// MODE 0: filter-append pass over all rows; MODE 1: threshold pass over the
// sample (one work item per query tile, top-16 kept in registers).
template <int PREC, int SPACE, int MODE, bool RESA>
__global__ void __launch_bounds__(kThreads, 1)
    bf_tc_kernel(const __grid_constant__ CUtensorMap qmap, const __grid_constant__ CUtensorMap xmap, TcArgs a) {
    extern __shared__ __align__(1024) unsigned char raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~(uintptr_t)1023);
    TcSmem& s = *reinterpret_cast<TcSmem*>(base + (size_t)kStages * kStageBytes);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // bf16 inner product needs no per-row helper (every scale is 1)
    constexpr bool NEEDH = !(PREC == 1 && SPACE == 1);

    const uint32_t q_tiles = (a.nq + kTileM - 1) / kTileM;
    const uint32_t n_tiles = (a.n_rows + kTileN - 1) / kTileN;
    const uint32_t chunk = MODE == 1 ? n_tiles : a.chunk_tiles;
    const uint32_t n_chunks = (n_tiles + chunk - 1) / chunk;
    const uint32_t items = q_tiles * n_chunks;
    const int kb_count = (int)a.k_blocks;

    if (threadIdx.x == 0) {
        for (int i = 0; i < kStages; i++) {
            mbar_init(&s.full[i], 1);
            mbar_init(&s.empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(&s.tfull[i], 1);
            mbar_init(&s.tempty[i], kEpiWarps * 32);
        }
        mbar_init(&s.done, 1);
        mbar_init(&s.afull, 1);
        mbar_init(&s.aempty, 1);
        s.error = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&s.tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s.tmem;
    volatile uint32_t* err = &s.error;

    if (warp == 0) {
        // ---- TMA producer
        if (lane == 0) {
            int stage = 0, hacc = 0;
            uint32_t phase = 0, haphase = 0, nitem = 0;
            const long long p0 = clock64();
            constexpr int nst = RESA ? kStagesB : kStages;
            for (uint32_t it = blockIdx.x; it < items && !*err; it += gridDim.x, nitem++) {
                const uint32_t qt = it % q_tiles, ck = it / q_tiles;
                const uint32_t t_end = min(n_tiles, (ck + 1) * chunk);
                if (RESA) {
                    // the previous item's MMAs have finished with the resident tile
                    if (nitem > 0 && !tc_wait(&s.aempty, (nitem - 1) & 1u)) {
                        *err = 1;
                        break;
                    }
                    mbar_arrive_expect_tx(&s.afull, (uint32_t)(kb_count * kABytes));
                    for (int kb = 0; kb < kb_count; kb++)
                        tma_load_2d(base + (size_t)kb * kABytes, &qmap, kb * kKBytes, (int)(qt * kTileM), &s.afull);
                }
                for (uint32_t t = ck * chunk; t < t_end && !*err; t++) {
                    // the helper slot of this tile is the one of its accumulator:
                    // free once the epilogue released that accumulator
                    if (NEEDH && !tc_wait(&s.tempty[hacc], haphase ^ 1u)) {
                        *err = 1;
                        break;
                    }
                    for (int kb = 0; kb < kb_count; kb++) {
                        const long long w0 = clock64();
                        if (!tc_wait(&s.empty[stage], phase ^ 1u)) {
                            *err = 1;
                            break;
                        }
                        TCT_ADD(0, clock64() - w0);
                        const bool with_h = NEEDH && kb == 0;
                        const int x = kb * (PREC == 1 ? kKBytes / 2 : kKBytes);
                        if (RESA) {
                            unsigned char* sb = base + (size_t)kResAKb * kABytes + (size_t)stage * kBBytes;
                            mbar_arrive_expect_tx(&s.full[stage], kBBytes + (with_h ? kTileN * 8 : 0));
                            tma_load_2d(sb, &xmap, x, (int)(t * kTileN), &s.full[stage]);
                        } else {
                            unsigned char* sa = base + (size_t)stage * kStageBytes;
                            mbar_arrive_expect_tx(&s.full[stage], kStageBytes + (with_h ? kTileN * 8 : 0));
                            tma_load_2d(sa, &qmap, x, (int)(qt * kTileM), &s.full[stage]);
                            tma_load_2d(sa + kABytes, &xmap, x, (int)(t * kTileN), &s.full[stage]);
                        }
                        if (with_h) bulk_g2s(&s.hinfo[hacc][0], a.rowinfo + (size_t)t * kTileN, kTileN * 8, &s.full[stage]);
                        if (++stage == nst) {
                            stage = 0;
                            phase ^= 1u;
                        }
                    }
                    if (++hacc == 2) {
                        hacc = 0;
                        haphase ^= 1u;
                    }
                }
            }
            TCT_ADD(1, clock64() - p0);
        }
    } else if (warp == 1) {
        // ---- MMA issuer
        if (lane == 0) {
            // D fp32 (bits 4-5), A/B bf16 (bits 7-9, 10-12) or e4m3 (0),
            // K-major A and B, N >> 3 at bit 17, M >> 4 at bit 24
            const uint32_t idesc = (1u << 4) | (PREC == 1 ? (1u << 7) | (1u << 10) : 0u) |
                                   ((uint32_t)(kTileN >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
            int stage = 0, acc = 0;
            uint32_t phase = 0, aphase = 0, nitem = 0;
            constexpr int nst = RESA ? kStagesB : kStages;
            const long long m0 = clock64();
            for (uint32_t it = blockIdx.x; it < items && !*err; it += gridDim.x, nitem++) {
                const uint32_t ck = it / q_tiles;
                const uint32_t t_end = min(n_tiles, (ck + 1) * chunk);
                if (RESA && !tc_wait(&s.afull, nitem & 1u)) {
                    *err = 1;
                    break;
                }
                for (uint32_t t = ck * chunk; t < t_end && !*err; t++) {
                    const long long w1 = clock64();
                    if (!tc_wait(&s.tempty[acc], aphase ^ 1u)) {
                        *err = 1;
                        break;
                    }
                    TCT_ADD(3, clock64() - w1);
                    tc_fence_after();
                    const uint32_t d = tmem + (uint32_t)acc * kTileN;
                    for (int kb = 0; kb < kb_count; kb++) {
                        const long long w2 = clock64();
                        if (!tc_wait(&s.full[stage], phase)) {
                            *err = 1;
                            break;
                        }
                        TCT_ADD(2, clock64() - w2);
                        tc_fence_after();
                        uint64_t da, db;
                        if (RESA) {
                            da = umma_desc(smem_u32(base + (size_t)kb * kABytes));
                            db = umma_desc(smem_u32(base + (size_t)kResAKb * kABytes + (size_t)stage * kBBytes));
                        } else {
                            const uint32_t sa = smem_u32(base + (size_t)stage * kStageBytes);
                            da = umma_desc(sa);
                            db = umma_desc(sa + kABytes);
                        }
#pragma unroll
                        for (int ks = 0; ks < 4; ks++)  // 32 bytes of K per MMA
                            umma<PREC>(d, da + 2 * ks, db + 2 * ks, idesc, (kb | ks) != 0);
                        umma_commit(&s.empty[stage]);
                        if (++stage == nst) {
                            stage = 0;
                            phase ^= 1u;
                        }
                    }
                    umma_commit(&s.tfull[acc]);
                    if (++acc == 2) {
                        acc = 0;
                        aphase ^= 1u;
                    }
                }
                // the resident query tile is free once this item's MMAs complete
                if (RESA) umma_commit(&s.aempty);
            }
            TCT_ADD(4, clock64() - m0);
            // every MMA issued has completed before TMEM is released
            umma_commit(&s.done);
            tc_wait(&s.done, 0);
        }
        __syncwarp();
    } else {
        // ---- epilogue: warps 2-9, TMEM lane quarter = warp % 4; half h of
        // them reads the tile's columns [128 h, 128 h + 128) (the threshold
        // pass: half 0 reads all 256, half 1 only releases the accumulator)
        const int quarter = warp & 3;
        const int half = (warp - 2) >> 2;
        const int r = quarter * 32 + lane;  // query row within the tile
        const int cb_begin = MODE == 1 ? 0 : 2 * half;
        const int cb_end = MODE == 1 ? (half == 0 ? 4 : 0) : 2 * half + 2;
        int acc = 0;
        uint32_t aphase = 0;
        const long long e0 = clock64();
        for (uint32_t it = blockIdx.x; it < items && !*err; it += gridDim.x) {
            const uint32_t qt = it % q_tiles, ck = it / q_tiles;
            const uint32_t q = qt * kTileM + r;
            const bool qok = q < a.nq;
            // queries past nq get tau = -inf: no candidate passes
            const float tau = !qok ? -__int_as_float(0x7f800000)
                                   : (MODE == 0 ? a.tau[q] : __int_as_float(0x7f800000));
            const float sq = qok ? a.qscale[q] : 0.f;
            // IP: d = -(s sq sc); L2: d = |x|^2 - 2 s sq sc
            const float coef = (SPACE == 0 ? -2.0f : -1.0f) * sq;
            // candidates of a tile are staged, then claimed with one atomic
            // whose result is used a tile later (its latency hidden)
            uint64_t* cst = &s.cst[half][r][0][0];
            int cb_cur = 0, n_cur = 0, n_prev = 0;
            uint32_t prev_slot = 0;
            float top[kTopT];
#pragma unroll
            for (int i = 0; i < kTopT; i++) top[i] = __int_as_float(0x7f800000);
            const uint32_t t_end = min(n_tiles, (ck + 1) * chunk);
            for (uint32_t t = ck * chunk; t < t_end; t++) {
                const long long w3 = clock64();
                if (!tc_wait(&s.tfull[acc], aphase)) {
                    *err = 1;
                    break;
                }
                const long long b0 = clock64();
                if (lane == 0) TCT_ADD(5, b0 - w3);
                tc_fence_after();
                const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)acc * kTileN;
                const float2* hinfo = s.hinfo[acc];
#pragma unroll 1
                for (int cb = cb_begin; cb < cb_end; cb++) {
                    float v[64];
#ifdef HNSWGPU_TC_TIMING
                    const long long l0 = clock64();
#endif
                    tmem_ld64(taddr + (uint32_t)(cb * 64), v);
#ifdef HNSWGPU_TC_TIMING
                    if (lane == 0) TCT_ADD(8, clock64() - l0);
#endif
                    // (1) unrolled and small: distances and a mask of the
                    // columns under the threshold (rare)
                    const float thr = MODE == 0 ? tau : top[kTopT - 1];
                    uint32_t m_lo = 0, m_hi = 0;
#pragma unroll
                    for (int j = 0; j < 64; j++) {
                        float dd;
                        if (!NEEDH) {
                            dd = v[j] * coef;
                        } else {
                            const float2 h = hinfo[cb * 64 + j];  // one broadcast shared-memory load
                            const float sv = PREC == 1 ? v[j] : v[j] * h.y;
                            dd = SPACE == 0 ? fmaf(sv, coef, h.x) : sv * coef;
                        }
                        const bool p = MODE == 0 ? dd <= thr : dd < thr;
                        if (j < 32) m_lo |= (uint32_t)p << j;
                        else m_hi |= (uint32_t)p << (j - 32);
                    }
                    // (2) rolled, warp-uniform: each column some lane passes;
                    // its score is read again from TMEM (one column)
                    uint64_t any = ((uint64_t)__reduce_or_sync(0xffffffffu, m_hi) << 32) |
                                   __reduce_or_sync(0xffffffffu, m_lo);
                    const uint64_t mine = ((uint64_t)m_hi << 32) | m_lo;
                    while (any) {
                        const int j = __ffsll((long long)any) - 1;
                        any &= any - 1;
                        const int col = cb * 64 + j;
                        __syncwarp();  // converge after the previous iteration's divergent tail
                        const float sc = tmem_ld1(taddr + (uint32_t)col);
                        if (!((mine >> j) & 1)) continue;
                        float dd;
                        if (!NEEDH) {
                            dd = sc * coef;
                        } else {
                            const float2 h = hinfo[col];
                            const float sv = PREC == 1 ? sc : sc * h.y;
                            dd = SPACE == 0 ? fmaf(sv, coef, h.x) : sv * coef;
                        }
                        const uint32_t lr = t * kTileN + (uint32_t)col;
                        const uint64_t g = (uint64_t)lr * a.row_step;
                        if (lr >= a.n_rows || (a.allow && !a.allow[g])) continue;
                        if (MODE == 0) {
                            const uint64_t key = mkkey(dd, (uint32_t)g);
                            if (n_cur < kStageC) {
                                cst[cb_cur * kStageC + n_cur++] = key;
                            } else {  // more than kStageC in one tile: direct append
                                const uint32_t slot = atomicAdd(a.cnt + q, 1u);
                                if (slot < a.cap) a.buf[(size_t)q * a.cap + slot] = key;
                            }
                        } else if (dd < top[kTopT - 1]) {
#pragma unroll
                            for (int i = 0; i < kTopT; i++) {
                                const float lo = fminf(dd, top[i]), hi = fmaxf(dd, top[i]);
                                top[i] = lo;
                                dd = hi;
                            }
                        }
                    }
                }
#ifdef HNSWGPU_TC_TIMING
                const long long f0 = clock64();
#endif
                if (MODE == 0) {
                    // write the previous tile's candidates (their slots were
                    // claimed a tile ago), then claim this tile's
                    for (int i = 0; i < n_prev; i++)
                        if (prev_slot + i < a.cap)
                            a.buf[(size_t)q * a.cap + prev_slot + i] = cst[(cb_cur ^ 1) * kStageC + i];
                    n_prev = n_cur;
                    if (n_cur) prev_slot = atomicAdd(a.cnt + q, (uint32_t)n_cur);
                    n_cur = 0;
                    cb_cur ^= 1;
                }
#ifdef HNSWGPU_TC_TIMING
                if (lane == 0) TCT_ADD(9, clock64() - f0);
#endif
                if (lane == 0) TCT_ADD(6, clock64() - b0);
                tc_fence_before();
                tc_arrive(&s.tempty[acc]);
                if (++acc == 2) {
                    acc = 0;
                    aphase ^= 1u;
                }
            }
            if (MODE == 1 && qok && half == 0) a.tau[q] = top[kTopT - 1];
            if (MODE == 0)  // the item's last claimed batch
                for (int i = 0; i < n_prev; i++)
                    if (prev_slot + i < a.cap)
                        a.buf[(size_t)q * a.cap + prev_slot + i] = cst[(cb_cur ^ 1) * kStageC + i];
        }
        if (lane == 0) TCT_ADD(7, clock64() - e0);
    }
    __syncthreads();
    if (threadIdx.x == 0 && *err) atomicOr(a.status, HNSWGPU_STATUS_TIMEOUT_BIT);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// ---------------------------------------------------------------------------
// Per-row helpers of the low-precision copy: (|x|^2 of the float32 row,
// per-row scale: the fp8 row's tail, 1 for bf16).
__global__ void tc_rowinfo_kernel(const float* __restrict__ vecs, uint32_t count, uint32_t dim, uint32_t row_floats,
                                  const unsigned char* __restrict__ tcopy, uint32_t trow_bytes, uint32_t prec,
                                  float2* __restrict__ out) {
    const uint64_t row = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= count) return;
    const float* x = vecs + row * row_floats;
    float s = 0.f;
    for (uint32_t i = lane; i < dim; i += 32) s = fmaf(x[i], x[i], s);
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const float sc = prec == 2 ? *reinterpret_cast<const float*>(tcopy + row * trow_bytes + trow_bytes - 16) : 1.f;
        out[row] = make_float2(s, sc);
    }
}

// Query prep: optional normalisation (the reference's normalize_vector order),
// then the low-precision row exactly as the index copy is made; per-query
// scale out.
__global__ void tc_query_prep_kernel(const float* __restrict__ q, uint32_t nq, uint32_t dim, uint32_t normalize,
                                     uint32_t prec, uint32_t trow_bytes, float* __restrict__ qf,
                                     unsigned char* __restrict__ qt, float* __restrict__ qscale) {
    const uint64_t row = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (row >= nq) return;
    const float* x = q + row * dim;
    float* y = qf + row * dim;
    const float sc = normalize ? norm_scale(x, (int)dim) : 1.f;
    for (uint32_t i = lane; i < dim; i += 32) y[i] = normalize ? x[i] * sc : x[i];
    __syncwarp();
    unsigned char* o = qt + row * trow_bytes;
    if (prec == 1) {
        __nv_bfloat16* ob = reinterpret_cast<__nv_bfloat16*>(o);
        for (uint32_t i = lane; i < trow_bytes / 2; i += 32) ob[i] = __float2bfloat16_rn(i < dim ? y[i] : 0.f);
        if (lane == 0) qscale[row] = 1.f;
        return;
    }
    float amax = 0.f;
    for (uint32_t i = lane; i < dim; i += 32) amax = fmaxf(amax, fabsf(y[i]));
#pragma unroll
    for (int of = 16; of; of >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, of));
    const float scale = amax > 0.f ? amax / 448.0f : 1.0f;
    const float inv = 1.0f / scale;
    const uint32_t data_bytes = trow_bytes - 16;
    for (uint32_t i = 2 * lane; i < data_bytes; i += 64) {
        float2 v = make_float2(i < dim ? y[i] * inv : 0.f, i + 1 < dim ? y[i + 1] * inv : 0.f);
        *reinterpret_cast<__nv_fp8x2_storage_t*>(o + i) = __nv_cvt_float2_to_fp8x2(v, __NV_SATFINITE, __NV_E4M3);
    }
    if (lane < 4) reinterpret_cast<float*>(o + data_bytes)[lane] = lane == 0 ? scale : 0.f;
    if (lane == 0) qscale[row] = scale;
}

// Helpers of the sampled rows, contiguous (the threshold pass reads them
// tile by tile with bulk copies).
__global__ void tc_gather_info_kernel(const float2* __restrict__ info, uint64_t n_sample, uint64_t step,
                                      float2* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_sample) out[i] = info[i * step];
}

// Row mask of an exact scan over an index with deleted elements: allowed by
// the caller's mask (if any) and not deleted.
__global__ void scan_mask_kernel(const uint32_t* __restrict__ deleted_bits, const uint8_t* __restrict__ allow,
                                 uint64_t n, uint8_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool del = (deleted_bits[i >> 5] >> (i & 31)) & 1u;
    out[i] = (!del && (!allow || allow[i])) ? 1 : 0;
}

__global__ void tc_fill_kernel(float* p, uint64_t n, float v) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// Step 3: one CTA per query.
template <int SPACE>
__global__ void __launch_bounds__(256) tc_select_rerank_kernel(TcSelectArgs a) {
    extern __shared__ __align__(1024) unsigned char sel_raw[];
    const uint32_t q = blockIdx.x;
    const int t = threadIdx.x;
    uint64_t* keys = reinterpret_cast<uint64_t*>(sel_raw);                    // pow2 >= min(cnt, cap)
    float* qv = reinterpret_cast<float*>(keys + a.sort_cap);             // dim
    uint64_t* ek = reinterpret_cast<uint64_t*>(qv + ((a.dim + 3) & ~3u));  // R pow2
    __shared__ uint32_t s_m, s_flag;
    const uint32_t cnt = a.cnt[q];
    const uint32_t m = min(cnt, a.cap);
    if (t == 0) {
        s_m = m;
        // overflowed, or a sampled threshold let fewer than R rows through
        s_flag = (cnt > a.cap || (a.sampled && cnt < a.R)) ? 1u : 0u;
        a.flags[q] = (uint8_t)s_flag;
        if (a.trace) a.trace[(size_t)q * 4] = cnt;
    }
    __syncthreads();
    if (s_flag) return;
    uint32_t P = 1;
    while (P < m) P <<= 1;
    for (uint32_t i = t; i < P; i += blockDim.x) keys[i] = i < m ? a.buf[(size_t)q * a.cap + i] : ~0ull;
    for (uint32_t i = t; i < a.dim; i += blockDim.x) qv[i] = a.qf[(size_t)q * a.dim + i];
    __syncthreads();
    // bitonic sort, ascending
    for (uint32_t kk = 2; kk <= P; kk <<= 1)
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
            for (uint32_t i = t; i < P; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const uint64_t x = keys[i], y = keys[l];
                    const bool up = (i & kk) == 0;
                    if ((x > y) == up) {
                        keys[i] = y;
                        keys[l] = x;
                    }
                }
            }
            __syncthreads();
        }
    const uint32_t R = min(m, a.R);
    uint32_t P2 = 1;
    while (P2 < R) P2 <<= 1;
    // exact float32 distances of the R best, reference summation order
    if (R > 0 && (a.dim & 15) == 0) {
        // 4 lanes per row (coalesced 64-byte reads), 8 rows per warp step
        const int warp = t >> 5, lane = t & 31, nw = blockDim.x >> 5;
        for (uint32_t b = (uint32_t)warp * 8; b < P2; b += (uint32_t)nw * 8) {
            const uint32_t i = b + (lane >> 2);
            const uint32_t row = i < R ? (uint32_t)keys[i] : (uint32_t)keys[0];
            const float d = group4_dist16<SPACE>(qv, a.vecs + (size_t)row * a.row_floats, (int)(a.dim >> 4), lane & 3);
            if ((lane & 3) == 0 && i < P2) ek[i] = i < R ? (((uint64_t)fkey(d) << 32) | i) : ~0ull;
        }
    } else {
        for (uint32_t i = t; i < P2; i += blockDim.x) {
            uint64_t e = ~0ull;
            if (i < R) {
                const uint32_t row = (uint32_t)keys[i];  // the candidate's row
                const float d = distance<SPACE>(qv, a.vecs + (size_t)row * a.row_floats, (int)a.dim);
                e = ((uint64_t)fkey(d) << 32) | i;
            }
            ek[i] = e;
        }
    }
    __syncthreads();
    for (uint32_t kk = 2; kk <= P2; kk <<= 1)
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
            for (uint32_t i = t; i < P2; i += blockDim.x) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const uint64_t x = ek[i], y = ek[l];
                    const bool up = (i & kk) == 0;
                    if ((x > y) == up) {
                        ek[i] = y;
                        ek[l] = x;
                    }
                }
            }
            __syncthreads();
        }
    if (t == 0) {
        // (distance, label) order: equal distances by label, as the
        // reference's max-heap of (distance, label) pairs keeps them
        const uint32_t kk = min(a.k, R);
        uint64_t* lab = a.out_labels + (size_t)q * a.k;
        float* dist = a.out_dists + (size_t)q * a.k;
        uint32_t i = 0;
        while (i < kk) {
            uint32_t e = i + 1;
            while (e < R && (uint32_t)(ek[e] >> 32) == (uint32_t)(ek[i] >> 32)) e++;
            // sort the run [i, e) by label (insertion; runs are short)
            for (uint32_t x = i + 1; x < e; x++) {
                const uint64_t v = ek[x];
                const uint64_t lv = a.labels[(uint32_t)keys[(uint32_t)v]];
                uint32_t y = x;
                while (y > i) {
                    const uint64_t w = ek[y - 1];
                    const uint64_t lw = a.labels[(uint32_t)keys[(uint32_t)w]];
                    if (lw <= lv) break;
                    ek[y] = w;
                    y--;
                }
                ek[y] = v;
            }
            for (uint32_t x = i; x < e && x < kk; x++) {
                lab[x] = a.labels[(uint32_t)keys[(uint32_t)ek[x]]];
                dist[x] = funkey((uint32_t)(ek[x] >> 32));
            }
            i = e;
        }
        for (uint32_t x = kk; x < a.k; x++) {
            lab[x] = ~0ull;
            dist[x] = __int_as_float(0x7f800000);
        }
        a.out_counts[q] = (int32_t)kk;
    }
}

__global__ void tc_gather_rows_kernel(const float* __restrict__ src, const uint32_t* __restrict__ idx, uint32_t n,
                                      uint32_t dim, float* __restrict__ dst) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < (uint64_t)n * dim) dst[i] = src[(uint64_t)idx[i / dim] * dim + i % dim];
}

__global__ void tc_scatter_results_kernel(const uint32_t* __restrict__ idx, uint32_t n, uint32_t k,
                                          const uint64_t* __restrict__ l, const float* __restrict__ d,
                                          const int32_t* __restrict__ c, uint64_t* __restrict__ ol,
                                          float* __restrict__ od, int32_t* __restrict__ oc) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)n * k) return;
    const uint32_t r = (uint32_t)(i / k), j = (uint32_t)(i % k);
    ol[(uint64_t)idx[r] * k + j] = l[i];
    od[(uint64_t)idx[r] * k + j] = d[i];
    if (j == 0) oc[idx[r]] = c[r];
}

// Ground-truth oracle: float64 distances of (query, row) pairs, one warp per
// pair (the only float64 arithmetic of the library).  space 0: squared L2;
// 1: 1 - inner product, the query normalised in float64 when `normalize`.
__global__ void fp64_distance_kernel(const float* __restrict__ q, uint64_t npairs, uint32_t m, uint32_t dim,
                                     const float* __restrict__ vecs, uint32_t row_floats,
                                     const uint32_t* __restrict__ rows, int space, int normalize,
                                     double* __restrict__ out) {
    const uint64_t pair = (uint64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (pair >= npairs) return;
    const uint32_t row = rows[pair];
    if (row == 0xffffffffu) {
        if (lane == 0) out[pair] = __longlong_as_double(0x7ff8000000000000ll);
        return;
    }
    const float* qv = q + (pair / m) * dim;
    const float* xv = vecs + (uint64_t)row * row_floats;
    double qs = 1.0;
    if (normalize) {
        double n2 = 0.0;
        for (uint32_t i = lane; i < dim; i += 32) n2 = fma((double)qv[i], (double)qv[i], n2);
#pragma unroll
        for (int o = 16; o; o >>= 1) n2 += __shfl_xor_sync(0xffffffffu, n2, o);
        qs = n2 > 0.0 ? 1.0 / sqrt(n2) : 1.0;
    }
    double acc = 0.0;
    for (uint32_t i = lane; i < dim; i += 32) {
        const double a = (double)qv[i] * qs, b = (double)xv[i];
        acc = space == 0 ? fma(a - b, a - b, acc) : fma(a, b, acc);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[pair] = space == 0 ? acc : 1.0 - acc;
}

template <int PREC, int SPACE, int MODE>
cudaError_t launch_tc(const CUtensorMap& qm, const CUtensorMap& xm, const TcArgs& a, int grid, cudaStream_t st) {
    const bool resa = PREC == 2 && a.k_blocks <= (uint32_t)kResAKb;
    auto fn = resa ? bf_tc_kernel<PREC, SPACE, MODE, PREC == 2> : bf_tc_kernel<PREC, SPACE, MODE, false>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    if (e != cudaSuccess) return e;
    fn<<<grid, kThreads, kSmemBytes, st>>>(qm, xm, a);
    return cudaGetLastError();
}

}  // namespace

size_t tc_smem_bytes() { return kSmemBytes; }

#ifdef HNSWGPU_TC_TIMING
cudaError_t tc_timing_read(unsigned long long* out) {
    cudaError_t e = cudaMemcpyFromSymbol(out, g_tc_timing, sizeof(unsigned long long) * 256 * 10);
    if (e != cudaSuccess) return e;
    static unsigned long long z[256][10];
    return cudaMemcpyToSymbol(g_tc_timing, z, sizeof(z));
}
#endif

cudaError_t launch_fp64_distances(const float* q, uint64_t nq, uint32_t m, uint32_t dim, const float* vecs,
                                  uint32_t row_floats, const uint32_t* rows, int space, int normalize, double* out,
                                  cudaStream_t st) {
    const uint64_t npairs = nq * m;
    if (!npairs) return cudaSuccess;
    fp64_distance_kernel<<<(unsigned)((npairs + 7) / 8), 256, 0, st>>>(q, npairs, m, dim, vecs, row_floats, rows,
                                                                       space, normalize, out);
    return cudaGetLastError();
}

cudaError_t tc_encode_map(void* base, uint32_t prec, uint64_t rows, uint32_t dim, uint64_t row_pitch_bytes,
                          uint32_t box_rows, CUtensorMap* out) {
    // the driver entry point, looked up once (host threads may race here)
    static std::atomic<PFN_cuTensorMapEncodeTiled> encode_fn{nullptr};
    PFN_cuTensorMapEncodeTiled encode = encode_fn.load(std::memory_order_acquire);
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void* fp = nullptr;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fp, cudaEnableDefault, &q);
        if (e != cudaSuccess) return e;
        if (q != cudaDriverEntryPointSuccess || !fp) return cudaErrorNotSupported;
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fp);
        encode_fn.store(encode, std::memory_order_release);
    }
    const cuuint64_t gdim[2] = {dim, rows};
    const cuuint64_t gstride[1] = {row_pitch_bytes};
    const cuuint32_t box[2] = {prec == 1 ? (cuuint32_t)(kKBytes / 2) : (cuuint32_t)kKBytes, box_rows};
    const cuuint32_t estride[2] = {1, 1};
    CUresult r = encode(out, prec == 1 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base,
                        gdim, gstride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_tc_scores(const CUtensorMap& qm, const CUtensorMap& xm, const TcArgs& a, uint32_t prec, int space,
                             int mode, int num_sms, cudaStream_t st) {
    const uint32_t q_tiles = (a.nq + kTileM - 1) / kTileM;
    const uint32_t n_tiles = (a.n_rows + kTileN - 1) / kTileN;
    const uint32_t items = mode == 1 ? q_tiles : q_tiles * ((n_tiles + a.chunk_tiles - 1) / a.chunk_tiles);
    const int grid = (int)std::min<uint32_t>(items, (uint32_t)num_sms);
    if (grid == 0) return cudaSuccess;
    if (prec == 1) {
        if (space == 0) return mode ? launch_tc<1, 0, 1>(qm, xm, a, grid, st) : launch_tc<1, 0, 0>(qm, xm, a, grid, st);
        return mode ? launch_tc<1, 1, 1>(qm, xm, a, grid, st) : launch_tc<1, 1, 0>(qm, xm, a, grid, st);
    }
    if (space == 0) return mode ? launch_tc<2, 0, 1>(qm, xm, a, grid, st) : launch_tc<2, 0, 0>(qm, xm, a, grid, st);
    return mode ? launch_tc<2, 1, 1>(qm, xm, a, grid, st) : launch_tc<2, 1, 0>(qm, xm, a, grid, st);
}

cudaError_t launch_tc_rowinfo(const float* vecs, uint32_t count, uint32_t dim, uint32_t row_floats,
                              const unsigned char* tcopy, uint32_t trow_bytes, uint32_t prec, float2* out,
                              cudaStream_t st) {
    if (!count) return cudaSuccess;
    tc_rowinfo_kernel<<<(count + 7) / 8, 256, 0, st>>>(vecs, count, dim, row_floats, tcopy, trow_bytes, prec, out);
    return cudaGetLastError();
}

cudaError_t launch_tc_query_prep(const float* q, uint32_t nq, uint32_t dim, uint32_t normalize, uint32_t prec,
                                 uint32_t trow_bytes, float* qf, unsigned char* qt, float* qscale, cudaStream_t st) {
    if (!nq) return cudaSuccess;
    tc_query_prep_kernel<<<(nq + 7) / 8, 256, 0, st>>>(q, nq, dim, normalize, prec, trow_bytes, qf, qt, qscale);
    return cudaGetLastError();
}

cudaError_t launch_tc_gather_info(const float2* info, uint64_t n_sample, uint64_t step, float2* out,
                                  cudaStream_t st) {
    if (!n_sample) return cudaSuccess;
    tc_gather_info_kernel<<<(unsigned)((n_sample + 255) / 256), 256, 0, st>>>(info, n_sample, step, out);
    return cudaGetLastError();
}

cudaError_t launch_scan_mask(const uint32_t* deleted_bits, const uint8_t* allow, uint64_t n, uint8_t* out,
                             cudaStream_t st) {
    if (!n) return cudaSuccess;
    scan_mask_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(deleted_bits, allow, n, out);
    return cudaGetLastError();
}

cudaError_t launch_tc_fill(float* p, uint64_t n, float v, cudaStream_t st) {
    if (!n) return cudaSuccess;
    tc_fill_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

size_t tc_select_smem(uint32_t sort_cap, uint32_t dim, uint32_t R) {
    uint32_t P2 = 1;
    while (P2 < R) P2 <<= 1;
    return (size_t)sort_cap * 8 + ((dim + 3) & ~3u) * 4 + (size_t)P2 * 8;
}

cudaError_t launch_tc_select(const TcSelectArgs& a, int space, cudaStream_t st) {
    if (!a.nq) return cudaSuccess;
    const size_t smem = tc_select_smem(a.sort_cap, a.dim, a.R);
    auto fn = space == 0 ? tc_select_rerank_kernel<0> : tc_select_rerank_kernel<1>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    fn<<<a.nq, 256, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_tc_gather(const float* src, const uint32_t* idx, uint32_t n, uint32_t dim, float* dst,
                             cudaStream_t st) {
    const uint64_t tot = (uint64_t)n * dim;
    if (!tot) return cudaSuccess;
    tc_gather_rows_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(src, idx, n, dim, dst);
    return cudaGetLastError();
}

cudaError_t launch_tc_scatter(const uint32_t* idx, uint32_t n, uint32_t k, const uint64_t* l, const float* d,
                              const int32_t* c, uint64_t* ol, float* od, int32_t* oc, cudaStream_t st) {
    const uint64_t tot = (uint64_t)n * k;
    if (!tot) return cudaSuccess;
    tc_scatter_results_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(idx, n, k, l, d, c, ol, od, oc);
    return cudaGetLastError();
}

}  // namespace hnswgpu
