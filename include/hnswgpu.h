/*
 * hnswgpu.h -- C ABI of the B200 (sm_100a) query path for hnswlib indexes.
 *
 * The library (hnsw_rabitq_b200/libhnswgpu.so) loads index files written by
 * hnswlib 0.9.0 (HierarchicalNSW::saveIndex, BruteforceSearch::saveIndex),
 * keeps them resident in GPU memory and answers k-nearest-neighbour queries
 * with hand-written CUDA kernels.  Every entry point returns an int status
 * (HNSWGPU_OK == 0, negative on failure); hnswgpu_last_error() gives the
 * message of the calling thread's last failure.  No torch types, no C++
 * types: plain pointers and sizes only.
 *
 * Which reference interface each entry point replaces is cited per function
 * (paths are relative to the hnswlib source tree).
 */
#ifndef HNSWGPU_H_
#define HNSWGPU_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HNSWGPU_API __attribute__((visibility("default")))
#else
#define HNSWGPU_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define HNSWGPU_OK 0
#define HNSWGPU_ERR_ARG -1        /* invalid argument (null handle, k == 0 ...)      */
#define HNSWGPU_ERR_IO -2         /* "Cannot open file"                              */
#define HNSWGPU_ERR_FORMAT -3     /* "Index seems to be corrupted or unsupported"    */
#define HNSWGPU_ERR_CUDA -4       /* a CUDA runtime call failed                      */
#define HNSWGPU_ERR_NOMEM -5      /* device or host allocation failed                */
#define HNSWGPU_ERR_LABEL -6      /* "Label not found"                               */
#define HNSWGPU_ERR_STATE -7      /* already deleted / not deleted                   */
#define HNSWGPU_ERR_KERNEL -8     /* a kernel reported a failure (see last_error)    */
#define HNSWGPU_ERR_UNSUPPORTED -9

/* spaces: hnswlib::L2Space, hnswlib::InnerProductSpace, and the Python
 * binding's "cosine" (inner product over normalised vectors,
 * python_bindings/bindings.cpp:160-172). */
#define HNSWGPU_SPACE_L2 0
#define HNSWGPU_SPACE_IP 1
#define HNSWGPU_SPACE_COSINE 2
/* hnswlib::L2SpaceI (hnswlib/space_l2.h:255-323): an HNSW index of uint8
 * vectors with integer squared-L2 distances (HierarchicalNSW<int>).  Queries
 * are passed as float32 rows holding the uint8 values; distances come back as
 * float32 holding the reference's integer distances exactly (needs
 * dim * 255^2 < 2^24, i.e. dim <= 258).  HNSW indexes only. */
#define HNSWGPU_SPACE_L2_UINT8 3

/* search flags */
#define HNSWGPU_DEVICE_PTRS 0x1u  /* queries / outputs / allow mask are device
                                     pointers; the call is asynchronous on
                                     `stream` and does not synchronise.  Without
                                     it they are host pointers and the call
                                     copies, launches and synchronises.
                                     Tie-exact searches (HNSWGPU_EXACT_TIES,
                                     hnswgpu_search_epsilon) of one index share
                                     its scratch (candidate-heap tails, the tie
                                     list): asynchronous ones must not overlap
                                     on the GPU, so issue them on one stream or
                                     order their streams (the serving loop runs
                                     one at a time).                            */
#define HNSWGPU_TRACE 0x2u        /* write per-query work counters to `trace`   */
#define HNSWGPU_EXACT_TIES 0x4u   /* HNSW: replay the reference's heap order so
                                     that exact distance ties resolve as in
                                     hnswlib (results identical to searchKnn);
                                     without it ties break by internal id.
                                     Runs in two passes: the id-order beam for
                                     every query, then the heap replay only for
                                     the queries whose run met a distance tie
                                     that can steer the reference's heaps.     */
#define HNSWGPU_REPLAY_ALL 0x20u  /* with HNSWGPU_EXACT_TIES: one pass, the
                                     heap replay for every query (same results;
                                     for testing and measurement).             */
#define HNSWGPU_LEARNED_STOP 0x8u /* HNSW: end each query's level-0 beam when
                                     the termination network set by
                                     hnswgpu_set_termination_model judges its
                                     top-k final; ef is then the cap.  Needs
                                     the id tie order (no HNSWGPU_EXACT_TIES). */
#define HNSWGPU_EXACT_SCAN 0x10u  /* HNSW: answer by an exhaustive scan of the
                                     index's resident vectors (exact k-NN,
                                     the ground truth of recall measurements;
                                     the allow mask applies and deleted
                                     elements are never returned).             */

/* kernel status bits (hnswgpu_search_opts.status / hnswgpu_get_status) */
#define HNSWGPU_STATUS_TIMEOUT 0x1u   /* a bounded wait gave up; results invalid   */
#define HNSWGPU_STATUS_OVERFLOW 0x2u  /* a search overflowed a candidate list
                                         (filtered search, or the shared-memory
                                         heap of hnswgpu_search_noalloc); results
                                         may differ from the reference for the
                                         flagged queries                        */

typedef struct hnswgpu_index hnswgpu_index;

typedef struct hnswgpu_info {
    uint64_t count;            /* cur_element_count                             */
    uint64_t max_elements;     /* max_elements_ after load                      */
    uint64_t dim;
    uint64_t M, maxM, maxM0;
    uint64_t ef_construction;
    uint64_t ef;               /* current ef_ (reset to 10 by load, as hnswalg.h:794) */
    uint64_t num_deleted;
    int32_t maxlevel;
    uint32_t enterpoint;
    int32_t space;
    int32_t is_bruteforce;
    uint64_t device_bytes;     /* bytes of index data resident on the GPU       */
} hnswgpu_info;

typedef struct hnswgpu_search_opts {
    uint32_t flags;            /* HNSWGPU_DEVICE_PTRS | HNSWGPU_TRACE | ...     */
    uint32_t precision;        /* HNSWGPU_PREC_FP32 (the reference's search),
                                  _BF16 or _FP8.  HNSW: the beam traverses
                                  that copy of the vectors; brute force: the
                                  scan runs on the tensor cores over that
                                  copy (sampled threshold, fused candidate
                                  filter; synchronises).  Both re-rank the
                                  best `rerank` candidates with exact FP32
                                  distances before returning k.  The HNSW
                                  form needs dim % 16 == 0, maxM0 <= 32 and
                                  the id tie order; deletes and `allow` are
                                  honoured.  FP8 with no deleted element and
                                  no `allow` / filter runs the lean beam and
                                  takes maxM0 <= 64.                           */
    uint64_t ef;               /* 0: use the index's ef_ (setEf)               */
    const uint8_t* allow;      /* optional per-internal-id byte mask: nonzero =
                                  the filter functor accepts that node's label.
                                  Internal ids are positions in
                                  hnswgpu_get_labels().                        */
    uint32_t* trace;           /* HNSWGPU_TRACE: 4 uint32 per query: upper-layer
                                  link lists read, upper-layer distances,
                                  level-0 expansions, level-0 distances.
                                  Same memory kind as the queries.            */
    void* stream;              /* cudaStream_t; NULL = the index's own stream  */
    uint32_t rerank;           /* low precision: candidates re-ranked; HNSW:
                                  0 = ef; brute force: the over-fetch of the
                                  tensor-core scan, 0 = 4 k, at most 1024     */
    uint32_t filter;           /* 0, or a filter id from hnswgpu_filter_create
                                  (its device-resident mask is used instead of
                                  `allow`, which must then be NULL)           */
} hnswgpu_search_opts;

/* traversal precisions (hnswgpu_search_opts.precision) */
#define HNSWGPU_PREC_FP32 0u
#define HNSWGPU_PREC_BF16 1u      /* bf16 copy of every vector                  */
#define HNSWGPU_PREC_FP8 2u       /* e4m3 copy with one fp32 scale per vector   */

/* Message of this thread's last failure ("" if none). */
HNSWGPU_API const char* hnswgpu_last_error(void);

/* Library version string. */
HNSWGPU_API const char* hnswgpu_version(void);

/* Load a HierarchicalNSW index file.  Replaces the load constructor
 * HierarchicalNSW(SpaceInterface*, const std::string& location, bool nmslib,
 * size_t max_elements, bool allow_replace_deleted) (hnswlib/hnswalg.h:78-86)
 * and HierarchicalNSW::loadIndex (hnswlib/hnswalg.h:715-821).  The space and
 * dimension are not stored in the file and are supplied by the caller, as in
 * the reference.  ef starts at 10. */
HNSWGPU_API int hnswgpu_load_hnsw(const char* path, int space, uint64_t dim, uint64_t max_elements, int device,
                      hnswgpu_index** out);

/* The same from an index image in memory (`size` bytes laid out as the file):
 * the Python binding's unpickling (createFromParams, bindings.cpp:485-519)
 * goes through it without a file.  The buffer is read during the call only.
 * hnswgpu_save_hnsw has no source to rewrite for such an index (the caller
 * holds the image). */
HNSWGPU_API int hnswgpu_load_hnsw_buffer(const void* data, uint64_t size, int space, uint64_t dim,
                                         uint64_t max_elements, int device, hnswgpu_index** out);

/* Load a BruteforceSearch index file.  Replaces
 * BruteforceSearch(SpaceInterface*, const std::string& location)
 * (hnswlib/bruteforce.h:35-43) and BruteforceSearch::loadIndex
 * (hnswlib/bruteforce.h:142-161). */
HNSWGPU_API int hnswgpu_load_bf(const char* path, int space, uint64_t dim, int device, hnswgpu_index** out);

/* Build a BruteforceSearch index from rows in host memory: the state that
 * BruteforceSearch(space, maxElements) + addPoint (hnswlib/bruteforce.h:46-83)
 * reaches after adding `n` rows with these labels, rows in this order.  For
 * the cosine space the rows are normalised as the Python binding's add_items
 * does (python_bindings/bindings.cpp:241-248, 790-800). */
HNSWGPU_API int hnswgpu_create_bf(int space, uint64_t dim, const float* data, const uint64_t* labels, uint64_t n,
                                  uint64_t max_elements, int device, hnswgpu_index** out);

/* Build (once) the low-precision traversal copy of an HNSW index's vectors
 * (precision HNSWGPU_PREC_BF16 or HNSWGPU_PREC_FP8), derived on the GPU from
 * the resident float32 rows.  Searches with that precision build it on first
 * use; calling this first keeps the allocation out of the timed path.  No
 * counterpart in the reference (which searches float32 only). */
HNSWGPU_API int hnswgpu_build_traversal_copy(hnswgpu_index* index, uint32_t precision);

/* Release the index and its device memory. */
HNSWGPU_API int hnswgpu_free(hnswgpu_index* index);

/* Index metadata. */
HNSWGPU_API int hnswgpu_get_info(const hnswgpu_index* index, hnswgpu_info* out);

/* setEf (hnswlib/hnswalg.h:173-175); the Python ef property
 * (python_bindings/bindings.cpp:979-987). */
HNSWGPU_API int hnswgpu_set_ef(hnswgpu_index* index, uint64_t ef);

/* Labels of all elements in internal-id order (count entries); the
 * positions are the internal ids used by hnswgpu_search_opts.allow.
 * Mirrors getExternalLabel (hnswlib/hnswalg.h:185-189). */
HNSWGPU_API int hnswgpu_get_labels(const hnswgpu_index* index, uint64_t* out);

/* markDelete / unmarkDelete (hnswlib/hnswalg.h:852-927): set or clear the
 * delete mark of the element with this label.  Deleted elements are still
 * traversed but never returned.  Errors as the reference: unknown label
 * (HNSWGPU_ERR_LABEL), already deleted / not deleted (HNSWGPU_ERR_STATE). */
HNSWGPU_API int hnswgpu_mark_deleted(hnswgpu_index* index, uint64_t label);
HNSWGPU_API int hnswgpu_unmark_deleted(hnswgpu_index* index, uint64_t label);

/* Batched HierarchicalNSW::searchKnn (hnswlib/hnswalg.h:1269-1323) or
 * BruteforceSearch::searchKnn (hnswlib/bruteforce.h:106-125), depending on
 * the index kind.  queries: nq x dim float32, row-major.  Outputs: nq x k
 * labels and distances, closest first (the order of
 * AlgorithmInterface::searchKnnCloserFirst, hnswlib/hnswlib.h:203-221, and of
 * the Python knn_query rows, bindings.cpp:649-654); counts[i] = number of
 * results found for query i (< k when the index or the filter yields fewer;
 * unused slots hold label UINT64_MAX and distance +inf).  For the cosine
 * space the queries are normalised exactly as bindings.cpp:241-248. */
HNSWGPU_API int hnswgpu_search(hnswgpu_index* index, const float* queries, uint64_t nq, uint64_t k,
                   const hnswgpu_search_opts* opts, uint64_t* out_labels, float* out_dists,
                   int32_t* out_counts);

/* Multi-vector indexes: a HierarchicalNSW over a MultiVectorL2Space
 * (hnswlib/stop_condition.h:7-76), whose elements carry a 32-bit document id
 * right after the vector.  The loader is hnswgpu_load_hnsw's with that
 * element layout (L2 space). */
HNSWGPU_API int hnswgpu_load_hnsw_multivector(const char* path, uint64_t dim, uint64_t max_elements, int device,
                                              hnswgpu_index** out);

/* searchStopConditionClosest with a MultiVectorSearchStopCondition(space,
 * num_docs, ef_collection) (hnswlib/hnswalg.h:1326-1377,
 * hnswlib/stop_condition.h:146-216): per query, the elements of the num_docs
 * nearest documents as the reference returns them -- closest first, equal
 * distances in its heap's pop order, INTERNAL ids (the reference copies
 * top_candidates' ids unchanged).  Host buffers: out_ids / out_dists nq x cap,
 * out_counts[i] = the result's size, or -1 when it has more than cap entries
 * or the query outgrew the kernel's fixed heaps (HNSWGPU_STATUS_OVERFLOW is
 * then raised too).  Indexes with deleted elements are not supported. */
HNSWGPU_API int hnswgpu_search_multivector(hnswgpu_index* index, const float* queries, uint64_t nq,
                                           uint64_t num_docs, uint64_t ef_collection, uint64_t cap,
                                           uint64_t* out_ids, float* out_dists, int32_t* out_counts);

/* A filter functor evaluated once over the index's labels and kept on the
 * device: `allow` holds a byte per internal id (hnswgpu_get_labels order),
 * nonzero = the functor accepts that label (hnswlib/hnswlib.h:128-132 calls
 * the functor per candidate instead).  Searches name it by the returned id in
 * hnswgpu_search_opts.filter, so repeated filtered searches copy no mask.
 * hnswgpu_filter_destroy waits for the index's stream, then frees it. */
HNSWGPU_API int hnswgpu_filter_create(hnswgpu_index* index, const uint8_t* allow, uint32_t* out_id);
HNSWGPU_API int hnswgpu_filter_destroy(hnswgpu_index* index, uint32_t filter_id);

/* HierarchicalNSW::saveIndex (hnswlib/hnswalg.h:685-712) of an index loaded
 * from a file: the file it was loaded from, re-read, with every element's
 * delete mark set as it is now (mark_deleted / unmark_deleted since the
 * load), written to `path`. */
HNSWGPU_API int hnswgpu_save_hnsw(hnswgpu_index* index, const char* path);

/* Replaces HierarchicalNSW::searchStopConditionClosest with an
 * EpsilonSearchStopCondition(epsilon, min_candidates, max_candidates)
 * (hnswlib/hnswalg.h:1326-1377, hnswlib/stop_condition.h:219-275): every
 * query's beam runs with ef = max_candidates and also stops at a candidate
 * beyond epsilon once min_candidates results are held; the results within
 * epsilon are returned.  epsilon is a distance (squared for L2).  Outputs:
 * nq x max_candidates ids and distances in the reference's result order
 * (closest first; equal distances in the order its heap pops them), counts[i]
 * = results kept, unused slots UINT64_MAX / +inf.  As in the reference, the
 * ids are INTERNAL ids (searchStopConditionClosest copies top_candidates'
 * internal ids into its result); they equal the labels when labels were
 * assigned 0, 1, 2, ... in insertion order.  Always the reference's heap
 * order.  opts: only HNSWGPU_DEVICE_PTRS, `allow` and `stream` apply. */
HNSWGPU_API int hnswgpu_search_epsilon(hnswgpu_index* index, const float* queries, uint64_t nq, float epsilon,
                                       uint64_t min_candidates, uint64_t max_candidates,
                                       const hnswgpu_search_opts* opts, uint64_t* out_ids, float* out_dists,
                                       int32_t* out_counts);

/* HNSW search that allocates no memory, for callers that cannot call
 * cudaMalloc: code running under a device-memory budget it does not own (a
 * framework's caching allocator or a serving process that reserves all of its
 * memory up front and treats any later allocation as a failure), and code
 * that must not risk the implicit device synchronisation an allocation or
 * free can cause.  It has no counterpart in the reference.
 *
 * Same search as hnswgpu_search with HNSWGPU_DEVICE_PTRS: queries, outputs and
 * the optional allow mask are device pointers, `ef` 0 means the index's ef,
 * flags may only hold HNSWGPU_EXACT_TIES (which here always runs the one-pass
 * heap replay: the two-pass form needs a per-query list); the call is
 * asynchronous on `stream`.  It holds the index's lock while it reads the
 * index, so it may run beside set_ef / mark_deleted in other threads.
 * The kernel's scratch (work counter, finished-CTA counter, status word) is a
 * fixed 256-byte array in the library's device image instead of per-index
 * memory; nq >= 2^31 is rejected.  Every GPU that loads the library holds that
 * array until the process exits.  The first call on a device resolves the
 * array's device address (cudaGetSymbolAddress with that device current): make
 * it before any stream capture; after a cudaDeviceReset the library must be
 * loaded again.  All calls on a device share the array, so calls that overlap
 * on the GPU (other streams, or a graph replay while another call runs) race
 * and must not be issued; each call clears the two counters before its launch.
 *
 * With HNSWGPU_EXACT_TIES the reference's candidate heap has no global tail
 * here: it lives in shared memory only, max(512, 12 * ef) entries, fewer (down
 * to 4 * ef) where the per-query shared memory runs short, against 28 * ef in
 * hnswgpu_search.  A query whose heap outgrows it drops pushes and raises
 * HNSWGPU_STATUS_OVERFLOW; its results may then differ from the reference.
 * The status bits of these calls (overflow; a bounded wait that timed out,
 * which invalidates the results) accumulate in the array's status word until
 * hnswgpu_noalloc_get_status reads them. */
HNSWGPU_API int hnswgpu_search_noalloc(const hnswgpu_index* index, const float* d_queries, uint64_t nq, uint64_t k,
                                       uint64_t ef, uint32_t flags, const uint8_t* d_allow, uint64_t* d_labels,
                                       float* d_dists, int32_t* d_counts, void* stream);

/* OR of the status bits (HNSWGPU_STATUS_*) raised by hnswgpu_search_noalloc
 * calls on `device` since the last read; clears them.  Ordered after the work
 * queued on `stream` and synchronises it; allocates nothing.  No counterpart in
 * the reference. */
HNSWGPU_API int hnswgpu_noalloc_get_status(int device, void* stream, uint32_t* out_bits);

/* Self-test of the kernels' bounded waits: launches one warp that waits on a
 * copy that never arrives, gives up after a few milliseconds and reports
 * HNSWGPU_STATUS_TIMEOUT in *out_bits, the way a search whose copy stalled
 * reports it; the device stays usable afterwards.  No counterpart in the
 * reference (its searches never wait on a device). */
HNSWGPU_API int hnswgpu_selftest_wait_timeout(int device, uint32_t* out_bits);

/* Ground-truth oracle: float64 distances between each query and m rows
 * given by label (labels: nq x m; out: nq x m doubles, NaN for an unknown
 * label), in the index's space (squared L2; 1 - inner product; cosine with
 * the query normalised in float64).  The only float64 arithmetic of the
 * library; used to measure recall and the error of returned float32
 * distances.  No counterpart in the reference. */
HNSWGPU_API int hnswgpu_fp64_distances(hnswgpu_index* index, const float* queries, uint64_t nq,
                                       const uint64_t* labels, uint64_t m, double* out);

/* ------------------------------------------------ learned early termination
 * No counterpart in the reference, whose beam always runs until its
 * candidate queue is exhausted (hnswlib/hnswalg.h:368-376).
 *
 * Every `period` level-0 expansions (at the first state from then on where
 * the top-k has not changed for `period` expansions and no waiting
 * candidate is closer than the k-th result) the beam forms a feature vector
 * of its state, with a = |d_k|:
 *   f0 log2(1 + expansions)            f8..f10 log2(1 + n(x)), x = 0.1, 0.25, 0.5
 *   f1 d_1 / a                         f11 waiting candidates / ef
 *   f2 (d_next - d_k) / a              f12 beam size / ef
 *   f3 log2(1 + d_entry / a)           f13 log2(1 + expansions that changed the top-k)
 *   f4 log2(1 + |q|^2)                 f14 distance evaluations per expansion
 *   f5 expansions since the top-k          since the previous checkpoint
 *      last changed / period           f15 (d_median - d_k) / a
 *   f6 (d_wait - d_k) / a
 *   f7 (d_worst - d_k) / a
 * d_1, d_k = best and k-th distances in the beam, d_next = the candidate
 * expanded next, d_entry = the level-0 entry point, waiting candidates =
 * beam entries not expanded yet (d_wait the closest of them after those
 * taken for expansion; n(x) how many are closer than d_k + x a), d_worst /
 * d_median = the beam's last and middle entries; ratios clamped to [-4, 4].
 * A 16 -> 64 -> 64 -> 1 ReLU network maps it to the logit of "the top-k is
 * final".  Parameters: HNSWGPU_TERM_PARAMS float32 in the order
 * mu[16], inv_sigma[16] (x = (f - mu) * inv_sigma), W1[64][16], b1[64],
 * W2[64][64], b2[64], w3[64], b3. */
#define HNSWGPU_TERM_FEATURES 16
#define HNSWGPU_TERM_HIDDEN 64
#define HNSWGPU_TERM_PARAMS 5345

/* Install (params != NULL) or remove (NULL) the index's termination network;
 * HNSWGPU_LEARNED_STOP searches evaluate it every `period` expansions and
 * stop when the logit exceeds `logit_threshold` (+inf: never, and the
 * network is not evaluated -- the plain beam).  The search runs the network
 * with fp16 weights and fp32 accumulation. */
HNSWGPU_API int hnswgpu_set_termination_model(hnswgpu_index* index, const float* params, uint32_t period,
                                              float logit_threshold);

/* Training data: the same search as hnswgpu_search (host pointers, id tie
 * order, opts->precision / rerank / ef honoured) that also records, at every
 * checkpoint, the feature vector (out_feat: nq x max_ckpt x
 * HNSWGPU_TERM_FEATURES) and the internal ids of the first W beam entries
 * (out_ids: nq x max_ckpt x W, W = ids_width, or k when 0; 0xffffffff
 * where the beam holds fewer); out_ckpt_dists (optional, same shape): their
 * float32 distances recomputed from the float32 rows (+inf for missing
 * entries), so that a low-precision beam can be labelled by what its
 * re-rank of those W entries would return.  out_nckpt[i] = rows written for
 * query i (1..max_ckpt when max_ckpt > 0).  The last row of each query
 * (out_nckpt[i] - 1) holds the state at the end of the beam (its first W
 * entries before any re-rank), the reference for labelling the earlier rows;
 * checkpoints beyond max_ckpt - 1 are dropped. */
HNSWGPU_API int hnswgpu_search_checkpoints(hnswgpu_index* index, const float* queries, uint64_t nq, uint64_t k,
                                           const hnswgpu_search_opts* opts, uint32_t period, uint32_t max_ckpt,
                                           uint32_t ids_width, float* out_feat, uint32_t* out_ids,
                                           float* out_ckpt_dists, uint32_t* out_nckpt, uint64_t* out_labels,
                                           float* out_dists, int32_t* out_counts);

typedef struct hnswgpu_term_train_opts {
    uint32_t epochs;
    uint32_t batch;            /* samples per Adam step (0: 1024)             */
    float lr;                  /* Adam step size                              */
    float pos_weight;          /* weight of the label-1 term of the loss      */
    float weight_decay;        /* decoupled, on the weight matrices           */
    uint32_t reserved;
    uint64_t seed;             /* mini-batch shuffling                        */
} hnswgpu_term_train_opts;

/* Train the network on the GPU (forward / backward / Adam kernels) from n
 * samples (feats: n x 6, labels: n floats in {0, 1}); `params` holds the
 * initial values (mu / inv_sigma set by the caller) and receives the
 * trained ones; out_epoch_loss (optional): mean batch loss per epoch. */
HNSWGPU_API int hnswgpu_term_train(int device, const float* feats, const float* labels, uint64_t n,
                                   const hnswgpu_term_train_opts* opts, float* params, float* out_epoch_loss);

/* Mean loss and its gradient (HNSWGPU_TERM_PARAMS floats; zero for
 * mu / inv_sigma) over n samples, computed by the training kernels. */
HNSWGPU_API int hnswgpu_term_loss_grad(int device, const float* params, const float* feats, const float* labels,
                                       uint64_t n, float pos_weight, float* out_loss, float* out_grad);

/* Logits of n feature vectors by the search's own in-warp inference. */
HNSWGPU_API int hnswgpu_term_logits(int device, const float* params, const float* feats, uint64_t n,
                                    float* out_logits);

/* ------------------------------------------------------------ serving loop
 * Continuous batching of single-query requests over one HNSW index (no
 * counterpart in the reference, where each caller thread runs its own
 * searchKnn).  A scheduler thread batches waiting requests that share a
 * search configuration (k, ef, filter, flags, precision, re-rank), launches
 * each batch on one of `max_inflight` CUDA streams so that batches overlap on
 * the device, and admits a batch only while the shared-memory footprint of
 * the queries in flight (one warp and its configuration's per-warp layout
 * each) stays within `smem_budget`; a finished batch frees its share at
 * once.  A request's results are those of hnswgpu_search for the same query
 * and settings, whatever else is in flight. */
typedef struct hnswgpu_server hnswgpu_server;

typedef struct hnswgpu_server_opts {
    uint32_t max_inflight;     /* concurrent batches (streams); 0: 32         */
    uint32_t max_batch;        /* queries per batch; 0: 4096                  */
    uint64_t smem_budget;      /* admission budget in bytes of per-query
                                  shared-memory footprint in flight; 0: twice
                                  the device's shared memory (SMs x per SM)  */
} hnswgpu_server_opts;

typedef struct hnswgpu_request {
    uint32_t k;
    uint32_t ef;               /* 0: the index's ef                          */
    int32_t filter;            /* hnswgpu_server_add_filter id, or -1        */
    uint32_t flags;            /* HNSWGPU_EXACT_TIES or HNSWGPU_LEARNED_STOP  */
    uint32_t precision;        /* HNSWGPU_PREC_*                              */
    uint32_t rerank;           /* as hnswgpu_search_opts.rerank               */
} hnswgpu_request;

typedef struct hnswgpu_server_stats {
    uint64_t submitted, completed, batches;
    double mean_batch;         /* queries per batch                           */
    double p50_us, p99_us, mean_us, max_us; /* submission -> results on the
                                  host, over requests completed since the
                                  last reset                                  */
} hnswgpu_server_stats;

HNSWGPU_API int hnswgpu_server_create(hnswgpu_index* index, const hnswgpu_server_opts* opts, hnswgpu_server** out);
/* Register a filter: a byte per internal id (hnswgpu_get_labels order),
 * nonzero = the label may be returned; out_id names it in requests. */
HNSWGPU_API int hnswgpu_server_add_filter(hnswgpu_server* server, const uint8_t* allow, int32_t* out_id);
/* Queue one query (dim floats, copied); returns at once with a ticket. */
HNSWGPU_API int hnswgpu_server_submit(hnswgpu_server* server, const float* query, const hnswgpu_request* req,
                                      uint64_t* out_ticket);
/* Block until the ticket's results are ready (req.k labels / distances,
 * closest first, count, latency in microseconds); releases the ticket. */
HNSWGPU_API int hnswgpu_server_wait(hnswgpu_server* server, uint64_t ticket, uint64_t* labels, float* dists,
                                    int32_t* count, double* latency_us);
/* Open-loop load: submit request i (queries + i * dim, reqs[i]) at
 * arrival_us[i] microseconds after the call starts, from the calling thread,
 * then collect every result (rows of k_stride labels / distances, padded
 * with UINT64_MAX / +inf) and its latency. */
HNSWGPU_API int hnswgpu_server_replay(hnswgpu_server* server, const float* queries, uint64_t n,
                                      const hnswgpu_request* reqs, const double* arrival_us, uint32_t k_stride,
                                      uint64_t* labels, float* dists, int32_t* counts, double* latency_us);
HNSWGPU_API int hnswgpu_server_get_stats(hnswgpu_server* server, hnswgpu_server_stats* out, int reset);
/* Finish every queued request, then release the server (not the index). */
HNSWGPU_API int hnswgpu_server_destroy(hnswgpu_server* server);

/* OR of the kernel status bits raised by searches on this index since the
 * last call (synchronises the index's stream); clears them. */
HNSWGPU_API int hnswgpu_get_status(hnswgpu_index* index, uint32_t* out_bits);

#ifdef __cplusplus
}
#endif
#endif /* HNSWGPU_H_ */
