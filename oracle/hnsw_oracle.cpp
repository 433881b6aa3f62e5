// CPU oracle for the hnswlib query path -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain C++, the arithmetic and the search algorithms
// of hnswlib 0.9.0 (the reference) so that tests, the smoke check and the CPU
// baseline leg of the benchmark can check the CUDA path against it.  Nothing
// in the product (hnsw_rabitq_b200/) links, loads or calls this code.
//
// Parity is pinned: tests/test_oracle_pins.py compares every function here
// against the reference's own compiled extension (oracle/_ref, built from the
// reference sources by oracle/Makefile) and against the committed fixtures
// under tests/golden/.
//
// Contents
//   * distances  -- L2Sqr / InnerProductDistance in the exact floating-point
//                   order the reference produces when built with its setup.py
//                   flags (-O3 -march=native) on an AVX-512 x86 host:
//                   hnswlib/space_l2.h:6-253, hnswlib/space_ip.h:6-398.
//                   Compiled with -ffp-contract=off; every fused multiply-add
//                   the reference's compiler forms is written as std::fma.
//   * loaders    -- the saved-index formats: HierarchicalNSW::loadIndex
//                   (hnswlib/hnswalg.h:715-821) and BruteforceSearch::loadIndex
//                   (hnswlib/bruteforce.h:142-161).
//   * search     -- mode 0 "reference": searchKnn (hnswalg.h:1269-1323) with
//                   searchBaseLayerST (hnswalg.h:308-440) on std::priority_queue
//                   exactly as the reference, ties included;
//                   mode 1 "canonical": the same algorithm with ties broken by
//                   (distance, internal id) and a sorted candidate pool, which
//                   is what the GPU kernel computes (see canonical_search()).
//   * brute force -- BruteforceSearch::searchKnn (bruteforce.h:106-125).
//   * stop conditions -- searchStopConditionClosest (hnswalg.h:1326-1377) with
//                   EpsilonSearchStopCondition and MultiVectorSearchStopCondition
//                   (stop_condition.h), pinned to the reference by the harnesses
//                   oracle/ref_stopcond.cpp and oracle/ref_multivec.cpp.
//   * L2SpaceI   -- space 3: uint8 elements, integer squared L2
//                   (space_l2.h:255-323), pinned by oracle/ref_l2u8.cpp.
//   * listing    -- mode 1 also marks the runs the GPU's two-pass tie-exact
//                   search lists for the heap replay (Trace::listed).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <queue>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

// ---------------------------------------------------------------- distances
// L2, dim % 16 == 0 (space_l2.h:25-54): 16 lane accumulators, each updated
// acc = fma(t, t, acc) over consecutive 16-float chunks, then the 16 lanes are
// summed left to right (space_l2.h:49-51).
float l2_simd16(const float* a, const float* b, size_t qty) {
    float acc[16] = {0};
    size_t n16 = qty >> 4;
    for (size_t c = 0; c < n16; c++)
        for (int l = 0; l < 16; l++) {
            float t = a[16 * c + l] - b[16 * c + l];
            acc[l] = std::fma(t, t, acc[l]);
        }
    float r = acc[0];
    for (int l = 1; l < 16; l++) r = r + acc[l];
    return r;
}

// L2, SSE 4-lane body (space_l2.h:165-190).
float l2_simd4(const float* a, const float* b, size_t qty) {
    float acc[4] = {0};
    size_t n4 = qty >> 2;
    for (size_t c = 0; c < n4; c++)
        for (int l = 0; l < 4; l++) {
            float t = a[4 * c + l] - b[4 * c + l];
            acc[l] = std::fma(t, t, acc[l]);
        }
    return ((acc[0] + acc[1]) + acc[2]) + acc[3];
}

// Scalar L2Sqr (space_l2.h:6-20).  GCC 13 at -O3 -march=native vectorises
// this loop 4 floats wide as an in-order reduction: the first (qty/4)*4 terms
// are added left to right as rounded products (no fusion), the remaining
// qty%4 terms by the scalar epilogue as fma.  Measured against the reference
// build for every tail length 1..15 (tests/test_oracle_pins.py).
float l2_scalar(const float* a, const float* b, size_t qty) {
    float r = 0.f;
    size_t n4 = qty / 4 * 4;
    for (size_t i = 0; i < n4; i++) {
        float t = a[i] - b[i];
        float p = t * t;
        r = r + p;
    }
    for (size_t i = n4; i < qty; i++) {
        float t = a[i] - b[i];
        r = std::fma(t, t, r);
    }
    return r;
}

// L2Space dispatch (space_l2.h:214-238).
float dist_l2(const float* a, const float* b, size_t dim) {
    if (dim % 16 == 0) return l2_simd16(a, b, dim);
    if (dim % 4 == 0) return l2_simd4(a, b, dim);
    if (dim > 16) {
        size_t d16 = dim >> 4 << 4;
        return l2_simd16(a, b, d16) + l2_scalar(a + d16, b + d16, dim - d16);
    }
    if (dim > 4) {
        size_t d4 = dim >> 2 << 2;
        return l2_simd4(a, b, d4) + l2_scalar(a + d4, b + d4, dim - d4);
    }
    return l2_scalar(a, b, dim);
}

// Inner product, AVX-512 body (space_ip.h:146-199): 16 lanes of fma chains
// over 16-float chunks, then GCC's _mm512_reduce_add_ps tree:
// (i, i+8) -> (i, i+4) -> (0,2),(1,3) -> final pair.
float ip_simd16(const float* a, const float* b, size_t qty) {
    float acc[16] = {0};
    size_t n16 = qty / 16;
    for (size_t c = 0; c < n16; c++)
        for (int l = 0; l < 16; l++) acc[l] = std::fma(a[16 * c + l], b[16 * c + l], acc[l]);
    float t3[8], t6[4];
    for (int i = 0; i < 8; i++) t3[i] = acc[i + 8] + acc[i];
    for (int i = 0; i < 4; i++) t6[i] = t3[i + 4] + t3[i];
    float t80 = t6[0] + t6[2], t81 = t6[1] + t6[3];
    return t80 + t81;
}

// Inner product, AVX 4-lane body (space_ip.h:24-69): 8 lanes over each
// 16-float chunk (two 8-float halves), folded to 4 lanes (i + i+4), then
// 4-lane fma over the remaining 4-float chunks, then a left-to-right sum.
float ip_simd4(const float* a, const float* b, size_t qty) {
    size_t n16 = qty / 16, n4 = qty / 4;
    float acc8[8] = {0};
    for (size_t c = 0; c < n16; c++) {
        for (int i = 0; i < 8; i++) acc8[i] = std::fma(a[16 * c + i], b[16 * c + i], acc8[i]);
        for (int i = 0; i < 8; i++) acc8[i] = std::fma(a[16 * c + 8 + i], b[16 * c + 8 + i], acc8[i]);
    }
    float s[4];
    for (int i = 0; i < 4; i++) s[i] = acc8[i] + acc8[i + 4];
    for (size_t c = 16 * n16; c < 4 * n4; c += 4)
        for (int i = 0; i < 4; i++) s[i] = std::fma(a[c + i], b[c + i], s[i]);
    return ((s[0] + s[1]) + s[2]) + s[3];
}

// Scalar InnerProduct (space_ip.h:6-14).
float ip_scalar(const float* a, const float* b, size_t qty) {
    float r = 0.f;
    for (size_t i = 0; i < qty; i++) r = std::fma(a[i], b[i], r);
    return r;
}

// InnerProductSpace dispatch (space_ip.h:348-383); distance = 1 - <a, b>.
float dist_ip(const float* a, const float* b, size_t dim) {
    if (dim % 16 == 0) return 1.0f - ip_simd16(a, b, dim);
    if (dim % 4 == 0) return 1.0f - ip_simd4(a, b, dim);
    if (dim > 16) {
        size_t d16 = dim >> 4 << 4;
        return 1.0f - (ip_simd16(a, b, d16) + ip_scalar(a + d16, b + d16, dim - d16));
    }
    if (dim > 4) {
        size_t d4 = dim >> 2 << 2;
        return 1.0f - (ip_simd4(a, b, d4) + ip_scalar(a + d4, b + d4, dim - d4));
    }
    return 1.0f - ip_scalar(a, b, dim);
}

// L2SpaceI (space_l2.h:255-323): uint8 elements, integer sum of squared
// differences, in any order exact; here over uint8 values held in floats.
float dist_l2_u8(const float* a, const float* b, size_t dim) {
    int64_t res = 0;
    for (size_t i = 0; i < dim; i++) {
        const int t = (int)(unsigned char)a[i] - (int)(unsigned char)b[i];
        res += t * t;
    }
    return (float)(int)res;
}

// space: 0 L2, 1 and 2 inner product (cosine: normalised vectors), 3 uint8 L2
inline float dist(int space, const float* a, const float* b, size_t dim) {
    if (space == 3) return dist_l2_u8(a, b, dim);
    return space == 0 ? dist_l2(a, b, dim) : dist_ip(a, b, dim);
}

// -------------------------------------------------------------- HNSW index
struct Hnsw {
    uint64_t offsetLevel0 = 0, max_elements = 0, cur = 0, size_data = 0, label_offset = 0, offsetData = 0;
    int32_t maxlevel = 0;
    uint32_t ep = 0;
    uint64_t maxM = 0, maxM0 = 0, M = 0;
    double mult = 0;
    uint64_t efc = 0;
    uint64_t size_links = 0, size_links0 = 0;
    std::vector<char> l0;
    std::vector<std::vector<char>> upper;
    std::vector<int> levels;
    std::unordered_map<uint64_t, uint32_t> lookup;
    int space = 0;
    uint64_t dim = 0;
    uint64_t num_deleted = 0;

    std::vector<float> u8f;  // space 3: the uint8 elements widened to float
    const char* rec(uint32_t i) const { return l0.data() + (size_t)i * size_data; }
    const float* vec(uint32_t i) const {
        return space == 3 ? u8f.data() + (size_t)i * dim : (const float*)(rec(i) + offsetData);
    }
    uint64_t label(uint32_t i) const {
        uint64_t v;
        memcpy(&v, rec(i) + label_offset, 8);
        return v;
    }
    const uint32_t* links0(uint32_t i) const { return (const uint32_t*)(rec(i) + offsetLevel0); }
    const uint32_t* links(uint32_t i, int level) const {
        return (const uint32_t*)(upper[i].data() + (size_t)(level - 1) * size_links);
    }
    static unsigned count(const uint32_t* ll) { return *(const uint16_t*)ll; }
    bool deleted(uint32_t i) const { return (((const unsigned char*)links0(i))[2] & 1) != 0; }
};

template <class T>
void rd(std::ifstream& in, T& v) { in.read((char*)&v, sizeof(T)); }

// HierarchicalNSW::loadIndex (hnswalg.h:715-821), including the file-length
// walk at :753-769.
Hnsw* load_hnsw(const char* path, int space, uint64_t dim) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) throw std::runtime_error("Cannot open file");
    in.seekg(0, in.end);
    std::streampos total = in.tellg();
    in.seekg(0, in.beg);
    auto* h = new Hnsw();
    h->space = space;
    h->dim = dim;
    rd(in, h->offsetLevel0);
    rd(in, h->max_elements);
    rd(in, h->cur);
    rd(in, h->size_data);
    rd(in, h->label_offset);
    rd(in, h->offsetData);
    rd(in, h->maxlevel);
    rd(in, h->ep);
    rd(in, h->maxM);
    rd(in, h->maxM0);
    rd(in, h->M);
    rd(in, h->mult);
    rd(in, h->efc);
    if (!in) { delete h; throw std::runtime_error("Index seems to be corrupted or unsupported"); }
    auto pos = in.tellg();
    in.seekg((std::streamoff)(h->cur * h->size_data), in.cur);
    for (uint64_t i = 0; i < h->cur; i++) {
        if (in.tellg() < 0 || in.tellg() >= total) { delete h; throw std::runtime_error("Index seems to be corrupted or unsupported"); }
        uint32_t sz;
        rd(in, sz);
        if (sz) in.seekg(sz, in.cur);
    }
    if (in.tellg() != total) { delete h; throw std::runtime_error("Index seems to be corrupted or unsupported"); }
    in.clear();
    in.seekg(pos, in.beg);
    h->l0.resize(h->cur * h->size_data);
    in.read(h->l0.data(), h->l0.size());
    h->size_links = h->maxM * 4 + 4;
    h->size_links0 = h->maxM0 * 4 + 4;
    h->upper.resize(h->cur);
    h->levels.assign(h->cur, 0);
    for (uint64_t i = 0; i < h->cur; i++) {
        h->lookup[h->label((uint32_t)i)] = (uint32_t)i;
        uint32_t sz;
        rd(in, sz);
        if (sz) {
            h->levels[i] = (int)(sz / h->size_links);
            h->upper[i].resize(sz);
            in.read(h->upper[i].data(), sz);
        }
    }
    for (uint64_t i = 0; i < h->cur; i++)
        if (h->deleted((uint32_t)i)) h->num_deleted++;
    if (space == 3) {
        h->u8f.resize(h->cur * dim);
        for (uint64_t i = 0; i < h->cur; i++) {
            const unsigned char* u = (const unsigned char*)(h->rec((uint32_t)i) + h->offsetData);
            for (uint64_t c = 0; c < dim; c++) h->u8f[i * dim + c] = (float)u[c];
        }
    }
    return h;
}

struct Trace {
    int64_t upper_hops = 0, upper_dists = 0, l0_expansions = 0, l0_dists = 0, ties = 0, max_cand = 0;
    int64_t listed = 0;  // mode 1: the run met a tie that can steer the reference's heaps (see below)
};

// Upper-layer greedy descent (hnswalg.h:1274-1302).  Shared by both modes.
uint32_t descend(const Hnsw& h, const float* q, Trace& tr) {
    uint32_t cur = h.ep;
    float curd = dist(h.space, q, h.vec(cur), h.dim);
    tr.upper_dists++;
    for (int level = h.maxlevel; level > 0; level--) {
        bool changed = true;
        while (changed) {
            changed = false;
            const uint32_t* ll = h.links(cur, level);
            int size = (int)Hnsw::count(ll);
            tr.upper_hops++;
            const uint32_t* nb = ll + 1;
            for (int i = 0; i < size; i++) {
                uint32_t c = nb[i];
                if (c > h.max_elements) throw std::runtime_error("cand error");
                float d = dist(h.space, q, h.vec(c), h.dim);
                tr.upper_dists++;
                if (d < curd) {
                    curd = d;
                    cur = c;
                    changed = true;
                }
            }
        }
    }
    return cur;
}

struct CompareByFirst {
    bool operator()(const std::pair<float, uint32_t>& a, const std::pair<float, uint32_t>& b) const {
        return a.first < b.first;
    }
};
using HeapQ = std::priority_queue<std::pair<float, uint32_t>, std::vector<std::pair<float, uint32_t>>, CompareByFirst>;

// Mode 0: the reference algorithm on the reference's own heap discipline:
// std::priority_queue is push_heap / pop_heap over a vector with the same
// comparator, used here directly so that the root's children can be read.
// searchBaseLayerST (hnswalg.h:308-440) without a stop condition.
//
// Tie events: the only decisions on which mode 0 and mode 1 can differ are
//  (a) a pop from either heap whose root ties one of its children (the heap
//      then picks among equal distances by its internal layout, mode 1 by id),
//  (b) the expansion of a candidate that had been evicted from
//      top_candidates, which the stop test only allows when its distance
//      equals lowerBound (mode 1 forgets evicted candidates).
// They are counted in Trace::ties; a query without tie events returns the
// same result in both modes.
//
// With `es` (searchStopConditionClosest with an EpsilonSearchStopCondition,
// hnswalg.h:1326-1377 and stop_condition.h:219-275) the loop is the
// non-bare-bone one (searchBaseLayerST<false>) with ef = max_num_candidates:
// the stop condition's item count is top_candidates' size, its
// should_consider_candidate and should_remove_extra are the ef tests, and its
// stop test adds "candidate beyond epsilon once min_num_candidates are held".
struct EpsStop {
    float eps;
    size_t min_c, max_c;
};
std::vector<std::pair<float, uint32_t>> base_layer_reference(const Hnsw& h, uint32_t ep, const float* q, size_t ef,
                                                             bool bare, const uint8_t* allow,
                                                             std::vector<uint32_t>& vis, uint32_t tag, Trace& tr,
                                                             const EpsStop* es = nullptr) {
    if (es) {
        ef = es->max_c;
        bare = false;
    }
    using P = std::pair<float, uint32_t>;
    CompareByFirst cmp;
    std::vector<P> top, cand;
    std::unordered_map<uint32_t, int> in_top;
    auto root_tied = [](const std::vector<P>& v) {
        return (v.size() > 1 && v[1].first == v[0].first) || (v.size() > 2 && v[2].first == v[0].first);
    };
    auto push = [&](std::vector<P>& v, P e) {
        v.push_back(e);
        std::push_heap(v.begin(), v.end(), cmp);
        if (&v == &cand && (int64_t)v.size() > tr.max_cand) tr.max_cand = (int64_t)v.size();
    };
    auto pop = [&](std::vector<P>& v) {
        if (root_tied(v)) tr.ties++;
        std::pop_heap(v.begin(), v.end(), cmp);
        v.pop_back();
    };
    auto allowed = [&](uint32_t id) { return !h.deleted(id) && (!allow || allow[id]); };
    float lb;
    if (bare || allowed(ep)) {
        float d = dist(h.space, q, h.vec(ep), h.dim);
        tr.l0_dists++;
        lb = d;
        push(top, {d, ep});
        in_top[ep]++;
        push(cand, {-d, ep});
    } else {
        lb = std::numeric_limits<float>::max();
        push(cand, {-lb, ep});
    }
    vis[ep] = tag;
    while (!cand.empty()) {
        P cp = cand.front();
        float cd = -cp.first;
        bool stop = bare ? (cd > lb) : (cd > lb && top.size() == ef);
        if (es && cd > es->eps && top.size() >= es->min_c) stop = true;
        if (stop) break;
        if (cd == lb && !in_top.count(cp.second) && (bare || allowed(cp.second))) tr.ties++;
        pop(cand);
        const uint32_t* ll = h.links0(cp.second);
        size_t size = Hnsw::count(ll);
        tr.l0_expansions++;
        for (size_t j = 1; j <= size; j++) {
            uint32_t c = ll[j];
            if (vis[c] == tag) continue;
            vis[c] = tag;
            float d = dist(h.space, q, h.vec(c), h.dim);
            tr.l0_dists++;
            if (top.size() < ef || lb > d) {
                push(cand, {-d, c});
                if (bare || allowed(c)) {
                    push(top, {d, c});
                    in_top[c]++;
                }
                while (top.size() > ef) {
                    uint32_t gone = top.front().second;
                    pop(top);
                    if (--in_top[gone] == 0) in_top.erase(gone);
                }
                if (!top.empty()) lb = top.front().first;
            }
        }
    }
    return top;
}

// Order-preserving 32-bit key of a float (monotone for all non-NaN values).
inline uint32_t fkey(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
struct Ent {
    float d;
    uint32_t id;
    bool exp;
    uint64_t key() const { return ((uint64_t)fkey(d) << 32) | id; }
};

// Mode 1: the canonical form of the same search, which the CUDA kernel
// implements.  It differs from mode 0 only where distances tie exactly:
//  * candidates are a pool sorted by (distance, internal id), each with an
//    "expanded" flag; the next expansion is the smallest unexpanded entry
//    (the reference pops its min-heap, hnswalg.h:343-359);
//  * the pool keeps the ef smallest (distance, id) allowed entries
//    (top_candidates, hnswalg.h:406-429); an insertion is accepted when the
//    pool holds fewer than ef entries or distance < lowerBound, exactly as
//    hnswalg.h:395;
//  * disallowed (deleted or filtered-out) accepted nodes go to a second sorted
//    list; they are expanded in (distance, id) order together with the pool,
//    and the search stops when the smallest remaining one lies beyond
//    lowerBound while the pool is full (hnswalg.h:353);
//  * evicted pool entries are forgotten: in the reference they stay in the
//    candidate heap but can only be expanded when they tie lowerBound.
// Trace::listed marks a bare run that meets one of the ties after which the
// reference's heaps may decide differently (the rule the GPU's two-pass
// tie-exact search lists queries by; the caller adds the top-k boundary):
//  (a) the entry popped next shares its distance with another unexpanded one;
//  (b) the entries dropped from the full pool by one expansion's insertions
//      include one whose distance equals the pool's new worst.
// A run with neither (and no boundary tie) makes the reference's decisions.
// A filtered run is always listed.
std::vector<Ent> base_layer_canonical(const Hnsw& h, uint32_t ep, const float* q, size_t ef, bool bare,
                                      const uint8_t* allow, std::vector<uint32_t>& vis, uint32_t tag, Trace& tr) {
    std::vector<Ent> pool, extra;
    auto allowed = [&](uint32_t id) { return !h.deleted(id) && (!allow || allow[id]); };
    auto ins = [](std::vector<Ent>& v, Ent e) {
        auto it = std::lower_bound(v.begin(), v.end(), e, [](const Ent& a, const Ent& b) { return a.key() < b.key(); });
        v.insert(it, e);
    };
    if (bare || allowed(ep)) {
        float d = dist(h.space, q, h.vec(ep), h.dim);
        tr.l0_dists++;
        pool.push_back({d, ep, false});
    } else {
        extra.push_back({std::numeric_limits<float>::max(), ep, false});
    }
    vis[ep] = tag;
    if (!bare) tr.listed = 1;
    while (true) {
        Ent* cp = nullptr;
        bool from_extra = false;
        for (auto& e : pool) if (!e.exp) { cp = &e; break; }
        for (auto& e : extra)
            if (!e.exp) {
                if (!cp || e.key() < cp->key()) { cp = &e; from_extra = true; }
                break;
            }
        if (!cp) break;
        float lb = pool.empty() ? std::numeric_limits<float>::max() : pool.back().d;
        if (!bare && from_extra && cp->d > lb && pool.size() == ef) break;
        if (bare)
            for (auto& e : pool)
                if (&e != cp && !e.exp && e.d == cp->d) tr.listed = 1;  // (a)
        cp->exp = true;
        uint32_t cid = cp->id;
        const uint32_t* ll = h.links0(cid);
        size_t size = Hnsw::count(ll);
        tr.l0_expansions++;
        bool dropped = false;
        float min_dropped = 0.f;
        for (size_t j = 1; j <= size; j++) {
            uint32_t c = ll[j];
            if (vis[c] == tag) continue;
            vis[c] = tag;
            float d = dist(h.space, q, h.vec(c), h.dim);
            tr.l0_dists++;
            float lbn = pool.empty() ? std::numeric_limits<float>::max() : pool.back().d;
            if (pool.size() < ef || lbn > d) {
                if (bare || allowed(c)) {
                    ins(pool, {d, c, false});
                    if (pool.size() > ef) {
                        if (!dropped || pool.back().d < min_dropped) min_dropped = pool.back().d;
                        dropped = true;
                        pool.pop_back();
                    }
                } else {
                    ins(extra, {d, c, false});
                }
            }
        }
        if (dropped && pool.back().d == min_dropped) tr.listed = 1;  // (b)
    }
    return pool;
}

struct SearchOut {
    std::vector<std::pair<float, uint64_t>> res;  // closest first
};

// searchStopConditionClosest with an EpsilonSearchStopCondition: the same
// upper-layer descent, the loop above, then top_candidates popped into a
// vector filled from the back (closest first; equal distances in the heap's
// pop order) and filter_results: trailing entries beyond epsilon dropped,
// then at most max_num_candidates kept.  The reference copies
// top_candidates' (distance, internal id) pairs into its (distance, label)
// result unchanged (hnswalg.h:1367-1371), so the second member is the
// internal id; it equals the label when labels were assigned 0, 1, 2, ... in
// insertion order.
void search_epsilon(const Hnsw& h, const float* q, const EpsStop& es, const uint8_t* allow, std::vector<uint32_t>& vis,
                    uint32_t& tag, SearchOut& out) {
    out.res.clear();
    if (h.cur == 0) return;
    Trace tr;
    uint32_t cur = descend(h, q, tr);
    tag++;
    if (tag == 0) { std::fill(vis.begin(), vis.end(), 0u); tag = 1; }
    std::vector<std::pair<float, uint32_t>> top =
        base_layer_reference(h, cur, q, es.max_c, false, allow, vis, tag, tr, &es);
    CompareByFirst cmp;
    std::vector<std::pair<float, uint64_t>> res(top.size());
    size_t sz = top.size();
    while (!top.empty()) {
        res[--sz] = {top.front().first, (uint64_t)top.front().second};
        std::pop_heap(top.begin(), top.end(), cmp);
        top.pop_back();
    }
    while (!res.empty() && res.back().first > es.eps) res.pop_back();
    while (res.size() > es.max_c) res.pop_back();
    out.res = std::move(res);
}

void search_one(const Hnsw& h, const float* q, size_t k, size_t ef, int mode, const uint8_t* allow,
                std::vector<uint32_t>& vis, uint32_t& tag, Trace& tr, SearchOut& out) {
    out.res.clear();
    if (h.cur == 0) return;
    uint32_t cur = descend(h, q, tr);
    bool bare = h.num_deleted == 0 && !allow;
    size_t ef2 = std::max(ef, k);
    tag++;
    if (tag == 0) { std::fill(vis.begin(), vis.end(), 0u); tag = 1; }
    if (mode == 0) {
        std::vector<std::pair<float, uint32_t>> top = base_layer_reference(h, cur, q, ef2, bare, allow, vis, tag, tr);
        CompareByFirst cmp;
        auto pop_top = [&] {
            if ((top.size() > 1 && top[1].first == top[0].first) || (top.size() > 2 && top[2].first == top[0].first))
                tr.ties++;
            std::pop_heap(top.begin(), top.end(), cmp);
            top.pop_back();
        };
        while (top.size() > k) pop_top();
        std::priority_queue<std::pair<float, uint64_t>> result;
        while (!top.empty()) {
            result.emplace(top.front().first, h.label(top.front().second));
            std::pop_heap(top.begin(), top.end(), cmp);
            top.pop_back();
        }
        out.res.resize(result.size());
        size_t n = result.size();
        while (!result.empty()) { out.res[--n] = result.top(); result.pop(); }
    } else {
        std::vector<Ent> pool = base_layer_canonical(h, cur, q, ef2, bare, allow, vis, tag, tr);
        if (pool.size() > k && pool[k - 1].d == pool[k].d) tr.listed = 1;  // the top-k boundary
        size_t n = std::min(k, pool.size());
        for (size_t i = 0; i < n; i++) out.res.emplace_back(pool[i].d, h.label(pool[i].id));
        std::sort(out.res.begin(), out.res.end());
    }
}

// ------------------------------------------------------------- brute force
struct Bf {
    uint64_t maxelements = 0, size_per = 0, cur = 0;
    std::vector<char> data;
    int space = 0;
    uint64_t dim = 0;
    const float* vec(size_t i) const { return (const float*)(data.data() + i * size_per); }
    uint64_t label(size_t i) const {
        uint64_t v;
        memcpy(&v, data.data() + i * size_per + dim * 4, 8);
        return v;
    }
};

// BruteforceSearch::loadIndex (bruteforce.h:142-161).
Bf* load_bf(const char* path, int space, uint64_t dim) {
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) throw std::runtime_error("Cannot open file");
    auto* b = new Bf();
    b->space = space;
    b->dim = dim;
    rd(in, b->maxelements);
    rd(in, b->size_per);
    rd(in, b->cur);
    b->size_per = dim * 4 + 8;
    b->data.resize(b->maxelements * b->size_per);
    in.read(b->data.data(), b->data.size());
    return b;
}

// BruteforceSearch::searchKnn (bruteforce.h:106-125).
void bf_one(const Bf& b, const float* q, size_t k, const uint8_t* allow, SearchOut& out) {
    std::priority_queue<std::pair<float, uint64_t>> top;
    float last = std::numeric_limits<float>::max();
    for (size_t i = 0; i < b.cur; i++) {
        float d = dist(b.space, q, b.vec(i), b.dim);
        if (d <= last || top.size() < k) {
            if (!allow || allow[i]) {
                top.emplace(d, b.label(i));
                if (top.size() > k) top.pop();
                if (!top.empty()) last = top.top().first;
            }
        }
    }
    out.res.resize(top.size());
    size_t n = top.size();
    while (!top.empty()) { out.res[--n] = top.top(); top.pop(); }
}

thread_local std::string g_err;

template <class F>
void parallel_for(size_t n, int nthreads, F fn) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    if (nthreads <= 1 || n <= 1) {
        for (size_t i = 0; i < n; i++) fn(i, 0);
        return;
    }
    std::atomic<size_t> next(0);
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++)
        th.emplace_back([&, t] {
            while (true) {
                size_t i = next.fetch_add(1);
                if (i >= n) break;
                fn(i, t);
            }
        });
    for (auto& t : th) t.join();
}

}  // namespace

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

float orc_distance(int space, const float* a, const float* b, uint64_t dim) { return dist(space, a, b, dim); }

void orc_distances(int space, const float* q, const float* x, uint64_t n, uint64_t dim, float* out) {
    for (uint64_t i = 0; i < n; i++) out[i] = dist(space, q, x + i * dim, dim);
}

// normalize_vector of python_bindings/bindings.cpp:241-248 (cosine space).
// The squared-norm loop compiles like L2Sqr's scalar loop: 4-wide in-order
// rounded products, then fma for the last dim%4 terms.
void orc_normalize(const float* in, float* out, uint64_t n, uint64_t dim) {
    for (uint64_t r = 0; r < n; r++) {
        const float* x = in + r * dim;
        float s = 0.f;
        uint64_t n4 = dim / 4 * 4;
        for (uint64_t i = 0; i < n4; i++) {
            float p = x[i] * x[i];
            s = s + p;
        }
        for (uint64_t i = n4; i < dim; i++) s = std::fma(x[i], x[i], s);
        s = 1.0f / (sqrtf(s) + 1e-30f);
        for (uint64_t i = 0; i < dim; i++) out[r * dim + i] = x[i] * s;
    }
}

void* orc_hnsw_load(const char* path, int space, uint64_t dim) {
    try {
        return load_hnsw(path, space, dim);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void orc_hnsw_free(void* p) { delete (Hnsw*)p; }
uint64_t orc_hnsw_count(void* p) { return ((Hnsw*)p)->cur; }
uint64_t orc_hnsw_num_deleted(void* p) { return ((Hnsw*)p)->num_deleted; }
uint64_t orc_hnsw_maxM0(void* p) { return ((Hnsw*)p)->maxM0; }
int orc_hnsw_maxlevel(void* p) { return ((Hnsw*)p)->maxlevel; }

void orc_hnsw_labels(void* p, uint64_t* out) {
    auto* h = (Hnsw*)p;
    for (uint64_t i = 0; i < h->cur; i++) out[i] = h->label((uint32_t)i);
}

// markDelete / unmarkDelete (hnswalg.h:852-927): byte 2, bit 0 of the level-0
// record.  Returns 0 on success, -1 for an unknown label, -2 when the mark is
// already in the requested state.
int orc_hnsw_set_deleted(void* p, uint64_t label, int flag) {
    auto* h = (Hnsw*)p;
    auto it = h->lookup.find(label);
    if (it == h->lookup.end()) return -1;
    unsigned char* b = (unsigned char*)h->links0(it->second) + 2;
    bool cur = (*b & 1) != 0;
    if (cur == (flag != 0)) return -2;
    if (flag) { *b |= 1; h->num_deleted++; }
    else { *b &= (unsigned char)~1u; h->num_deleted--; }
    return 0;
}

// Batched searchKnn.  mode 0 = reference heaps, 1 = canonical pool.
// allow: optional per-internal-id byte mask (the filter functor evaluated on
// each node's label).  Outputs are closest first; counts[i] = results found.
// trace (optional) receives 7 int64 per query: upper-layer link lists read,
// upper-layer distances, level-0 expansions, level-0 distances, tie events
// (mode 0 only; see base_layer_reference), largest candidate-heap size (mode 0),
// listed for the heap replay (mode 1; see base_layer_canonical).
int orc_hnsw_search(void* p, const float* q, uint64_t nq, uint64_t k, uint64_t ef, int mode,
                    const uint8_t* allow, uint64_t* labels, float* dists, int32_t* counts,
                    int64_t* trace, int nthreads) {
    auto* h = (Hnsw*)p;
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    std::vector<std::vector<uint32_t>> vis(nthreads, std::vector<uint32_t>());
    std::vector<uint32_t> tags(nthreads, 0);
    std::vector<SearchOut> outs(nthreads);
    std::atomic<int> failed(0);
    parallel_for(nq, nthreads, [&](size_t i, int t) {
        if (vis[t].size() != h->cur) vis[t].assign(h->cur + 1, 0);
        Trace tr;
        try {
            search_one(*h, q + i * h->dim, k, ef, mode, allow, vis[t], tags[t], tr, outs[t]);
        } catch (const std::exception& e) {
            failed = 1;
            return;
        }
        auto& r = outs[t].res;
        counts[i] = (int32_t)r.size();
        for (size_t j = 0; j < k; j++) {
            labels[i * k + j] = j < r.size() ? r[j].second : ~0ull;
            dists[i * k + j] = j < r.size() ? r[j].first : std::numeric_limits<float>::infinity();
        }
        if (trace) {
            trace[i * 7 + 0] = tr.upper_hops;
            trace[i * 7 + 1] = tr.upper_dists;
            trace[i * 7 + 2] = tr.l0_expansions;
            trace[i * 7 + 3] = tr.l0_dists;
            trace[i * 7 + 4] = tr.ties;
            trace[i * 7 + 5] = tr.max_cand;
            trace[i * 7 + 6] = tr.listed;
        }
    });
    if (failed) { g_err = "cand error"; return -1; }
    return 0;
}

// searchStopConditionClosest with a MultiVectorSearchStopCondition
// (stop_condition.h:146-216) over a multi-vector index, whose elements carry
// a uint32 document id right after the vector.  The loop is the non-bare-bone
// one of base_layer_reference, but its size tests count distinct documents
// among top_candidates (curr_num_docs against ef_collection =
// max(ef_collection, num_docs)), and the condition keeps its own max-heap of
// (distance, document) pairs, popped on every eviction and by
// filter_results, which trims the result until num_docs documents remain.
void search_multivector(const Hnsw& h, const float* q, size_t num_docs, size_t ef_coll_in,
                        std::vector<uint32_t>& vis, uint32_t& tag, SearchOut& out) {
    out.res.clear();
    if (h.cur == 0) return;
    Trace tr;
    uint32_t ep = descend(h, q, tr);
    tag++;
    if (tag == 0) { std::fill(vis.begin(), vis.end(), 0u); tag = 1; }
    const size_t ef_coll = std::max(ef_coll_in, num_docs);
    auto doc = [&](uint32_t id) {
        uint32_t d;
        memcpy(&d, (const char*)h.vec(id) + h.dim * sizeof(float), 4);
        return d;
    };
    using P = std::pair<float, uint32_t>;
    CompareByFirst cmp;
    std::vector<P> top, cand;
    std::unordered_map<uint32_t, size_t> doc_counter;
    size_t cur_docs = 0;
    std::priority_queue<std::pair<float, uint32_t>> results;  // (distance, document)
    auto add_point = [&](uint32_t id, float d) {
        const uint32_t dc = doc(id);
        if (doc_counter[dc] == 0) cur_docs++;
        results.emplace(d, dc);
        doc_counter[dc]++;
    };
    auto remove_point = [&](uint32_t id) {
        const uint32_t dc = doc(id);
        if (--doc_counter[dc] == 0) cur_docs--;
        results.pop();
    };
    const float d0 = dist(h.space, q, h.vec(ep), h.dim);
    float lb = d0;
    top.push_back({d0, ep});
    std::push_heap(top.begin(), top.end(), cmp);
    add_point(ep, d0);
    cand.push_back({-d0, ep});
    std::push_heap(cand.begin(), cand.end(), cmp);
    vis[ep] = tag;
    while (!cand.empty()) {
        const P cp = cand.front();
        const float cd = -cp.first;
        if (cd > lb && cur_docs == ef_coll) break;
        std::pop_heap(cand.begin(), cand.end(), cmp);
        cand.pop_back();
        const uint32_t* ll = h.links0(cp.second);
        const size_t size = Hnsw::count(ll);
        for (size_t j = 1; j <= size; j++) {
            const uint32_t c = ll[j];
            if (vis[c] == tag) continue;
            vis[c] = tag;
            const float d = dist(h.space, q, h.vec(c), h.dim);
            if (cur_docs < ef_coll || lb > d) {
                cand.push_back({-d, c});
                std::push_heap(cand.begin(), cand.end(), cmp);
                top.push_back({d, c});
                std::push_heap(top.begin(), top.end(), cmp);
                add_point(c, d);
                while (cur_docs > ef_coll) {
                    const uint32_t gone = top.front().second;
                    std::pop_heap(top.begin(), top.end(), cmp);
                    top.pop_back();
                    remove_point(gone);
                }
                if (!top.empty()) lb = top.front().first;
            }
        }
    }
    std::vector<std::pair<float, uint64_t>> res(top.size());
    size_t sz = top.size();
    while (!top.empty()) {
        res[--sz] = {top.front().first, (uint64_t)top.front().second};
        std::pop_heap(top.begin(), top.end(), cmp);
        top.pop_back();
    }
    while (cur_docs > num_docs && !res.empty()) {
        const uint32_t dc = results.top().second;
        if (--doc_counter[dc] == 0) cur_docs--;
        results.pop();
        res.pop_back();
    }
    out.res = std::move(res);
}

// Batched multi-vector search; up to `cap` results per query (internal ids,
// as the reference returns them), counts[i] = result size or -1 beyond cap.
int orc_hnsw_search_multivector(void* p, const float* q, uint64_t nq, uint64_t num_docs, uint64_t ef_coll,
                                uint64_t cap, uint64_t* ids, float* dists, int32_t* counts, int nthreads) {
    auto* h = (Hnsw*)p;
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    std::vector<std::vector<uint32_t>> vis(nthreads, std::vector<uint32_t>());
    std::vector<uint32_t> tags(nthreads, 0);
    std::vector<SearchOut> outs(nthreads);
    parallel_for(nq, nthreads, [&](size_t i, int t) {
        if (vis[t].size() != h->cur) vis[t].assign(h->cur + 1, 0);
        search_multivector(*h, q + i * h->dim, num_docs, ef_coll, vis[t], tags[t], outs[t]);
        auto& r = outs[t].res;
        counts[i] = r.size() <= cap ? (int32_t)r.size() : -1;
        for (size_t j = 0; j < cap; j++) {
            ids[i * cap + j] = j < r.size() ? r[j].second : ~0ull;
            dists[i * cap + j] = j < r.size() ? r[j].first : std::numeric_limits<float>::infinity();
        }
    });
    return 0;
}

// Batched epsilon search (searchStopConditionClosest with
// EpsilonSearchStopCondition).  Outputs max_c slots per query in the
// reference's result order; counts[i] = results kept.
int orc_hnsw_search_epsilon(void* p, const float* q, uint64_t nq, float eps, uint64_t min_c, uint64_t max_c,
                            const uint8_t* allow, uint64_t* labels, float* dists, int32_t* counts, int nthreads) {
    auto* h = (Hnsw*)p;
    if (min_c > max_c || max_c == 0) { g_err = "need 0 < max_num_candidates and min <= max"; return -1; }
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    std::vector<std::vector<uint32_t>> vis(nthreads, std::vector<uint32_t>());
    std::vector<uint32_t> tags(nthreads, 0);
    std::vector<SearchOut> outs(nthreads);
    const EpsStop es{eps, (size_t)min_c, (size_t)max_c};
    parallel_for(nq, nthreads, [&](size_t i, int t) {
        if (vis[t].size() != h->cur) vis[t].assign(h->cur + 1, 0);
        search_epsilon(*h, q + i * h->dim, es, allow, vis[t], tags[t], outs[t]);
        auto& r = outs[t].res;
        counts[i] = (int32_t)r.size();
        for (size_t j = 0; j < max_c; j++) {
            labels[i * max_c + j] = j < r.size() ? r[j].second : ~0ull;
            dists[i * max_c + j] = j < r.size() ? r[j].first : std::numeric_limits<float>::infinity();
        }
    });
    return 0;
}

void* orc_bf_load(const char* path, int space, uint64_t dim) {
    try {
        return load_bf(path, space, dim);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}
void orc_bf_free(void* p) { delete (Bf*)p; }
uint64_t orc_bf_count(void* p) { return ((Bf*)p)->cur; }

int orc_bf_search(void* p, const float* q, uint64_t nq, uint64_t k, const uint8_t* allow, uint64_t* labels,
                  float* dists, int32_t* counts, int nthreads) {
    auto* b = (Bf*)p;
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    std::vector<SearchOut> outs(nthreads);
    parallel_for(nq, nthreads, [&](size_t i, int t) {
        bf_one(*b, q + i * b->dim, k, allow, outs[t]);
        auto& r = outs[t].res;
        counts[i] = (int32_t)r.size();
        for (size_t j = 0; j < k; j++) {
            labels[i * k + j] = j < r.size() ? r[j].second : ~0ull;
            dists[i * k + j] = j < r.size() ? r[j].first : std::numeric_limits<float>::infinity();
        }
    });
    return 0;
}

// Brute force over a plain row-major float matrix (no index file): exact top-k
// by (distance, row) -- the BruteforceSearch result when labels are row ids.
int orc_bf_matrix(int space, const float* x, uint64_t n, uint64_t dim, const float* q, uint64_t nq, uint64_t k,
                  uint64_t* labels, float* dists, int nthreads) {
    if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
    parallel_for(nq, nthreads, [&](size_t i, int) {
        std::priority_queue<std::pair<float, uint64_t>> top;
        float last = std::numeric_limits<float>::max();
        for (uint64_t r = 0; r < n; r++) {
            float d = dist(space, q + i * dim, x + r * dim, dim);
            if (d <= last || top.size() < k) {
                top.emplace(d, r);
                if (top.size() > k) top.pop();
                last = top.top().first;
            }
        }
        size_t m = top.size();
        for (size_t j = m; j < k; j++) { labels[i * k + j] = ~0ull; dists[i * k + j] = INFINITY; }
        while (!top.empty()) {
            --m;
            labels[i * k + m] = top.top().second;
            dists[i * k + m] = top.top().first;
            top.pop();
        }
    });
    return 0;
}

}  // extern "C"
