// Test infrastructure only (a CPU checker, never part of the product): the
// reference's multi-vector search, HierarchicalNSW::searchStopConditionClosest
// with MultiVectorSearchStopCondition over MultiVectorL2Space /
// MultiVectorInnerProductSpace (hnswlib/stop_condition.h:1-217), compiled from
// the reference's headers by oracle/Makefile into oracle/_ref/libref_multivec.so.
// Each stored element carries a document id after its vector; the Python
// bindings cannot build such an index, so this builds one with addPoint,
// saves it, and searches it, for the golden-fixture script and the tests.
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "hnswlib.h"

namespace {

using DocId = unsigned int;

std::unique_ptr<hnswlib::BaseMultiVectorSpace<DocId>> make_space(int space, uint64_t dim) {
    if (space == 0) return std::unique_ptr<hnswlib::BaseMultiVectorSpace<DocId>>(new hnswlib::MultiVectorL2Space<DocId>(dim));
    return std::unique_ptr<hnswlib::BaseMultiVectorSpace<DocId>>(new hnswlib::MultiVectorInnerProductSpace<DocId>(dim));
}

}  // namespace

extern "C" {

// Build (single-threaded addPoint in row order) and save an index of n
// vectors with their document ids and labels.  space 0 = L2, 1 = inner product.
int ref_mv_build(const char* path, int space, const float* vecs, const uint32_t* docs, const uint64_t* labels,
                 uint64_t n, uint64_t dim, uint64_t M, uint64_t efc, uint64_t seed) {
    try {
        auto sp = make_space(space, dim);
        hnswlib::HierarchicalNSW<float> alg(sp.get(), n, M, efc, seed);
        std::vector<char> point(sp->get_data_size());
        for (uint64_t i = 0; i < n; i++) {
            memcpy(point.data(), vecs + i * dim, dim * sizeof(float));
            sp->set_doc_id(point.data(), docs[i]);
            alg.addPoint(point.data(), labels[i]);
        }
        alg.saveIndex(std::string(path));
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// searchStopConditionClosest with MultiVectorSearchStopCondition(space,
// num_docs, ef_collection) for nq queries of dim floats; up to `cap` results
// per query in the reference's order (internal ids, as the reference's result
// holds them), counts[i] = its result size (-1 if larger than cap).
int ref_mv_search(const char* path, int space, uint64_t dim, const float* q, uint64_t nq, uint64_t num_docs,
                  uint64_t ef_collection, uint64_t cap, uint64_t* ids, float* dists, int32_t* counts) {
    try {
        auto sp = make_space(space, dim);
        hnswlib::HierarchicalNSW<float> alg(sp.get(), std::string(path));
        for (uint64_t i = 0; i < nq; i++) {
            hnswlib::MultiVectorSearchStopCondition<DocId, float> stop(*sp, num_docs, ef_collection);
            auto r = alg.searchStopConditionClosest(q + i * dim, stop);
            counts[i] = r.size() <= cap ? (int32_t)r.size() : -1;
            for (uint64_t j = 0; j < cap; j++) {
                ids[i * cap + j] = j < r.size() ? (uint64_t)r[j].second : ~0ull;
                dists[i * cap + j] = j < r.size() ? r[j].first : __builtin_inff();
            }
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
