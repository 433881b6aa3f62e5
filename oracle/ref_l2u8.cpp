// Test infrastructure only (a CPU checker, never part of the product): the
// reference's HierarchicalNSW<int> over hnswlib::L2SpaceI (uint8 vectors,
// integer squared-L2; hnswlib/space_l2.h:255-323), compiled from the
// reference's headers by oracle/Makefile into oracle/_ref/libref_l2u8.so.
// The Python bindings cannot build such an index, so this builds one with the
// reference's addPoint, saves it with saveIndex, and runs searchKnn on it, for
// the golden-fixture script and the tests.
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "hnswlib.h"

namespace {

class LabelMask : public hnswlib::BaseFilterFunctor {
 public:
    LabelMask(const uint8_t* mask, uint64_t n) : mask_(mask), n_(n) {}
    bool operator()(hnswlib::labeltype label) override { return label < n_ && mask_[label] != 0; }

 private:
    const uint8_t* mask_;
    uint64_t n_;
};

}  // namespace

extern "C" {

// Build (single-threaded addPoint in row order) and save an index of n uint8
// rows with the given labels.  Returns 0, or -1 on an exception.
int ref_l2u8_build(const char* path, const uint8_t* data, const uint64_t* labels, uint64_t n, uint64_t dim,
                   uint64_t M, uint64_t efc, uint64_t seed) {
    try {
        hnswlib::L2SpaceI space(dim);
        hnswlib::HierarchicalNSW<int> alg(&space, n, M, efc, seed);
        for (uint64_t i = 0; i < n; i++) alg.addPoint(data + i * dim, labels[i]);
        alg.saveIndex(std::string(path));
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// searchKnn on a saved index (queries: nq x dim uint8) after marking the
// `deleted` labels, with an optional per-label filter.  Outputs k slots per
// query, closest first (the reference's priority queue popped in reverse);
// distances as int.  Returns 0, or -1 on an exception.
int ref_l2u8_search(const char* path, uint64_t dim, const uint8_t* q, uint64_t nq, uint64_t k, uint64_t ef,
                    const uint64_t* deleted, uint64_t ndel, const uint8_t* allow, uint64_t nallow, uint64_t* labels,
                    int32_t* dists, int32_t* counts) {
    try {
        hnswlib::L2SpaceI space(dim);
        hnswlib::HierarchicalNSW<int> alg(&space, std::string(path));
        alg.setEf(ef);
        for (uint64_t i = 0; i < ndel; i++) alg.markDelete(deleted[i]);
        LabelMask filter(allow, nallow);
        for (uint64_t i = 0; i < nq; i++) {
            auto pq = alg.searchKnn(q + i * dim, k, allow ? &filter : nullptr);
            const size_t c = pq.size();
            counts[i] = (int32_t)c;
            for (size_t j = c; j < k; j++) {
                labels[i * k + j] = ~0ull;
                dists[i * k + j] = -1;
            }
            for (size_t j = c; j-- > 0;) {
                labels[i * k + j] = (uint64_t)pq.top().second;
                dists[i * k + j] = pq.top().first;
                pq.pop();
            }
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
