// Test infrastructure only (a CPU checker, never part of the product): the
// reference's own HierarchicalNSW::searchStopConditionClosest with its
// EpsilonSearchStopCondition (hnswlib/hnswalg.h:1326-1377,
// hnswlib/stop_condition.h:219-275), compiled from the reference's headers by
// oracle/Makefile into oracle/_ref/libref_stopcond.so and called through the
// C function below by the tests and by the golden-fixture script.
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "hnswlib.h"

namespace {

// The reference's filter functor over labels, from a per-label byte mask.
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

// space 0 = L2, 1 = inner product.  `deleted` labels are marked deleted after
// loading; `allow` (nallow bytes, indexed by label) is the filter, or null.
// Outputs max_c slots per query, in the order searchStopConditionClosest
// returns; counts[i] = its result size.  Returns 0, or -1 on an exception.
int ref_epsilon_search(const char* path, int space, uint64_t dim, const uint64_t* deleted, uint64_t ndel,
                       const uint8_t* allow, uint64_t nallow, const float* q, uint64_t nq, float eps, uint64_t min_c,
                       uint64_t max_c, uint64_t* labels, float* dists, int32_t* counts) {
    try {
        std::unique_ptr<hnswlib::SpaceInterface<float>> sp;
        if (space == 0) sp.reset(new hnswlib::L2Space(dim));
        else sp.reset(new hnswlib::InnerProductSpace(dim));
        hnswlib::HierarchicalNSW<float> alg(sp.get(), std::string(path));
        for (uint64_t i = 0; i < ndel; i++) alg.markDelete(deleted[i]);
        LabelMask filter(allow, nallow);
        for (uint64_t i = 0; i < nq; i++) {
            hnswlib::EpsilonSearchStopCondition<float> stop(eps, min_c, max_c);
            std::vector<std::pair<float, hnswlib::labeltype>> r =
                alg.searchStopConditionClosest(q + i * dim, stop, allow ? &filter : nullptr);
            counts[i] = (int32_t)r.size();
            for (uint64_t j = 0; j < max_c; j++) {
                labels[i * max_c + j] = j < r.size() ? (uint64_t)r[j].second : ~0ull;
                dists[i * max_c + j] = j < r.size() ? r[j].first : __builtin_inff();
            }
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
