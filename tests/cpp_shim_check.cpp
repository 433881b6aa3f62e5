// Drives the C++ shim (include/hnswgpu.hpp) the way hnswlib's own C++ tests
// drive hnswlib (tests/cpp/searchKnnCloserFirst_test.cpp,
// tests/cpp/searchKnnWithFilter_test.cpp): prints the closest-first results
// of searchKnn for every query so the Python side can compare them with the
// reference's recorded outputs, and checks closer-first ordering, filter
// functors and delete marks.  With three more arguments it then prints a line
// "EPS" and, per query, searchStopConditionClosest's results for an
// EpsilonSearchStopCondition(eps, min, max) (tests/cpp/epsilon_search_test.cpp
// drives the reference the same way).
// Usage: cpp_shim_check index.bin queries.f32 dim nq k ef [eps min max]
//        cpp_shim_check --timed index.bin queries.f32 dim nq k ef out.bin
// The second form runs nq single-query searchKnn calls with a filter functor
// of a type unrelated to hnswgpu::BaseFilterFunctor (the shape of
// hnswlib::BaseFilterFunctor: even labels only), prints each result and, last,
// the seconds the calls took; it also checks the ef_ proxy and writes the
// index with one delete mark through saveIndex to out.bin.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "hnswgpu.hpp"

// A filter functor as hnswlib declares one (hnswlib/hnswlib.h:128-132),
// not derived from hnswgpu::BaseFilterFunctor.
namespace hnswlib_like {
class BaseFilterFunctor {
 public:
    virtual bool operator()(size_t) { return true; }
    virtual ~BaseFilterFunctor() {}
};
}  // namespace hnswlib_like
struct PickEven : public hnswlib_like::BaseFilterFunctor {
    bool operator()(size_t l) override { return l % 2 == 0; }
};

static int timed(int argc, char** argv) {
    if (argc != 9) return 2;
    const char* path = argv[2];
    size_t dim = atoi(argv[4]), nq = atoi(argv[5]), k = atoi(argv[6]), ef = atoi(argv[7]);
    std::vector<float> q(nq * dim);
    FILE* f = fopen(argv[3], "rb");
    if (!f || fread(q.data(), 4, q.size(), f) != q.size()) return 3;
    fclose(f);
    hnswgpu::L2Space space(dim);
    hnswgpu::HierarchicalNSW<float> alg(&space, path);
    alg.ef_ = ef;
    if ((size_t)alg.ef_ != ef) return 20;
    PickEven even;
    hnswlib_like::BaseFilterFunctor* filter = &even;
    std::vector<std::vector<std::pair<float, size_t>>> res(nq);
    const auto t0 = std::chrono::steady_clock::now();
    for (size_t i = 0; i < nq; i++) res[i] = alg.searchKnnCloserFirst(q.data() + i * dim, k, filter);
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (auto& r : res) {
        for (auto& e : r) {
            if (e.second % 2) return 21;
            printf("%llu %.9g ", (unsigned long long)e.second, e.first);
        }
        printf("\n");
    }
    alg.markDelete(res[0][0].second);
    alg.saveIndex(argv[8]);
    printf("SECONDS %.6f\n", secs);
    return 0;
}

struct PickNothing : public hnswgpu::BaseFilterFunctor {
    bool operator()(hnswgpu::labeltype) override { return false; }
};
struct PickDivisible : public hnswgpu::BaseFilterFunctor {
    size_t div;
    explicit PickDivisible(size_t d) : div(d) {}
    bool operator()(hnswgpu::labeltype l) override { return l % div == 0; }
};

int main(int argc, char** argv) {
    if (argc > 1 && strcmp(argv[1], "--timed") == 0) return timed(argc, argv);
    if (argc != 7 && argc != 10) return 2;
    const char* path = argv[1];
    size_t dim = atoi(argv[3]), nq = atoi(argv[4]), k = atoi(argv[5]), ef = atoi(argv[6]);
    std::vector<float> q(nq * dim);
    FILE* f = fopen(argv[2], "rb");
    if (!f || fread(q.data(), 4, q.size(), f) != q.size()) return 3;
    fclose(f);
    hnswgpu::L2Space space(dim);
    auto* alg = new hnswgpu::HierarchicalNSW<float>(&space, path);
    alg->setEf(ef);
    for (size_t i = 0; i < nq; i++) {
        auto pq = alg->searchKnn(q.data() + i * dim, k);
        auto cf = alg->searchKnnCloserFirst(q.data() + i * dim, k);
        if (cf.size() != pq.size()) return 4;
        // closer first == the heap popped into reverse order
        for (size_t j = cf.size(); j-- > 0;) {
            if (cf[j] != pq.top()) return 5;
            pq.pop();
        }
        for (auto& r : cf) printf("%llu %.9g ", (unsigned long long)r.second, r.first);
        printf("\n");
    }
    if (argc == 10) {
        hnswgpu::EpsilonSearchStopCondition sc((float)atof(argv[7]), atoi(argv[8]), atoi(argv[9]));
        printf("EPS\n");
        for (size_t i = 0; i < nq; i++) {
            auto r = alg->searchStopConditionClosest(q.data() + i * dim, sc);
            for (size_t j = 0; j < r.size(); j++) {
                if (r[j].first > sc.epsilon() || (j && r[j].first < r[j - 1].first)) return 13;
                printf("%llu %.9g ", (unsigned long long)r[j].second, r[j].first);
            }
            printf("\n");
        }
    }
    PickNothing none;
    if (!alg->searchKnn(q.data(), k, &none).empty()) return 6;
    PickDivisible d3(3);
    for (auto& r : alg->searchKnnCloserFirst(q.data(), k, &d3))
        if (r.second % 3) return 7;
    auto first = alg->searchKnnCloserFirst(q.data(), 1)[0].second;
    alg->markDelete(first);
    for (auto& r : alg->searchKnnCloserFirst(q.data(), k))
        if (r.second == first) return 8;
    try {
        alg->markDelete(first);
        return 9;
    } catch (const std::runtime_error&) {
    }
    alg->unmarkDelete(first);
    if (alg->searchKnnCloserFirst(q.data(), 1)[0].second != first) return 10;
    try {
        hnswgpu::HierarchicalNSW<float> bad(&space, "/nonexistent/index.bin");
        return 11;
    } catch (const std::runtime_error& e) {
        if (std::string(e.what()) != "Cannot open file") return 12;
    }
    delete alg;
    return 0;
}
