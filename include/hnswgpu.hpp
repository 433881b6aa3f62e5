// hnswgpu.hpp -- header-only C++ classes over the C ABI (hnswgpu.h) with the
// shape of hnswlib's query API, so that C++ code written against hnswlib
// 0.9.0 switches by changing the namespace and the space type:
//
//   hnswlib::L2Space space(dim);                    hnswgpu::L2Space space(dim);
//   auto* a = new hnswlib::HierarchicalNSW<float>(  auto* a = new hnswgpu::HierarchicalNSW<float>(
//       &space, "index.bin");                           &space, "index.bin");
//   a->setEf(64);                                   a->setEf(64);
//   auto pq = a->searchKnn(q, 10, &filter);         auto pq = a->searchKnn(q, 10, &filter);
//
// Replaced interfaces: HierarchicalNSW load constructor, setEf and the public
// ef_, searchKnn, searchKnnCloserFirst, saveIndex, markDelete / unmarkDelete
// (hnswlib/hnswalg.h:78-86, 173-175, 685-712, 852-927, 1269-1323;
// hnswlib/hnswlib.h:186-221 -- both classes derive from an AlgorithmInterface
// of the same shape), BruteforceSearch load constructor and searchKnn
// (hnswlib/bruteforce.h:35-43, 106-125), BaseFilterFunctor
// (hnswlib/hnswlib.h:128-132).  searchKnn takes any filter functor type with
// bool operator()(size_t) -- hnswlib::BaseFilterFunctor included, without
// including hnswlib.  Errors are thrown as std::runtime_error with the
// reference's messages.  Index construction (addPoint) stays with hnswlib:
// build and save there, load here; addPoint throws.
//
// Filters: the GPU cannot call a C++ functor per candidate, so a functor is
// evaluated once over the index's labels at its first use with an index and
// its answers are kept on the device (one mask per functor object): later
// searches with the same functor copy nothing.  A functor whose answers
// change must be passed to refreshFilter (or forgetFilter) first.
#pragma once
#include <cstdint>
#include <queue>
#include <unordered_map>
#include <type_traits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "hnswgpu.h"

namespace hnswgpu {

typedef size_t labeltype;

// Same contract as hnswlib::BaseFilterFunctor: true = the label may be
// returned.  The GPU path evaluates it for every label of the index at its
// first use with that index and keeps the answers on the device (the
// reference calls it per candidate).
class BaseFilterFunctor {
 public:
    virtual bool operator()(labeltype) { return true; }
    virtual ~BaseFilterFunctor() {}
};

// The parameters of hnswlib::EpsilonSearchStopCondition
// (hnswlib/stop_condition.h:219-233); the search itself runs on the GPU.
class EpsilonSearchStopCondition {
 public:
    EpsilonSearchStopCondition(float epsilon, size_t min_num_candidates, size_t max_num_candidates)
        : eps_(epsilon), min_(min_num_candidates), max_(max_num_candidates) {
        if (min_num_candidates > max_num_candidates)
            throw std::runtime_error("min_num_candidates must not exceed max_num_candidates");
    }
    float epsilon() const { return eps_; }
    size_t min_num_candidates() const { return min_; }
    size_t max_num_candidates() const { return max_; }

 private:
    float eps_;
    size_t min_, max_;
};

class SpaceInterface {
 public:
    virtual int space_kind() const = 0;
    virtual size_t dim() const = 0;
    size_t get_data_size() const { return dim() * sizeof(float); }
    virtual ~SpaceInterface() {}
};

class L2Space : public SpaceInterface {
    size_t dim_;

 public:
    explicit L2Space(size_t dim) : dim_(dim) {}
    int space_kind() const override { return HNSWGPU_SPACE_L2; }
    size_t dim() const override { return dim_; }
};

class InnerProductSpace : public SpaceInterface {
    size_t dim_;

 public:
    explicit InnerProductSpace(size_t dim) : dim_(dim) {}
    int space_kind() const override { return HNSWGPU_SPACE_IP; }
    size_t dim() const override { return dim_; }
};

// The Python binding's "cosine" space: inner product with queries
// normalised on the way in (stored vectors are expected normalised).
class CosineSpace : public SpaceInterface {
    size_t dim_;

 public:
    explicit CosineSpace(size_t dim) : dim_(dim) {}
    int space_kind() const override { return HNSWGPU_SPACE_COSINE; }
    size_t dim() const override { return dim_; }
};

// The shape of hnswlib::AlgorithmInterface (hnswlib/hnswlib.h:186-221) with
// this library's filter type; searchKnn / searchKnnCloserFirst also accept
// any other functor type through the derived classes' templates.
template <typename dist_t>
class AlgorithmInterface {
 public:
    virtual void addPoint(const void* datapoint, labeltype label, bool replace_deleted = false) = 0;
    virtual std::priority_queue<std::pair<dist_t, labeltype>> searchKnn(const void*, size_t,
                                                                        BaseFilterFunctor* isIdAllowed = nullptr) const = 0;
    virtual std::vector<std::pair<dist_t, labeltype>> searchKnnCloserFirst(
        const void* query_data, size_t k, BaseFilterFunctor* isIdAllowed = nullptr) const = 0;
    virtual void saveIndex(const std::string& location) = 0;
    virtual ~AlgorithmInterface() {}
};

namespace detail {
inline void check(int rc) {
    if (rc != HNSWGPU_OK) throw std::runtime_error(hnswgpu_last_error());
}

class IndexBase {
 protected:
    hnswgpu_index* h_ = nullptr;
    size_t dim_ = 0;
    uint32_t flags_ = 0;
    // device-resident masks of the functors used with this index
    mutable std::unordered_map<const void*, uint32_t> filters_;

    template <class F>
    uint32_t filter_id(F* f) const {
        if (!f) return 0;
        auto it = filters_.find(static_cast<const void*>(f));
        if (it != filters_.end()) return it->second;
        hnswgpu_info info;
        check(hnswgpu_get_info(h_, &info));
        std::vector<uint64_t> labels(info.count);
        if (info.count) check(hnswgpu_get_labels(h_, labels.data()));
        std::vector<uint8_t> m(info.count);
        for (size_t i = 0; i < labels.size(); i++) m[i] = (*f)((labeltype)labels[i]) ? 1 : 0;
        uint32_t id = 0;
        check(hnswgpu_filter_create(h_, m.data(), &id));
        filters_.emplace(static_cast<const void*>(f), id);
        return id;
    }

    // host mask of a functor (the epsilon search takes the mask itself)
    template <class F>
    std::vector<uint8_t> mask(F* f) const {
        std::vector<uint8_t> m;
        if (!f) return m;
        hnswgpu_info info;
        check(hnswgpu_get_info(h_, &info));
        std::vector<uint64_t> labels(info.count);
        if (info.count) check(hnswgpu_get_labels(h_, labels.data()));
        m.resize(info.count);
        for (size_t i = 0; i < labels.size(); i++) m[i] = (*f)((labeltype)labels[i]) ? 1 : 0;
        return m;
    }

    void batch(const float* queries, size_t nq, size_t k, labeltype* labels, float* dists, int32_t* counts,
               uint32_t filter) const {
        hnswgpu_search_opts o{};
        o.flags = flags_;
        o.filter = filter;
        static_assert(sizeof(labeltype) == sizeof(uint64_t), "labeltype must be 64-bit");
        check(hnswgpu_search(h_, queries, nq, k, &o, reinterpret_cast<uint64_t*>(labels), dists, counts));
    }

    std::priority_queue<std::pair<float, labeltype>> knn(const void* query, size_t k, uint32_t filter) const {
        std::vector<labeltype> l(k);
        std::vector<float> d(k);
        int32_t c = 0;
        batch(static_cast<const float*>(query), 1, k, l.data(), d.data(), &c, filter);
        std::priority_queue<std::pair<float, labeltype>> out;
        for (int32_t i = 0; i < c; i++) out.emplace(d[i], l[i]);
        return out;
    }

    static std::vector<std::pair<float, labeltype>> closer_first(std::priority_queue<std::pair<float, labeltype>> pq) {
        std::vector<std::pair<float, labeltype>> r(pq.size());
        size_t n = pq.size();
        while (!pq.empty()) {
            r[--n] = pq.top();
            pq.pop();
        }
        return r;
    }

 public:
    IndexBase() = default;
    IndexBase(const IndexBase&) = delete;
    IndexBase& operator=(const IndexBase&) = delete;
    virtual ~IndexBase() {
        if (h_) hnswgpu_free(h_);
    }

    // Batched search (an extension): nq queries, closest-first rows of k
    // labels / distances, counts[i] = results found (rest: UINT64_MAX / +inf).
    template <class F = BaseFilterFunctor>
    void searchKnnBatch(const float* queries, size_t nq, size_t k, labeltype* labels, float* dists,
                        int32_t* counts, F* f = nullptr) const {
        batch(queries, nq, k, labels, dists, counts, filter_id(f));
    }

    // Evaluate the functor again (its answers changed since its first use).
    template <class F>
    void refreshFilter(F* f) {
        forgetFilter(f);
        filter_id(f);
    }
    // Drop the functor's device mask (before the functor object is destroyed
    // and its address reused).
    template <class F>
    void forgetFilter(F* f) {
        auto it = filters_.find(static_cast<const void*>(f));
        if (it == filters_.end()) return;
        check(hnswgpu_filter_destroy(h_, it->second));
        filters_.erase(it);
    }

    size_t getCurrentElementCount() const {
        hnswgpu_info info;
        check(hnswgpu_get_info(h_, &info));
        return info.count;
    }
    size_t getMaxElements() const {
        hnswgpu_info info;
        check(hnswgpu_get_info(h_, &info));
        return info.max_elements;
    }
    hnswgpu_index* handle() const { return h_; }
};
}  // namespace detail

template <typename dist_t = float>
class HierarchicalNSW : public detail::IndexBase, public AlgorithmInterface<dist_t> {
    static_assert(sizeof(dist_t) == sizeof(float), "the GPU path computes float distances");

 public:
    // The public ef_ of the reference: reads and assignments go to the
    // index's ef (setEf / the ef the next searchKnn uses).
    class EfProxy {
        HierarchicalNSW* o_;

     public:
        explicit EfProxy(HierarchicalNSW* o) : o_(o) {}
        operator size_t() const { return o_->getEf(); }
        EfProxy& operator=(size_t ef) {
            o_->setEf(ef);
            return *this;
        }
    };
    EfProxy ef_{this};

    // HierarchicalNSW(SpaceInterface*, location, nmslib, max_elements,
    // allow_replace_deleted) -- loads a file written by saveIndex.
    HierarchicalNSW(const SpaceInterface* s, const std::string& location, bool nmslib = false,
                    size_t max_elements = 0, bool allow_replace_deleted = false, int device = 0) {
        (void)nmslib;
        (void)allow_replace_deleted;
        dim_ = s->dim();
        flags_ = HNSWGPU_EXACT_TIES;
        detail::check(hnswgpu_load_hnsw(location.c_str(), s->space_kind(), dim_, max_elements, device, &h_));
    }

    void setEf(size_t ef) { detail::check(hnswgpu_set_ef(h_, ef)); }

    // hnswlib's searchKnn: a max-heap of (distance, label), farthest on top.
    std::priority_queue<std::pair<dist_t, labeltype>> searchKnn(const void* query, size_t k,
                                                                BaseFilterFunctor* f = nullptr) const override {
        return knn(query, k, filter_id(f));
    }
    template <class F, class = typename std::enable_if<!std::is_base_of<BaseFilterFunctor, F>::value>::type>
    std::priority_queue<std::pair<dist_t, labeltype>> searchKnn(const void* query, size_t k, F* f) const {
        return knn(query, k, filter_id(f));
    }
    // AlgorithmInterface::searchKnnCloserFirst (hnswlib/hnswlib.h:203-221).
    std::vector<std::pair<dist_t, labeltype>> searchKnnCloserFirst(const void* query, size_t k,
                                                                   BaseFilterFunctor* f = nullptr) const override {
        return closer_first(knn(query, k, filter_id(f)));
    }
    template <class F, class = typename std::enable_if<!std::is_base_of<BaseFilterFunctor, F>::value>::type>
    std::vector<std::pair<dist_t, labeltype>> searchKnnCloserFirst(const void* query, size_t k, F* f) const {
        return closer_first(knn(query, k, filter_id(f)));
    }

    // saveIndex (hnswlib/hnswalg.h:685-712): the loaded file with the current
    // delete marks.
    void saveIndex(const std::string& location) override { detail::check(hnswgpu_save_hnsw(h_, location.c_str())); }

    // Index construction stays with hnswlib.
    void addPoint(const void*, labeltype, bool = false) override {
        throw std::runtime_error("addPoint is not supported on the GPU path: build the index with hnswlib");
    }

    // searchStopConditionClosest with an EpsilonSearchStopCondition
    // (hnswlib/hnswalg.h:1326-1377): the results within epsilon, closest
    // first, in the reference's order; like the reference, the second member
    // is the internal id.
    std::vector<std::pair<float, labeltype>> searchStopConditionClosest(const void* query,
                                                                        const EpsilonSearchStopCondition& sc,
                                                                        BaseFilterFunctor* f = nullptr) const {
        std::vector<uint8_t> m = mask(f);
        hnswgpu_search_opts o{};
        o.allow = f ? m.data() : nullptr;
        const size_t cap = sc.max_num_candidates();
        std::vector<uint64_t> ids(cap);
        std::vector<float> d(cap);
        int32_t c = 0;
        detail::check(hnswgpu_search_epsilon(h_, static_cast<const float*>(query), 1, sc.epsilon(),
                                             sc.min_num_candidates(), cap, &o, ids.data(), d.data(), &c));
        std::vector<std::pair<float, labeltype>> r((size_t)c);
        for (int32_t i = 0; i < c; i++) r[(size_t)i] = {d[(size_t)i], (labeltype)ids[(size_t)i]};
        return r;
    }
    size_t getEf() const {
        hnswgpu_info info;
        detail::check(hnswgpu_get_info(h_, &info));
        return info.ef;
    }
    // true (default): equal distances resolve exactly as hnswlib's heaps do;
    // false: ties break by internal id (faster, identical without ties).
    void setReferenceTieOrder(bool on) { flags_ = on ? HNSWGPU_EXACT_TIES : 0u; }

    void markDelete(labeltype label) { detail::check(hnswgpu_mark_deleted(h_, label)); }
    void unmarkDelete(labeltype label) { detail::check(hnswgpu_unmark_deleted(h_, label)); }
    size_t getDeletedCount() const {
        hnswgpu_info info;
        detail::check(hnswgpu_get_info(h_, &info));
        return info.num_deleted;
    }
};

template <typename dist_t = float>
class BruteforceSearch : public detail::IndexBase, public AlgorithmInterface<dist_t> {
    static_assert(sizeof(dist_t) == sizeof(float), "the GPU path computes float distances");

 public:
    // BruteforceSearch(SpaceInterface*, location) -- loads a file written by
    // BruteforceSearch::saveIndex.
    BruteforceSearch(const SpaceInterface* s, const std::string& location, int device = 0) {
        dim_ = s->dim();
        detail::check(hnswgpu_load_bf(location.c_str(), s->space_kind(), dim_, device, &h_));
    }

    std::priority_queue<std::pair<dist_t, labeltype>> searchKnn(const void* query, size_t k,
                                                                BaseFilterFunctor* f = nullptr) const override {
        return knn(query, k, filter_id(f));
    }
    template <class F, class = typename std::enable_if<!std::is_base_of<BaseFilterFunctor, F>::value>::type>
    std::priority_queue<std::pair<dist_t, labeltype>> searchKnn(const void* query, size_t k, F* f) const {
        return knn(query, k, filter_id(f));
    }
    std::vector<std::pair<dist_t, labeltype>> searchKnnCloserFirst(const void* query, size_t k,
                                                                   BaseFilterFunctor* f = nullptr) const override {
        return closer_first(knn(query, k, filter_id(f)));
    }
    template <class F, class = typename std::enable_if<!std::is_base_of<BaseFilterFunctor, F>::value>::type>
    std::vector<std::pair<dist_t, labeltype>> searchKnnCloserFirst(const void* query, size_t k, F* f) const {
        return closer_first(knn(query, k, filter_id(f)));
    }
    void saveIndex(const std::string&) override {
        throw std::runtime_error("saveIndex of a brute-force index: use the Python BFIndex.save_index");
    }
    void addPoint(const void*, labeltype, bool = false) override {
        throw std::runtime_error("addPoint is not supported on the GPU path: build the index with hnswlib");
    }
};

}  // namespace hnswgpu
