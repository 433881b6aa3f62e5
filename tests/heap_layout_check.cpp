// Compares the tie-exact heap routines (hnsw_rabitq_b200/csrc/ref_heap.h)
// with std::push_heap / std::pop_heap on random operation sequences whose
// keys tie often.  Prints "ok" or the first mismatch; exit status 0 on ok.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "ref_heap.h"

using hnswgpu::CandLess;
using hnswgpu::TopLess;

struct PairTop {  // CompareByFirst on (distance, id), as the reference
    bool operator()(const std::pair<float, uint32_t>& a, const std::pair<float, uint32_t>& b) const {
        return a.first < b.first;
    }
};

static uint64_t enc(float d, uint32_t id) {
    uint32_t u;
    std::memcpy(&u, &d, 4);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((uint64_t)u << 32) | id;
}

template <class Less>
static int run(bool cand, unsigned seed) {
    std::mt19937 rng(seed);
    std::vector<std::pair<float, uint32_t>> ref;
    std::vector<uint64_t> mine(4096);
    int n = 0;
    Less less;
    for (int step = 0; step < 8000; step++) {
        bool push = ref.empty() || (rng() % 100) < 55 || n > 4000;
        if (n > 4000) push = false;
        if (push) {
            float d = (float)(rng() % 9);  // heavy ties
            uint32_t id = rng() % 100000;
            ref.push_back({cand ? -d : d, id});
            std::push_heap(ref.begin(), ref.end(), PairTop());
            hnswgpu::ref_heap_push(mine.data(), n, enc(d, id), less);
        } else {
            std::pop_heap(ref.begin(), ref.end(), PairTop());
            auto gone = ref.back();
            ref.pop_back();
            uint64_t g = hnswgpu::ref_heap_pop(mine.data(), n, less);
            if ((uint32_t)g != gone.second) {
                std::printf("pop mismatch at step %d\n", step);
                return 1;
            }
        }
        if ((int)ref.size() != n) return 1;
        for (int i = 0; i < n; i++)
            if ((uint32_t)mine[i] != ref[i].second) {
                std::printf("layout mismatch at step %d index %d\n", step, i);
                return 1;
            }
    }
    return 0;
}

int main() {
    for (unsigned s = 1; s <= 6; s++) {
        if (run<TopLess>(false, s) || run<CandLess>(true, s)) return 1;
    }
    std::printf("ok\n");
    return 0;
}
