// Binary heaps with exactly the element layout of the reference's
// std::priority_queue (libstdc++: push_heap sifts the new element up while
// its parent compares lower; pop_heap moves the last element out, walks the
// hole from the root to a leaf along the higher child -- the right child wins
// ties -- and sifts the moved element back up from there).  With equal keys
// the order in which entries leave the heap depends on this layout, so the
// tie-exact search mode replays the reference's two heaps
// (hnswlib/hnswalg.h:321-322, CompareByFirst at :165-170) operation by
// operation.  Usable from host code for testing.
#pragma once
#include <cstdint>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#endif

namespace hnswgpu {

// Entries are (distance key << 32 | id); only the distance key is compared,
// as CompareByFirst compares only .first.
// top_candidates: max-heap on distance.
struct TopLess {
    __host__ __device__ __forceinline__ bool operator()(uint64_t a, uint64_t b) const {
        return (uint32_t)(a >> 32) < (uint32_t)(b >> 32);
    }
};
// candidate_set stores (-distance, id) under the same comparator, i.e. the
// entry with the smaller distance has the higher priority.
struct CandLess {
    __host__ __device__ __forceinline__ bool operator()(uint64_t a, uint64_t b) const {
        return (uint32_t)(a >> 32) > (uint32_t)(b >> 32);
    }
};

// `A` is a pointer or any type whose operator[] returns a uint64_t& (the
// search keeps the top levels of its candidate heap in shared memory and
// the deeper ones in a global spill area).
template <class A, class Less>
__host__ __device__ __forceinline__ void ref_heap_push(A h, int& n, uint64_t v, Less less) {
    int hole = n++;
    while (hole > 0) {
        int parent = (hole - 1) / 2;
        if (!less(h[parent], v)) break;
        h[hole] = h[parent];
        hole = parent;
    }
    h[hole] = v;
}

// Removes and returns the top entry (n >= 1).
template <class A, class Less>
__host__ __device__ __forceinline__ uint64_t ref_heap_pop(A h, int& n, Less less) {
    const uint64_t top = h[0];
    const int len = n - 1;
    if (len > 0) {
        const uint64_t v = h[len];
        int hole = 0, child = 0;
        while (child < (len - 1) / 2) {
            child = 2 * (child + 1);
            if (less(h[child], h[child - 1])) child--;
            h[hole] = h[child];
            hole = child;
        }
        if ((len & 1) == 0 && child == (len - 2) / 2) {
            child = 2 * (child + 1);
            h[hole] = h[child - 1];
            hole = child - 1;
        }
        while (hole > 0) {
            int parent = (hole - 1) / 2;
            if (!less(h[parent], v)) break;
            h[hole] = h[parent];
            hole = parent;
        }
        h[hole] = v;
    }
    n = len;
    return top;
}

// Heap storage split between a shared-memory head (entries [0, cap_s)) and a
// global-memory tail (entries [cap_s, cap_s + cap_g)).
struct SplitHeap {
    uint64_t* s;
    uint64_t* g;
    int cap_s;
    __host__ __device__ __forceinline__ uint64_t& operator[](int i) const { return i < cap_s ? s[i] : g[i - cap_s]; }
};

}  // namespace hnswgpu
