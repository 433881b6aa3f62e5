// Per-device cache of a kernel's launch set-up: the opt-in dynamic shared
// memory already granted (cudaFuncSetAttribute applies to the current
// device's context) and the resident CTAs per SM for the last block size and
// shared-memory size asked.  One cache per kernel instantiation; safe to use from several
// host threads and with indexes on several devices in one process.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>

namespace hnswgpu {

class LaunchCache {
public:
    static constexpr int kMaxDevices = 64;

    LaunchCache() {
        for (int d = 0; d < kMaxDevices; d++) {
            attr_[d] = -1;
            occ_smem_[d] = 0;
            occ_threads_[d] = 0;
            occ_blocks_[d] = -1;
        }
    }

    // Resident CTAs per SM of `fn` launched with `threads` threads and `smem`
    // bytes of dynamic shared memory on the current device, granting the
    // opt-in first when needed.
    cudaError_t blocks_per_sm(const void* fn, int threads, size_t smem, int* out) {
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        if (dev < 0 || dev >= kMaxDevices) return query(fn, threads, smem, out);
        std::lock_guard<std::mutex> g(mu_);
        if ((int)smem > attr_[dev]) {
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            attr_[dev] = (int)smem;
        }
        if (occ_blocks_[dev] < 0 || occ_smem_[dev] != smem || occ_threads_[dev] != threads) {
            int b = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, threads, smem);
            if (e != cudaSuccess) return e;
            occ_smem_[dev] = smem;
            occ_threads_[dev] = threads;
            occ_blocks_[dev] = b;
        }
        *out = occ_blocks_[dev];
        return cudaSuccess;
    }

private:
    static cudaError_t query(const void* fn, int threads, size_t smem, int* out) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, fn, threads, smem);
    }

    std::mutex mu_;
    int attr_[kMaxDevices];
    size_t occ_smem_[kMaxDevices];
    int occ_threads_[kMaxDevices];
    int occ_blocks_[kMaxDevices];
};

}  // namespace hnswgpu
