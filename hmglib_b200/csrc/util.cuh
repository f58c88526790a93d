// util.cuh -- device-wide primitives used by setup and planning: exclusive scans
// and a stable LSD radix sort (64-bit keys, 32-bit values).
#pragma once

#include "hmg_internal.cuh"
#include "../../include/hmg.h"

namespace hmg {

// Stream-ordered device allocation helpers (cudaMallocAsync pool).
template <typename T>
hmg_status dalloc(T** p, size_t count, cudaStream_t s)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocAsync((void**)p, count * sizeof(T), s);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("device allocation of %zu bytes failed: %s", count * sizeof(T),
                  cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? HMG_ERR_NOMEM : HMG_ERR_CUDA;
    }
    return HMG_OK;
}

template <typename T>
void dfree(T*& p, cudaStream_t s)
{
    if (p) cudaFreeAsync((void*)p, s);
    p = nullptr;
}

// out[i] = sum_{k<i} in[k]; optionally *total_dev = sum of all (device pointer).
// T = int or long long.  in and out may alias.
template <typename T>
hmg_status scan_exclusive(const T* in, T* out, long long n, T* total_dev, cudaStream_t s);

// Stable LSD radix sort, 8-bit digits, in place (uses n-sized temporaries).
hmg_status radix_sort_pairs(uint64_t* keys, uint32_t* vals, int n, int key_bits,
                            cudaStream_t s);

}  // namespace hmg
