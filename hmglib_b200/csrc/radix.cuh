// radix.cuh -- the per-tile steps of the stable LSD radix sort (8-bit digits), as
// device functions shared by the allocating sort (util.cu) and the sort that
// allocates nothing (noalloc.cu).  A tile is RS_TILE consecutive keys handled by one
// CTA of RS_THREADS threads.
#pragma once

#include <stdint.h>

namespace hmg {

static constexpr int RS_THREADS = 256;                 // 8 warps
static constexpr int RS_ITEMS = 16;                    // items per lane
static constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 4096 keys per tile
static constexpr int RS_WARP_SPAN = 32 * RS_ITEMS;     // contiguous keys per warp

// digit counts of tile `tile`, stored digit-major: counts[digit * ntiles + tile]
__device__ __forceinline__ void rs_tile_hist(const uint64_t* keys, int n, int shift, int ntiles, int tile,
                                             unsigned* counts)
{
    __shared__ unsigned h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    long long base = (long long)tile * RS_TILE;
#pragma unroll 4
    for (int k = 0; k < RS_ITEMS; k++) {
        long long i = base + (long long)k * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    counts[(size_t)threadIdx.x * ntiles + tile] = h[threadIdx.x];
}

// stable scatter of tile `tile` to the scanned (digit, tile) offsets; every warp
// ranks its keys with __match_any_sync
__device__ __forceinline__ void rs_scatter(const uint64_t* kin, const uint32_t* vin, uint64_t* kout,
                                           uint32_t* vout, int n, int shift, int ntiles, int tile,
                                           const unsigned* offsets)
{
    __shared__ unsigned wcount[8][256];
    __shared__ unsigned wbase[8][256];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int t = lane; t < 256; t += 32) wcount[warp][t] = 0;
    __syncwarp();
    long long wstart = (long long)tile * RS_TILE + (long long)warp * RS_WARP_SPAN;
    uint64_t key[RS_ITEMS];
    uint32_t val[RS_ITEMS];
    unsigned rank[RS_ITEMS];
    unsigned lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int it = 0; it < RS_ITEMS; it++) {
        long long i = wstart + it * 32 + lane;
        bool valid = i < n;
        key[it] = valid ? kin[i] : 0;
        val[it] = valid ? vin[i] : 0;
        unsigned digit = valid ? (unsigned)((key[it] >> shift) & 255u) : 256u;
        unsigned peers = __match_any_sync(0xffffffffu, digit);
        unsigned before = __popc(peers & lt_mask);
        unsigned cnt = __popc(peers);
        unsigned basecnt = valid ? wcount[warp][digit] : 0u;
        rank[it] = basecnt + before;
        __syncwarp();
        if (valid && before == 0) wcount[warp][digit] = basecnt + cnt;
        __syncwarp();
    }
    __syncthreads();
    {
        int d = threadIdx.x;  // 256 threads, one digit each
        unsigned run = offsets[(size_t)d * ntiles + tile];
#pragma unroll
        for (int w = 0; w < 8; w++) {
            wbase[w][d] = run;
            run += wcount[w][d];
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < RS_ITEMS; it++) {
        long long i = wstart + it * 32 + lane;
        if (i < n) {
            unsigned digit = (unsigned)((key[it] >> shift) & 255u);
            unsigned pos = wbase[warp][digit] + rank[it];
            kout[pos] = key[it];
            vout[pos] = val[it];
        }
    }
}

}  // namespace hmg
