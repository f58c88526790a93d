// noalloc.cu -- a radix-sort entry point that allocates no device memory.
//
// hmg_radix_sort_u64 allocates its ping-pong buffers and per-tile counters on
// every call.  Some callers cannot do that: code that runs while another
// component owns the device allocator (a host application that reserves all
// device memory up front for its own pool, or a real-time loop in which a
// cudaMalloc, with its implicit device synchronisation, is not allowed).  For
// them, hmg_radix_sort_u64_noalloc sorts with scratch that lives in a fixed,
// file-scope device array of this library instead:
//
//   * capacity: NA_MAX_KEYS = 2^20 keys; larger n is rejected with
//     HMG_ERR_INVALID and nothing is touched;
//   * every GPU that loads the library holds the array (12 MB + 0.27 MB) until
//     the process exits;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it, so make that
//     first call before any stream capture on the device; the cached address is
//     not looked up again, so a cudaDeviceReset on that device ends the entry
//     point's use in this process;
//   * all calls share the one array: calls whose work overlaps on the GPU (two
//     streams, two host threads) race on it and corrupt each other's results --
//     order them on one stream or synchronise between them;
//   * the array keeps the previous call's contents; the counters that must start
//     at zero are cleared on the stream by each call;
//   * the call only enqueues work on `stream` and returns: it neither copies to
//     the host nor waits for the stream.  Every digit pass is launched; a pass
//     whose digit is the same for all keys (read on the device from the histogram
//     of all digits) skips its counting and scan and copies the keys through
//     unchanged, which is what the stable pass would produce.
// The sort is the same stable LSD radix sort as hmg_radix_sort_u64, with the same
// per-tile steps, and gives bit-identical results.
#include <mutex>

#include "hmg_internal.cuh"
#include "radix.cuh"
#include "../../include/hmg.h"

namespace hmg {

// histogram of all eight digits (util.cu)
__global__ void k_rs_hist_all(const uint64_t* keys, int n, unsigned* hist);

static constexpr int NA_MAX_KEYS = 1 << 20;
static constexpr int NA_TILE = RS_TILE;  // keys per tile of the radix steps
static constexpr int NA_MAX_TILES = NA_MAX_KEYS / NA_TILE;
static constexpr int NA_COUNTS = 256 * NA_MAX_TILES;

struct NoAllocScratch {
    uint64_t keys[NA_MAX_KEYS];
    uint32_t vals[NA_MAX_KEYS];
    unsigned counts[NA_COUNTS];  // per (digit, tile), scanned in place
    unsigned hist[8 * 256];
};

static __device__ __align__(256) NoAllocScratch g_sort_scratch;

// A pass is trivial when every key has the same digit: the histogram of all
// digits (of the input keys; any permutation of them has the same one) then holds
// n for the digit of the current first key.
__device__ __forceinline__ bool na_pass_trivial(const unsigned* hist, const uint64_t* keys, int n, int shift)
{
    const unsigned d = (unsigned)((keys[0] >> shift) & 255u);
    return hist[(shift >> 3) * 256 + d] == (unsigned)n;
}

__global__ void k_na_tile_hist(const uint64_t* keys, int n, int shift, int ntiles, unsigned* counts,
                               const unsigned* hist)
{
    if (na_pass_trivial(hist, keys, n, shift)) return;
    rs_tile_hist(keys, n, shift, ntiles, blockIdx.x, counts);
}

// stable scatter of the pass, or a plain copy of the tile when the pass is trivial
// (the stable order of equal digits is the input order)
__global__ void k_na_scatter(const uint64_t* kin, const uint32_t* vin, uint64_t* kout, uint32_t* vout, int n,
                             int shift, int ntiles, const unsigned* offsets, const unsigned* hist)
{
    if (na_pass_trivial(hist, kin, n, shift)) {
        const long long base = (long long)blockIdx.x * RS_TILE;
        for (int k = threadIdx.x; k < RS_TILE; k += blockDim.x) {
            const long long i = base + k;
            if (i < n) {
                kout[i] = kin[i];
                vout[i] = vin[i];
            }
        }
        return;
    }
    rs_scatter(kin, vin, kout, vout, n, shift, ntiles, blockIdx.x, offsets);
}

// exclusive scan of the (digit, tile) counts in place: one CTA, 1024 threads,
// each owning a contiguous run; nothing to do for a trivial pass
__global__ void __launch_bounds__(1024) k_na_scan(unsigned* a, int n, const uint64_t* keys, int nkeys,
                                                  int shift, const unsigned* hist)
{
    if (na_pass_trivial(hist, keys, nkeys, shift)) return;
    __shared__ unsigned warp_tot[32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int per = (n + 1023) / 1024;
    const int b = t * per, e = min(n, b + per);
    unsigned sum = 0;
    for (int i = b; i < e; i++) sum += a[i];
    unsigned x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned w = warp_tot[lane];
        for (int o = 1; o < 32; o <<= 1) {
            unsigned y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        warp_tot[lane] = w;
    }
    __syncthreads();
    unsigned run = (warp ? warp_tot[warp - 1] : 0u) + x - sum;
    for (int i = b; i < e; i++) {
        unsigned v = a[i];
        a[i] = run;
        run += v;
    }
}

static std::mutex g_na_mutex;
static NoAllocScratch* g_na_ptr[256];  // device address per device ordinal

static hmg_status scratch_for_current_device(NoAllocScratch** out)
{
    int dev = 0;
    HMG_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 256) {
        set_error("hmg_radix_sort_u64_noalloc: device ordinal %d out of range", dev);
        return HMG_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || !p) {
            set_error("hmg_radix_sort_u64_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return HMG_ERR_CUDA;
        }
        g_na_ptr[dev] = static_cast<NoAllocScratch*>(p);
    }
    *out = g_na_ptr[dev];
    return HMG_OK;
}

}  // namespace hmg

using namespace hmg;

extern "C" hmg_status hmg_radix_sort_u64_noalloc(uint64_t* keys, uint32_t* values, int n, int key_bits,
                                                 void* stream)
{
    if (n < 0 || n > NA_MAX_KEYS) {
        set_error("hmg_radix_sort_u64_noalloc: n=%d is outside [0, %d] (the fixed scratch capacity)", n,
                  NA_MAX_KEYS);
        return HMG_ERR_INVALID;
    }
    if (n > 0 && (!keys || !values)) {
        set_error("hmg_radix_sort_u64_noalloc: NULL argument");
        return HMG_ERR_INVALID;
    }
    NoAllocScratch* w = nullptr;
    hmg_status st = scratch_for_current_device(&w);
    if (st) return st;
    if (n <= 1) return HMG_OK;
    if (key_bits <= 0 || key_bits > 64) key_bits = 64;
    cudaStream_t s = (cudaStream_t)stream;
    const int ntiles = (n + NA_TILE - 1) / NA_TILE;
    HMG_CUDA_TRY(cudaMemsetAsync(w->hist, 0, sizeof(w->hist), s));
    const int hb = ntiles < 1184 ? ntiles : 1184;
    k_rs_hist_all<<<hb, RS_THREADS, 0, s>>>(keys, n, w->hist);
    HMG_LAUNCH_CHECK();
    uint64_t *ka = keys, *kb = w->keys;
    uint32_t *va = values, *vb = w->vals;
    const int npasses = (key_bits + 7) / 8;
    for (int p = 0; p < npasses; p++) {
        const int shift = 8 * p;
        k_na_tile_hist<<<ntiles, RS_THREADS, 0, s>>>(ka, n, shift, ntiles, w->counts, w->hist);
        HMG_LAUNCH_CHECK();
        k_na_scan<<<1, 1024, 0, s>>>(w->counts, 256 * ntiles, ka, n, shift, w->hist);
        HMG_LAUNCH_CHECK();
        k_na_scatter<<<ntiles, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, ntiles, w->counts, w->hist);
        HMG_LAUNCH_CHECK();
        uint64_t* tk = ka; ka = kb; kb = tk;
        uint32_t* tv = va; va = vb; vb = tv;
    }
    if (ka != keys) {
        HMG_CUDA_TRY(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(values, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
    return HMG_OK;
}
