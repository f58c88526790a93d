// util.cu -- device-wide exclusive scan and stable LSD radix sort.
//
// The radix sort replaces thrust::sort_by_key over (Morton code, index)
// (helper.cu:140-167).  Each 8-bit pass runs three kernels: per-tile digit
// histograms, one exclusive scan of the (digit, tile) counts in digit-major order,
// and a stable scatter in which every warp ranks its keys with __match_any_sync.
// Passes whose digit is identical for every key are skipped (decided from one
// up-front histogram of all eight digits), which is exact and removes the top
// pass of 3D codes (60 significant bits).
#include <cstdarg>

#include "radix.cuh"
#include "util.cuh"

namespace hmg {

// ---------------------------------------------------------------------------
// exclusive scan: reduce per 2048-element block, scan the block sums
// (recursively), then rescan each block with its offset.
// ---------------------------------------------------------------------------
static constexpr int SCAN_THREADS = 256;
static constexpr int SCAN_ITEMS = 8;
static constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem_warp, T* total)
{
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < (SCAN_THREADS / 32) ? smem_warp[lane] : T(0);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < (SCAN_THREADS / 32)) smem_warp[lane] = w;
    }
    __syncthreads();
    T warp_prefix = warp > 0 ? smem_warp[warp - 1] : T(0);
    if (total) *total = smem_warp[SCAN_THREADS / 32 - 1];
    return warp_prefix + x - v;
}

template <typename T>
__global__ void k_scan_reduce(const T* in, long long n, T* sums)
{
    __shared__ T sw[SCAN_THREADS / 32];
    long long base = (long long)blockIdx.x * SCAN_TILE;
    T acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + (long long)k * SCAN_THREADS + threadIdx.x;
        if (i < n) acc += in[i];
    }
    T tot;
    block_exclusive_scan<T>(acc, sw, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <typename T>
__global__ void k_scan_apply(const T* in, T* out, long long n, const T* offsets, T* total_dev,
                             long long nblocks_total)
{
    __shared__ T sw[SCAN_THREADS / 32];
    long long base = (long long)blockIdx.x * SCAN_TILE;
    T v[SCAN_ITEMS];
    T acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        v[k] = i < n ? in[i] : T(0);
        acc += v[k];
    }
    T tot;
    T pre = block_exclusive_scan<T>(acc, sw, &tot);
    T off = offsets ? offsets[blockIdx.x] : T(0);
    T run = off + pre;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (total_dev && blockIdx.x == nblocks_total - 1 && threadIdx.x == SCAN_THREADS - 1)
        *total_dev = run;
}

template <typename T>
hmg_status scan_exclusive(const T* in, T* out, long long n, T* total_dev, cudaStream_t s)
{
    if (n <= 0) {
        if (total_dev) HMG_CUDA_TRY(cudaMemsetAsync(total_dev, 0, sizeof(T), s));
        return HMG_OK;
    }
    long long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 1) {
        k_scan_apply<T><<<1, SCAN_THREADS, 0, s>>>(in, out, n, nullptr, total_dev, 1);
        HMG_LAUNCH_CHECK();
        return HMG_OK;
    }
    T* sums = nullptr;
    hmg_status st = dalloc(&sums, (size_t)nb, s);
    if (st) return st;
    k_scan_reduce<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, sums);
    HMG_LAUNCH_CHECK();
    st = scan_exclusive<T>(sums, sums, nb, nullptr, s);
    if (st) { dfree(sums, s); return st; }
    k_scan_apply<T><<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, out, n, sums, total_dev, nb);
    HMG_LAUNCH_CHECK();
    dfree(sums, s);
    return HMG_OK;
}

template hmg_status scan_exclusive<int>(const int*, int*, long long, int*, cudaStream_t);
template hmg_status scan_exclusive<long long>(const long long*, long long*, long long,
                                              long long*, cudaStream_t);

// ---------------------------------------------------------------------------
// radix sort
// ---------------------------------------------------------------------------
// histogram of all eight 8-bit digits over all keys
__global__ void k_rs_hist_all(const uint64_t* keys, int n, unsigned* hist /* [8][256] */)
{
    __shared__ unsigned h[8][256];
    for (int t = threadIdx.x; t < 8 * 256; t += blockDim.x) (&h[0][0])[t] = 0;
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        uint64_t k = keys[i];
#pragma unroll
        for (int p = 0; p < 8; p++) atomicAdd(&h[p][(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 8 * 256; t += blockDim.x) {
        unsigned v = (&h[0][0])[t];
        if (v) atomicAdd(&hist[t], v);
    }
}

// per-tile counts, stored digit-major: counts[digit * ntiles + tile]
__global__ void k_rs_tile_hist(const uint64_t* keys, int n, int shift, int ntiles,
                               unsigned* counts)
{
    rs_tile_hist(keys, n, shift, ntiles, blockIdx.x, counts);
}

__global__ void k_rs_scatter(const uint64_t* kin, const uint32_t* vin, uint64_t* kout,
                             uint32_t* vout, int n, int shift, int ntiles,
                             const unsigned* offsets /* scanned counts */)
{
    rs_scatter(kin, vin, kout, vout, n, shift, ntiles, blockIdx.x, offsets);
}

hmg_status radix_sort_pairs(uint64_t* keys, uint32_t* vals, int n, int key_bits,
                            cudaStream_t s)
{
    if (n <= 1) return HMG_OK;
    if (key_bits <= 0 || key_bits > 64) key_bits = 64;
    int ntiles = (n + RS_TILE - 1) / RS_TILE;
    unsigned *hist = nullptr, *counts = nullptr;
    uint64_t* k2 = nullptr;
    uint32_t* v2 = nullptr;
    hmg_status st;
    if ((st = dalloc(&hist, 8 * 256, s))) return st;
    if ((st = dalloc(&counts, (size_t)256 * ntiles, s))) { dfree(hist, s); return st; }
    if ((st = dalloc(&k2, (size_t)n, s)) || (st = dalloc(&v2, (size_t)n, s))) {
        dfree(hist, s); dfree(counts, s); dfree(k2, s); return st;
    }
    HMG_CUDA_TRY(cudaMemsetAsync(hist, 0, 8 * 256 * sizeof(unsigned), s));
    int hb = ntiles < 1184 ? ntiles : 1184;
    k_rs_hist_all<<<hb, 256, 0, s>>>(keys, n, hist);
    HMG_LAUNCH_CHECK();
    unsigned h_hist[8 * 256];
    HMG_CUDA_TRY(cudaMemcpyAsync(h_hist, hist, sizeof(h_hist), cudaMemcpyDeviceToHost, s));
    HMG_CUDA_TRY(cudaStreamSynchronize(s));
    uint64_t *ka = keys, *kb = k2;
    uint32_t *va = vals, *vb = v2;
    int npasses = (key_bits + 7) / 8;
    for (int p = 0; p < npasses; p++) {
        bool trivial = false;
        for (int d = 0; d < 256; d++)
            if (h_hist[p * 256 + d] == (unsigned)n) trivial = true;
        if (trivial) continue;
        int shift = 8 * p;
        k_rs_tile_hist<<<ntiles, RS_THREADS, 0, s>>>(ka, n, shift, ntiles, counts);
        HMG_LAUNCH_CHECK();
        st = scan_exclusive<int>((const int*)counts, (int*)counts, (long long)256 * ntiles,
                                 nullptr, s);
        if (st) break;
        k_rs_scatter<<<ntiles, RS_THREADS, 0, s>>>(ka, va, kb, vb, n, shift, ntiles, counts);
        HMG_LAUNCH_CHECK();
        uint64_t* tk = ka; ka = kb; kb = tk;
        uint32_t* tv = va; va = vb; vb = tv;
    }
    if (!st && ka != keys) {
        HMG_CUDA_TRY(cudaMemcpyAsync(keys, ka, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, s));
        HMG_CUDA_TRY(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, s));
    }
    dfree(hist, s); dfree(counts, s); dfree(k2, s); dfree(v2, s);
    return st;
}

// ---------------------------------------------------------------------------
// error recording
// ---------------------------------------------------------------------------
static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char* last_error() { return g_err; }

}  // namespace hmg
