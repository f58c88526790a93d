// stream.cu -- the H-matvec's two streaming kernels with bulk asynchronous copies.
//
// Both kernels are persistent (one CTA per SM, 8 consumer warps + 1 producer
// warp).  The producer lane walks the CTA's work list and streams every stored
// slice into a ring of shared-memory stages with cp.async.bulk (1-D, 16-byte
// aligned), together with the matching piece of the multiplied vector; consumer
// warps reduce out of shared memory.  The ring keeps ~200 KB per SM in flight,
// which is what HBM3e needs at full bandwidth, independent of how short the
// individual slices are.  Products are accumulated in FP64 from FP32 or FP64
// storage; every reduction has a fixed owner and order, so results are
// deterministic.
//
//   k_tiles_bulk  y(tile) = sum over the tile's pairs of slice * vector
//                 (dense slices with x, U slices with t = V^T x)
//   k_vtx_bulk    t_b = V_b^T x_b for every admissible block
#include <algorithm>
#include <vector>

#include "hmg_matrix.cuh"
#include "pipeline.cuh"
#include "stream.cuh"

namespace hmg {

static constexpr int NCW = 8;                    // consumer warps
static constexpr int NTH = (NCW + 1) * 32;       // + one producer warp
static constexpr int STAGES = 6;
static constexpr int STAGE_BYTES = 32768;
static constexpr int K2_MAXCOLS = 256;           // columns per stage (vector piece)
static constexpr int K2_WBYTES = K2_MAXCOLS * 8 + 48;
static constexpr int K1_CW_F = 1024;             // V^T row piece (float), elements
static constexpr int K1_CW_D = 512;              // (double)
static constexpr int K1_WBYTES = 4096 + 64;

enum { ST_DATA = 0, ST_END = 1, ST_DONE = 2 };

struct StageMeta {
    int kind;
    int unit;   // tile (K2) or block (K1)
    int nc;     // columns in the stage (K2) / row piece length (K1)
    int sp;     // padded tile rows (K2) / V^T row stride (K1)
    int woff;   // first element of the vector piece in the stage's vector buffer
    int last;   // last stage of a pair (K2) / last column piece of these rows (K1)
    int s;      // tile rows (K2) / first row (K1)
    int r0;     // first Z row of the tile (K2) / rows in the stage (K1)
    long long ro;  // (K1) offset of the block's t_b
};

__device__ __forceinline__ PairDesc shfl_desc(const PairDesc& d, int k)
{
    PairDesc o;
    o.data = reinterpret_cast<const void*>(
        __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(d.data), k));
    o.w = reinterpret_cast<const void*>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(d.w), k));
    o.ncol = __shfl_sync(0xffffffffu, d.ncol, k);
    o.kind = __shfl_sync(0xffffffffu, d.kind, k);
    o.c0 = 0;
    o.pad = 0;
    return o;
}

template <typename T>
__device__ __forceinline__ void load4(const T* p, double* v);
template <>
__device__ __forceinline__ void load4<float>(const float* p, double* v)
{
    float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
template <>
__device__ __forceinline__ void load4<double>(const double* p, double* v)
{
    double2 a = *reinterpret_cast<const double2*>(p);
    double2 b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// Producer-side stage acquisition: the k-th use of a stage waits for the consumers'
// release of use k-1 (parity trick: the first use passes immediately).
struct Ring {
    long long it = 0;
    __device__ __forceinline__ int acquire(uint64_t* empty, int* err)
    {
        int s = (int)(it % STAGES);
        unsigned par = (unsigned)(((it / STAGES) & 1) ^ 1);
        if (!mbar_wait(&empty[s], par, err, 1)) return -1;
        return s;
    }
};

// On a timed-out wait the producer still waits (bounded) for the copies it issued.
__device__ void drain(uint64_t* full, long long it, int* err)
{
    for (long long j = it - STAGES; j < it; j++) {
        if (j < 0) continue;
        mbar_wait(&full[j % STAGES], (unsigned)((j / STAGES) & 1), err, 3);
    }
}

// ---------------------------------------------------------------------------
// K2: row tiles
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NTH, 1)
k_tiles_bulk(const PairDesc* __restrict__ desc, const int* __restrict__ tile_pair_start,
             const int* __restrict__ tile_r0, const int* __restrict__ tile_s, int ntiles,
             const int* __restrict__ perm1, double* __restrict__ y, int* err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* data = smem;
    unsigned char* wbuf = data + STAGES * STAGE_BYTES;
    StageMeta* meta = reinterpret_cast<StageMeta*>(wbuf + STAGES * K2_WBYTES);
    uint64_t* full = reinterpret_cast<uint64_t*>(meta + STAGES);
    uint64_t* empty = full + STAGES;
    double* red = reinterpret_cast<double*>(empty + STAGES);  // [NCW][128]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == NCW) {
        // The whole producer warp fetches descriptors (32 at a time, the next batch
        // while the current one is issued) and the next tile index; lane 0 alone
        // arms the barriers and issues the copies.
        Ring ring;
        int t = lane == 0 ? atomicAdd(err + 1, 1) : 0;
        t = __shfl_sync(0xffffffffu, t, 0);
        while (t < ntiles) {
            int tn = lane == 0 ? atomicAdd(err + 1, 1) : 0;  // tiles are handed out dynamically
            const int s_rows = tile_s[t], sp = (s_rows + 3) & ~3, tr0 = tile_r0[t];
            const int colbytes = sp * (int)sizeof(T);
            const int cpc = min(K2_MAXCOLS, STAGE_BYTES / colbytes);
            const int pb = tile_pair_start[t], pe = tile_pair_start[t + 1];
            PairDesc cur = pb + lane < pe ? desc[pb + lane] : PairDesc{};
            for (int p0 = pb; p0 < pe; p0 += 32) {
                PairDesc nxt = p0 + 32 + lane < pe ? desc[p0 + 32 + lane] : PairDesc{};
                const int n = min(32, pe - p0);
                for (int k = 0; k < n; k++) {
                    const PairDesc d = shfl_desc(cur, k);
                    for (int c0 = 0; c0 < d.ncol; c0 += cpc) {
                        const int nc = min(cpc, d.ncol - c0);
                        int ok = 1;
                        if (lane == 0) {
                            const int s = ring.acquire(empty, err);
                            if (s < 0) {
                                ok = 0;
                            } else {
                                const uintptr_t a = reinterpret_cast<uintptr_t>(static_cast<const T*>(d.w) + c0);
                                const uintptr_t a16 = a & ~(uintptr_t)15;
                                const unsigned woffb = (unsigned)(a - a16);
                                const unsigned wbytes = (woffb + nc * (unsigned)sizeof(T) + 15u) & ~15u;
                                StageMeta m;
                                m.kind = ST_DATA; m.unit = t; m.nc = nc; m.sp = sp;
                                m.woff = (int)(woffb / sizeof(T)); m.last = (c0 + nc >= d.ncol);
                                m.s = s_rows; m.r0 = tr0; m.ro = 0;
                                meta[s] = m;
                                const unsigned dbytes = (unsigned)(nc * colbytes);
                                mbar_arrive_expect_tx(&full[s], dbytes + wbytes);
                                bulk_g2s(data + (size_t)s * STAGE_BYTES,
                                         static_cast<const char*>(d.data) + (size_t)c0 * colbytes, dbytes, &full[s]);
                                bulk_g2s(wbuf + (size_t)s * K2_WBYTES, reinterpret_cast<const void*>(a16), wbytes,
                                         &full[s]);
                            }
                        }
                        ok = __shfl_sync(0xffffffffu, ok, 0);
                        if (!ok) {
                            if (lane == 0) drain(full, ring.it, err);
                            return;
                        }
                        ring.it++;
                    }
                }
                cur = nxt;
            }
            int ok = 1;
            if (lane == 0) {
                const int s = ring.acquire(empty, err);
                if (s < 0) {
                    ok = 0;
                } else {
                    StageMeta m;
                    m.kind = ST_END; m.unit = t; m.nc = 0; m.sp = sp; m.woff = 0; m.last = 0;
                    m.s = s_rows; m.r0 = tr0; m.ro = 0;
                    meta[s] = m;
                    mbar_arrive(&full[s]);
                }
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) {
                if (lane == 0) drain(full, ring.it, err);
                return;
            }
            ring.it++;
            t = __shfl_sync(0xffffffffu, tn, 0);
        }
        if (lane == 0) {
            const int s = ring.acquire(empty, err);
            if (s < 0) { drain(full, ring.it, err); return; }
            meta[s].kind = ST_DONE;
            mbar_arrive(&full[s]);
        }
        return;
    }

    // consumers: lane owns padded rows 4*lane .. 4*lane+3 of the tile; a warp takes
    // columns warp, warp+8, ... of each stage, two at a time (independent chains)
    const int row0 = lane * 4;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    double part[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long it = 0;; it++) {
        const int s = (int)(it % STAGES);
        if (!mbar_wait(&full[s], (unsigned)((it / STAGES) & 1), err, 2)) break;
        const StageMeta m = meta[s];
        if (m.kind == ST_DONE) break;
        if (m.kind == ST_END) {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                red[warp * 128 + row0 + q] = acc[q];
                acc[q] = 0.0;
            }
            consumers_sync(NCW * 32);
            for (int i = threadIdx.x; i < m.s; i += NCW * 32) {
                double v = 0.0;
#pragma unroll
                for (int w = 0; w < NCW; w++) v += red[w * 128 + i];
                y[perm1[m.r0 + i]] = v;
            }
            consumers_sync(NCW * 32);
        } else {
            const T* buf = reinterpret_cast<const T*>(data + (size_t)s * STAGE_BYTES);
            const T* w = reinterpret_cast<const T*>(wbuf + (size_t)s * K2_WBYTES) + m.woff;
            if (row0 < m.sp) {
                double p2[4] = {0.0, 0.0, 0.0, 0.0};
                int j = warp;
                for (; j + NCW < m.nc; j += 2 * NCW) {
                    double v[4], u[4];
                    load4<T>(buf + (size_t)j * m.sp + row0, v);
                    load4<T>(buf + (size_t)(j + NCW) * m.sp + row0, u);
                    const double wj = (double)w[j], wk = (double)w[j + NCW];
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        part[q] = fma(v[q], wj, part[q]);
                        p2[q] = fma(u[q], wk, p2[q]);
                    }
                }
                if (j < m.nc) {
                    double v[4];
                    load4<T>(buf + (size_t)j * m.sp + row0, v);
                    const double wj = (double)w[j];
#pragma unroll
                    for (int q = 0; q < 4; q++) part[q] = fma(v[q], wj, part[q]);
                }
#pragma unroll
                for (int q = 0; q < 4; q++) part[q] += p2[q];
            }
            if (m.last) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    acc[q] += part[q];
                    part[q] = 0.0;
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// ---------------------------------------------------------------------------
// K1: t_b = V_b^T x_b
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(NTH, 1)
k_vtx_bulk(const int* __restrict__ blocks, int nblocks, const int* __restrict__ blk_c0,
           const int* __restrict__ blk_m2, const int* __restrict__ rank,
           const long long* __restrict__ rank_off, T* const* __restrict__ ptrV,
           const T* __restrict__ xs, T* __restrict__ tbuf, int* err)
{
    constexpr int CW = sizeof(T) == 4 ? K1_CW_F : K1_CW_D;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char* data = smem;
    unsigned char* wbuf = data + STAGES * STAGE_BYTES;
    StageMeta* meta = reinterpret_cast<StageMeta*>(wbuf + STAGES * K1_WBYTES);
    uint64_t* full = reinterpret_cast<uint64_t*>(meta + STAGES);
    uint64_t* empty = full + STAGES;
    double* rowacc = reinterpret_cast<double*>(empty + STAGES);  // [K1_MAXRANK]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NCW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = threadIdx.x; i < K1_MAXRANK; i += blockDim.x) rowacc[i] = 0.0;
    __syncthreads();

    if (warp == NCW) {
        // Blocks are handed out 32 at a time (err[2], zeroed before launch; coarse
        // levels come first in the list).  The producer warp loads the 32 blocks'
        // geometry in one go and the next chunk index ahead of time; lane 0 issues.
        Ring ring;
        int base = lane == 0 ? atomicAdd(err + 2, 32) : 0;
        base = __shfl_sync(0xffffffffu, base, 0);
        while (base < nblocks) {
            int nbase = lane == 0 ? atomicAdd(err + 2, 32) : 0;
            int mb = -1, mr = 0, mm2 = 0, mc0 = 0;
            long long mro = 0;
            unsigned long long mV = 0;
            if (base + lane < nblocks) {
                mb = blocks[base + lane];
                mr = rank[mb];
                mm2 = blk_m2[mb];
                mc0 = blk_c0[mb];
                mro = rank_off[mb];
                mV = reinterpret_cast<unsigned long long>(ptrV[mb]);
            }
            const int n = min(32, nblocks - base);
            for (int k = 0; k < n; k++) {
                const int b = __shfl_sync(0xffffffffu, mb, k);
                const int r = __shfl_sync(0xffffffffu, mr, k);
                const int m2 = __shfl_sync(0xffffffffu, mm2, k);
                const int c0 = __shfl_sync(0xffffffffu, mc0, k);
                const long long ro = __shfl_sync(0xffffffffu, mro, k);
                const T* V = reinterpret_cast<const T*>(__shfl_sync(0xffffffffu, mV, k));
                const int m2p = (m2 + 3) & ~3;
                const bool whole = m2p <= CW;
                const int cw = whole ? m2p : CW;
                // rows per stage: whole rows when they are short, else 8 pieces of CW
                const int rps = whole ? max(1, min(r, STAGE_BYTES / (m2p * (int)sizeof(T)))) : 8;
                for (int l0 = 0; l0 < r; l0 += rps) {
                    const int nr = min(rps, r - l0);
                    for (int j0 = 0; j0 < m2p; j0 += cw) {
                        const int nc = min(cw, m2p - j0);
                        int ok = 1;
                        if (lane == 0) {
                            const int s = ring.acquire(empty, err);
                            if (s < 0) {
                                ok = 0;
                            } else {
                                const uintptr_t a = reinterpret_cast<uintptr_t>(xs + c0 + j0);
                                const uintptr_t a16 = a & ~(uintptr_t)15;
                                const unsigned woffb = (unsigned)(a - a16);
                                const unsigned wbytes = (woffb + nc * (unsigned)sizeof(T) + 15u) & ~15u;
                                StageMeta m;
                                m.kind = ST_DATA; m.unit = b; m.nc = nc; m.sp = whole ? m2p : nc;
                                m.woff = (int)(woffb / sizeof(T)); m.last = (j0 + nc >= m2p);
                                m.s = l0; m.r0 = nr; m.ro = ro;
                                meta[s] = m;
                                const unsigned rowbytes = (unsigned)(nc * sizeof(T));
                                mbar_arrive_expect_tx(&full[s], rowbytes * nr + wbytes);
                                unsigned char* dst = data + (size_t)s * STAGE_BYTES;
                                if (whole) {
                                    bulk_g2s(dst, V + (size_t)l0 * m2p, rowbytes * nr, &full[s]);
                                } else {
                                    for (int i = 0; i < nr; i++)
                                        bulk_g2s(dst + (size_t)i * rowbytes, V + (size_t)(l0 + i) * m2p + j0, rowbytes,
                                                 &full[s]);
                                }
                                bulk_g2s(wbuf + (size_t)s * K1_WBYTES, reinterpret_cast<const void*>(a16), wbytes,
                                         &full[s]);
                            }
                        }
                        ok = __shfl_sync(0xffffffffu, ok, 0);
                        if (!ok) {
                            if (lane == 0) drain(full, ring.it, err);
                            return;
                        }
                        ring.it++;
                    }
                }
            }
            base = __shfl_sync(0xffffffffu, nbase, 0);
        }
        if (lane == 0) {
            const int s = ring.acquire(empty, err);
            if (s < 0) { drain(full, ring.it, err); return; }
            meta[s].kind = ST_DONE;
            mbar_arrive(&full[s]);
        }
        return;
    }

    // consumers: row l of a block belongs to warp l % NCW (fixed order of
    // accumulation); lanes take elements lane, lane+32, ... (conflict-free) in four
    // independent FP64 chains
    for (long long it = 0;; it++) {
        const int s = (int)(it % STAGES);
        if (!mbar_wait(&full[s], (unsigned)((it / STAGES) & 1), err, 2)) break;
        const StageMeta m = meta[s];
        if (m.kind == ST_DONE) break;
        const T* buf = reinterpret_cast<const T*>(data + (size_t)s * STAGE_BYTES);
        const T* w = reinterpret_cast<const T*>(wbuf + (size_t)s * K1_WBYTES) + m.woff;
        for (int i = (warp - m.s % NCW + NCW) % NCW; i < m.r0; i += NCW) {
            const int l = m.s + i;
            const T* row = buf + (size_t)i * m.sp;
            double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
            int j = lane;
            for (; j + 96 < m.nc; j += 128) {
                p0 = fma((double)row[j], (double)w[j], p0);
                p1 = fma((double)row[j + 32], (double)w[j + 32], p1);
                p2 = fma((double)row[j + 64], (double)w[j + 64], p2);
                p3 = fma((double)row[j + 96], (double)w[j + 96], p3);
            }
            for (; j < m.nc; j += 32) p0 = fma((double)row[j], (double)w[j], p0);
            double part = (p0 + p1) + (p2 + p3);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            if (lane == 0) {
                double tot = rowacc[l] + part;
                if (m.last) {
                    tbuf[m.ro + l] = (T)tot;
                    rowacc[l] = 0.0;
                } else {
                    rowacc[l] = tot;
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

size_t k2_smem_bytes()
{
    return (size_t)STAGES * (STAGE_BYTES + K2_WBYTES) + STAGES * sizeof(StageMeta) + 2 * STAGES * 8 +
           NCW * 128 * 8;
}

size_t k1_smem_bytes()
{
    return (size_t)STAGES * (STAGE_BYTES + K1_WBYTES) + STAGES * sizeof(StageMeta) + 2 * STAGES * 8 +
           K1_MAXRANK * 8;
}

hmg_status launch_tiles_bulk(hmg_matrix* h, bool fp64, double* y)
{
    const size_t smem = k2_smem_bytes();
    const int grid = std::min(h->nsm, std::max(1, h->ntiles));
    HMG_CUDA_TRY(cudaMemsetAsync(h->dev_err + 1, 0, sizeof(int), h->stream));
    if (fp64) {
        HMG_CUDA_TRY(cudaFuncSetAttribute(k_tiles_bulk<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_tiles_bulk<double><<<grid, NTH, smem, h->stream>>>((const PairDesc*)h->pair_desc, h->tile_pair_start,
                                                              h->tile_r0, h->tile_s, h->ntiles, h->perm[0], y,
                                                              h->dev_err);
    } else {
        HMG_CUDA_TRY(cudaFuncSetAttribute(k_tiles_bulk<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_tiles_bulk<float><<<grid, NTH, smem, h->stream>>>((const PairDesc*)h->pair_desc, h->tile_pair_start,
                                                             h->tile_r0, h->tile_s, h->ntiles, h->perm[0], y,
                                                             h->dev_err);
    }
    HMG_LAUNCH_CHECK();
    return HMG_OK;
}

hmg_status launch_vtx_bulk(hmg_matrix* h, bool fp64)
{
    const size_t smem = k1_smem_bytes();
    const int grid = std::min(h->nsm, std::max(1, h->nfar_list));
    HMG_CUDA_TRY(cudaMemsetAsync(h->dev_err + 2, 0, sizeof(int), h->stream));
    if (fp64) {
        HMG_CUDA_TRY(cudaFuncSetAttribute(k_vtx_bulk<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_vtx_bulk<double><<<grid, NTH, smem, h->stream>>>(h->far_list, h->nfar_list, h->blk_c0, h->blk_m2, h->rank,
                                                            h->rank_off, (double* const*)h->ptrV, h->xs64,
                                                            (double*)h->tbuf, h->dev_err);
    } else {
        HMG_CUDA_TRY(cudaFuncSetAttribute(k_vtx_bulk<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_vtx_bulk<float><<<grid, NTH, smem, h->stream>>>(h->far_list, h->nfar_list, h->blk_c0, h->blk_m2, h->rank,
                                                           h->rank_off, (float* const*)h->ptrV, h->xs32,
                                                           (float*)h->tbuf, h->dev_err);
    }
    HMG_LAUNCH_CHECK();
    return HMG_OK;
}

}  // namespace hmg
