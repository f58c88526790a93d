// stream.cuh -- descriptors shared by the product kernels (matvec.cu, stream.cu, multi.cu).
#pragma once

#include "hmg_internal.cuh"
#include "../../include/hmg.h"

struct hmg_matrix;

namespace hmg {

enum { PAIR_STORED = 0, PAIR_FAR = 1, PAIR_ONTHEFLY = 2, PAIR_FAR_MIXED = 3 };

// One (row tile, block) pair of the product: the block's slice for the tile and
// the vector piece it multiplies.  32 bytes, read once per product.
struct PairDesc {
    const void* data;  // tile slice (column-major, s_pad rows) or nullptr (on the fly)
    const void* w;     // vector multiplied: x_b (dense) or t_b (low rank), storage type
    int ncol;          // m2 (dense), rank (low rank), FP32 terms (mixed)
    int kind;          // PAIR_*
    int c0;            // first column (on the fly), FP16 terms (mixed)
    int pad;           // FP8 terms (mixed)
};

struct K1Unit {
    int b, l0, l1, tier;  // terms [l0, l1); tier: 0 storage type (FP32/FP64), 1 FP16, 2 FP8
};

// A K1 piece resolved to addresses: terms [l0, l1) of one storage tier of V_b^T, as
// rows of single terms (tier 0), interleaved pairs (FP16) or quads (FP8).
struct K1Desc {
    const void* v;       // first row of the piece
    const float* scal;   // the terms' scales (FP16/FP8 tiers), else null
    long long tout;      // tbuf index of term l0
    int c0, m2;          // the block's x segment
    int nrows, row_bytes;  // rows in the piece; row stride, a multiple of 16 bytes
    int pad[2];
};
static_assert(sizeof(K1Desc) == 48, "K1Desc layout");

// Loads of the stored near field and factors: each byte is read once per product, so
// they bypass L1 (which keeps the x and t_b values reused across rows) and ask L2 to
// fetch the whole 256-byte sector group (the neighbouring lanes' and steps' bytes).
__device__ __forceinline__ uint4 ld_stream(const void* p)
{
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.L2::256B.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p));
    return v;
}
// largest rank the streaming V^T x kernel accepts
static constexpr int K1_MAXRANK = 128;

hmg_status launch_tiles_bulk(hmg_matrix* h, bool fp64, double* y);
// pair and K1 descriptors for products in arithmetic of elem bytes (matvec.cu)
hmg_status ensure_desc(hmg_matrix* h, int elem);
// padded, zeroed Z-ordered x buffers (matvec.cu)
hmg_status ensure_xs(hmg_matrix* h);
hmg_status launch_vtx_bulk(hmg_matrix* h, bool fp64);
size_t k1_smem_bytes();
size_t k2_smem_bytes();

}  // namespace hmg
