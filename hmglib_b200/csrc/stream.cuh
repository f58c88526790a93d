// stream.cuh -- descriptors shared by the product kernels (matvec.cu, stream.cu).
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

// largest rank the streaming V^T x kernel accepts
static constexpr int K1_MAXRANK = 128;

hmg_status launch_tiles_bulk(hmg_matrix* h, bool fp64, double* y);
hmg_status launch_vtx_bulk(hmg_matrix* h, bool fp64);
size_t k1_smem_bytes();
size_t k2_smem_bytes();

}  // namespace hmg
