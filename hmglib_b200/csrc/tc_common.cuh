// tc_common.cuh -- tcgen05 building blocks shared by the tensor-core product passes
// (tc.cu: operands stored as BF16 copies; tcm.cu: operands converted on chip from the
// stored factors): shared-memory matrix descriptors, the instruction descriptor, MMA
// issue, tensor-memory loads, commits, and the conversion of X into BF16 operand cores.
#pragma once

#include <cuda_bf16.h>

#include "pipeline.cuh"

namespace hmg {

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100; base offset 0, no swizzle
    return d;
}

// kind::f16, D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28
template <int NV>
__host__ __device__ constexpr uint32_t tc_idesc()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NV >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void bulk_g2s_first(void* dst, const void* src, unsigned bytes, uint64_t* bar,
                                               uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
        "%4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred pd;\n setp.ne.b32 pd, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, pd;\n}" ::"r"(d),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
        "[%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}

__device__ __forceinline__ void tc_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
        "%13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}

__device__ __forceinline__ void tc_ld8(uint32_t taddr, uint32_t (&v)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}

// A from tensor memory (M = 128 lanes, the K pairs of a row packed in consecutive
// 32-bit columns), B from shared memory
__device__ __forceinline__ void tc_mma_ts(uint32_t d, uint32_t a_tmem, uint64_t bd, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred pd;\n setp.ne.b32 pd, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, pd;\n}" ::"r"(d),
        "r"(a_tmem), "l"(bd), "r"(idesc), "r"(acc));
}

// 16 consecutive 32-bit columns of this thread's tensor-memory lane
__device__ __forceinline__ void tc_st16(uint32_t taddr, const uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}

// (a0, a1) += (b0, b1), one packed FP32 add (each lane rounded as a scalar add)
__device__ __forceinline__ void add_f32x2(uint32_t& a0, uint32_t& a1, uint32_t b0, uint32_t b1)
{
    asm("{\n\t.reg .b64 x, y;\n\tmov.b64 x, {%0, %1};\n\tmov.b64 y, {%2, %3};\n\t"
        "add.rn.f32x2 x, x, y;\n\tmov.b64 {%0, %1}, x;\n\t}"
        : "+r"(a0), "+r"(a1)
        : "r"(b0), "r"(b1));
}
__device__ __forceinline__ void add_f32x2(float& a0, float& a1, uint32_t b0, uint32_t b1)
{
    asm("{\n\t.reg .b64 x, y;\n\tmov.b64 x, {%0, %1};\n\tmov.b64 y, {%2, %3};\n\t"
        "add.rn.f32x2 x, x, y;\n\tmov.b64 {%0, %1}, x;\n\t}"
        : "+f"(a0), "+f"(a1)
        : "r"(b0), "r"(b1));
}

__device__ __forceinline__ void tc_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// non-blocking: has the phase of this parity completed?
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// ---------------------------------------------------------------------------
// per product: X -> BF16 cores (Z-ordered columns), FP32 rows -> Y
// ---------------------------------------------------------------------------
// thread (g, j): columns 8g..8g+7 of vector j, one 16-byte row of K core g in each part
// (K core g holds its parts one after another, NV * 16 bytes each)
template <int NV>
__global__ void k_tc_x(const double* __restrict__ X, int ldx, int nrhs, const int* __restrict__ perm1, int n,
                       long long ngroups, uint4* xb, int parts)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= ngroups * NV) return;
    const long long g = idx / NV;
    const int j = (int)(idx % NV);
    float f[8];
#pragma unroll
    for (int e = 0; e < 8; e++) {
        const long long c = g * 8 + e;
        f[e] = c < n && j < nrhs ? (float)X[(size_t)perm1[c] + (size_t)j * ldx] : 0.0f;
    }
#pragma unroll
    for (int q = 0; q < 3; q++)
        if (q < parts) {
            __nv_bfloat16 v[8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                v[e] = __float2bfloat16_rn(f[e]);
                f[e] -= __bfloat162float(v[e]);
            }
            xb[(g * parts + q) * NV + j] = *reinterpret_cast<const uint4*>(v);
        }
}

}  // namespace hmg
