/*
 * tp_tcgen05.cuh - device helpers for the fifth-generation tensor cores
 * (sm_100a): shared-memory operand layouts and descriptors, the MMA, its
 * commit, bounded mbarrier waits, TMA / bulk loads and tensor-memory loads.
 * Used by the tensor-core inference of the learned residual and by the
 * tensor-core (hi + lo split) forms of the CLT stages.
 *
 * Operand layout: canonical K-major, no swizzle: 8-row x 16-byte core
 * matrices, the 8-row groups of one K chunk 128 bytes apart (SBO), K chunks
 * (rows / 8) x 128 bytes apart (LBO).
 */
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace tp {

/* byte offset of BF16 element (row r, k) in a canonical K-major block of `rows` rows */
__host__ __device__ constexpr uint32_t tc_off(int r, int k, int rows)
{
    return (uint32_t)((k >> 3) * (rows / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

/* byte offset of TF32 element (row r, k) in a canonical K-major block of `rows` rows */
__host__ __device__ constexpr uint32_t tc_off32(int r, int k, int rows)
{
    return (uint32_t)((k >> 2) * (rows / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

/* shared-memory matrix descriptor: no swizzle, K-major, version 1 */
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

/* K-major, 128-byte swizzle: rows of 128 bytes, 8-row groups 1024 bytes apart
 * (SBO), LBO unused (1); layout type 2 */
__device__ __forceinline__ uint64_t tc_desc_sw128(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

/* instruction descriptor: FP32 accumulator, A and B both of format `fmt`
 * (1 = BF16 for kind::f16, 2 = TF32 for kind::tf32), both K-major, M x N */
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N, uint32_t fmt = 1u)
{
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
                 "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tc_mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
                 "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

/* bounded wait for phase `parity` of the mbarrier; false when it ran out */
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity)
{
    for (int it = 0; it < (1 << 22); it++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, P;\n\t}\n"
                     : "=r"(done)
                     : "r"(mbar), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

/* the producer's arrival on a `full` mbarrier, announcing `bytes` of copies */
__device__ __forceinline__ void tc_expect(uint32_t mbar, uint32_t bytes)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(mbar),
                 "r"(bytes)
                 : "memory");
}

/* 2-D TMA tensor load of the box at (x, y) (elements) into shared memory */
__device__ __forceinline__ void tc_tma_load_2d(uint32_t dst, const void *tmap, int x, int y, uint32_t mbar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                 "[%4];" ::"r"(dst),
                 "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(mbar)
                 : "memory");
}

/* bulk copy of `bytes` (multiple of 16, both ends 16-byte aligned) into shared memory */
__device__ __forceinline__ void tc_bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

/* 32 consecutive TMEM columns of this thread's lane, one wait */
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float v[32])
{
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                 "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                 "[%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(a));
    const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(b));
    return lo | (hi << 16);
}

/* FP32 -> TF32 (round to nearest, ties away; low 13 bits zero) */
__device__ __forceinline__ float to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}


/* tcgen05.ld of 8 consecutive TMEM columns of this thread's lane, one wait */
__device__ __forceinline__ void tc_ld8(uint32_t taddr, float v[8])
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

} /* namespace tp */
