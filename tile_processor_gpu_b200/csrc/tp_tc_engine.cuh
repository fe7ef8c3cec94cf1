/*
 * tp_tc_engine.cuh - the batched 8x8 transforms of the CLT stages on the
 * tensor cores, with FP32 accuracy from split 16-bit operands.
 *
 * Each stage of the path applies, per job (one tile and camera / pair and
 * colour), a separable 2-D transform to each of its 8x8 quadrants:
 * Y_q = V_q X_q H_q^T, V and H one of the 8-point DCT-IV / DST-IV / DCT-II /
 * DST-II of the reference (src/dtt8x8.cuh:382-463, :621-745).  Flattened
 * row-major, that is one 64 x 64 matrix per quadrant,
 *     vec(Y_q) = K_q vec(X_q),   K_q[(i, j)][(m, n)] = V_q[i][m] H_q[j][n],
 * so 128 jobs' quadrant q is one M = 128, N = 64, K = 64 GEMM.  The operands
 * are split into 16-bit halves, x = x_hi + x_lo (FP16 with the rows scaled by
 * a power of two, or BF16), and each product is the sum of three MMAs,
 * A_hi B_hi + A_hi B_lo + A_lo B_hi, accumulated in FP32 in tensor memory:
 * 22 (FP16) or 16 (BF16) significant bits per operand instead of 11 or 8.
 *
 * Shared-memory operand images: 128-byte-swizzled K-major.  One quadrant of
 * 128 A rows is 128 rows x 128 bytes (64 halves), 16 KB; the Q quadrants of
 * the hi part follow each other, then those of the lo part.  B_q (64 rows of
 * N x 64 K) is 8 KB; a stage's table (64 KB in global memory) holds the four
 * B_q hi, then the four lo; the kernel copies the hi and lo of its Q
 * quadrants.  Byte of half k of row r in a quadrant: r * 128 + ((k / 8) ^
 * (r % 8)) * 16 + (k % 8) * 2.  An MMA's K step of 16 halves advances the
 * descriptor's start by 32 bytes inside the swizzle atom.
 *
 * k_tc_stage<S, FMT> is the pipeline every stage shares; S supplies the
 * work (rows, producer, epilogue).  Persistent, one CTA per SM (512 or 768
 * threads: the producers' loads and the epilogues' per-job work are latency
 * bound, so the stages take as many warps as their registers allow), blocks
 * of 128 rows (jobs):
 *   producer warps: one 8-lane group per row writes its quadrants, split,
 *     into the A image and (lane 0) the row's metadata words; after a named
 *     barrier thread 0 issues the block's 12 Q MMAs into accumulator buffer
 *     (block & 1) and commits them to mma[block & 1];
 *   epilogue warps: thread t of epilogue warp e owns row 32 (e % 4) + t of
 *     the block, read from tensor-memory lane 32 (e % 4) + t (with eight
 *     epilogue warps, warps e and e + 4 share the rows and split the work:
 *     part e / 4); it waits for meta[block & 1] and mma[block & 1], runs
 *     S::epilogue, and the warp then releases the buffer (free[block & 1]).
 * Before the producers fill block b, thread 0 waits for the epilogue of
 * block b-2 (its accumulator and metadata buffer are free) and, with one A
 * image, for the MMAs of block b-1 (the A image is free; a stage with two
 * quadrant slots keeps two A images, block b filling image b % 2, whose last
 * reader, block b-2's MMAs, completed before that block's epilogue ran), and
 * publishes the outcome before a named
 * barrier, so all producer threads go on or leave together; each epilogue
 * warp agrees on its waits with a vote.  The metadata reach the epilogue
 * through the meta mbarrier's release / acquire.  Every wait is bounded: one
 * that runs out sets the abort flag, every role leaves its loop, the CTA
 * drains the MMAs in flight (bounded), sets *err and frees its tensor memory.
 * Tensor memory: accumulator buffer b at column 64 Q b, quadrant q at 64 q.
 */
#pragma once
#include "tp_common.cuh"
#include "tp_tcgen05.cuh"

namespace tp {

constexpr int kTcRows = 128;                         /* jobs per block (MMA M)          */
constexpr int kTcQuadBytes = kTcRows * 128;          /* one quadrant of 128 A rows       */
constexpr int kTcBQuadBytes = 64 * 128;              /* one B_q, hi or lo                */
constexpr int kTcBBytes = 8 * kTcBQuadBytes;         /* a stage's table: 4 hi, then 4 lo */
constexpr int kTcBTableHalves = kTcBBytes / 2;       /* halves per table                 */

/* operand formats: TP_TC_FP16X2 -> FP16 halves (kind::f16 format 0), TP_TC_BF16X2 -> BF16 (format 1) */
__host__ __device__ constexpr uint32_t tc_idesc_fmt(int fmt) { return fmt == TP_TC_BF16X2 ? 1u : 0u; }

/* byte offset of half k (0..63) of row r in a 128-byte-swizzled quadrant image */
__host__ __device__ constexpr uint32_t tc_sw_off(int r, int k)
{
    return (uint32_t)(r * 128 + (((k >> 3) ^ (r & 7)) << 4) + ((k & 7) << 1));
}

/* x -> (hi, lo) 16-bit halves of format FMT, packed in pairs: a in the low
 * 16 bits, b in the high */
template <int FMT>
__device__ __forceinline__ void tc_split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
    if constexpr (FMT == TP_TC_BF16X2) {
        const __nv_bfloat16 ah = __float2bfloat16_rn(a), bh = __float2bfloat16_rn(b);
        const __nv_bfloat16 al = __float2bfloat16_rn(a - __bfloat162float(ah));
        const __nv_bfloat16 bl = __float2bfloat16_rn(b - __bfloat162float(bh));
        hi = (uint32_t)__bfloat16_as_ushort(ah) | ((uint32_t)__bfloat16_as_ushort(bh) << 16);
        lo = (uint32_t)__bfloat16_as_ushort(al) | ((uint32_t)__bfloat16_as_ushort(bl) << 16);
    } else {
        const __half ah = __float2half_rn(a), bh = __float2half_rn(b);
        const __half al = __float2half_rn(a - __half2float(ah));
        const __half bl = __float2half_rn(b - __half2float(bh));
        hi = (uint32_t)__half_as_ushort(ah) | ((uint32_t)__half_as_ushort(bh) << 16);
        lo = (uint32_t)__half_as_ushort(al) | ((uint32_t)__half_as_ushort(bl) << 16);
    }
}

/* A image of a stage with Q quadrants: hi at [0, Q quads), lo after */
template <int Q>
struct TcA {
    unsigned char *img;
    /* 8 consecutive K values (halves k0 .. k0 + 7 of quadrant q, k0 a multiple
     * of 8) of row r, scaled by s, as a hi and a lo 16-byte chunk */
    template <int FMT>
    __device__ __forceinline__ void put8(int r, int q, int k0, const float v[8], float s) const
    {
        uint32_t h[4], lo[4];
#pragma unroll
        for (int i = 0; i < 4; i++) tc_split2<FMT>(v[2 * i] * s, v[2 * i + 1] * s, h[i], lo[i]);
        const uint32_t off = (uint32_t)q * kTcQuadBytes + tc_sw_off(r, k0);
        *reinterpret_cast<uint4 *>(img + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(img + Q * kTcQuadBytes + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
    /* zeros for row r, quadrant q, halves k0 .. k0 + 7 */
    __device__ __forceinline__ void zero8(int r, int q, int k0) const
    {
        const uint32_t off = (uint32_t)q * kTcQuadBytes + tc_sw_off(r, k0);
        *reinterpret_cast<uint4 *>(img + off) = make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4 *>(img + Q * kTcQuadBytes + off) = make_uint4(0u, 0u, 0u, 0u);
    }
};

/* The 12 Q MMAs of one block: for each quadrant, A_hi B_hi, A_hi B_lo, A_lo
 * B_hi over the four K steps, into accumulator columns d + 64 q. */
template <int Q>
__device__ __forceinline__ void tc_issue_block(uint32_t d, uint32_t a_s, uint32_t b_s, uint32_t idesc)
{
#pragma unroll
    for (int q = 0; q < Q; q++) {
        const uint32_t aq = a_s + (uint32_t)q * kTcQuadBytes, bq = b_s + (uint32_t)q * kTcBQuadBytes;
#pragma unroll
        for (int pass = 0; pass < 3; pass++) {
            const uint32_t ap = aq + (pass == 2 ? (uint32_t)(Q * kTcQuadBytes) : 0u);
            const uint32_t bp = bq + (pass == 1 ? (uint32_t)(Q * kTcBQuadBytes) : 0u);
#pragma unroll
            for (int s = 0; s < 4; s++)
                tc_mma(d + 64u * q, tc_desc_sw128(ap + 32u * s), tc_desc_sw128(bp + 32u * s), idesc,
                       (pass > 0 || s > 0) ? 1u : 0u);
        }
    }
}

/* tcgen05.ld of 4 x 8 consecutive columns of this thread's lane (four loads, one wait) */
__device__ __forceinline__ void tc_ld8x4(uint32_t t0, uint32_t t1, uint32_t t2, uint32_t t3, float v[4][8])
{
    uint32_t r[4][8];
#define TP_TC_LD8(T, R)                                                                                       \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"              \
                 : "=r"(R[0]), "=r"(R[1]), "=r"(R[2]), "=r"(R[3]), "=r"(R[4]), "=r"(R[5]), "=r"(R[6]), "=r"(R[7]) \
                 : "r"(T))
    TP_TC_LD8(t0, r[0]);
    TP_TC_LD8(t1, r[1]);
    TP_TC_LD8(t2, r[2]);
    TP_TC_LD8(t3, r[3]);
#undef TP_TC_LD8
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int i = 0; i < 8; i++) v[q][i] = __uint_as_float(r[q][i]);
}

/* bounded mbarrier wait that also gives up when another role has aborted */
__device__ __forceinline__ bool tc_wait_or_abort(uint32_t mbar, uint32_t parity, volatile int *abort_flag)
{
    for (int it = 0; it < (1 << 22); it++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, P;\n\t}\n"
                     : "=r"(done)
                     : "r"(mbar), "r"(parity)
                     : "memory");
        if (done) return true;
        if ((it & 1023) == 1023 && *abort_flag) return false;
    }
    return false;
}

/* mbarrier arrive (release: this thread's earlier shared-memory writes are
 * visible to a thread whose wait observes the phase) */
__device__ __forceinline__ void tc_arrive(uint32_t mbar)
{
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(mbar) : "memory");
}

/* named barrier over the producer warps (id 1) */
__device__ __forceinline__ void tc_producer_sync(int nthreads)
{
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

/* dynamic shared memory of k_tc_stage for a stage of Q quadrants, M
 * metadata words per row and AS A images */
__host__ __device__ constexpr int tc_stage_smem(int Q, int M, int AS)
{
    return 1024 + AS * 2 * Q * kTcQuadBytes + 2 * Q * kTcBQuadBytes + 2 * kTcRows * M * 4 + 8 * 8 + 32;
}

template <class S, int FMT>
__global__ void __launch_bounds__(S::kThreads, 1) k_tc_stage(const S st, const unsigned char *__restrict__ btab,
                                                             int *__restrict__ err)
{
    constexpr int Q = S::kQuads;
    constexpr int kMetaWords = S::kMeta;
    constexpr int kProd = 32 * S::kProdWarps;
    constexpr int kAStages = S::kAStages; /* 1, or 2: block b fills A image b % 2 */
    static_assert(kAStages == 1 || kAStages == 2, "A images");
    constexpr int kAImage = 2 * Q * kTcQuadBytes, kABytes = kAStages * kAImage, kBBytes = 2 * Q * kTcBQuadBytes;
    constexpr uint32_t kCols = (uint32_t)(2 * 64 * Q); /* 256 or 512 */
    enum { kBarB = 0, kBarMma = 1, kBarMeta = 3, kBarFree = 5, kBarDrain = 7, kBars = 8 };
    extern __shared__ __align__(1024) unsigned char tcs_smem[];
    const uint32_t base_s = (uint32_t)__cvta_generic_to_shared(tcs_smem);
    const uint32_t pad = (1024 - (base_s & 1023)) & 1023;
    unsigned char *sm = tcs_smem + pad;
    const uint32_t aA = base_s + pad, aB = aA + kABytes;
    uint32_t *meta = reinterpret_cast<uint32_t *>(sm + kABytes + kBBytes); /* [2][128][kMetaWords] */
    uint64_t *mbar = reinterpret_cast<uint64_t *>(meta + 2 * kTcRows * kMetaWords);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + kBars);
    volatile int *flags = reinterpret_cast<volatile int *>(tmem_slot + 1); /* [0] abort, [1] producers go */
    const uint32_t aBar = (uint32_t)__cvta_generic_to_shared(mbar);
    auto bar = [&](int b) { return aBar + 8u * (uint32_t)b; };

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = warp < S::kProdWarps;
    const bool issuer = tid == 0;
    if (issuer) {
        for (int b = 0; b < kBars; b++) {
            uint32_t count = 1u;
            if (b == kBarMeta || b == kBarMeta + 1) count = (uint32_t)kProd;
            if (b == kBarFree || b == kBarFree + 1) count = (uint32_t)S::kEpiWarps;
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar(b)), "r"(count) : "memory");
        }
        flags[0] = 0;
        flags[1] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == S::kProdWarps) { /* the first epilogue warp owns the allocation */
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const long long nrows = st.rows();
    const long long nblocks = (nrows + kTcRows - 1) / kTcRows;
    bool b_loaded = false, b_issued = false;
    int issued = 0;

    if (producer) {
        const int l = tid & 7, grp = tid >> 3;
        const unsigned gm = group_mask();
        if (issuer && blockIdx.x < nblocks) {
            tc_expect(bar(kBarB), (uint32_t)kBBytes);
            tc_bulk_load(aB, btab, (uint32_t)(Q * kTcBQuadBytes), bar(kBarB));
            tc_bulk_load(aB + Q * kTcBQuadBytes, btab + 4 * kTcBQuadBytes, (uint32_t)(Q * kTcBQuadBytes), bar(kBarB));
            b_issued = true;
        }
        int lb = 0;
        for (long long blk = blockIdx.x; blk < nblocks; blk += gridDim.x, lb++) {
            if (issuer) {
                bool ok = !flags[0];
                /* one A image: free once the previous block's MMAs completed.  Two:
                 * image lb % 2 was last read by the MMAs of block lb - 2, which
                 * completed before that block's epilogue ran (waited for below) */
                if (kAStages == 1 && ok && lb > 0)
                    ok = tc_wait_or_abort(bar(kBarMma + ((lb - 1) & 1)), (uint32_t)(((lb - 1) >> 1) & 1), flags);
                /* accumulator and metadata buffer: free once block lb - 2's epilogue released them */
                if (ok && lb >= 2)
                    ok = tc_wait_or_abort(bar(kBarFree + (lb & 1)), (uint32_t)(((lb >> 1) - 1) & 1), flags);
                if (!ok) flags[0] = 1;
                flags[1] = ok ? 1 : 0;
            }
            tc_producer_sync(kProd);
            if (!flags[1]) break;
            uint32_t *mb = meta + (lb & 1) * kTcRows * kMetaWords;
            const TcA<Q> A{sm + (lb % kAStages) * kAImage};
#pragma unroll 1
            for (int row = grp; row < kTcRows; row += kProd / 8)
                st.template produce<FMT>(blk * kTcRows + row, row, l, gm, A, mb + row * kMetaWords);
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_arrive(bar(kBarMeta + (lb & 1)));
            tc_producer_sync(kProd);
            if (issuer) {
                bool ok = !flags[0];
                if (ok && !b_loaded) {
                    ok = tc_wait_or_abort(bar(kBarB), 0u, flags);
                    b_loaded = ok;
                }
                if (!ok) {
                    flags[0] = 1;
                } else {
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    tc_issue_block<Q>(tmem + 64u * Q * (uint32_t)(lb & 1), aA + (uint32_t)((lb % kAStages) * kAImage),
                                      aB, tc_idesc(kTcRows, 64, tc_idesc_fmt(FMT)));
                    tc_commit(bar(kBarMma + (lb & 1)));
                    issued++;
                }
            }
        }
    } else {
        static_assert(S::kProdWarps % 4 == 0 && (S::kEpiWarps == 4 || S::kEpiWarps == 8), "warp roles");
        const int e = (warp - S::kProdWarps) & 3; /* == warp % 4: this warp's tensor-memory lanes */
        const int part = (warp - S::kProdWarps) >> 2;
        const int row = 32 * e + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(32 * e) << 16);
        int lb = 0;
        for (long long blk = blockIdx.x; blk < nblocks; blk += gridDim.x, lb++) {
            const uint32_t par = (uint32_t)((lb >> 1) & 1);
            bool ok = tc_wait_or_abort(bar(kBarMeta + (lb & 1)), par, flags);
            if (ok) ok = tc_wait_or_abort(bar(kBarMma + (lb & 1)), par, flags);
            if (!__all_sync(0xffffffffu, ok)) {
                flags[0] = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            st.epilogue(blk * kTcRows + row, lane_base + 64u * Q * (uint32_t)(lb & 1),
                        meta + ((lb & 1) * kTcRows + row) * kMetaWords, part);
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) tc_arrive(bar(kBarFree + (lb & 1)));
        }
    }
    /* ---- teardown ---- */
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (issuer) {
        if (flags[0] && err) atomicExch(err, 1);
        /* every MMA this CTA issued has completed before its memory is freed */
        if (issued > 0) {
            tc_commit(bar(kBarDrain));
            (void)tc_wait(bar(kBarDrain), 0u);
        }
        if (b_issued && !b_loaded) (void)tc_wait(bar(kBarB), 0u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == S::kProdWarps)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

} /* namespace tp */
