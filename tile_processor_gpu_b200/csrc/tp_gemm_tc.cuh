/*
 * tp_gemm_tc.cuh - the learned residual's training GEMM on the tensor cores:
 * C = op(A) op(B) (+ bias, + beta C, optional pre-activation z and GELU), the
 * operation of k_gemm, with FP32 operands split into two TF32 parts,
 *   x = hi + lo,  hi = tf32(x),  lo = tf32(x - hi),
 * and each product formed as three tcgen05 TF32 MMAs, A_hi B_hi + A_hi B_lo +
 * A_lo B_hi (about 21 significant bits per operand; the dropped A_lo B_lo
 * term is below 2^-21 of a product).  Each K chunk of 32 is accumulated in
 * its own tensor-memory buffer and added into FP32 registers: one
 * accumulator over all of K (169 MMA steps for K = 1350, sums up to ~170
 * times a product) loses about 1e-5 of the result, the per-chunk sums stay
 * within 2e-6.
 *
 * One CTA of 128 threads per 128 x 64 tile of C; K in chunks of 32.  Every
 * thread loads its share of the chunk's op(A) (128 x 32) and op(B) (64 x 32)
 * from global memory in whichever order is contiguous for the operand's
 * transpose, splits it and stores both parts as K-major 128-byte-swizzled
 * images (rows of 32 TF32 values, the 16-byte chunk index XOR the row's low
 * three bits); after a barrier thread 0 issues the chunk's 12 MMAs (four K
 * steps of 8) into the chunk's tensor-memory buffer (two, by chunk parity)
 * and commits them to the stage's mbarrier.  Two stages: the threads fill one
 * while the tensor cores read the other; before overwriting a stage they wait
 * (bounded) for the MMAs of chunk c - 2, read that chunk's 64 columns of
 * their own lane (warp w: lanes 32 w .. 32 w + 31, one row of C per thread)
 * with tcgen05.ld and add them into 64 registers.  The epilogue applies bias,
 * beta C and GELU to the registers.
 * A wait that runs out sets *err, drains the issued MMAs (one more bounded
 * wait), frees the tensor memory and leaves C unwritten.
 */
#pragma once
#include "tp_tcgen05.cuh"

namespace tp {

constexpr int kGtM = 128, kGtN = 64, kGtK = 32;
constexpr int kGtABytes = kGtM * kGtK * 4; /* one TF32 part of the A chunk: 16 KB */
constexpr int kGtBBytes = kGtN * kGtK * 4; /* one TF32 part of the B chunk: 8 KB  */
constexpr int kGtStageBytes = 2 * kGtABytes + 2 * kGtBBytes;
constexpr int kGtStages = 2;
constexpr size_t kGtSmemBytes = (size_t)kGtStages * kGtStageBytes + 1024; /* + alignment of the swizzle atoms */
static_assert(kGtABytes % 1024 == 0 && kGtBBytes % 1024 == 0, "images start on 1024-byte swizzle atoms");

/* byte offset of element (row r, k) in a K-major image with 128-byte rows and
 * the 128-byte swizzle */
__device__ __forceinline__ uint32_t gt_sw_off(int r, int k)
{
    return (uint32_t)(r * 128 + ((((k >> 2) ^ (r & 7)) & 7) << 4) + (k & 3) * 4);
}

__device__ __forceinline__ void gt_put(unsigned char *hi_img, unsigned char *lo_img, uint32_t off, float v)
{
    const float h = to_tf32(v);
    *reinterpret_cast<float *>(hi_img + off) = h;
    *reinterpret_cast<float *>(lo_img + off) = to_tf32(v - h);
}

__global__ void __launch_bounds__(128, 1) k_gemm_tc(int M, int N, int K, const float *__restrict__ A, int lda,
                                                    int ta, const float *__restrict__ B, int ldb, int tb, float beta,
                                                    float *__restrict__ C, int ldc, const float *__restrict__ bias,
                                                    float *__restrict__ z, int ldz, int *__restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char gt_smem[];
    __shared__ __align__(8) uint64_t bars[kGtStages + 2]; /* MMA done per stage, (unused), drain */
    __shared__ uint32_t tmem_slot;
    const uint32_t base_s = (uint32_t)__cvta_generic_to_shared(gt_smem);
    const uint32_t pad = (1024 - (base_s & 1023)) & 1023;
    unsigned char *sm = gt_smem + pad;
    const uint32_t a_sm = base_s + pad;
    const uint32_t a_bar = (uint32_t)__cvta_generic_to_shared(bars);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * kGtM, n0 = blockIdx.x * kGtN;

    if (tid == 0) {
        for (int b = 0; b < kGtStages + 2; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a_bar + 8 * b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(&tmem_slot)),
                     "n"(2 * kGtN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = tc_idesc(kGtM, kGtN, 2u);
    /* this CTA's chunks: the K range blockIdx.z of gridDim.z (several only
     * for a plain product into a zeroed C, see tp_mlp_gemm_tc) */
    const int nch = (K + kGtK - 1) / kGtK;
    const int per = (nch + (int)gridDim.z - 1) / (int)gridDim.z;
    const int c_begin = min(nch, (int)blockIdx.z * per);
    const int nloc = min(nch, c_begin + per) - c_begin;

    auto stage_ptr = [&](int s) { return sm + (size_t)s * kGtStageBytes; };
    auto stage_addr = [&](int s) { return a_sm + (uint32_t)(s * kGtStageBytes); };
    /* One chunk of op(A) and op(B): load (all of this thread's 48 values in
     * flight at once) into registers, then split them into stage s.  The
     * loop below loads chunk c + 1 right after storing chunk c, so the loads'
     * latency overlaps the barrier, the MMA issue and the next chunk's wait. */
    constexpr int kAE = kGtM * kGtK / 128, kBE = kGtN * kGtK / 128;
    auto a_rk = [&](int i, int *r, int *k) {
        const int e = tid + 128 * i; /* consecutive threads walk the contiguous index */
        *r = ta ? (e & (kGtM - 1)) : (e >> 5);
        *k = ta ? (e >> 7) : (e & 31);
    };
    auto b_nk = [&](int i, int *n, int *k) {
        const int e = tid + 128 * i;
        *n = tb ? (e >> 5) : (e & (kGtN - 1));
        *k = tb ? (e & 31) : (e >> 6);
    };
    auto load_chunk = [&](int c, float ra[kAE], float rb[kBE]) {
        const int k0 = c * kGtK;
#pragma unroll
        for (int i = 0; i < kAE; i++) {
            int r, k;
            a_rk(i, &r, &k);
            const int gm = m0 + r, gk = k0 + k;
            ra[i] = (gm < M && gk < K) ? (ta ? __ldg(A + (size_t)gk * lda + gm) : __ldg(A + (size_t)gm * lda + gk))
                                       : 0.0f;
        }
#pragma unroll
        for (int i = 0; i < kBE; i++) {
            int n, k;
            b_nk(i, &n, &k);
            const int gn = n0 + n, gk = k0 + k;
            rb[i] = (gn < N && gk < K) ? (tb ? __ldg(B + (size_t)gn * ldb + gk) : __ldg(B + (size_t)gk * ldb + gn))
                                       : 0.0f;
        }
    };
    auto store_chunk = [&](int s, const float ra[kAE], const float rb[kBE]) {
        unsigned char *ahi = stage_ptr(s), *alo = ahi + kGtABytes;
        unsigned char *bhi = alo + kGtABytes, *blo = bhi + kGtBBytes;
#pragma unroll
        for (int i = 0; i < kAE; i++) {
            int r, k;
            a_rk(i, &r, &k);
            gt_put(ahi, alo, gt_sw_off(r, k), ra[i]);
        }
#pragma unroll
        for (int i = 0; i < kBE; i++) {
            int n, k;
            b_nk(i, &n, &k);
            gt_put(bhi, blo, gt_sw_off(n, k), rb[i]);
        }
    };

    bool ok = true, failed = false;
    bool issued = false; /* thread 0: MMAs issued */
    float acc[kGtN];     /* this thread's row of the tile: the sum of the chunks read so far */
#pragma unroll
    for (int i = 0; i < kGtN; i++) acc[i] = 0.0f;
    const uint32_t t_lane = (uint32_t)(warp * 32) << 16;
    /* local chunk c's partial sums (buffer c & 1) into acc; its MMAs have completed */
    auto gather = [&](int c) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int c0 = 0; c0 < kGtN; c0 += 32) {
            float v[32];
            tc_ld32(tmem + t_lane + (uint32_t)((c & 1) * kGtN + c0), v);
#pragma unroll
            for (int i = 0; i < 32; i++) acc[c0 + i] += v[i];
        }
    };
    float ra[kAE], rb[kBE];
    if (nloc > 0) load_chunk(c_begin, ra, rb);
    for (int i = 0; i < nloc; i++) {
        const int s = i & 1;
        /* the MMAs of local chunk i - 2 have read stage s and filled buffer s */
        if (i >= 2 && ok) ok = tc_wait(a_bar + 8u * s, (uint32_t)(((i - 2) >> 1) & 1));
        if (!__syncthreads_and(ok ? 1 : 0)) {
            failed = true;
            break;
        }
        if (i >= 2) gather(i - 2);
        store_chunk(s, ra, rb);
        if (i + 1 < nloc) load_chunk(c_begin + i + 1, ra, rb);
        /* the generic-proxy stores visible to the tensor cores' reads, and
         * this thread's reads of buffer s ordered before the next MMAs */
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a = stage_addr(s);
            const uint32_t ahi = a, alo = a + kGtABytes, bhi = a + 2 * kGtABytes, blo = bhi + kGtBBytes;
            const uint32_t d = tmem + (uint32_t)(s * kGtN);
#pragma unroll
            for (int j = 0; j < kGtK / 8; j++) {
                const uint32_t o = 32u * j;
                tc_mma_tf32(d, tc_desc_sw128(ahi + o), tc_desc_sw128(bhi + o), idesc, j > 0 ? 1u : 0u);
                tc_mma_tf32(d, tc_desc_sw128(ahi + o), tc_desc_sw128(blo + o), idesc, 1u);
                tc_mma_tf32(d, tc_desc_sw128(alo + o), tc_desc_sw128(bhi + o), idesc, 1u);
            }
            tc_commit(a_bar + 8u * s);
            issued = true;
        }
    }
    /* the last two chunks */
    for (int i = nloc - 2; i < nloc && !failed; i++) {
        if (i < 0) continue;
        const int s = i & 1;
        if (ok) ok = tc_wait(a_bar + 8u * s, (uint32_t)((i >> 1) & 1));
        if (!__syncthreads_and(ok ? 1 : 0)) {
            failed = true;
            break;
        }
        gather(i);
    }
    if (!failed) {
        /* epilogue: warp w holds rows m0 + 32 w .. + 31, one per lane */
        const int gm = m0 + warp * 32 + lane;
        /* (loops fully unrolled: acc stays in registers) */
        if (gm < M && gridDim.z > 1) {
            /* one of several K ranges: its partial sums into the zeroed C */
#pragma unroll
            for (int i = 0; i < kGtN; i++) {
                const int gn = n0 + i;
                if (gn < N) atomicAdd(C + (size_t)gm * ldc + gn, acc[i]);
            }
        } else if (gm < M) {
#pragma unroll
            for (int i = 0; i < kGtN; i++) {
                const int gn = n0 + i;
                if (gn >= N) continue;
                float x = acc[i];
                if (bias) x += bias[gn];
                if (beta != 0.0f) x = __fmaf_rn(beta, C[(size_t)gm * ldc + gn], x);
                if (z) {
                    z[(size_t)gm * ldz + gn] = x;
                    x = gelu_f(x);
                }
                C[(size_t)gm * ldc + gn] = x;
            }
        }
    } else if (tid == 0) {
        /* MMAs issued so far complete before the tensor memory is freed */
        if (issued) {
            tc_commit(a_bar + 8u * (kGtStages + 1));
            (void)tc_wait(a_bar + 8u * (kGtStages + 1), 0u);
        }
        if (err) atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(2 * kGtN) : "memory");
}

} /* namespace tp */
