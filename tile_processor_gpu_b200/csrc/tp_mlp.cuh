/*
 * tp_mlp.cuh - the learned disparity residual: features, a small MLP and its
 * training, as plain CUDA kernels.
 *
 * New work: the reference stops at the correlation tiles; its Java caller
 * (absent) fits disparity.  The library's plain fit (tp_disparity_fit) is
 * refined by a network that maps a tile's six (2r+1)^2 correlation planes to
 * a correction of the plain fit and a log-variance (its confidence):
 *   features  x = the six planes of the tile (pair p in slot p, missing pairs
 *             zero) divided by their largest magnitude;
 *   network   h1 = gelu(x W1 + b1), h2 = gelu(h1 W2 + b2), [d, s] = h2 W3 + b3
 *             (1350 -> 256 -> 128 -> 2 for r = 7);
 *   estimate  rho = plain + d, variance exp(s);
 *   loss      mean of 0.5 exp(-s) (plain + d - truth)^2 + 0.5 s (Gaussian
 *             negative log-likelihood), s clamped to [-12, 12].
 * Kernels: feature gather, a tiled FP32 GEMM with optional transposes and a
 * bias / GELU epilogue (forward and the three backward products), the GELU
 * derivative, column sums (bias gradients), the loss with its gradient, and
 * Adam.  Rows are samples; matrices are row-major with leading dimensions.
 */
#pragma once
#include <cuda_bf16.h>

#include "tp_common.cuh"

namespace tp {

/* ---- features ------------------------------------------------------------- */

/* One warp per correlation entry; the warp holding the first entry of a
 * tile's run (entries of one tile adjacent) writes the tile's row:
 * feat[tile][p * n2 + k] = C_p[k] / max |C| over the run, zeros for pairs the
 * run does not list. */
__global__ void __launch_bounds__(256) k_mlp_features(int ntiles, const float *__restrict__ corrs,
                                                      size_t corr_stride, int n2, long long num,
                                                      const int *__restrict__ idx, float *__restrict__ feat,
                                                      size_t feat_stride)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long e = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < num; e += warps) {
        const int tile = __ldg(&idx[e]) >> 8;
        if (e > 0 && (__ldg(&idx[e - 1]) >> 8) == tile) continue;
        if (tile < 0 || tile >= ntiles) continue;
        long long end = e;
        float mx = 0.0f;
        while (end < num && (__ldg(&idx[end]) >> 8) == tile) {
            const int p = __ldg(&idx[end]) & 0xff;
            if (p < 6)
                for (int k = lane; k < n2; k += 32) mx = fmaxf(mx, fabsf(__ldg(&corrs[(size_t)end * corr_stride + k])));
            end++;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        const float sc = mx > 0.0f ? 1.0f / mx : 0.0f;
        float *row = feat + (size_t)tile * feat_stride;
        for (int k = lane; k < 6 * n2; k += 32) row[k] = 0.0f;
        __syncwarp();
        for (long long e2 = e; e2 < end; e2++) {
            const int p = __ldg(&idx[e2]) & 0xff;
            if (p >= 6) continue;
            for (int k = lane; k < n2; k += 32) row[p * n2 + k] = __ldg(&corrs[(size_t)e2 * corr_stride + k]) * sc;
        }
    }
}

/* ---- GEMM ----------------------------------------------------------------- */

/* C[M][N] = beta C + op(A) op(B) (+ bias[n]); op(A) is M x K (A[m][k], or
 * A[k][m] when ta), op(B) K x N (B[k][n], or B[n][k] when tb).  With z given,
 * z = the pre-activation and C = gelu(z).  64 x 64 output tile per block,
 * 256 threads with 4 x 4 outputs each, K in steps of 16 through shared
 * memory; every access bounds-checked. */
constexpr int kGB = 64, kGK = 16;

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float x)
{
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

__global__ void __launch_bounds__(256) k_gemm(int M, int N, int K, const float *__restrict__ A, int lda, int ta,
                                              const float *__restrict__ B, int ldb, int tb, float beta,
                                              float *__restrict__ C, int ldc, const float *__restrict__ bias,
                                              float *__restrict__ z, int ldz)
{
    __shared__ float sA[kGK][kGB + 4];
    __shared__ float sB[kGK][kGB + 4];
    const int tid = threadIdx.x;
    const int m0 = blockIdx.y * kGB, n0 = blockIdx.x * kGB;
    const int tr = tid >> 4, tc = tid & 15; /* 16 x 16 threads, 4 x 4 outputs */
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += kGK) {
        /* 64 x 16 of op(A) and 16 x 64 of op(B), 4 elements per thread each */
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int e = tid + 256 * i;
            {
                /* consecutive threads walk the operand's contiguous index */
                const int mm = ta ? (e & 63) : (e >> 4), kk = ta ? (e >> 6) : (e & 15);
                const int gm = m0 + mm, gk = k0 + kk;
                float v = 0.0f;
                if (gm < M && gk < K) v = ta ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
                sA[kk][mm] = v;
            }
            {
                const int nn = tb ? (e >> 4) : (e & 63), kk = tb ? (e & 15) : (e >> 6);
                const int gk = k0 + kk, gn = n0 + nn;
                float v = 0.0f;
                if (gk < K && gn < N) v = tb ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
                sB[kk][nn] = v;
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kGK; kk++) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = sA[kk][tr * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = sB[kk][tc * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gm = m0 + tr * 4 + i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gn = n0 + tc * 4 + j;
            if (gn >= N) continue;
            float v = acc[i][j];
            if (bias) v += bias[gn];
            if (beta != 0.0f) v = __fmaf_rn(beta, C[(size_t)gm * ldc + gn], v);
            if (z) {
                z[(size_t)gm * ldz + gn] = v;
                v = gelu_f(v);
            }
            C[(size_t)gm * ldc + gn] = v;
        }
    }
}

/* ---- element-wise and reductions ------------------------------------------ */

/* dz = dh * gelu'(z), [rows][cols] with leading dimension ld */
__global__ void k_gelu_backward(long long n, int cols, int ld, const float *__restrict__ z,
                                const float *__restrict__ dh, float *__restrict__ dz)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / cols, c = i - r * cols;
        const size_t o = (size_t)r * ld + c;
        dz[o] = dh[o] * gelu_grad_f(z[o]);
    }
}

/* out[c] = scale * sum over rows of x[r][c] (one thread per column, fixed order) */
__global__ void k_colsum(int rows, int cols, int ld, const float *__restrict__ x, float scale,
                         float *__restrict__ out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; r++) s += x[(size_t)r * ld + c];
    out[c] = s * scale;
}

/* Gaussian NLL of out[r] = [d, s] against target[r] = truth - plain, with the
 * gradient dout = d loss / d out for the mean over rows (weights w[r] in
 * {0, 1} select the rows that count; count = their number).  loss_rows[r]
 * receives the per-row loss. */
__global__ void k_nll(int rows, const float *__restrict__ out, const float *__restrict__ target,
                      const float *__restrict__ w, float inv_count, float *__restrict__ dout,
                      float *__restrict__ loss_rows)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const float d = out[2 * r], s = fminf(12.0f, fmaxf(-12.0f, out[2 * r + 1]));
    const float wr = w ? w[r] : 1.0f;
    const float e = d - target[r];
    const float ivar = expf(-s);
    loss_rows[r] = wr * (0.5f * ivar * e * e + 0.5f * s);
    dout[2 * r] = wr * inv_count * ivar * e;
    const float ds = 0.5f - 0.5f * ivar * e * e;
    const bool live = out[2 * r + 1] > -12.0f && out[2 * r + 1] < 12.0f;
    dout[2 * r + 1] = live ? wr * inv_count * ds : 0.0f;
}

/* Adam: m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2; p -= lr mhat / (sqrt(vhat) + eps) */
__global__ void k_adam(long long n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}



/* ---- inference on the tensor cores (tcgen05) -------------------------------
 *
 * out[r] = the network at feature row r, layers 1 and 2 as BF16 x BF16 -> FP32
 * tcgen05 MMAs with the accumulators in tensor memory, layer 3 and the
 * activations on the CUDA cores.  Persistent: one 128-thread CTA per SM walks
 * 128-row tiles.  Per tile:
 *   layer 1: for each 64-wide K block, the features (FP32 -> BF16) and W1^T
 *     (packed BF16) are written to shared memory in the canonical K-major,
 *     non-swizzled layout (8-row x 16-byte core matrices; the 16-byte K chunks
 *     LBO apart, 8-row groups 128 bytes apart); one thread issues four
 *     M=128, N=256, K=16 MMAs into TMEM columns 0..255 and commits them to an
 *     mbarrier that every thread waits on (bounded) before the next block;
 *   epilogue 1: warp w reads its 32 rows (TMEM lanes 32w..) in 8-column
 *     pieces, adds b1, applies GELU and writes BF16 rows of H1 to shared
 *     memory in the same layout -- the A operand of layer 2;
 *   layer 2: sixteen M=128, N=128, K=16 MMAs against W2^T (loaded once per
 *     CTA) into TMEM columns 256..383;
 *   epilogue 2: + b2, GELU, then layer 3 (128 -> 2) per row in registers.
 * A wait that runs out sets *err and the CTA stops after freeing its TMEM.
 */
constexpr int kTcM = 128, kTcK = 64, kTcN1 = 256, kTcN2 = 128;
constexpr int kTcKPad = 1408;                        /* 1350 padded to a multiple of 64 */
constexpr int kTcBytesA = kTcM * kTcK * 2;           /* features block, 16 KB          */
constexpr int kTcBytesB1 = kTcN1 * kTcK * 2;         /* W1^T block, 32 KB              */
constexpr int kTcBytesH1 = kTcM * kTcN1 * 2;         /* H1, 64 KB                      */
constexpr int kTcBytesW2 = kTcN2 * kTcN1 * 2;        /* W2^T, 64 KB                    */
constexpr int kTcSmemBytes = 1024 + kTcBytesA + kTcBytesB1 + kTcBytesH1 + kTcBytesW2 +
                             4 * (kTcN1 + kTcN2 + 2 * kTcN2 + 2) + 128;

/* byte offset of element (row r, k) in a canonical K-major block of `rows` rows */
__device__ __forceinline__ uint32_t tc_off(int r, int k, int rows)
{
    return (uint32_t)((k >> 3) * (rows / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

/* shared-memory matrix descriptor: no swizzle, K-major, version 1 */
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

/* instruction descriptor: BF16 x BF16 -> F32, both K-major, M x N */
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
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

__device__ __forceinline__ uint32_t pack_bf16(float a, float b)
{
    const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(a));
    const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(b));
    return lo | (hi << 16);
}

/* W1 [1350][256] -> W1^T BF16 [256][1408] (zero padded); W2 [256][128] ->
 * W2^T BF16 [128][256] */
__global__ void k_mlp_pack(const float *__restrict__ W1, const float *__restrict__ W2,
                           __nv_bfloat16 *__restrict__ w1t, __nv_bfloat16 *__restrict__ w2t)
{
    const int n1 = kTcN1 * kTcKPad, n2 = kTcN2 * kTcN1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1 + n2; i += gridDim.x * blockDim.x) {
        if (i < n1) {
            const int n = i / kTcKPad, k = i - n * kTcKPad;
            w1t[i] = __float2bfloat16_rn(k < 1350 ? W1[(size_t)k * kTcN1 + n] : 0.0f);
        } else {
            const int j = i - n1, n = j / kTcN1, k = j - n * kTcN1;
            w2t[j] = __float2bfloat16_rn(W2[(size_t)k * kTcN2 + n]);
        }
    }
}

__global__ void __launch_bounds__(128, 1) k_mlp_infer_tc(int rows, const float *__restrict__ x, int ldx,
                                                         const __nv_bfloat16 *__restrict__ w1t,
                                                         const float *__restrict__ b1,
                                                         const __nv_bfloat16 *__restrict__ w2t,
                                                         const float *__restrict__ b2,
                                                         const float *__restrict__ W3,
                                                         const float *__restrict__ b3, float *__restrict__ out,
                                                         int *__restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    /* 1024-byte aligned operand buffers, then the small tables */
    const uint32_t base_s = (uint32_t)__cvta_generic_to_shared(tc_smem);
    const uint32_t pad = (1024 - (base_s & 1023)) & 1023;
    unsigned char *sm = tc_smem + pad;
    unsigned char *sA = sm, *sB1 = sA + kTcBytesA, *sH1 = sB1 + kTcBytesB1, *sW2 = sH1 + kTcBytesH1;
    float *sb1 = reinterpret_cast<float *>(sW2 + kTcBytesW2);
    float *sb2 = sb1 + kTcN1, *sW3 = sb2 + kTcN2, *sb3 = sW3 + 2 * kTcN2;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sb3 + 2) + 1; /* 8-byte aligned */
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 1);
    const uint32_t aA = (uint32_t)__cvta_generic_to_shared(sA), aB1 = (uint32_t)__cvta_generic_to_shared(sB1);
    const uint32_t aH1 = (uint32_t)__cvta_generic_to_shared(sH1), aW2 = (uint32_t)__cvta_generic_to_shared(sW2);
    const uint32_t aMbar = (uint32_t)__cvta_generic_to_shared(mbar);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    /* tables and W2^T (K-major, 128 rows of N) once per CTA */
    for (int i = tid; i < kTcN1; i += 128) sb1[i] = b1[i];
    for (int i = tid; i < kTcN2; i += 128) sb2[i] = b2[i];
    for (int i = tid; i < 2 * kTcN2; i += 128) sW3[i] = W3[i];
    if (tid < 2) sb3[tid] = b3[tid];
    for (int i = tid; i < kTcN2 * kTcN1 / 2; i += 128) {
        const int n = (2 * i) / kTcN1, k = (2 * i) - n * kTcN1;
        const uint32_t v = *reinterpret_cast<const uint32_t *>(w2t + (size_t)n * kTcN1 + k);
        *reinterpret_cast<uint32_t *>(sW2 + tc_off(n, k, kTcN2)) = v;
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(aMbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    uint32_t phase = 0;
    bool ok = true;
    const uint32_t idesc1 = tc_idesc(kTcM, kTcN1), idesc2 = tc_idesc(kTcM, kTcN2);
    const int tiles = (rows + kTcM - 1) / kTcM;

    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int r0 = t * kTcM;
        /* ---- layer 1 ---- */
        for (int kb = 0; kb < kTcKPad / kTcK && ok; kb++) {
            const int k0 = kb * kTcK;
            /* features: warp w rows 32w..32w+31, lane = k pair */
            for (int rr = 0; rr < 32; rr++) {
                const int r = warp * 32 + rr, gr = r0 + r, k = k0 + 2 * lane;
                float2 v = make_float2(0.0f, 0.0f);
                if (gr < rows) {
                    const float *px = x + (size_t)gr * ldx + k;
                    if (k < 1350) v.x = px[0];
                    if (k + 1 < 1350) v.y = px[1];
                }
                *reinterpret_cast<uint32_t *>(sA + tc_off(r, 2 * lane, kTcM)) = pack_bf16(v.x, v.y);
            }
            /* W1^T block: 256 rows x 64 k, 16 bytes (8 k) per thread-step */
            for (int i = tid; i < kTcN1 * (kTcK / 8); i += 128) {
                const int n = i >> 3, kc = i & 7;
                const uint4 v = *reinterpret_cast<const uint4 *>(w1t + (size_t)n * kTcKPad + k0 + kc * 8);
                *reinterpret_cast<uint4 *>(sB1 + tc_off(n, kc * 8, kTcN1)) = v;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                for (int j = 0; j < kTcK / 16; j++) {
                    const uint64_t da = tc_desc(aA + j * 2 * (kTcM / 8) * 128, (kTcM / 8) * 128, 128);
                    const uint64_t db = tc_desc(aB1 + j * 2 * (kTcN1 / 8) * 128, (kTcN1 / 8) * 128, 128);
                    tc_mma(tmem, da, db, idesc1, (kb > 0 || j > 0) ? 1u : 0u);
                }
                tc_commit(aMbar);
            }
            /* every thread takes the same branch after a wait */
            ok = __syncthreads_and(tc_wait(aMbar, phase) ? 1 : 0) != 0;
            phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        }
        if (!ok) break;
        /* ---- epilogue 1: H1 = gelu(D1 + b1) as BF16 rows of the layer-2 A operand ---- */
        {
            const int r = warp * 32 + lane;
            for (int c0 = 0; c0 < kTcN1; c0 += 8) {
                float v[8];
                tc_ld8(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
                uint32_t w[4];
#pragma unroll
                for (int i = 0; i < 4; i++)
                    w[i] = pack_bf16(gelu_f(v[2 * i] + sb1[c0 + 2 * i]), gelu_f(v[2 * i + 1] + sb1[c0 + 2 * i + 1]));
                *reinterpret_cast<uint4 *>(sH1 + tc_off(r, c0, kTcM)) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        /* ---- layer 2 ---- */
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int j = 0; j < kTcN1 / 16; j++) {
                const uint64_t da = tc_desc(aH1 + j * 2 * (kTcM / 8) * 128, (kTcM / 8) * 128, 128);
                const uint64_t db = tc_desc(aW2 + j * 2 * (kTcN2 / 8) * 128, (kTcN2 / 8) * 128, 128);
                tc_mma(tmem + kTcN1, da, db, idesc2, j > 0 ? 1u : 0u);
            }
            tc_commit(aMbar);
        }
        ok = __syncthreads_and(tc_wait(aMbar, phase) ? 1 : 0) != 0;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!ok) break;
        /* ---- epilogue 2 and layer 3 ---- */
        {
            const int r = warp * 32 + lane, gr = r0 + r;
            float o0 = sb3[0], o1 = sb3[1];
            for (int c0 = 0; c0 < kTcN2; c0 += 8) {
                float v[8];
                tc_ld8(tmem + ((uint32_t)(warp * 32) << 16) + kTcN1 + c0, v);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const float h = gelu_f(v[i] + sb2[c0 + i]);
                    o0 = __fmaf_rn(h, sW3[2 * (c0 + i)], o0);
                    o1 = __fmaf_rn(h, sW3[2 * (c0 + i) + 1], o1);
                }
            }
            if (gr < rows) {
                out[2 * (size_t)gr] = o0;
                out[2 * (size_t)gr + 1] = o1;
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads(); /* H1 and TMEM free for the next tile */
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (!ok && tid == 0 && err) atomicExch(err, 1);
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

} /* namespace tp */
