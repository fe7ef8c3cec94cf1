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
#include <cuda.h>
#include <cuda_bf16.h>

#include "tp_common.cuh"
#include "tp_tcgen05.cuh"

namespace tp {

/* ---- features ------------------------------------------------------------- */

/* One warp per correlation entry; the warp holding the first entry of a
 * tile's run (entries of one tile adjacent) writes the tile's row:
 * feat[tile][p * n2 + k] = C_p[k] / max |C| over the run, zeros for pairs the
 * run does not list (a pair listed twice: the later entry's plane, both in
 * the maximum; entries with p >= 6 are skipped).  The warp reads idx[e ..
 * e + 31] at once to find the run; a run of at most 32 entries without a
 * repeated pair is read once into registers (lane l holds k = l + 32 i of
 * every pair) and written once; other runs take the two-pass loop. */
__global__ void __launch_bounds__(256) k_mlp_features(int ntiles, const float *__restrict__ corrs,
                                                      size_t corr_stride, int n2, long long num,
                                                      const int *__restrict__ idx, float *__restrict__ feat,
                                                      size_t feat_stride)
{
    constexpr int kPer = 8; /* ceil(225 / 32): n2 <= 225 */
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long e = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < num; e += warps) {
        const int tile = __ldg(&idx[e]) >> 8;
        if (e > 0 && (__ldg(&idx[e - 1]) >> 8) == tile) continue;
        if (tile < 0 || tile >= ntiles) continue;
        /* the run: lanes holding entries e + lane of the same tile */
        const int code = e + lane < num ? __ldg(&idx[e + lane]) : -1;
        const unsigned other = __ballot_sync(0xffffffffu, e + lane >= num || (code >> 8) != tile);
        const int len = other ? __ffs(other) - 1 : 32;
        const int pl = lane < len ? (code & 0xff) : 255;
        bool simple = len < 32 || e + 32 >= num || (__ldg(&idx[e + 32]) >> 8) != tile;
        int where[6];
#pragma unroll
        for (int pp = 0; pp < 6; pp++) {
            const unsigned m = __ballot_sync(0xffffffffu, pl == pp);
            where[pp] = m ? __ffs(m) - 1 : -1;
            simple = simple && __popc(m) <= 1;
        }
        float *row = feat + (size_t)tile * feat_stride;
        if (simple) {
            float v[6][kPer];
            float mx = 0.0f;
#pragma unroll
            for (int pp = 0; pp < 6; pp++) {
                const float *src = corrs + (size_t)(e + (where[pp] < 0 ? 0 : where[pp])) * corr_stride;
#pragma unroll
                for (int i = 0; i < kPer; i++) {
                    const int k = lane + 32 * i;
                    v[pp][i] = (where[pp] >= 0 && k < n2) ? __ldg(&src[k]) : 0.0f;
                    mx = fmaxf(mx, fabsf(v[pp][i]));
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            const float sc = mx > 0.0f ? 1.0f / mx : 0.0f;
#pragma unroll
            for (int pp = 0; pp < 6; pp++)
#pragma unroll
                for (int i = 0; i < kPer; i++) {
                    const int k = lane + 32 * i;
                    if (k < n2) row[pp * n2 + k] = v[pp][i] * sc;
                }
            continue;
        }
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
        for (int k = lane; k < 6 * n2; k += 32) row[k] = 0.0f;
        __syncwarp();
        for (long long e2 = e; e2 < end; e2++) {
            const int p = __ldg(&idx[e2]) & 0xff;
            if (p >= 6) continue;
            for (int k = lane; k < n2; k += 32) row[p * n2 + k] = __ldg(&corrs[(size_t)e2 * corr_stride + k]) * sc;
        }
    }
}

/* ---- the learned estimate with the plain fit as fallback -------------------
 * rho[i] = plain[i] + d_i where the network's log-variance s_i < gate, else
 * plain[i] (out[i] = {d_i, s_i}). */
__global__ void __launch_bounds__(256) k_mlp_combine(long long n, const float *__restrict__ plain,
                                                     const float *__restrict__ out, float gate,
                                                     float *__restrict__ rho)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float2 o = reinterpret_cast<const float2 *>(out)[i];
        rho[i] = plain[i] + (o.y < gate ? o.x : 0.0f);
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

/* out[c] = scale * sum over rows of x[r][c].  Block (32, kColLanes): 32
 * columns, each summed by kColLanes threads over rows lane, lane + kColLanes,
 * ... and the lanes' partial sums added in a fixed tree order, so the
 * result does not depend on scheduling. */
constexpr int kColLanes = 16;
__global__ void __launch_bounds__(32 * kColLanes) k_colsum(int rows, int cols, int ld, const float *__restrict__ x,
                                                           float scale, float *__restrict__ out)
{
    __shared__ float part[kColLanes][33];
    const int c = blockIdx.x * 32 + threadIdx.x, lane = threadIdx.y;
    float s = 0.0f;
    if (c < cols)
        for (int r = lane; r < rows; r += kColLanes) s += x[(size_t)r * ld + c];
    part[lane][threadIdx.x] = s;
    __syncthreads();
    for (int h = kColLanes / 2; h > 0; h >>= 1) {
        if (lane < h) part[lane][threadIdx.x] += part[lane + h][threadIdx.x];
        __syncthreads();
    }
    if (lane == 0 && c < cols) out[c] = part[0][threadIdx.x] * scale;
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



/* ---- inference on the tensor cores (tcgen05 + TMA) --------------------------
 *
 * out[r] = the network at feature row r: layer 1 as TF32 x TF32 -> FP32 and
 * layer 2 as BF16 x BF16 -> FP32 tcgen05 MMAs with the accumulators in tensor
 * memory (columns 0..255 and 256..383), layer 3 and the activations on the
 * CUDA cores.  Persistent: one 128-thread CTA per SM walks 128-row tiles.
 *
 * Layer 1 runs over 43 K blocks of 32 through a three-stage ring of shared
 * memory.  Thread 32 is the producer: per block one TMA tensor load of the
 * 128 x 32 FP32 feature box (128-byte swizzle; columns past 1349 and rows past
 * `rows` arrive as zeros) and one bulk copy of the 32 KB W1^T block, which
 * k_mlp_pack stores already in the canonical K-major, non-swizzled image
 * (8-row x 16-byte core matrices, K chunks 4096 bytes apart), both completing
 * on the stage's `full` mbarrier.  Thread 0 issues the block's four M=128,
 * N=256, K=8 MMAs once `full` flips and commits them to the stage's `empty`
 * mbarrier, which the producer waits on before refilling the stage; after
 * the last block it commits `acc`.  The other threads wait on `acc`.
 * Epilogue 1: warp w reads its 32 rows (TMEM lanes 32w..) in 32-column pieces,
 * adds b1, applies GELU and writes BF16 rows of H1 over the first 64 KB of the
 * ring (stages 0 and 1); block kb of every tile uses stage (kb + 2) % 3, so the
 * next tile's block 0 (stage 2) is loading meanwhile.  Layer 2: sixteen
 * M=128, N=128, K=16 MMAs against W2^T (one bulk copy per CTA, also stored
 * pre-laid-out) committed to `l2`; once it flips the next tile's block 1 may
 * overwrite stage 0.  Epilogue 2: + b2, GELU, layer 3 (128 -> 2) per row.
 * Every commit and every load completion is waited exactly once, in order,
 * so one parity bit per mbarrier tracks its phase.  A wait that runs out
 * makes its thread stop issuing; the CTA leaves the loop together at the next
 * barrier, waits (bounded) for its copies and MMAs in flight, sets *err and
 * frees its TMEM.
 */
constexpr int kTcM = 128, kTcN1 = 256, kTcN2 = 128;
constexpr int kTcKB = 32;                         /* TF32 elements of K per block    */
constexpr int kTcBlocks = 43;                     /* 1350 -> 1376 = 43 x 32          */
constexpr int kTcKPad = kTcBlocks * kTcKB;
constexpr int kTcStages = 3;
constexpr int kTcBytesA = kTcM * kTcKB * 4;       /* feature box, 16 KB              */
constexpr int kTcBytesB1 = kTcN1 * kTcKB * 4;     /* W1^T block, 32 KB               */
constexpr int kTcBytesStage = kTcBytesA + kTcBytesB1;
constexpr int kTcBytesRing = kTcStages * kTcBytesStage; /* 144 KB                   */
constexpr int kTcBytesH1 = kTcM * kTcN1 * 2;      /* H1 in BF16, 64 KB, over stages 0-1 */
constexpr int kTcBytesW2 = kTcN2 * kTcN1 * 2;     /* W2^T in BF16, 64 KB             */
static_assert(kTcBytesH1 <= 2 * kTcBytesStage, "H1 must stay clear of stage 2");
static_assert(kTcBytesStage % 1024 == 0, "stages start on 1024-byte boundaries (128-byte swizzle)");
static_assert(kTcKPad >= 1350 && kTcKPad - kTcKB < 1350, "K blocking");
constexpr int kTcTableFloats = kTcN1 + kTcN2 + 2 * kTcN2 + 2;
enum { kBarFull = 0, kBarEmpty = 3, kBarAcc = 6, kBarL2 = 7, kBarW2 = 8, kBarDrain = 9, kTcBars = 10 };
constexpr int kTcSmemBytes = 1024 + kTcBytesRing + kTcBytesW2 + 4 * kTcTableFloats + 8 * kTcBars + 64;

/* W1 [1350][256] -> 43 blocks of 256 x 32 TF32 (W1^T, zero past row 1349),
 * each the byte image of a canonical non-swizzled K-major B operand;
 * W2 [256][128] -> the image of W2^T in BF16 (128 x 256, same layout) */
__global__ void k_mlp_pack(const float *__restrict__ W1, const float *__restrict__ W2, float *__restrict__ w1img,
                           __nv_bfloat16 *__restrict__ w2img)
{
    const int n1 = kTcBlocks * kTcN1 * kTcKB, n2 = kTcN2 * kTcN1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n1 + n2; i += gridDim.x * blockDim.x) {
        if (i < n1) {
            const int kb = i / (kTcN1 * kTcKB), e = i - kb * (kTcN1 * kTcKB);
            const int n = e / kTcKB, kk = e - n * kTcKB, k = kb * kTcKB + kk;
            w1img[(size_t)kb * (kTcN1 * kTcKB) + tc_off32(n, kk, kTcN1) / 4] =
                k < 1350 ? to_tf32(W1[(size_t)k * kTcN1 + n]) : 0.0f;
        } else {
            const int j = i - n1, n = j / kTcN1, k = j - n * kTcN1;
            w2img[tc_off(n, k, kTcN2) / 2] = __float2bfloat16_rn(W2[(size_t)k * kTcN2 + n]);
        }
    }
}

__global__ void __launch_bounds__(128, 1) k_mlp_infer_tc(const __grid_constant__ CUtensorMap tmap_x, int rows,
                                                         const float *__restrict__ w1img,
                                                         const float *__restrict__ b1,
                                                         const __nv_bfloat16 *__restrict__ w2img,
                                                         const float *__restrict__ b2,
                                                         const float *__restrict__ W3,
                                                         const float *__restrict__ b3, float *__restrict__ out,
                                                         int *__restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    /* 1024-byte aligned ring (H1 over its start), W2^T, then the small tables */
    const uint32_t base_s = (uint32_t)__cvta_generic_to_shared(tc_smem);
    const uint32_t pad = (1024 - (base_s & 1023)) & 1023;
    unsigned char *sm = tc_smem + pad;
    unsigned char *sH1 = sm;
    float *sb1 = reinterpret_cast<float *>(sm + kTcBytesRing + kTcBytesW2);
    float *sb2 = sb1 + kTcN1, *sW3 = sb2 + kTcN2, *sb3 = sW3 + 2 * kTcN2;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sb3 + 2);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + kTcBars);
    const uint32_t aRing = base_s + pad, aH1 = aRing, aW2 = aRing + kTcBytesRing;
    const uint32_t aBar = (uint32_t)__cvta_generic_to_shared(mbar);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const bool producer = tid == 32, issuer = tid == 0;
    for (int i = tid; i < kTcN1; i += 128) sb1[i] = b1[i];
    for (int i = tid; i < kTcN2; i += 128) sb2[i] = b2[i];
    for (int i = tid; i < 2 * kTcN2; i += 128) sW3[i] = W3[i];
    if (tid < 2) sb3[tid] = b3[tid];
    if (issuer) {
        for (int b = 0; b < kTcBars; b++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(aBar + 8 * b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (producer) asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tmap_x)) : "memory");
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
    const uint32_t idesc1 = tc_idesc(kTcM, kTcN1, 2u), idesc2 = tc_idesc(kTcM, kTcN2, 1u);
    const int tiles = (rows + kTcM - 1) / kTcM;
    auto stage_of = [](int kb) { return (kb + 2) % kTcStages; };
    auto sA = [&](int s) { return aRing + (uint32_t)(s * kTcBytesStage); };
    auto sB = [&](int s) { return aRing + (uint32_t)(s * kTcBytesStage + kTcBytesA); };
    auto bar = [&](int b) { return aBar + 8u * (uint32_t)b; };

    bool ok = true;          /* this thread's waits so far */
    bool failed = false;     /* CTA-uniform */
    uint32_t ph = 0;         /* parity bit per mbarrier, this thread's view */
    int nload[kTcStages] = {0, 0, 0}; /* producer: loads issued per stage */
    bool w2_issued = false;
    auto wait_bar = [&](int b) {
        if (ok) ok = tc_wait(bar(b), (ph >> b) & 1u);
        ph ^= 1u << b;
    };
    auto load_block = [&](int tile, int kb) {
        const int s = stage_of(kb);
        tc_expect(bar(kBarFull + s), (uint32_t)kTcBytesStage);
        tc_tma_load_2d(sA(s), &tmap_x, kb * kTcKB, tile * kTcM, bar(kBarFull + s));
        tc_bulk_load(sB(s), w1img + (size_t)kb * (kTcN1 * kTcKB), (uint32_t)kTcBytesB1, bar(kBarFull + s));
        nload[s]++;
    };

    int t = blockIdx.x;
    if (producer && t < tiles) {
        tc_expect(bar(kBarW2), (uint32_t)kTcBytesW2);
        tc_bulk_load(aW2, w2img, (uint32_t)kTcBytesW2, bar(kBarW2));
        w2_issued = true;
        load_block(t, 0);
        load_block(t, 1);
    }
    bool first = true;
    for (; t < tiles; t += gridDim.x) {
        const int r0 = t * kTcM, tn = t + (int)gridDim.x;
        /* ---- layer 1 ---- */
        if (producer) {
            for (int kb = 2; kb < kTcBlocks && ok; kb++) {
                if (kb >= 3) wait_bar(kBarEmpty + stage_of(kb)); /* MMAs of block kb - 3 */
                if (ok) load_block(t, kb);
            }
            /* the last three blocks' MMAs, in commit order */
            for (int kb = kTcBlocks - 3; kb < kTcBlocks; kb++) wait_bar(kBarEmpty + stage_of(kb));
            if (ok && tn < tiles) load_block(tn, 0); /* stage 2: clear of H1 */
        } else if (issuer) {
            for (int kb = 0; kb < kTcBlocks && ok; kb++) {
                const int s = stage_of(kb);
                wait_bar(kBarFull + s);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                for (int j = 0; j < kTcKB / 8; j++) {
                    const uint64_t da = tc_desc_sw128(sA(s) + 32u * j);
                    const uint64_t db = tc_desc(sB(s) + j * 2 * (kTcN1 / 8) * 128, (kTcN1 / 8) * 128, 128);
                    tc_mma_tf32(tmem, da, db, idesc1, (kb > 0 || j > 0) ? 1u : 0u);
                }
                tc_commit(bar(kBarEmpty + s));
            }
            if (ok) tc_commit(bar(kBarAcc));
        }
        __syncwarp();
        wait_bar(kBarAcc);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!__syncthreads_and(ok ? 1 : 0)) {
            failed = true;
            break;
        }
        __syncwarp();
        /* ---- epilogue 1: H1 = gelu(D1 + b1) as BF16 rows of the layer-2 A operand ---- */
        {
            const int r = warp * 32 + lane;
            for (int c0 = 0; c0 < kTcN1; c0 += 32) {
                float v[32];
                tc_ld32(tmem + ((uint32_t)(warp * 32) << 16) + c0, v);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    uint32_t w[4];
#pragma unroll
                    for (int i = 0; i < 4; i++) {
                        const int c = c0 + 8 * q + 2 * i;
                        w[i] = pack_bf16(gelu_f(v[8 * q + 2 * i] + sb1[c]), gelu_f(v[8 * q + 2 * i + 1] + sb1[c + 1]));
                    }
                    *reinterpret_cast<uint4 *>(sH1 + tc_off(r, c0 + 8 * q, kTcM)) = make_uint4(w[0], w[1], w[2], w[3]);
                }
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        /* ---- layer 2 ---- */
        if (issuer) {
            if (first) wait_bar(kBarW2);
            if (ok) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
                for (int j = 0; j < kTcN1 / 16; j++) {
                    const uint64_t da = tc_desc(aH1 + j * 2 * (kTcM / 8) * 128, (kTcM / 8) * 128, 128);
                    const uint64_t db = tc_desc(aW2 + j * 2 * (kTcN2 / 8) * 128, (kTcN2 / 8) * 128, 128);
                    tc_mma(tmem + kTcN1, da, db, idesc2, j > 0 ? 1u : 0u);
                }
                tc_commit(bar(kBarL2));
            }
        }
        first = false;
        __syncwarp();
        wait_bar(kBarL2);
        /* H1 consumed: the next tile's block 1 may overwrite stage 0 */
        if (producer && ok && tn < tiles) load_block(tn, 1);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (!__syncthreads_and(ok ? 1 : 0)) {
            failed = true;
            break;
        }
        /* ---- epilogue 2 and layer 3 ---- */
        {
            const int r = warp * 32 + lane, gr = r0 + r;
            float o0 = sb3[0], o1 = sb3[1];
            for (int c0 = 0; c0 < kTcN2; c0 += 32) {
                float v[32];
                tc_ld32(tmem + ((uint32_t)(warp * 32) << 16) + kTcN1 + c0, v);
#pragma unroll
                for (int i = 0; i < 32; i++) {
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
        /* TMEM columns 256.. are rewritten only after the next tile's layer 1 */
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (failed) {
        /* copies still in flight land before the CTA exits; MMAs get one more bounded wait */
        if (producer) {
            for (int s = 0; s < kTcStages; s++)
                if (nload[s] > 0) (void)tc_wait(bar(kBarFull + s), (uint32_t)(nload[s] - 1) & 1u);
            if (w2_issued) (void)tc_wait(bar(kBarW2), 0u);
        }
        if (issuer) {
            tc_commit(bar(kBarDrain));
            (void)tc_wait(bar(kBarDrain), 0u);
            if (err) atomicExch(err, 1);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

} /* namespace tp */
