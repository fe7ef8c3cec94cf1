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

} /* namespace tp */
