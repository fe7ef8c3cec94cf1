/*
 * tp_corr_tc.cuh - pairwise phase correlation with the pixel-domain transform
 * on the tensor cores (the precision form of correlate2D,
 * src/TileProcessor.cuh:1176-1443).
 *
 * Same arithmetic as k_correlate2D up to the normalised, low-pass-filtered
 * CLT-domain product of a pair (correlateAccumulateTiles :2829-2890,
 * normalizeTileAmplitude :2915-2942); its four 8x8 quadrants then go through
 * the DCT-II / DST-II pairs of dttii_shared_mem_nonortho as four 64 x 64
 * GEMMs on the tensor cores (tp_tc_engine.cuh: split FP16 or BF16 operands,
 * FP32 accumulation), and corrUnfoldTile (:2950-3008) folds the pixel-domain
 * quadrants into the (2r+1)^2 output.
 *
 * Runs in the shared pipeline k_tc_stage (tp_tc_engine.cuh) over blocks of
 * 128 index entries: twelve producer warps, one 8-lane group per entry,
 * compute row l of the four accumulated quadrants and write them split into
 * the A image; four epilogue warps, one thread per entry, read the
 * pixel-domain quadrants row by row from tensor memory, unfold and store
 * them.
 *
 * FP16 rows are scaled by `up` (a power of two chosen by the host from the
 * final LPF's largest entry, which bounds the normalised product) so the hi
 * halves stay below 2^15; BF16 needs no scale.
 */
#pragma once
#include "tp_correlate.cuh"
#include "tp_tc_engine.cuh"

namespace tp {

/* The normalised, low-pass-filtered CLT-domain product of one (tile, pair)
 * entry, row l of the four quadrants in acc (k_correlate2D's first half). */
__device__ __forceinline__ void corr_product_rows(const float *a, const float *b, int cstride, int colors,
                                                  float scale0, float scale1, float scale2, float fat_zero,
                                                  int l, float acc[4][8])
{
    const bool al16 = !((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
                         (uintptr_t)(cstride * sizeof(float))) & 15);
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int k = 0; k < 8; k++) acc[q][k] = 0.0f;
    for (int color = 0; color < colors; color++) {
        const float s = color == 0 ? scale0 : color == 1 ? scale1 : scale2;
        float A[4][8], B[4][8];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            load_row8(a + color * cstride + q * 64 + l * 8, al16, A[q]);
            load_row8(b + color * cstride + q * 64 + l * 8, al16, B[q]);
        }
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const float a0 = A[0][k], a1 = A[1][k], a2 = A[2][k], a3 = A[3][k];
            const float b0 = B[0][k], b1 = B[1][k], b2 = B[2][k], b3 = B[3][k];
            const float r0 = __fmaf_rn(a3, b3, __fmaf_rn(a2, b2, __fmaf_rn(a1, b1, a0 * b0)));
            const float r1 = __fmaf_rn(a2, b3, __fmaf_rn(-a3, b2, __fmaf_rn(a0, b1, -a1 * b0)));
            const float r2 = __fmaf_rn(a1, b3, __fmaf_rn(a0, b2, __fmaf_rn(-a3, b1, -a2 * b0)));
            const float r3 = __fmaf_rn(a0, b3, __fmaf_rn(-a1, b2, __fmaf_rn(-a2, b1, a3 * b0)));
            acc[0][k] = __fmaf_rn(s, r0, acc[0][k]);
            acc[1][k] = __fmaf_rn(s, r1, acc[1][k]);
            acc[2][k] = __fmaf_rn(s, r2, acc[2][k]);
            acc[3][k] = __fmaf_rn(s, r3, acc[3][k]);
        }
        if (color == 1) {
            float f[8];
            load_row8(&d_lpf[4][l * 8], true, f);
#pragma unroll
            for (int k = 0; k < 8; k++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[q][k] *= f[k];
        }
    }
    float f[8];
    load_row8(&d_lpf[5][l * 8], true, f);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        float s2 = fat_zero * fat_zero;
#pragma unroll
        for (int q = 0; q < 4; q++) s2 = __fmaf_rn(acc[q][k], acc[q][k], s2);
        const float sc = rsqrtf(s2);
#pragma unroll
        for (int q = 0; q < 4; q++) acc[q][k] = (acc[q][k] * sc) * f[k];
    }
}

/* The correlation as a tensor-core stage (k_tc_stage): rows are index
 * entries; twelve producer warps (the CLT products are the heavy part), four
 * epilogue warps (512 threads, at most 128 registers each). */
struct CorrTcStage {
    static constexpr int kQuads = 4, kProdWarps = 12, kEpiWarps = 4;
    static constexpr int kThreads = 32 * (kProdWarps + kEpiWarps);
    static constexpr int kMeta = 1;
    static constexpr int kAStages = 1;
    Geom g;
    float *const *clt;
    int colors;
    float scale0, scale1, scale2, fat_zero;
    long long num;
    const int *idx;
    size_t stride;
    int radius;
    float *corrs;
    float up; /* FP16 row scale (a power of two); 1 for BF16 */

    __host__ __device__ __forceinline__ long long rows() const { return num; }

    __device__ __forceinline__ int entry(long long n, int *tile, int *pair) const
    {
        const int code = n < num ? __ldg(&idx[n]) : -1;
        *tile = code >> 8;
        *pair = code & 0xff;
        return code >= 0 && *pair < 6 && *tile < g.TX * g.TY;
    }

    template <int FMT>
    __device__ __forceinline__ void produce(long long n, int row, int l, unsigned gm, const TcA<4> &A,
                                            uint32_t *meta) const
    {
        (void)gm;
        (void)meta;
        int tile, pair;
        float acc[4][8];
        if (entry(n, &tile, &pair)) {
            corr_product_rows(clt[c_pairs[pair][0]] + (size_t)tile * 768, clt[c_pairs[pair][1]] + (size_t)tile * 768,
                              256, colors, scale0, scale1, scale2, fat_zero, l, acc);
        } else {
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int k = 0; k < 8; k++) acc[q][k] = 0.0f;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) A.template put8<FMT>(row, q, l * 8, acc[q], up);
    }

    /* corrUnfoldTile: R[+-i][+-j] from q0[i][j], q1[i][j-1], q2[i-1][j],
     * q3[i-1][j-1], x 1/4 (all lanes of the warp run it: the tensor-memory
     * loads are warp-wide) */
    __device__ __forceinline__ void epilogue(long long n, uint32_t tb, const uint32_t *meta, int part) const
    {
        (void)meta;
        (void)part;
        int tile, pair;
        const bool valid = entry(n, &tile, &pair);
        const int r = radius, sz = 2 * r + 1;
        const float down = 1.0f / up; /* a power of two: exact */
        float *dst = corrs + (size_t)(valid ? n : 0) * stride;
        float prev2[8], prev3[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            prev2[j] = 0.0f;
            prev3[j] = 0.0f;
        }
#pragma unroll 1
        for (int i = 0; i <= r; i++) {
            float v[4][8];
            tc_ld8x4(tb + 8u * i, tb + 64u + 8u * i, tb + 128u + 8u * i, tb + 192u + 8u * i, v);
            if (valid) {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if (j > r) break;
                    const float q0 = v[0][j] * down;
                    const float q1 = j > 0 ? v[1][j - 1] * down : 0.0f;
                    const float q2 = prev2[j];
                    const float q3 = j > 0 ? prev3[j - 1] : 0.0f;
                    dst[(r + i) * sz + (r + j)] = 0.25f * ((q0 + q1) + (q2 + q3));
                    dst[(r + i) * sz + (r - j)] = 0.25f * ((q0 - q1) + (q2 - q3));
                    dst[(r - i) * sz + (r + j)] = 0.25f * ((q0 + q1) - (q2 + q3));
                    dst[(r - i) * sz + (r - j)] = 0.25f * ((q0 - q1) - (q2 - q3));
                }
            }
#pragma unroll
            for (int j = 0; j < 8; j++) {
                prev2[j] = v[2][j] * down;
                prev3[j] = v[3][j] * down;
            }
        }
    }
};

} /* namespace tp */
