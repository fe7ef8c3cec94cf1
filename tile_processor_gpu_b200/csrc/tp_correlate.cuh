/*
 * tp_correlate.cuh - pairwise phase correlation (the drop-in for the
 * reference's correlate2D, src/TileProcessor.cuh:1176-1443, with its helpers
 * correlateAccumulateTiles :2829-2890, normalizeTileAmplitude :2915-2942 and
 * corrUnfoldTile :2950-3008).
 *
 * One 8-lane group per (tile, pair) entry of the index list.  Lane l holds
 * row l of the four accumulated quadrants, loaded as 16-byte vectors; the
 * color accumulation, the two LPFs and the amplitude normalisation are per
 * coefficient; the horizontal DCT-II/DST-II runs on the held row, one
 * shared-memory transpose per quadrant gives columns for the vertical pass
 * (the separable transform in the other order), and the unfold into the
 * (2r+1)^2 output reads the pixel-domain quadrants back from shared memory.
 * The output tile is staged in shared memory and written as consecutive
 * floats.
 */
#pragma once
#include "tp_common.cuh"

namespace tp {

/* per-group buffer: four 8x9 quadrant transposes; 296 % 32 == 8 */
constexpr int kCorrBuf = 4 * 72 + 8;

/* 4 consecutive floats at p (16-byte aligned when al16) */
__device__ __forceinline__ void load_row4(const float *p, bool al16, float v[4])
{
    if (al16) {
        const float4 x = *reinterpret_cast<const float4 *>(p);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] = p[k];
    }
}

/* 8 consecutive floats at p (16-byte aligned when al16) */
__device__ __forceinline__ void load_row8(const float *p, bool al16, float v[8])
{
    if (al16) {
        const float4 x = *reinterpret_cast<const float4 *>(p), y = *reinterpret_cast<const float4 *>(p + 4);
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w; v[4] = y.x; v[5] = y.y; v[6] = y.z; v[7] = y.w;
    } else {
#pragma unroll
        for (int k = 0; k < 8; k++) v[k] = p[k];
    }
}

/* One (tile, pair) correlation on an 8-lane group.  a, b: the two cameras'
 * CLT of the tile, colour c at a + c * cstride (4 x 64 floats, row stride 8);
 * global or shared.  tb: kCorrBuf floats of this group.  dst: (2r+1)^2
 * floats.  KC: coefficients of the held rows loaded at a time (8: all 64
 * of both tiles' colour at once, as many loads in flight as possible from
 * global memory; 4: half the registers, for shared-memory sources).  The
 * arithmetic and its order do not depend on KC. */
template <int KC = 8>
__device__ __forceinline__ void corr_job(const float *a, const float *b, int cstride, int colors, float scale0,
                                         float scale1, float scale2, float fat_zero, int r, float *tb,
                                         float *__restrict__ dst, int l, unsigned gm)
{
    const int sz = 2 * r + 1;
    const bool al16 = !((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b) |
                         (uintptr_t)(cstride * sizeof(float))) & 15);
    float acc[4][8]; /* row l of each quadrant */
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int k = 0; k < 8; k++) acc[q][k] = 0.0f;
    for (int color = 0; color < colors; color++) {
        const float s = color == 0 ? scale0 : color == 1 ? scale1 : scale2;
        static_assert(KC == 8 || KC == 4, "chunk");
#pragma unroll
        for (int k0 = 0; k0 < 8; k0 += KC) {
            float A[4][8], B[4][8];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const float *pa = a + color * cstride + q * 64 + l * 8 + k0;
                const float *pb = b + color * cstride + q * 64 + l * 8 + k0;
                if (KC == 8) {
                    load_row8(pa, al16, A[q]);
                    load_row8(pb, al16, B[q]);
                } else {
                    load_row4(pa, al16, A[q]);
                    load_row4(pb, al16, B[q]);
                }
            }
#pragma unroll
            for (int kk = 0; kk < KC; kk++) {
                const int k = k0 + kk;
                const float a0 = A[0][kk], a1 = A[1][kk], a2 = A[2][kk], a3 = A[3][kk];
                const float b0 = B[0][kk], b1 = B[1][kk], b2 = B[2][kk], b3 = B[3][kk];
                /* CLT-domain correlation of the two tiles */
                const float r0 = __fmaf_rn(a3, b3, __fmaf_rn(a2, b2, __fmaf_rn(a1, b1, a0 * b0)));
                const float r1 = __fmaf_rn(a2, b3, __fmaf_rn(-a3, b2, __fmaf_rn(a0, b1, -a1 * b0)));
                const float r2 = __fmaf_rn(a1, b3, __fmaf_rn(a0, b2, __fmaf_rn(-a3, b1, -a2 * b0)));
                const float r3 = __fmaf_rn(a0, b3, __fmaf_rn(-a1, b2, __fmaf_rn(-a2, b1, a3 * b0)));
                acc[0][k] = __fmaf_rn(s, r0, acc[0][k]);
                acc[1][k] = __fmaf_rn(s, r1, acc[1][k]);
                acc[2][k] = __fmaf_rn(s, r2, acc[2][k]);
                acc[3][k] = __fmaf_rn(s, r3, acc[3][k]);
            }
        }
        if (color == 1) { /* LPF after red and blue */
            float f[8];
            load_row8(&d_lpf[4][l * 8], true, f);
#pragma unroll
            for (int k = 0; k < 8; k++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[q][k] *= f[k];
        }
    }
    /* amplitude normalisation with fat zero, then the final LPF */
    {
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
    /* pixel domain: horizontal DCT-II (q0,q2) / DST-II (q1,q3) on the held
     * row, transpose, vertical DCT-II (q0,q1) / DST-II (q2,q3) on the held
     * column: lane l ends holding column l of each quadrant, p[q][i] = row i */
    float p[4][8];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float v[8], col[8];
        if (q & 1) dtt8<3>(acc[q], v); else dtt8<2>(acc[q], v);
#pragma unroll
        for (int k = 0; k < 8; k++) tb[TBI(q, l, k)] = v[k];
        __syncwarp(gm);
#pragma unroll
        for (int k = 0; k < 8; k++) col[k] = tb[TBI(q, k, l)];
        if (q >> 1) dtt8<3>(col, p[q]); else dtt8<2>(col, p[q]);
    }
    __syncwarp(gm); /* the transpose buffer free for the group's next job */
    /* unfold, lane j = columns r +- j: R[+-i][+-j] from q0[i][j], q1[i][j-1]
     * (lane j - 1), q2[i-1][j], q3[i-1][j-1], scaled by 1/4, stored straight
     * to dst (each store of a group covers 8 consecutive floats of a row) */
    float q1l[8], q3l[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        q1l[i] = __shfl_up_sync(gm, p[1][i], 1, 8);
        q3l[i] = __shfl_up_sync(gm, p[3][i], 1, 8);
    }
    if (l <= r) {
        const int j = l;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if (i > r) break;
            const float q0 = p[0][i];
            const float q1 = j > 0 ? q1l[i] : 0.0f;
            const float q2 = i > 0 ? p[2][i - 1] : 0.0f;
            const float q3 = (i > 0 && j > 0) ? q3l[i - 1] : 0.0f;
            /* in this order: where i or j is 0 the later store to the same
             * element is the one that stays */
            float *up = dst + (r + i) * sz + r, *dn = dst + (r - i) * sz + r;
            up[j] = 0.25f * ((q0 + q1) + (q2 + q3));
            up[-j] = 0.25f * ((q0 - q1) + (q2 - q3));
            dn[j] = 0.25f * ((q0 + q1) - (q2 + q3));
            dn[-j] = 0.25f * ((q0 - q1) - (q2 - q3));
        }
    }
}

__global__ void __launch_bounds__(128, 4) k_correlate2D(Geom g, float *const *clt, int colors,
                                                        float scale0, float scale1, float scale2,
                                                        float fat_zero, long long num_corr_tiles,
                                                        const int *__restrict__ corr_indices,
                                                        size_t corr_stride, int corr_radius,
                                                        float *__restrict__ corrs)
{
    __shared__ float tbuf[128 / 8][kCorrBuf];
    const int l = threadIdx.x & 7;
    const int grp = threadIdx.x >> 3;
    const unsigned gm = group_mask();
    const long long groups_total = (long long)gridDim.x * (blockDim.x >> 3);
    const int ntiles = g.TX * g.TY;
    for (long long n = (long long)blockIdx.x * (blockDim.x >> 3) + grp; n < num_corr_tiles; n += groups_total) {
        const int code = corr_indices[n];
        const int tile = code >> 8, pair = code & 0xff;
        if (pair >= 6 || tile < 0 || tile >= ntiles) continue;
        const float *ta = clt[c_pairs[pair][0]] + (size_t)tile * 768;
        const float *tb2 = clt[c_pairs[pair][1]] + (size_t)tile * 768;
        corr_job(ta, tb2, 256, colors, scale0, scale1, scale2, fat_zero, corr_radius, tbuf[grp],
                 corrs + (size_t)n * corr_stride, l, gm);
    }
}

} /* namespace tp */
