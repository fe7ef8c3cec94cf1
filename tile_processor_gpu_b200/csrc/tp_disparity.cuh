/*
 * tp_disparity.cuh - residual disparity of each tile from its pair
 * correlations (the consumer of correlate2D).
 *
 * The reference stops at the correlation tiles (src/TileProcessor.cuh:
 * 1176-1443) and leaves the disparity fit to its Java caller, which is not
 * part of it; this is the plain fit the library defines.  Pair p = (i, j) of a
 * tile correlates with its peak at rho * b_p, b_p = port_offsets[j] -
 * port_offsets[i] (pairs as src/TileProcessor.cuh:484-490) and rho the
 * residual disparity (true minus task disparity).  The tile's profile is
 *   S(k) = sum over its listed pairs in pair_mask of C_p(k * b_p),
 * k = -r..r, C_p sampled bilinearly in the centred (2r+1)^2 tile; a k whose
 * sample of any contributing pair leaves the tile is not used.  rho is the
 * sub-pixel maximum of S around its first integer argmax k* (double
 * precision):
 *   mode 0: parabola through S(k*-1), S(k*), S(k*+1);
 *   mode 1: least-squares parabola through the valid S(k*-2 .. k*+2);
 *   mode 2: centroid of S - min over k*-1 .. k*+1.
 * The sub-pixel offset is kept within [-1, 1]; a fit without a maximum gives
 * k*.  strength = the fitted peak value / number of pairs.
 *
 * One warp per correlation entry; the warp that holds the first entry of a
 * tile's run (entries of one tile adjacent in the list) fits the tile, lane k
 * evaluating S(k - r).
 */
#pragma once
#include "tp_common.cuh"

namespace tp {

/* bilinear sample of a centred (2r+1)^2 tile c at (x, y); false outside */
__device__ __forceinline__ bool corr_sample(const float *__restrict__ c, int r, float x, float y, float *out)
{
    const float fx0 = floorf(x), fy0 = floorf(y);
    const int ix = (int)fx0, iy = (int)fy0;
    const float fx = x - fx0, fy = y - fy0;
    const int n = 2 * r + 1;
    if (ix < -r || iy < -r || ix > r || iy > r) return false;
    if ((fx > 0.0f && ix + 1 > r) || (fy > 0.0f && iy + 1 > r)) return false;
    const float *p = c + (iy + r) * n + ix + r;
    float v = (1.0f - fx) * (1.0f - fy) * __ldg(p);
    if (fx > 0.0f) v = __fmaf_rn(fx * (1.0f - fy), __ldg(p + 1), v);
    if (fy > 0.0f) v = __fmaf_rn((1.0f - fx) * fy, __ldg(p + n), v);
    if (fx > 0.0f && fy > 0.0f) v = __fmaf_rn(fx * fy, __ldg(p + n + 1), v);
    *out = v;
    return true;
}

/* sub-pixel step on s[t + 2] = S(k* + t), t = -2..2 (ok[]: usable) */
__device__ __forceinline__ void fit_peak(const double s[5], const bool ok[5], int mode, double *off_out,
                                         double *peak_out)
{
    double off = 0.0, pk = s[2];
    if (mode == 0) {
        if (ok[1] && ok[3]) {
            const double a = s[1], b = s[2], c = s[3];
            const double den = a - 2.0 * b + c;
            if (den < 0.0) {
                off = fmin(1.0, fmax(-1.0, 0.5 * (a - c) / den));
                pk = b - 0.25 * (a - c) * off;
            }
        }
    } else if (mode == 1) {
        /* normal equations of y = a + b t + c t^2 over the usable points */
        double m0 = 0, m1 = 0, m2 = 0, m3 = 0, m4 = 0, z0 = 0, z1 = 0, z2 = 0;
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < 5; i++) {
            if (!ok[i]) continue;
            const double t = i - 2, t2 = t * t;
            m0 += 1.0; m1 += t; m2 += t2; m3 += t2 * t; m4 += t2 * t2;
            z0 += s[i]; z1 += t * s[i]; z2 += t2 * s[i];
            cnt++;
        }
        if (cnt >= 3) {
            /* Cramer's rule on [m0 m1 m2; m1 m2 m3; m2 m3 m4] */
            const double c00 = m2 * m4 - m3 * m3, c01 = m1 * m4 - m3 * m2, c02 = m1 * m3 - m2 * m2;
            const double det = m0 * c00 - m1 * c01 + m2 * c02;
            if (det != 0.0) {
                const double a = (z0 * c00 - m1 * (z1 * m4 - m3 * z2) + m2 * (z1 * m3 - m2 * z2)) / det;
                const double b = (m0 * (z1 * m4 - z2 * m3) - z0 * c01 + m2 * (m1 * z2 - z1 * m2)) / det;
                const double c = (m0 * (m2 * z2 - m3 * z1) - m1 * (m1 * z2 - m3 * z0) + z0 * c02) / det;
                if (c < 0.0) {
                    off = fmin(1.0, fmax(-1.0, -b / (2.0 * c)));
                    pk = a + b * off + c * off * off;
                }
            }
        }
    } else {
        if (ok[1] && ok[3]) {
            const double a = s[1], b = s[2], c = s[3];
            const double m = fmin(a, fmin(b, c));
            const double w = (a - m) + (b - m) + (c - m);
            if (w > 0.0) off = ((c - m) - (a - m)) / w;
        }
    }
    *off_out = off;
    *peak_out = pk;
}

__global__ void __launch_bounds__(256) k_disparity_fit(int ntiles, const float *__restrict__ corrs,
                                                       size_t corr_stride, int r, long long num,
                                                       const int *__restrict__ idx,
                                                       const float *__restrict__ port_offsets, int pair_mask,
                                                       int mode, float *__restrict__ disparity,
                                                       float *__restrict__ strength)
{
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    float bx[6], by[6];
#pragma unroll
    for (int p = 0; p < 6; p++) {
        const int i = c_pairs[p][0], j = c_pairs[p][1];
        bx[p] = __ldg(&port_offsets[2 * j]) - __ldg(&port_offsets[2 * i]);
        by[p] = __ldg(&port_offsets[2 * j + 1]) - __ldg(&port_offsets[2 * i + 1]);
    }
    const int n = 2 * r + 1;
    for (long long e = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); e < num; e += warps) {
        const int tile = __ldg(&idx[e]) >> 8;
        if (e > 0 && (__ldg(&idx[e - 1]) >> 8) == tile) continue; /* not the first entry of the tile */
        if (tile < 0 || tile >= ntiles) continue;
        const float k = (float)(lane - r);
        float S = 0.0f;
        bool valid = lane < n;
        int npairs = 0;
        /* the first 8 entries of the run in one load, lane j holding e + j */
        const int mycode = (lane < 8 && e + lane < num) ? __ldg(&idx[e + lane]) : -1;
        const unsigned same = __ballot_sync(0xffffffffu, lane < 8 && e + lane < num && (mycode >> 8) == tile);
        const int m = __ffs(~same) - 1; /* run length within the first 8 */
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int code = __shfl_sync(0xffffffffu, mycode, j);
            if (j >= m) break;
            const int p = code & 0xff;
            if (p > 5 || !((pair_mask >> p) & 1)) continue;
            npairs++;
            if (lane < n) {
                float v;
                if (corr_sample(corrs + (size_t)(e + j) * corr_stride, r, k * bx[p], k * by[p], &v))
                    S += v;
                else
                    valid = false;
            }
        }
        /* runs longer than 8 (repeated pairs) */
        for (long long e2 = e + 8; m == 8 && e2 < num; e2++) {
            const int code = __ldg(&idx[e2]);
            if ((code >> 8) != tile) break;
            const int p = code & 0xff;
            if (p > 5 || !((pair_mask >> p) & 1)) continue;
            npairs++;
            if (lane < n) {
                float v;
                if (corr_sample(corrs + (size_t)e2 * corr_stride, r, k * bx[p], k * by[p], &v))
                    S += v;
                else
                    valid = false;
            }
        }
        if (!npairs) continue;
        /* first (lowest k) maximum over the usable lanes */
        float best = valid ? S : -INFINITY;
        int bk = valid ? lane : 64;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_down_sync(0xffffffffu, best, o);
            const int ok = __shfl_down_sync(0xffffffffu, bk, o);
            if (ok < 64 && (bk == 64 || ob > best || (ob == best && ok < bk))) { best = ob; bk = ok; }
        }
        const int km = __shfl_sync(0xffffffffu, bk, 0);
        if (km == 64) continue; /* no usable k */
        double s5[5];
        bool ok5[5];
#pragma unroll
        for (int t = -2; t <= 2; t++) {
            const int src = km + t;
            const int srcc = src < 0 ? 0 : (src > 31 ? 31 : src);
            const float sv = __shfl_sync(0xffffffffu, S, srcc);
            const int vv = __shfl_sync(0xffffffffu, (int)valid, srcc);
            s5[t + 2] = (double)sv;
            ok5[t + 2] = src >= 0 && src < n && vv;
        }
        if (lane == 0) {
            double off, pk;
            fit_peak(s5, ok5, mode, &off, &pk);
            disparity[tile] = (float)((double)(km - r) + off);
            strength[tile] = (float)(pk / npairs);
        }
    }
}

} /* namespace tp */
