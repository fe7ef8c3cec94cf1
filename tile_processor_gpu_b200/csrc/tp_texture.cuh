/*
 * tp_texture.cuh - texture tiles (the drop-in for the reference's
 * textures_accumulate, src/TileProcessor.cuh:2207-2579, with imclt8threads
 * :3847-4017, debayer_shot / debayer :4019-4199 and tile_combine_rgba
 * :4202-4665).
 *
 * One 128-thread block per listed tile (grid-stride).  Stage 1: twelve 8-lane
 * groups, one per (camera, color), low-pass the CLT tile, invert it (vertical
 * DCT-IV/DST-IV on the held column, transpose, horizontal pass on the held
 * row) and unfold it into a windowed 16x16 tile in shared memory.  Stage 2:
 * every thread takes pixels of all twelve tiles for the un-window / 3x3
 * debayer / shot-noise square root / re-window chain.  Stage 3: one thread per
 * pixel fuses the four cameras.  Stage 4: the slices are written as
 * non-overlapping 16x16 tiles and/or faded by the neighbour mask and added into
 * the overlapped RGBA image.
 */
#pragma once
#include "tp_common.cuh"

namespace tp {

struct TextureParams {
    int colors;
    float min_shot, scale_shot, diff_sigma;
    float w0, w1, w2;
    int dust_remove, keep_weights;
};

/* windowed inverse CLT of one job into a [16][17] tile (w * d, no accumulate).
 * Quadrant signs of the unfold (idct_signs, src/TileProcessor.cuh:399-420)
 * factor into a vertical and a horizontal sign vector. */
__device__ __forceinline__ void imclt_job(const float *__restrict__ src, const float *lpf,
                                          float *tb, float (*mout)[17], int l, unsigned gm)
{
    float y[4][8];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float col[8], v[8], row[8];
#pragma unroll
        for (int m = 0; m < 8; m++) {
            float x = __ldg(src + q * 64 + m * 8 + l);
            col[m] = lpf ? x * lpf[m * 8 + l] : x;
        }
        if (q >> 1) dtt8<1>(col, v); else dtt8<0>(col, v);
#pragma unroll
        for (int k = 0; k < 8; k++) tb[TBI(q, k, l)] = v[k];
        __syncwarp(gm);
#pragma unroll
        for (int k = 0; k < 8; k++) row[k] = tb[TBI(q, l, k)];
        __syncwarp(gm);
        if (q & 1) dtt8<1>(row, y[q]); else dtt8<0>(row, y[q]);
    }
    /* output rows whose fold index is l */
    const int ra = (l >= 4) ? l - 4 : 11 - l;
    const int rb = (l >= 4) ? 11 - l : 12 + l;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int r = h ? rb : ra;
        const int rq = r >> 2;
        const float svc = (rq == 0) ? 1.0f : -1.0f; /* cosine vertical */
        const float svs = (rq == 3) ? -1.0f : 1.0f; /* sine vertical   */
        const float wr = 0.5f * c_hwin[r];
#pragma unroll
        for (int c = 0; c < 16; c++) {
            const int v = (c < 4) ? c + 4 : (c < 12) ? 11 - c : c - 12;
            const int cq = c >> 2;
            const float shc = (cq == 0) ? 1.0f : -1.0f;
            const float shs = (cq == 3) ? -1.0f : 1.0f;
            const float d01 = (svc * shc) * y[0][v] + (svc * shs) * y[1][v];
            const float d23 = (svs * shc) * y[2][v] + (svs * shs) * y[3][v];
            const float w = wr * (0.5f * c_hwin[c]);
            mout[r][c] = w * (d01 + d23);
        }
    }
}

__device__ __forceinline__ int sym8(int i) { return (i & 8) ? (i ^ 15) : i; }

__global__ void __launch_bounds__(128) k_textures(
    Geom g, const int *__restrict__ woi, float *const *clt, long long num_texture_tiles,
    const int *__restrict__ list, const int *__restrict__ dev_counts, int count_slot, int list_cap,
    int border_quarter, const float *__restrict__ port_offsets, TextureParams p,
    size_t texture_rbg_stride, float *__restrict__ texture_rbg, size_t texture_stride,
    float *__restrict__ texture_tiles)
{
    __shared__ float s_m[12][16][17];      /* IMCLT tiles (not debayered)  */
    __shared__ float s_t[12][16][17];      /* un-windowed; later the slices */
    __shared__ union {
        float tb[12][kTB4];                /* stage-1 transposes           */
        float d[12][16][17];               /* debayered tiles              */
    } s_u;
    __shared__ float s_hsq[16], s_hsqi[16];

    const int tid = threadIdx.x;
    const int l = tid & 7, grp = tid >> 3;
    const unsigned gm = group_mask();
    const int colors = p.colors;
    const int njobs = 4 * colors;
    if (tid < 16) {
        const float s = c_hwin[tid];
        s_hsq[tid] = s * s;
        s_hsqi[tid] = 1.0f / (s * s);
    }

    long long count = num_texture_tiles;
    const int *lst = list;
    if (dev_counts) {
        /* sub-list length from the list builder, kept inside its quarter */
        count = dev_counts[count_slot];
        count = count < 0 ? 0 : (count > list_cap ? list_cap : count);
        if (border_quarter) lst = list + (border_quarter - count);
    }
    int wx0 = 0, wy0 = 0, wh = 0;
    if (texture_rbg && texture_rbg_stride) { wx0 = woi[0]; wy0 = woi[1]; wh = woi[3]; }
    const size_t slice_stride = texture_rbg_stride * (size_t)(wh + 1) * 8;
    const float ksigma = (float)(1.0 / (2.0 * (double)p.diff_sigma * (double)p.diff_sigma));
    float pd2r[6];
    {
        int k = 0;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = i + 1; j < 4; j++) {
                const float dx = port_offsets[2 * j] - port_offsets[2 * i];
                const float dy = port_offsets[2 * j + 1] - port_offsets[2 * i + 1];
                pd2r[k++] = ksigma / (dx * dx + dy * dy);
            }
    }
    const float chw[3] = {p.w0, p.w1, p.w2};
    __syncthreads();

    for (long long n = blockIdx.x; n < count; n += gridDim.x) {
        const int code = lst[n];
        const int tile = code >> 8;
        if (!(code & (1 << 7)) || tile < 0 || tile >= g.TX * g.TY) continue;

        /* ---- stage 1: LPF + inverse CLT per (camera, color) ---- */
        if (grp < njobs) {
            const int cam = grp / colors, color = grp - cam * colors;
            const float *src = clt[cam] + ((size_t)tile * 3 + color) * 256;
            imclt_job(src, c_lpf[colors > 1 ? color : 3], s_u.tb[grp], s_m[grp], l, gm);
        }
        __syncthreads();

        /* ---- stage 2: debayer with shot-noise correction ---- */
        if (colors > 1) {
            for (int e = tid; e < 12 * 256; e += 128) {
                const int j = e >> 8, r = (e >> 4) & 15, c = e & 15;
                s_t[j][r][c] = (s_m[j][r][c] * s_hsqi[sym8(c)]) * s_hsqi[sym8(r)];
            }
            __syncthreads();
            const float kshot = rsqrtf(p.min_shot);
            for (int e = tid; e < 12 * 256; e += 128) {
                const int j = e >> 8, r = (e >> 4) & 15, c = e & 15;
                const int color = j % 3;
                float v;
                if (r == 0 || r == 15 || c == 0 || c == 15) {
                    v = s_t[j][r][c];
                } else {
                    const float orth = ((s_t[j][r - 1][c] + s_t[j][r + 1][c]) + s_t[j][r][c - 1]) + s_t[j][r][c + 1];
                    if (color < 2) {
                        const float diag = ((s_t[j][r - 1][c - 1] + s_t[j][r - 1][c + 1]) + s_t[j][r + 1][c - 1]) + s_t[j][r + 1][c + 1];
                        v = (float)(0.0625 * (double)diag + 0.125 * (double)orth + 0.25 * (double)s_t[j][r][c]);
                    } else {
                        v = (float)(0.125 * (double)orth + 0.5 * (double)s_t[j][r][c]);
                    }
                }
                if (p.scale_shot > 0.0f) v = p.scale_shot * ((v > p.min_shot) ? sqrtf(v) : (kshot * v));
                s_u.d[j][r][c] = v * (s_hsq[sym8(c)] * s_hsq[sym8(r)]);
            }
        } else {
            for (int e = tid; e < 4 * 256; e += 128) {
                const int j = e >> 8, r = (e >> 4) & 15, c = e & 15;
                s_u.d[j][r][c] = s_m[j][r][c];
            }
        }
        __syncthreads();

        /* ---- stage 3: fuse the four cameras, one thread per pixel ---- */
        float(*out)[16][17] = s_t; /* 12 slices */
        for (int px = tid; px < 256; px += 128) {
            const int r = px >> 4, c = px & 15;
            float D[4][3], M[4][3];
#pragma unroll
            for (int cam = 0; cam < 4; cam++)
#pragma unroll
                for (int col = 0; col < 3; col++) {
                    if (col < colors) {
                        D[cam][col] = s_u.d[cam * colors + col][r][c];
                        M[cam][col] = s_m[cam * colors + col][r][c];
                    } else {
                        D[cam][col] = 0.0f;
                        M[cam][col] = 0.0f;
                    }
                }
            if (p.keep_weights) {
                float sw = 0.0f;
#pragma unroll
                for (int col = 0; col < 3; col++) {
                    if (col >= colors) break;
                    float s0 = 0.0f, s1 = 0.0f, s2 = 0.0f;
#pragma unroll
                    for (int cam = 0; cam < 4; cam++) {
                        s0 += 1.0f;
                        s1 += D[cam][col];
                        s2 = __fmaf_rn(D[cam][col], D[cam][col], s2);
                    }
                    const float mse = (s0 * s2 - s1 * s1) / (s0 * s0);
                    out[colors + 5 + col][r][c] = sqrtf(mse);
                    sw = __fmaf_rn(chw[col], mse, sw);
                }
                out[colors + 5 + colors][r][c] = sqrtf(sw);
            }
            const float wnd2 = s_hsq[sym8(r)] * s_hsq[sym8(c)];
            const float wi = (float)(1.0 / (double)wnd2);
            float pw[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            {
                int k = 0;
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = i + 1; j < 4; j++) {
                        float d = 0.0f;
#pragma unroll
                        for (int col = 0; col < 3; col++) {
                            if (col >= colors) break;
                            const float dc = (D[i][col] - D[j][col]) * wi;
                            d = __fmaf_rn(chw[col] * dc, dc, d);
                        }
                        const float e = (float)((double)expf(-pd2r[k] * d) + 0.0001);
                        pw[i] += e;
                        pw[j] += e;
                        k++;
                    }
            }
            int b1 = 0;
#pragma unroll
            for (int cam = 1; cam < 4; cam++) if (pw[cam] > pw[b1]) b1 = cam;
            int b2 = (b1 == 0) ? 1 : 0;
#pragma unroll
            for (int cam = 1; cam < 4; cam++) if (cam > b2 && cam != b1 && pw[cam] > pw[b2]) b2 = cam;
            const float w1 = pw[b1] / (pw[b1] + pw[b2]);
            const float w2 = 1.0f - w1;
            float avg[3];
#pragma unroll
            for (int col = 0; col < 3; col++) avg[col] = w1 * D[b1][col] + w2 * D[b2][col];
#pragma unroll
            for (int cam = 0; cam < 4; cam++) {
                float d2 = 0.0f;
#pragma unroll
                for (int col = 0; col < 3; col++) {
                    if (col >= colors) break;
                    const float dc = (D[cam][col] - avg[col]) * wi;
                    d2 = __fmaf_rn(chw[col] * dc, dc, d2);
                }
                pw[cam] = (float)((double)expf(-ksigma * d2) + 0.0001);
            }
            if (p.dust_remove) {
                int worst = 0;
#pragma unroll
                for (int cam = 1; cam < 4; cam++) if (pw[cam] < pw[worst]) worst = cam;
                const float wv = pw[worst];
                float a = -wv;
#pragma unroll
                for (int cam = 0; cam < 4; cam++) a += pw[cam];
                a /= 3.0f;
                const float scale = (float)(1.0 + (double)(wv * (a - wv) / (a * a * 3.0f)));
#pragma unroll
                for (int cam = 0; cam < 4; cam++) if (cam != worst) pw[cam] *= scale;
                pw[worst] *= wv / a;
            }
            float ksum = 0.0f;
#pragma unroll
            for (int cam = 0; cam < 4; cam++) ksum += pw[cam];
            const float kinv = (float)(1.0 / (double)ksum);
#pragma unroll
            for (int col = 0; col < 3; col++) {
                if (col >= colors) break;
                float v = 0.0f;
#pragma unroll
                for (int cam = 0; cam < 4; cam++) v = __fmaf_rn(kinv * pw[cam], M[cam][col], v);
                out[col][r][c] = v;
            }
            out[colors][r][c] = wnd2 * ksum / 4.0f;
#pragma unroll
            for (int cam = 0; cam < 4; cam++) out[colors + 1 + cam][r][c] = pw[cam];
        }
        __syncthreads();

        /* ---- stage 4: outputs ---- */
        if (texture_tiles && texture_stride) {
            const int ns = (colors == 3) ? (p.keep_weights ? 12 : 4) : (p.keep_weights ? 8 : 2);
            float *dst = texture_tiles + (size_t)n * texture_stride;
            for (int e = tid; e < ns * 256; e += 128) {
                const int s = e >> 8, r = (e >> 4) & 15, c = e & 15;
                dst[e] = out[s][r][c];
            }
        }
        const int nbr = code & TP_TASK_TEXTURE_BITS;
        if (texture_rbg && texture_rbg_stride && nbr) {
            const int ty = tile / g.TX, tx = tile - ty * g.TX;
            const long long x0 = (long long)(tx - wx0) * 8, y0 = (long long)(ty - wy0) * 8;
            for (int e = tid; e < (colors + 1) * 256; e += 128) {
                const int s = e >> 8, r = (e >> 4) & 15, c = e & 15;
                float v = out[s][r][c];
                if (nbr != TP_TASK_TEXTURE_BITS) v *= c_alpha_fade[nbr][r * 16 + c];
                const long long gy = y0 + r, gx = x0 + c;
                if (gy < 0 || gx < 0) continue;
                float *pdst = texture_rbg + (size_t)s * slice_stride + (size_t)gy * texture_rbg_stride + (size_t)gx;
                *pdst += v;
            }
        }
        __syncthreads();
    }
}

} /* namespace tp */
