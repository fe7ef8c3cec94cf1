/*
 * tp_imclt.cuh - inverse CLT of one color plane into an image by overlap-add
 * (the drop-in for the reference's imclt_rbg, src/TileProcessor.cuh:2588-2710,
 * with imclt :3700-3835).
 *
 * One 8-lane group per tile of the parity pass.  The group inverts the four
 * quadrants (vertical pass on held columns, transpose, horizontal pass on held
 * rows), stages the signed unfolded 16x16 tile in its shared buffer and then
 * read-modify-writes the image with each lane owning two columns, so every row
 * access of the group is two 32-byte segments.  Accumulation uses the
 * reference's round-down fused multiply-add, w * d + previous.
 */
#pragma once
#include "tp_common.cuh"

namespace tp {

__global__ void __launch_bounds__(256) k_imclt_rbg(Geom g, const float *__restrict__ clt,
                                                   float *__restrict__ rbg, int color, int v_offset,
                                                   int h_offset, size_t dstride)
{
    __shared__ float tbuf[256 / 8][kTB4];
    const int l = threadIdx.x & 7;
    const int grp = threadIdx.x >> 3;
    const unsigned gm = group_mask();
    float *tb = tbuf[grp];
    const int txh = (g.TX + (h_offset ^ 1)) >> 1;
    const int tyh = (g.TY + (v_offset ^ 1)) >> 1;
    const long long ntl = (long long)txh * tyh;
    const long long groups_total = (long long)gridDim.x * (blockDim.x >> 3);
    const int pass = (v_offset << 1) + h_offset;
    float *plane = rbg + dstride * (size_t)(g.H + 8) * color;
    for (long long n = (long long)blockIdx.x * (blockDim.x >> 3) + grp; n < ntl; n += groups_total) {
        const int ty = 2 * (int)(n / txh) + v_offset;
        const int tx = 2 * (int)(n % txh) + h_offset;
        const float *src = clt + (((size_t)ty * g.TX + tx) * 3 + color) * 256;
        float y[4][8];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            float col[8], v[8], row[8];
#pragma unroll
            for (int m = 0; m < 8; m++) col[m] = __ldg(src + q * 64 + m * 8 + l);
            if (q >> 1) dtt8<1>(col, v); else dtt8<0>(col, v);
#pragma unroll
            for (int k = 0; k < 8; k++) tb[TBI(q, k, l)] = v[k];
            __syncwarp(gm);
#pragma unroll
            for (int k = 0; k < 8; k++) row[k] = tb[TBI(q, l, k)];
            __syncwarp(gm);
            if (q & 1) dtt8<1>(row, y[q]); else dtt8<0>(row, y[q]);
        }
        /* signed unfold (idct_signs) into the group buffer as [16][17] */
        const int ra = (l >= 4) ? l - 4 : 11 - l;
        const int rb = (l >= 4) ? 11 - l : 12 + l;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int r = h ? rb : ra;
            const int rq = r >> 2;
            const float svc = (rq == 0) ? 1.0f : -1.0f;
            const float svs = (rq == 3) ? -1.0f : 1.0f;
#pragma unroll
            for (int c = 0; c < 16; c++) {
                const int v = (c < 4) ? c + 4 : (c < 12) ? 11 - c : c - 12;
                const int cq = c >> 2;
                const float shc = (cq == 0) ? 1.0f : -1.0f;
                const float shs = (cq == 3) ? -1.0f : 1.0f;
                const float d01 = (svc * shc) * y[0][v] + (svc * shs) * y[1][v];
                const float d23 = (svs * shc) * y[2][v] + (svs * shs) * y[3][v];
                tb[r * 17 + c] = d01 + d23;
            }
        }
        __syncwarp(gm);
        float *top = plane + (size_t)ty * 8 * dstride + (size_t)tx * 8;
        const bool mark0 = g.debug_marks && tx == 0 && ty == 0;
        const bool mark2 = g.debug_marks && tx == 161 && ty == 111;
#pragma unroll
        for (int hc = 0; hc < 2; hc++) {
            const int c = l + 8 * hc;
            const float wc = 0.5f * __ldg(&d_hwin[c]);
            for (int r = 0; r < 16; r++) {
                const float w = (0.5f * c_hwin[r]) * wc;
                float *px = top + (size_t)r * dstride + c;
                const float prev = pass ? *px : 0.0f;
                float val = __fmaf_rd(w, tb[r * 17 + c], prev);
                if (mark0) val = 100.0f;
                else if (mark2) val *= 2.0f;
                *px = val;
            }
        }
        __syncwarp(gm);
    }
}

} /* namespace tp */
