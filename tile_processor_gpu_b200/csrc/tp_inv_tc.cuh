/*
 * tp_inv_tc.cuh - the inverse CLT of the texture stage on the tensor cores
 * (the precision form of imclt8threads, src/TileProcessor.cuh:3847-4017, as
 * textures_accumulate :2207-2579 uses it).
 *
 * A stage of the shared pipeline k_tc_stage (tp_tc_engine.cuh).  Rows are
 * (entry, camera, colour) jobs, 12 per entry; an entry is a task with texture
 * bits (tasks mode, after the texture-list kernels rewrote them) or a texture
 * list code (list mode).  Per job:
 *   producer (8-lane group, lane l = row l of each quadrant): the job's CLT
 *     times the colour's low-pass filter, scaled for FP16 by a power of two
 *     that brings the job's largest coefficient just under 2^15, split into
 *     the A image; the inverse of that scale is the row's metadata word;
 *   tensor cores: per quadrant the vertical and horizontal DCT-IV / DST-IV,
 *     Y_q = V_q X_q H_q^T (DST-IV vertically for q2, q3, horizontally for q1,
 *     q3);
 *   epilogue (one thread per job; two warps share a job, fold rows 0-3 and
 *     4-7): the unfold of the four pixel-domain quadrants into the 16x16 tile
 *     with the quadrant signs of idct_signs (:399-420), times the per-pixel
 *     factor of the tile the texture kernel's next step wants: the
 *     un-windowed tile T = d / (4 sin r sin c) for colour textures, the
 *     windowed M = (w_r / 2)(w_c / 2) d for mono; stored row-major [16][16]
 *     at the job's CLT offset of the tile buffer (the same layout as the CLT).
 * k_textures<true> then runs the debayer and the camera fusion from those
 * tiles.
 */
#pragma once
#include "tp_correlate.cuh"
#include "tp_tc_engine.cuh"
#include "tp_texture.cuh"

namespace tp {

struct InvTcStage {
    static constexpr int kQuads = 4, kProdWarps = 16, kEpiWarps = 8;
    static constexpr int kThreads = 32 * (kProdWarps + kEpiWarps);
    static constexpr int kMeta = 2;
    static constexpr int kAStages = 1;
    Geom g;
    float *const *clt;   /* in: per camera [tiles][3][256]                  */
    float *const *tiles; /* out: per camera [tiles][3][16][16]              */
    const tp_task *tasks;
    long long num;       /* entries: tasks, or list codes                    */
    const int *list;     /* NULL: tasks mode                                 */
    int colors;

    __host__ __device__ __forceinline__ long long rows() const { return 12 * num; }

    /* the job of row n: tile (or -1), camera and colour */
    __device__ __forceinline__ int job(long long n, int *cam, int *color) const
    {
        const long long e = n / 12;
        const int j = (int)(n - 12 * e);
        *cam = j / 3;
        *color = j - 3 * (j / 3);
        if (e >= num || *color >= colors) return -1;
        int tile;
        if (list) {
            const int code = __ldg(&list[e]);
            if (!(code & (1 << 7))) return -1;
            tile = code >> 8;
        } else {
            const tp_task *t = tasks + e;
            if (!(__ldg(&t->task) & TP_TASK_TEXTURE_BITS)) return -1;
            const int txy = __ldg(&t->txy);
            const int tx = txy & 0xffff, ty = txy >> 16;
            if (tx >= g.TX || ty < 0 || ty >= g.TY) return -1;
            tile = ty * g.TX + tx;
        }
        return (tile >= 0 && tile < g.TX * g.TY) ? tile : -1;
    }

    template <int FMT>
    __device__ __forceinline__ void produce(long long n, int row, int l, unsigned gm, const TcA<4> &A,
                                            uint32_t *meta) const
    {
        int cam, color;
        const int tile = job(n, &cam, &color);
        float x[4][8];
        if (tile >= 0) {
            const float *src = clt[cam] + ((size_t)tile * 3 + color) * 256 + l * 8;
            const bool al16 = !(reinterpret_cast<uintptr_t>(src) & 15);
            const float *lpf = d_lpf[colors > 1 ? color : 3] + l * 8;
            float f[8];
            load_row8(lpf, true, f);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                load_row8(src + q * 64, al16, x[q]);
#pragma unroll
                for (int k = 0; k < 8; k++) x[q][k] *= f[k];
            }
        } else {
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int k = 0; k < 8; k++) x[q][k] = 0.0f;
        }
        float up = 1.0f;
        if constexpr (FMT == TP_TC_FP16X2) {
            float mx = 0.0f;
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int k = 0; k < 8; k++) mx = fmaxf(mx, fabsf(x[q][k]));
            mx = fmaxf(mx, __shfl_xor_sync(gm, mx, 1));
            mx = fmaxf(mx, __shfl_xor_sync(gm, mx, 2));
            mx = fmaxf(mx, __shfl_xor_sync(gm, mx, 4));
            /* mx < 2^e with e = biased exponent - 126: scale by 2^(15 - e) */
            if (mx > 0.0f) {
                const int e = ((__float_as_int(mx) >> 23) & 0xff) - 126;
                up = __int_as_float(min(254, max(1, 127 + 15 - e)) << 23);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) A.template put8<FMT>(row, q, l * 8, x[q], up);
        if (l == 0) {
            meta[0] = __float_as_uint(1.0f / up);
            meta[1] = (uint32_t)tile;
        }
    }

    __device__ __forceinline__ void epilogue(long long n, uint32_t tb, const uint32_t *meta, int part) const
    {
        int cam, color;
        (void)job(n, &cam, &color);
        const int tile = (int)meta[1];
        const float down = __uint_as_float(meta[0]);
        float *dst = tile >= 0 ? tiles[cam] + ((size_t)tile * 3 + color) * 256 : nullptr;
        const float *fac = colors > 1 ? d_tex_tfac : d_tex_mfac;
#pragma unroll 1
        for (int l = 4 * part; l < 4 * part + 4; l++) {
            float a[4][8];
            tc_ld8x4(tb + 8u * l, tb + 64u + 8u * l, tb + 128u + 8u * l, tb + 192u + 8u * l, a);
            if (!dst) continue;
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int v = 0; v < 8; v++) a[q][v] *= down;
            /* the two output rows folding onto row l (rows 0-3: +,+; 4-7: -,+;
             * 8-11: -,+; 12-15: -,-) */
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = (l >= 4) ? (h ? 11 - l : l - 4) : (h ? l + 12 : 11 - l);
                const int rq = r >> 2;
                const bool n01 = rq != 0, n23 = rq == 3;
                float o[16];
#pragma unroll
                for (int c = 0; c < 16; c++) {
                    const int v = (c < 4) ? c + 4 : (c < 12) ? 11 - c : c - 12;
                    const int cq = c >> 2;
                    const float e0 = (cq == 0) ? a[0][v] + a[1][v] : (cq == 3) ? -a[0][v] - a[1][v] : a[1][v] - a[0][v];
                    const float e1 = (cq == 0) ? a[2][v] + a[3][v] : (cq == 3) ? -a[2][v] - a[3][v] : a[3][v] - a[2][v];
                    const float d = (n01 ? -e0 : e0) + (n23 ? -e1 : e1);
                    o[c] = d * __ldg(&fac[r * 17 + c]);
                }
                if (!(reinterpret_cast<uintptr_t>(dst) & 15)) {
                    float4 *p = reinterpret_cast<float4 *>(dst + r * 16);
#pragma unroll
                    for (int k = 0; k < 4; k++) p[k] = make_float4(o[4 * k], o[4 * k + 1], o[4 * k + 2], o[4 * k + 3]);
                } else {
#pragma unroll
                    for (int c = 0; c < 16; c++) dst[r * 16 + c] = o[c];
                }
            }
        }
    }
};

} /* namespace tp */
