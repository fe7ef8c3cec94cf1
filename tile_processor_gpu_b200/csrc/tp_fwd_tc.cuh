/*
 * tp_fwd_tc.cuh - the forward CLT with aberration correction with its 2-D
 * DCT-IV / DST-IV on the tensor cores (the precision form of
 * convert_correct_tiles, src/TileProcessor.cuh:1859-1937, convertCorrectTile
 * :3106-3635).
 *
 * A stage of the shared pipeline k_tc_stage (tp_tc_engine.cuh), two
 * quadrant slots.  Rows are (task, camera, colour) jobs, 12 per task.
 *   producer (8-lane group, lane l): the job's kernel tile, window corner and
 *     residual shifts (job_geometry), the fold of the windowed Bayer samples
 *     into DTT row l (fold_rows: P for the CC quadrant, and for green Q, the
 *     sine-windowed fold for SC), scaled for FP16 by a power of two, split
 *     into the A image; lane l also computes the horizontal shift rotation of
 *     column l and the vertical one of row l.  Metadata words: the inverse
 *     scale, the kernel tile, the corner parities, the tile, then the 32
 *     rotation cosines and sines;
 *   tensor cores: CC = C4 P C4^T (slot 0) and, for green, SC = C4 Q S4^T
 *     (slot 1; red and blue give zeros there);
 *   epilogue (one thread per job; two warps share a job, CC rows {0, 7, 1, 6}
 *     and {2, 5, 3, 4}): the missing quadrants from the Bayer mirror
 *     symmetries (red / blue SC[i][j] = +-CC[i][7-j]; CS[i][j] =
 *     +-SC[7-i][7-j], SS[i][j] = +-CC[7-i][7-j], :3459-3504), the CLT-domain
 *     convolution with the kernel tile (convolveTiles :2778-2827), the
 *     horizontal then vertical shift rotations (shiftTileHor / shiftTileVert
 *     :2715-2776), the optional LPF, and the store of the job's 4 x 64
 *     coefficients.
 */
#pragma once
#include "tp_convert.cuh"
#include "tp_correlate.cuh"
#include "tp_tc_engine.cuh"

namespace tp {

struct FwdTcStage {
    static constexpr int kQuads = 2, kProdWarps = 16, kEpiWarps = 8;
    static constexpr int kThreads = 32 * (kProdWarps + kEpiWarps);
    static constexpr int kMeta = 36;
    /* One A image: a second slot (double buffering) measured 15% slower, the
     * larger shared-memory carve-out leaving less L1 for the producers' loads. */
    static constexpr int kAStages = 1;
    Geom g;
    size_t dstride;
    float *const *kernel_offsets;
    float *const *kernels;
    float *const *images;
    const tp_task *tasks;
    float *const *clt;
    int num_tiles;
    int lpf_mask;

    __host__ __device__ __forceinline__ long long rows() const { return 12LL * num_tiles; }

    /* task, camera and colour of row n; the tile (or -1) */
    __device__ __forceinline__ int job(long long n, int *cam, int *color, float *cx, float *cy) const
    {
        const long long t = n / 12;
        const int j = (int)(n - 12 * t);
        *cam = j / 3;
        *color = j - 3 * (j / 3);
        if (t >= num_tiles) return -1;
        const tp_task *tk = tasks + t;
        if (!__ldg(&tk->task)) return -1;
        const int txy = __ldg(&tk->txy);
        const int tx = txy & 0xfff, ty = txy >> 16;
        if (tx >= g.TX || ty < 0 || ty >= g.TY) return -1;
        *cx = __ldg(&tk->xy[*cam][0]);
        *cy = __ldg(&tk->xy[*cam][1]);
        return ty * g.TX + tx;
    }

    template <int FMT>
    __device__ __forceinline__ void produce(long long n, int row, int l, unsigned gm, const TcA<2> &A,
                                            uint32_t *meta) const
    {
        int cam, color;
        float cx = 0.0f, cy = 0.0f;
        const int tile = job(n, &cam, &color, &cx, &cy);
        float P[8], Q[8];
        float rot[4] = {1.0f, 0.0f, 1.0f, 0.0f};
        JobGeometry jg;
        jg.kidx = 0;
        jg.itlx = jg.itly = 0;
        if (tile >= 0) {
            jg = job_geometry(g, kernel_offsets[cam], cx, cy, color, nullptr);
            fold_rows(g, dstride, images[cam], jg, color, l, P, Q);
            /* the rotation angles of column l (horizontal) and row l (vertical) */
            sincospif((jg.shx * (float)(2 * l + 1)) * 0.0625f, &rot[1], &rot[0]);
            sincospif((jg.shy * (float)(2 * l + 1)) * 0.0625f, &rot[3], &rot[2]);
        } else {
#pragma unroll
            for (int v = 0; v < 8; v++) {
                P[v] = 0.0f;
                Q[v] = 0.0f;
            }
        }
        float up = 1.0f;
        if constexpr (FMT == TP_TC_FP16X2) {
            float mx = 0.0f;
#pragma unroll
            for (int v = 0; v < 8; v++) mx = fmaxf(mx, fmaxf(fabsf(P[v]), fabsf(Q[v])));
            mx = fmaxf(mx, __shfl_xor_sync(gm, mx, 1));
            mx = fmaxf(mx, __shfl_xor_sync(gm, mx, 2));
            mx = fmaxf(mx, __shfl_xor_sync(gm, mx, 4));
            if (mx > 0.0f) {
                const int e = ((__float_as_int(mx) >> 23) & 0xff) - 126;
                up = __int_as_float(min(254, max(1, 127 + 15 - e)) << 23);
            }
        }
        A.template put8<FMT>(row, 0, l * 8, P, up);
        A.template put8<FMT>(row, 1, l * 8, Q, up);
        if (l == 0) {
            meta[0] = __float_as_uint(1.0f / up);
            meta[1] = tile >= 0 ? (uint32_t)jg.kidx : 0xffffffffu;
            meta[2] = (uint32_t)((jg.itlx & 1) | ((jg.itly & 1) << 1));
            meta[3] = (uint32_t)tile;
        }
        meta[4 + l] = __float_as_uint(rot[0]);  /* cos, column l */
        meta[12 + l] = __float_as_uint(rot[1]); /* sin, column l */
        meta[20 + l] = __float_as_uint(rot[2]); /* cos, row l    */
        meta[28 + l] = __float_as_uint(rot[3]); /* sin, row l    */
    }

    __device__ __forceinline__ void epilogue(long long n, uint32_t tb, const uint32_t *meta, int part) const
    {
        const bool valid = meta[1] != 0xffffffffu;
        const long long t = n / 12;
        const int jj = (int)(n - 12 * t), cam = jj / 3, color = jj - 3 * (jj / 3);
        const float down = __uint_as_float(meta[0]);
        const int c1 = (color >> 1) & 1;
        const int px = (int)(meta[2] & 1u), py = (int)((meta[2] >> 1) & 1u);
        const float neg1 = 1.0f - 2.0f * (float)(px ^ (1 ^ color));
        const float neg2 = 1.0f - 2.0f * (float)(px ^ py ^ 1 ^ c1);
        const bool lpf = (lpf_mask >> color) & 1;
        const float *kr = valid ? kernels[cam] + (size_t)meta[1] * 256 : nullptr;
        float *out = valid ? clt[cam] + ((size_t)meta[3] * 3 + color) * 256 : nullptr;
        const bool k16 = valid && !(reinterpret_cast<uintptr_t>(kr) & 15);
        const bool o16 = valid && !(reinterpret_cast<uintptr_t>(out) & 15);
#pragma unroll 1
        for (int mm = 0; mm < 2; mm++) {
            const int m = 2 * part + mm;
            float v[4][8]; /* CC[m], CC[7-m], SC[m], SC[7-m] */
            tc_ld8x4(tb + 8u * m, tb + 8u * (7 - m), tb + 64u + 8u * m, tb + 64u + 8u * (7 - m), v);
            if (!valid) continue;
#pragma unroll
            for (int q = 0; q < 4; q++)
#pragma unroll
                for (int j = 0; j < 8; j++) v[q][j] *= down;
            if (!c1) { /* red, blue: SC[i][j] = +-CC[i][7-j] */
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    v[2][j] = neg1 * v[0][7 - j];
                    v[3][j] = neg1 * v[1][7 - j];
                }
            }
#pragma unroll
            for (int side = 0; side < 2; side++) {
                const int i = side ? 7 - m : m;
                const float *cc = v[side], *sc = v[2 + side], *ccm = v[1 - side], *scm = v[3 - side];
                const float cv = __uint_as_float(meta[20 + i]), sv = __uint_as_float(meta[28 + i]);
                float k[4][8];
#pragma unroll
                for (int q = 0; q < 4; q++) load_row8(kr + q * 64 + i * 8, k16, k[q]);
                float o[4][8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const float a0 = cc[j], a1 = sc[j];
                    const float a2 = neg2 * scm[7 - j], a3 = neg2 * ccm[7 - j];
                    const float k0 = k[0][j], k1 = k[1][j], k2 = k[2][j], k3 = k[3][j];
                    float x0 = __fmaf_rn(a3, k3, __fmaf_rn(-a2, k2, __fmaf_rn(-a1, k1, a0 * k0)));
                    float x1 = __fmaf_rn(-a2, k3, __fmaf_rn(-a3, k2, __fmaf_rn(a0, k1, a1 * k0)));
                    float x2 = __fmaf_rn(-a1, k3, __fmaf_rn(a0, k2, __fmaf_rn(-a3, k1, a2 * k0)));
                    float x3 = __fmaf_rn(a0, k3, __fmaf_rn(a1, k2, __fmaf_rn(a2, k1, a3 * k0)));
                    /* horizontal shift (column j), then vertical (row i) */
                    const float ch = __uint_as_float(meta[4 + j]), sh = __uint_as_float(meta[12 + j]);
                    const float y0 = x0 * ch - x1 * sh, y1 = x0 * sh + x1 * ch;
                    const float y2 = x2 * ch - x3 * sh, y3 = x2 * sh + x3 * ch;
                    o[0][j] = y0 * cv - y2 * sv;
                    o[2][j] = y0 * sv + y2 * cv;
                    o[1][j] = y1 * cv - y3 * sv;
                    o[3][j] = y1 * sv + y3 * cv;
                    if (lpf) {
                        const float f = __ldg(&d_lpf[color][i * 8 + j]);
#pragma unroll
                        for (int q = 0; q < 4; q++) o[q][j] *= f;
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    float *d = out + q * 64 + i * 8;
                    if (o16) {
                        reinterpret_cast<float4 *>(d)[0] = make_float4(o[q][0], o[q][1], o[q][2], o[q][3]);
                        reinterpret_cast<float4 *>(d)[1] = make_float4(o[q][4], o[q][5], o[q][6], o[q][7]);
                    } else {
#pragma unroll
                        for (int j = 0; j < 8; j++) d[j] = o[q][j];
                    }
                }
            }
        }
    }
};

} /* namespace tp */
