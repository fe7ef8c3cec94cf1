/*
 * tp_texture.cuh - texture tiles (the drop-in for the reference's
 * textures_accumulate, src/TileProcessor.cuh:2207-2579, with imclt8threads
 * :3847-4017, debayer_shot / debayer :4019-4199 and tile_combine_rgba
 * :4202-4665).
 *
 * One 96-thread block (three warps) per listed tile (grid-stride), seven
 * blocks per SM (at most 80 registers, 27 KB of shared memory each: the
 * tiles T and D only).  The CLT is read straight from global memory by the inverse
 * transform; the next tile's CLT and the RGBA rows it will update are
 * prefetched into L2 while the block works on the current tile.  Per
 * (camera, color) job one 8-lane group, working only with __syncwarp on its
 * own buffers:
 *   1. low-pass filter and invert the CLT tile (vertical DCT-IV/DST-IV on the
 *      held column, transpose, horizontal pass on the held row) and unfold it
 *      into the un-windowed tile T (colour) or the windowed tile M (mono);
 *   2. debayer T with the 3x3 stencil (a register window walked down each
 *      column), apply the shot-noise square root and re-window into D (lane l
 *      owns columns l and l + 8).
 * After one block barrier every thread fuses the four cameras at its pixels
 * (stage 3; the plain windowed tile is T times the squared window) and
 * writes them out itself (stage 4): as non-overlapping 16x16 tiles and/or
 * faded by the neighbour mask and added into the overlapped RGBA image.
 * Per-job buffers are 280 floats apart (280 % 32 == 24) so the four groups
 * of a warp never share a bank.
 */
#pragma once
#include "tp_common.cuh"
#include "tp_correlate.cuh"

namespace tp {

struct TextureParams {
    int colors;
    float min_shot, scale_shot, diff_sigma;
    float w0, w1, w2;
    int dust_remove, keep_weights;
};

constexpr int kJob = 280; /* floats per job tile (16 rows of at most 17), padded */
/* Pixel (r, c) of a job tile with row stride S.  The camera fusion reads 32
 * consecutive pixels (two rows) per warp: at stride 16 they fall on 32
 * distinct banks, at 17 the second row's last pixel shares the first row's
 * first bank.  The column-wise passes (unfold, debayer: one column per lane,
 * the four groups' tiles 280 floats apart) are conflict-free at either
 * stride.  Tiles copied in row by row (one row per lane, the tensor-core
 * inverse's output) keep stride 17, where those stores spread over the
 * banks. */
#define JTS(S, r, c) ((r) * (S) + (c))
constexpr int kJS = 16; /* row stride of tiles the inverse transform writes */

__device__ __forceinline__ int sym8(int i) { return (i & 8) ? (i ^ 15) : i; }

/* Per-pixel factors of the unfold, [16][17]:
 *   tfac[r][c] = (0.25 / w[c]) / w[r]     un-windowed tile T = d * tfac
 *   mfac[r][c] = (0.5 w[r]) (0.5 w[c])    windowed tile M = mfac * d
 * with w the half-sine window, as read-only tables in global memory for the
 * tensor-core inverse stage's epilogue (values bit-identical to the float
 * expressions, generated by gen_tables.py); and the squared window at each
 * of the 256 pixels with its reciprocal for the camera fusion. */
constexpr int kFac = 16 * 17;
__device__ float d_tex_tfac[kFac] = TP_TEX_TFAC_INIT;
__device__ float d_tex_mfac[kFac] = TP_TEX_MFAC_INIT;
__device__ float d_tex_wnd2[256] = TP_TEX_WND2_INIT;
__device__ float d_tex_wi[256] = TP_TEX_WI_INIT;

/* Windowed inverse CLT of one job (imclt8threads, :3847-4017) into the
 * [16][kJS] tile M = w * d (w the product of the two half-sine windows, no
 * accumulation), and, for the debayer, the same tile with the squared window
 * removed, T = M / (sin^2 r sin^2 c) = d / (4 sin r sin c), formed directly
 * from the signed sum d.  Lane l loads coefficient row l of each quadrant (two
 * 16-byte loads per row where the source allows); per quadrant it applies
 * the low-pass filter, runs
 * the horizontal DCT-IV/DST-IV on it, and after a transpose the vertical one
 * on column l: it ends holding pixel-domain column l of all four quadrants.
 * The unfold (fold column RIND[c] = l for exactly two output columns c) then
 * writes those two columns whole, the quadrant signs of idct_signs
 * (:399-420) factored into a horizontal sign pair per column (per lane) and
 * a vertical sign per row (compile-time); the window factors are a per-lane
 * column factor, carried by the horizontal sign pair, times a compile-time
 * row factor.  MONO: M (mono) instead of T (colour).  The first column a lane
 * writes is 11 - l: with job buffers 280 floats apart the four groups of a
 * warp then store to 32 distinct banks in both columns.  src: the job's
 * 4x64 coefficients (row stride 8), shared or global memory; tb: the
 * group's transpose buffer; out: the job's [16][kJS] output tile. */
template <bool MONO>
__device__ __forceinline__ void imclt_unfold_job(const float *src, const float *lpf, float *tb, float *out, int l,
                                                 unsigned gm)
{
    constexpr float kHwin[16] = TP_HWIN_INIT;
    float a[4][8]; /* pixel-domain column l of each quadrant */
    float f[8];    /* row l of the low-pass filter, shared by the quadrants */
    if (lpf)
        load_row8(lpf + l * 8, true, f);
    const bool al16 = !(reinterpret_cast<uintptr_t>(src) & 15);
    /* all four rows in flight before the first transform needs one */
    float raw[4][8];
#pragma unroll
    for (int q = 0; q < 4; q++) load_row8(src + q * 64 + l * 8, al16, raw[q]);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float row[8], v[8], col[8];
#pragma unroll
        for (int k = 0; k < 8; k++) row[k] = raw[q][k];
        if (lpf) {
#pragma unroll
            for (int k = 0; k < 8; k++) row[k] *= f[k];
        }
        if (q & 1) dtt8<1>(row, v); else dtt8<0>(row, v);
#pragma unroll
        for (int k = 0; k < 8; k++) tb[TBI(q, l, k)] = v[k];
        __syncwarp(gm);
#pragma unroll
        for (int k = 0; k < 8; k++) col[k] = tb[TBI(q, k, l)];
        if (q >> 1) dtt8<1>(col, a[q]); else dtt8<0>(col, a[q]);
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        /* the output column and its quarter (columns 0-3: (+,+); 4-11:
         * (-,+); 12-15: (-,-) on the (even, odd) quadrant of each pair) */
        const int c = h ? ((l < 4) ? l + 12 : l - 4) : 11 - l;
        const int cq = c >> 2;
        const float wc = __ldg(&d_hwin[c]);
        /* the column's window factor: 0.5 w[c] (M) or 0.25 / w[c] (T) */
        const float cf = MONO ? 0.5f * wc : 0.25f / wc;
        const float s0 = (cq == 0) ? cf : -cf, s1 = (cq == 3) ? -cf : cf;
        float e0[8], e1[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
            e0[u] = __fmaf_rn(s0, a[0][u], s1 * a[1][u]);
            e1[u] = __fmaf_rn(s0, a[2][u], s1 * a[3][u]);
        }
#pragma unroll
        for (int r = 0; r < 16; r++) {
            const int u = (r < 4) ? r + 4 : (r < 12) ? 11 - r : r - 12;
            const int rq = r >> 2;
            /* vertical signs: rows 0-3 (+,+); 4-11 (-,+); 12-15 (-,-) */
            const float d = ((rq != 0) ? -e0[u] : e0[u]) + ((rq == 3) ? -e1[u] : e1[u]);
            out[JTS(kJS, r, c)] = d * (MONO ? 0.5f * kHwin[r] : 1.0f / kHwin[r]);
        }
    }
}

/* 1 / sqrt(x) from the hardware's reciprocal square root (PTX
 * rsqrt.approx.ftz; x must be a normal float or zero) */
__device__ __forceinline__ float rsqrt_hw(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

/* 1 / x from the hardware's reciprocal (PTX rcp.approx.ftz, within one ulp
 * of the correctly rounded value for normal x) */
__device__ __forceinline__ float rcp_hw(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

/* 3x3 debayer of the un-windowed tile T (interior 14x14; border copied),
 * shot-noise square root, squared window re-applied: T -> D
 * (debayer_shot / debayer, :4019-4199).  Lane l: columns l and l + 8, each
 * walked down with a 3x3 register window.  The stencil's horizontal pair
 * t[r][c-1] + t[r][c+1] is summed once per row and shared by the three rows
 * that use it; red/blue (rb_mode) and green take one branch-free form (the
 * diagonal term's weight is 0 for green), so the groups of a warp, which
 * hold different colours, do not diverge; the border columns (copied
 * unchanged) take the same form with stencil weights 0, 0 and 1.  The
 * shot-noise scale and the two window factors are one product per pixel.
 * WINDOWED = false stores D without them (the camera fusion of the RGBA-only
 * path measures distances in D wi sqrt(w) scale_shot, where the squared
 * window cancels against wi = 1 / wnd2: it takes scale_shot with its colour
 * factors instead).  SHOT: scale_shot > 0, the shot-noise step applies.
 * S: the tiles' row stride. */
template <bool WINDOWED, bool SHOT, int S>
__device__ __forceinline__ void debayer_tile(const float *t, float *d, int rb_mode, float min_shot,
                                             float scale_shot, int l, unsigned gm)
{
    /* the window as compile-time constants (the values of c_hwin): the
     * squared window of an unrolled row folds into an immediate operand */
    constexpr float kHwin[16] = TP_HWIN_INIT;
    __syncwarp(gm);
    const float kdiag = rb_mode ? 0.0625f : 0.0f, kcenter = rb_mode ? 0.25f : 0.5f;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int c = l + 8 * h;
        const bool cborder = (c == 0) || (c == 15);
        const int cm = cborder ? c : c - 1, cp = cborder ? c : c + 1;
        /* per-lane stencil weights: diagonal, orthogonal, centre */
        const float kd = cborder ? 0.0f : kdiag, ko = cborder ? 0.0f : 0.125f, kc = cborder ? 1.0f : kcenter;
        const float hcc = __ldg(&d_hwin[c]);
        const float swx = (SHOT ? scale_shot : 1.0f) * (hcc * hcc);
        float a1 = t[JTS(S, 0, c)], ha = t[JTS(S, 0, cm)] + t[JTS(S, 0, cp)];
        float b1 = t[JTS(S, 1, c)], hb = t[JTS(S, 1, cm)] + t[JTS(S, 1, cp)];
#pragma unroll
        for (int r = 0; r < 16; r++) {
            float v;
            if (r == 0) {
                v = a1;
            } else if (r == 15) {
                v = b1;
            } else {
                const float e1 = t[JTS(S, r + 1, c)], he = t[JTS(S, r + 1, cm)] + t[JTS(S, r + 1, cp)];
                const float orth = (a1 + e1) + hb;
                const float diag = ha + he;
                v = __fmaf_rn(kd, diag, __fmaf_rn(ko, orth, kc * b1));
                a1 = b1; ha = hb;
                b1 = e1; hb = he;
            }
            /* shot-noise square root above min_shot, v / sqrt(min_shot) at or
             * below it: both are v * rsqrt(max(v, min_shot)) (min_shot is a
             * normal float > 0 whenever the transform applies), from the
             * hardware reciprocal square root (within 3e-7 of sqrtf) */
            if (SHOT) v = v * rsqrt_hw(fmaxf(v, min_shot));
            d[JTS(S, r, c)] = WINDOWED ? v * (swx * (kHwin[r] * kHwin[r])) : v;
        }
    }
    __syncwarp(gm);
}

/* debayer_tile with the shot-noise step compiled in (scale_shot > 0) or out:
 * one switch per job, outside the unrolled stencil */
template <bool WINDOWED, int S = kJS>
__device__ __forceinline__ void debayer_job(const float *t, float *d, int rb_mode, float min_shot,
                                            float scale_shot, int l, unsigned gm)
{
    if (scale_shot > 0.0f)
        debayer_tile<WINDOWED, true, S>(t, d, rb_mode, min_shot, scale_shot, l, gm);
    else
        debayer_tile<WINDOWED, false, S>(t, d, rb_mode, min_shot, scale_shot, l, gm);
}

/* log2(e): e^x = 2^(x log2 e) */
constexpr float kLog2e = 1.4426950408889634f;

/* 2^x from the hardware's base-2 exponential (PTX ex2.approx.ftz; results
 * below the smallest normal float flush to zero) */
__device__ __forceinline__ float exp2_hw(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

/* Fuse the four cameras at one pixel (tile_combine_rgba, one pixel).
 * sd: debayered tiles D; sm: the plain (not debayered) tiles, scaled by
 * m_scale (the plain tile is the un-windowed one times the squared window);
 * both [job = cam * colors + color] with the given strides, pixel offset e.
 * chw: the colour weights; chws: their square roots, times scale_shot when
 * the D tiles come without the window and the shot scale (D_WINDOWED false;
 * wi is then not applied to them).  pd2r (the six pairs'
 * 1 / (2 sigma^2 |offset|^2)) and ksigma (1 / (2 sigma^2)) come multiplied by
 * log2(e): each weight exp(-k d) is evaluated as 2^(-(k log2 e) d).
 * o: colours, alpha, 4 port weights and (keep_weights) colors + 1 rms.
 * The colour distances sum_col chw[col] ((X[col] - Y[col]) wi)^2 are formed
 * as sum_col (X'[col] - Y'[col])^2 in the scaled space X' = X wi sqrt(chw),
 * the same quantity with fewer operations per camera pair. */
template <int COLORS, bool D_WINDOWED = true>
__device__ __forceinline__ void combine_pixel(const float *sd, int sd_stride, const float *sm, int sm_stride,
                                              float m_scale, int e, const float *pd2r, float ksigma,
                                              const float *chw, const float *chws, float wnd2, float wi,
                                              int dust_remove, int keep_weights, float *o)
{
    float D[4][COLORS];
#pragma unroll
    for (int cam = 0; cam < 4; cam++)
#pragma unroll
        for (int col = 0; col < COLORS; col++) D[cam][col] = sd[(cam * COLORS + col) * sd_stride + e];
    if (keep_weights) {
        float sw = 0.0f;
#pragma unroll
        for (int col = 0; col < COLORS; col++) {
            /* variance of the four cameras, two-pass (the one-pass form of
             * the reference loses digits where the cameras agree) */
            const float mean = ((D[0][col] + D[1][col]) + (D[2][col] + D[3][col])) * 0.25f;
            float ss = 0.0f;
#pragma unroll
            for (int cam = 0; cam < 4; cam++) {
                const float dv = D[cam][col] - mean;
                ss = __fmaf_rn(dv, dv, ss);
            }
            const float mse = ss * 0.25f;
            o[COLORS + 5 + col] = sqrtf(mse);
            sw = __fmaf_rn(chw[col], mse, sw);
        }
        o[COLORS + 5 + COLORS] = sqrtf(sw);
    }
    /* D in the scaled space */
#pragma unroll
    for (int col = 0; col < COLORS; col++) {
        const float sc = D_WINDOWED ? wi * chws[col] : chws[col];
#pragma unroll
        for (int cam = 0; cam < 4; cam++) D[cam][col] *= sc;
    }
    /* wi = 1 / wnd2 correctly rounded (the reference forms it in double).
     * A weight is exp(...) plus the 1e-4 floor added in double and rounded
     * once to float, as the reference's double floor constant makes it: the
     * floor sum decides the best and worst cameras where every exponential
     * is tiny (high-contrast or high-dynamic-range tiles), and a float sum
     * with 1e-4f can land one ulp lower and break such ties the other way
     * (splitting the floor into two floats still rounds 1 in 2e6 tiny sums
     * differently).  The exponential is the hardware's base-2 one with the
     * log2(e) factor folded into pd2r and ksigma: its relative error (about
     * 2^-22) is under what float32 inputs already move a weight by, and a
     * flushed subnormal weight is lost in the 1e-4 floor. */
    float pw[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    {
        int k = 0;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = i + 1; j < 4; j++) {
                float d = 0.0f;
#pragma unroll
                for (int col = 0; col < COLORS; col++) {
                    const float dc = D[i][col] - D[j][col];
                    d = __fmaf_rn(dc, dc, d);
                }
                const float x = __double2float_rn((double)exp2_hw(-pd2r[k] * d) + 1e-4);
                pw[i] += x;
                pw[j] += x;
                k++;
            }
    }
    /* the best two cameras (first of equals), their weights carried beside
     * the indices: an array indexed by a run-time camera would live in local
     * memory */
    int b1 = 0;
    float p1 = pw[0];
#pragma unroll
    for (int cam = 1; cam < 4; cam++)
        if (pw[cam] > p1) { b1 = cam; p1 = pw[cam]; }
    int b2 = (b1 == 0) ? 1 : 0;
    float p2 = (b1 == 0) ? pw[1] : pw[0];
#pragma unroll
    for (int cam = 1; cam < 4; cam++)
        if (cam > b2 && cam != b1 && pw[cam] > p2) { b2 = cam; p2 = pw[cam]; }
    const float w1 = __fdividef(p1, p1 + p2);
    const float w2 = 1.0f - w1;
    float avg[COLORS];
#pragma unroll
    for (int col = 0; col < COLORS; col++) {
        float a = 0.0f, b = 0.0f;
#pragma unroll
        for (int cam = 0; cam < 4; cam++) {
            if (cam == b1) a = D[cam][col];
            if (cam == b2) b = D[cam][col];
        }
        avg[col] = w1 * a + w2 * b;
    }
#pragma unroll
    for (int cam = 0; cam < 4; cam++) {
        float d2 = 0.0f;
#pragma unroll
        for (int col = 0; col < COLORS; col++) {
            const float dc = D[cam][col] - avg[col];
            d2 = __fmaf_rn(dc, dc, d2);
        }
        pw[cam] = __double2float_rn((double)exp2_hw(-ksigma * d2) + 1e-4);
    }
    if (dust_remove) {
        int worst = 0;
        float wv = pw[0];
#pragma unroll
        for (int cam = 1; cam < 4; cam++)
            if (pw[cam] < wv) { worst = cam; wv = pw[cam]; }
        float a = -wv;
#pragma unroll
        for (int cam = 0; cam < 4; cam++) a += pw[cam];
        a *= (1.0f / 3.0f);
        const float ra = rcp_hw(a);
        const float scale = 1.0f + (wv * (a - wv)) * (ra * ra) * (1.0f / 3.0f);
        const float fw = wv * ra;
#pragma unroll
        for (int cam = 0; cam < 4; cam++) pw[cam] *= (cam == worst) ? fw : scale;
    }
    float ksum = 0.0f;
#pragma unroll
    for (int cam = 0; cam < 4; cam++) ksum += pw[cam];
    const float kinv = rcp_hw(ksum);
    float kw[4];
#pragma unroll
    for (int cam = 0; cam < 4; cam++) kw[cam] = kinv * pw[cam];
#pragma unroll
    for (int col = 0; col < COLORS; col++) {
        float v = 0.0f;
#pragma unroll
        for (int cam = 0; cam < 4; cam++) v = __fmaf_rn(kw[cam], sm[(cam * COLORS + col) * sm_stride + e], v);
        o[col] = v * m_scale;
    }
    o[COLORS] = wnd2 * ksum / 4.0f;
#pragma unroll
    for (int cam = 0; cam < 4; cam++) o[COLORS + 1 + cam] = pw[cam];
}

/* k_textures block: three warps, one 8-lane group per (camera, colour) job */
constexpr int kTexThreads = 96;
/* dynamic shared memory of k_textures, in floats: T (un-windowed tiles),
 * transposes then D (debayered tiles) */
constexpr int kTexSmemFloats = 12 * kJob + 12 * kTB4;
constexpr size_t kTexSmemBytes = sizeof(float) * kTexSmemFloats;

/* FROM_T: `clt` holds the jobs' pixel tiles instead of their CLT, as
 * k_tc_stage<InvTcStage> writes them (the un-windowed T for colour, the
 * windowed M for mono, [16][16] row-major at the job's CLT offset): stage 1
 * copies the tile into shared memory instead of inverting the CLT.
 * ALL: the texture-tile outputs and the keep-weights statistics are built
 * (false: the RGBA image only).  COLORS: the colour count, 1 or 3 (p.colors;
 * a compile-time count lets each form keep only its own colour path). */
template <bool FROM_T, bool ALL, int COLORS>
__global__ void __launch_bounds__(kTexThreads, 7) k_textures(
    Geom g, const int *__restrict__ woi, float *const *clt, long long num_texture_tiles,
    const int *__restrict__ list, const int *__restrict__ dev_counts, int count_slot, int list_cap,
    int border_quarter, const float *__restrict__ port_offsets, TextureParams p,
    size_t texture_rbg_stride, float *__restrict__ texture_rbg, size_t texture_stride,
    float *__restrict__ texture_tiles)
{
    extern __shared__ __align__(16) float smem[];
    float *s_t = smem;                 /* un-windowed tiles T (colour) or windowed M (mono) */
    float *s_x = s_t + 12 * kJob;      /* transposes, then the debayered tiles D            */
    __shared__ float *s_cp[4];
    __shared__ float s_pd2r[6], s_chw[3], s_chws[3];

    const int tid = threadIdx.x;
    const int l = tid & 7, grp = tid >> 3;
    const unsigned gm = group_mask();
    static_assert(COLORS == 1 || COLORS == 3, "colour count");
    constexpr int colors = COLORS;
    /* row stride of the T and D tiles: 17 where stage 1 copies T in row by
     * row (FROM_T), else that of the inverse transform's output */
    constexpr int kS = FROM_T ? 17 : kJS;
    const int njobs = 4 * colors;
    /* 1 / (2 sigma^2) times log2(e): the fusion's weights are powers of two */
    const float ksigma = (float)(1.0 / (2.0 * (double)p.diff_sigma * (double)p.diff_sigma)) * kLog2e;
    if (tid < 4) s_cp[tid] = clt[tid];
    if (tid == 0) {
        int k = 0;
        for (int i = 0; i < 4; i++)
            for (int j = i + 1; j < 4; j++) {
                const float dx = port_offsets[2 * j] - port_offsets[2 * i];
                const float dy = port_offsets[2 * j + 1] - port_offsets[2 * i + 1];
                s_pd2r[k++] = ksigma / (dx * dx + dy * dy);
            }
        s_chw[0] = p.w0; s_chw[1] = p.w1; s_chw[2] = p.w2;
        /* the RGBA-only colour path debayers without the window (see
         * debayer_job): its distance factors carry the shot scale */
        const float dsc = (!ALL && COLORS == 3 && p.scale_shot > 0.0f) ? p.scale_shot : 1.0f;
        for (int c = 0; c < 3; c++) s_chws[c] = sqrtf(s_chw[c]) * dsc;
    }
    /* D tiles come with the window and the shot scale in the ALL form and
     * for mono (the keep-weights statistics and mono need them as the
     * reference forms them); the RGBA-only colour form debayers without them */

    long long count = num_texture_tiles;
    const int *lst = list;
    /* entries at or past `split` sit `gap` further on in the list */
    int split = 0x7fffffff, gap = 0;
    if (dev_counts) {
        /* sub-list length from the list builder, kept inside its quarter */
        count = dev_counts[count_slot];
        count = count < 0 ? 0 : (count > list_cap ? list_cap : count);
        if (border_quarter > 0) {
            /* the border sub-list alone: it grows down from the quarter's end */
            lst = list + (border_quarter - count);
        } else if (border_quarter < 0) {
            /* inner (count_slot) then border (count_slot + 1) sub-lists of one
             * quarter of -border_quarter entries in one pass: tiles of one
             * parity never overlap, so their RGBA updates need no ordering */
            const int q = -border_quarter, ci = (int)count;
            int cb = dev_counts[count_slot + 1];
            cb = cb < 0 ? 0 : (cb > q - ci ? q - ci : cb);
            split = ci;
            gap = q - cb - ci;
            count += cb;
        }
    }
    /* list entry n of this pass */
    auto code_at = [&](long long n) -> int { return lst[n + (n >= split ? gap : 0)]; };
    const bool want_rbg = texture_rbg && texture_rbg_stride;
    const bool want_tiles = ALL && texture_tiles && texture_stride;
    const int keep_weights = ALL ? p.keep_weights : 0;
    const int ns_tiles = (colors == 3) ? (p.keep_weights ? 12 : 4) : (p.keep_weights ? 8 : 2);
    int wx0 = 0, wy0 = 0, wh = 0;
    if (want_rbg) { wx0 = woi[0]; wy0 = woi[1]; wh = woi[3]; }
    const size_t slice_stride = texture_rbg_stride * (size_t)(wh + 1) * 8;
    __syncthreads();
    const int ntiles = g.TX * g.TY;
    /* list entry -> tile index, or -1 when the entry is not a texture tile */
    auto tile_of = [&](long long n) -> int {
        if (n >= count) return -1;
        const int code = code_at(n);
        const int tile = code >> 8;
        return ((code & (1 << 7)) && tile >= 0 && tile < ntiles) ? tile : -1;
    };
    /* window position of a tile's top-left pixel (once per tile) */
    auto rgba_origin = [&](int tile, int *gy0, int *gx0) {
        const int ty = tile / g.TX, tx = tile - ty * g.TX;
        *gy0 = (ty - wy0) * 8;
        *gx0 = (tx - wx0) * 8;
    };
    /* RGBA address of pixel px (slice 0) of the tile at (gy0, gx0), or NULL
     * when it lies left of / above the window */
    auto rgba_at = [&](int gy0, int gx0, int px) -> float * {
        const int gy = gy0 + (px >> 4), gx = gx0 + (px & 15);
        if (gy < 0 || gx < 0) return nullptr;
        return texture_rbg + (size_t)gy * texture_rbg_stride + (size_t)gx;
    };
    /* The next tile's inputs are prefetched into L2 while the block works on
     * the current one: its CLT (one 128-byte line per thread: 24 lines of 768
     * floats per camera) and the RGBA rows its pixels update (both ends of
     * each 16-pixel row of each slice).  The RGBA prefetch comes after the
     * wait for the previous pass, which writes those rows. */
    auto prefetch_clt = [&](int tile) {
        const int cam = tid / 24, line = tid - cam * 24;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(s_cp[cam] + (size_t)tile * 768 + line * 32));
    };
    auto prefetch_rgba = [&](long long n) {
        if (!want_rbg || n >= count) return;
        const int code = code_at(n);
        const int tile = code >> 8;
        if (!(code & (1 << 7)) || tile < 0 || tile >= ntiles || !(code & TP_TASK_TEXTURE_BITS)) return;
        int gy0, gx0;
        rgba_origin(tile, &gy0, &gx0);
        const int r = tid & 15, sl = tid >> 4; /* row r of slice sl */
        if (sl <= colors) {
            const float *b = rgba_at(gy0, gx0, r * 16);
            if (b) {
                b += (size_t)sl * slice_stride;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(b));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(b + 15));
            }
        }
    };

    /* the next tile-parity pass may be scheduled on the SM slots this grid
     * frees as its blocks finish */
    grid_dependents_launch();
    {
        const long long n0 = blockIdx.x;
        const int t0 = tile_of(n0);
        if (t0 >= 0) prefetch_clt(t0);
        /* A pass launched as a programmatic dependent of the launch before it
         * (the RGBA clear, or the previous tile-parity pass) waits here for
         * it: that launch writes the RGBA image.  Everything read above (the
         * list and its counts, the window, the CLT, the port offsets) was
         * complete before that launch let this one start. */
        grid_dependency_wait();
        if (t0 >= 0) prefetch_rgba(n0);
    }

    for (long long n = blockIdx.x; n < count; n += gridDim.x) {
        const int code = code_at(n);
        const int tile = tile_of(n);
        const long long n_next = n + gridDim.x;
        __syncthreads(); /* the previous tile's buffers free */
        if (tile < 0) {
            const int tn = tile_of(n_next);
            if (tn >= 0) {
                prefetch_clt(tn);
                prefetch_rgba(n_next);
            }
            continue;
        }

        /* ---- stages 1-2: per (camera, color) group ---- */
        if (grp < njobs && FROM_T) {
            const int cam = grp / colors, color = grp - cam * colors;
            float *tj = s_t + grp * kJob, *xj = s_x + grp * kTB4;
            const float *src = s_cp[cam] + ((size_t)tile * 3 + color) * 256 + l * 32;
            const bool al16 = !(reinterpret_cast<uintptr_t>(src) & 15);
            /* lane l: rows 2 l and 2 l + 1 */
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float v[16];
                load_row8(src + 16 * h, al16, v);
                load_row8(src + 16 * h + 8, al16, v + 8);
#pragma unroll
                for (int c = 0; c < 16; c++) tj[JTS(kS, 2 * l + h, c)] = v[c];
            }
            if (colors > 1) debayer_job<ALL, kS>(tj, xj, color < 2, p.min_shot, p.scale_shot, l, gm);
        } else if (grp < njobs) {
            const int cam = grp / colors, color = grp - cam * colors;
            float *tj = s_t + grp * kJob, *xj = s_x + grp * kTB4;
            if (colors > 1) {
                /* T -> s_t, then the debayered D -> s_x (the transpose
                 * buffer, free once the unfold has read it) */
                imclt_unfold_job<false>(s_cp[cam] + ((size_t)tile * 3 + color) * 256, d_lpf[color], xj, tj, l, gm);
                debayer_job<ALL>(tj, xj, color < 2, p.min_shot, p.scale_shot, l, gm);
            } else {
                imclt_unfold_job<true>(s_cp[cam] + ((size_t)tile * 3 + color) * 256, d_lpf[3], xj, tj, l, gm);
            }
        }
        __syncthreads();
        {
            const int tn = tile_of(n_next);
            if (tn >= 0) prefetch_clt(tn);
        }

        /* ---- stages 3-4: fuse the four cameras at the thread's pixels and
         * write them out ---- */
        const int nbr = code & TP_TASK_TEXTURE_BITS;
        int gy0 = 0, gx0 = 0;
        if (want_rbg && nbr) rgba_origin(tile, &gy0, &gx0);
#pragma unroll 1
        for (int px = tid; px < 256; px += kTexThreads) {
            const int r = px >> 4, c = px & 15;
            const int e = JTS(kS, r, c);
            const float wnd2 = __ldg(&d_tex_wnd2[px]), wi = __ldg(&d_tex_wi[px]);
            /* the pixel's RGBA values are loaded before the fusion, whose
             * arithmetic then covers their latency */
            float old[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            float *b = (want_rbg && nbr) ? rgba_at(gy0, gx0, px) : nullptr;
            if (b) {
#pragma unroll
                for (int sl = 0; sl < 4; sl++)
                    if (sl <= colors) old[sl] = b[(size_t)sl * slice_stride];
            }
            float o[12];
            if (colors == 3)
                combine_pixel<3, ALL>(s_x, kTB4, s_t, kJob, wnd2, e, s_pd2r, ksigma, s_chw, s_chws, wnd2, wi,
                                      p.dust_remove, keep_weights, o);
            else
                combine_pixel<1>(s_t, kJob, s_t, kJob, 1.0f, e, s_pd2r, ksigma, s_chw, s_chws, wnd2, wi,
                                 p.dust_remove, keep_weights, o);
            if (want_tiles) {
                float *dst = texture_tiles + (size_t)n * texture_stride + px;
#pragma unroll
                for (int sl = 0; sl < 12; sl++)
                    if (sl < ns_tiles) dst[sl * 256] = o[sl];
            }
            if (b) {
                const float f = (nbr != TP_TASK_TEXTURE_BITS) ? __ldg(&d_alpha_fade[nbr][px]) : 1.0f;
#pragma unroll
                for (int sl = 0; sl < 4; sl++) {
                    if (sl > colors) break;
                    const float v = (nbr != TP_TASK_TEXTURE_BITS) ? o[sl] * f : o[sl];
                    b[(size_t)sl * slice_stride] = old[sl] + v;
                }
            }
        }
        prefetch_rgba(n_next);
    }
}

} /* namespace tp */
