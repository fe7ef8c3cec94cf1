/*
 * tp_convert.cuh - forward CLT with aberration correction (the drop-in for the
 * reference's convert_correct_tiles, src/TileProcessor.cuh:1859-1937 and
 * convertCorrectTile :3106-3635).
 *
 * One 8-lane group per (tile, camera, color) job; a warp holds four jobs of the
 * same camera and color for four consecutive tasks, so the green jobs (two
 * Bayer phases and a DST pass) never share a warp with the cheaper red/blue
 * ones.  Per job:
 *   lane u gathers DTT row u of the folded, windowed Bayer samples (one image
 *   row, 8 same-color pixels), applies the row DCT-IV (green: also the row
 *   DST-IV of the sine-windowed fold), transposes through shared memory and
 *   applies the column DCT-IV, ending with column u of CC (and SC);
 *   the remaining quadrants come from the Bayer mirror symmetries by lane
 *   shuffles; the CLT-domain kernel, the two residual-shift rotations and the
 *   optional LPF are per-coefficient and run in registers; the 256
 *   coefficients are stored as 32-byte row segments.
 */
#pragma once
#include "tp_common.cuh"

namespace tp {

/* Clamp of the integer tile corner (src/TileProcessor.cuh:3188-3193,
 * :3246-3252); `n` is the image size along the axis. */
__device__ __forceinline__ int corner_clamp(int itl, int n, bool horizontal, int mode)
{
    if (itl < 0) itl &= 1;
    if (itl >= n - 8) {
        if (mode == TP_BORDER_REFERENCE && horizontal)
            itl = itl & (1 + (n - 8 - 2)); /* the reference's `itlx & 1 +(W-10)` */
        else
            itl = (itl & 1) + (n - 8 - 2);
    }
    return itl;
}

__device__ __forceinline__ int pair_clamp(int idx, int n)
{
    if (idx < 0) return idx & 1;
    if (idx >= n) return (n - 2) + (idx & 1);
    return idx;
}

struct ConvertJob {
    int cam, color;
};

/* Where a job's window sits and how its kernel tile and shifts follow from
 * the task's tile centre (float32, as the reference computes them:
 * src/TileProcessor.cuh:3129-3255). */
struct JobGeometry {
    size_t kidx;    /* kernel tile (x, y, colour) index into the table   */
    int itlx, itly; /* integer corner of the 16x16 window                */
    float shx, shy; /* residual shifts                                   */
    float hc, hs, vc, vs; /* (cos, sin)(pi s / 16) of the shifted windows */
};

__device__ __forceinline__ JobGeometry job_geometry(const Geom &g, const float *__restrict__ extra_tab, float cx,
                                                    float cy, int color, const float *pre_ex)
{
    JobGeometry j;
    const float step_inv = __int_as_float((127 - g.ls) << 23);
    int ktx = __float2int_rn(__fmaf_rn(cx, step_inv, 1.0f));
    int kty = __float2int_rn(__fmaf_rn(cy, step_inv, 1.0f));
    ktx = min(g.KH - 1, max(0, ktx));
    kty = min(g.KV - 1, max(0, kty));
    const float kdx = (cx - (float)(ktx << g.ls)) + (float)(1 << (g.ls - 1));
    const float kdy = (cy - (float)(kty << g.ls)) + (float)(1 << (g.ls - 1));
    j.kidx = ((size_t)ktx + (size_t)kty * g.KH) * 3 + color;
    /* the kernel tile's offsets: prefetched by the caller (pre_ex[6]) or here */
    const float *ex = extra_tab + j.kidx * 8;
    const float data_x = pre_ex ? pre_ex[0] : __ldg(ex + 0), data_y = pre_ex ? pre_ex[1] : __ldg(ex + 1);
    const float dxc_dx = pre_ex ? pre_ex[2] : __ldg(ex + 4), dxc_dy = pre_ex ? pre_ex[3] : __ldg(ex + 5);
    const float dyc_dx = pre_ex ? pre_ex[4] : __ldg(ex + 6), dyc_dy = pre_ex ? pre_ex[5] : __ldg(ex + 7);
    const float px = (cx - 8.0f) - __fmaf_rn(dxc_dy, kdy, __fmaf_rn(dxc_dx, kdx, data_x));
    const float py = (cy - 8.0f) - __fmaf_rn(dyc_dy, kdy, __fmaf_rn(dyc_dx, kdx, data_y));
    j.itlx = corner_clamp(__float2int_rd(px + 0.5f), g.W, true, g.border_mode);
    j.itly = corner_clamp(__float2int_rd(py + 0.5f), g.H, false, g.border_mode);
    j.shx = (float)j.itlx - px;
    j.shy = (float)j.itly - py;
    /* (cos, sin)(pi s / 16) for the shifted windows */
    const float xh = j.shx * (1.0f / 16.0f), xv = j.shy * (1.0f / 16.0f);
    sincospif(xh, &j.hs, &j.hc);
    sincospif(xv, &j.vs, &j.vc);
    return j;
}

/* A job's window staged in shared memory (the TMA-fed convert kernel): 16
 * rows of 20 floats from the 16-byte boundary at or left of the corner */
constexpr int kCvWinW = 20, kCvWinH = 16;

/* The fold: lane l builds DTT row l of the folded, windowed Bayer samples of
 * the job's colour (P: the cosine fold; Q: the sine-windowed fold of green,
 * zeros for red and blue), both Bayer phases of green summed
 * (src/TileProcessor.cuh:3257-3416).  win (may be NULL): the job's window in
 * shared memory, used for windows inside the image (the same samples). */
__device__ __forceinline__ void fold_rows(const Geom &g, size_t dstride, const float *__restrict__ img,
                                          const JobGeometry &j, int color, int l, float P[8], float Q[8],
                                          const float *win = nullptr, int win_dx = 0)
{
    const int itlx = j.itlx, itly = j.itly;
    const int c0 = color & 1, c1 = (color >> 1) & 1;
    const bool fast = (itlx >= 0) && (itlx < g.W - 16) && (itly >= 0) && (itly < g.H - 16);
    const long long last = (long long)g.image_rows * (long long)dstride - 1;
#pragma unroll
    for (int v = 0; v < 8; v++) { P[v] = 0.0f; Q[v] = 0.0f; }
#pragma unroll
    for (int gp = 0; gp < 2; gp++) {
        if (gp > c1) break;
        const int colp = (itlx & 1) ^ (1 ^ c0 ^ c1 ^ gp);
        const int rowp = (itly & 1) ^ (c0 ^ gp);
        const int lr = fold_sample(l, rowp);
        const float wv = fold_sign_c(lr) * shifted_window_lane(lr, j.vc, j.vs);
        long long rowbase;
        int eff_col = 0;
        if (fast) {
            rowbase = (long long)(itly + lr) * (long long)dstride + itlx;
        } else if (g.border_mode == TP_BORDER_CLAMP) {
            rowbase = (long long)pair_clamp(itly + lr, g.H) * (long long)dstride;
        } else {
            /* src/TileProcessor.cuh:3328-3361: columns clamped by IMG_HEIGHT/2,
             * rows by IMG_WIDTH/2, row offset `rowp` added once */
            const int i = (lr - rowp) >> 1;
            int rp = min(g.W / 2 - 1, max(0, (itly >> 1) + i));
            int cp = min(g.H / 2 - 1, max(0, itlx >> 1));
            eff_col = (cp << 1) + (itlx & 1);
            rowbase = (long long)(rowp + (rp << 1) + (itly & 1)) * (long long)dstride + eff_col;
        }
#pragma unroll
        for (int v = 0; v < 8; v++) {
            /* the sample's column for either Bayer phase and its window values
             * are compile-time constants; the job's phase selects one (the
             * groups of a warp hold jobs of either phase, so a table indexed
             * by the run-time column would serialise their reads) */
            constexpr float kW[16] = TP_HWIN_INIT, kWc[16] = TP_HWINC_INIT;
            const int lc0 = fold_sample(v, 0), lc1 = fold_sample(v, 1);
            const int lc = colp ? lc1 : lc0;
            const float ww = colp ? kW[lc1] : kW[lc0], wwc = colp ? kWc[lc1] : kWc[lc0];
            const float whs_raw = __fmaf_rn(ww, j.hc, wwc * j.hs);
            float pix;
            if (fast && win) {
                /* the window staged in shared memory: rows of kCvWinW floats from
                 * column itlx - win_dx */
                pix = win[lr * kCvWinW + win_dx + lc];
            } else if (fast) {
                pix = __ldg(img + rowbase + lc);
            } else if (g.border_mode == TP_BORDER_CLAMP) {
                pix = __ldg(img + rowbase + pair_clamp(itlx + lc, g.W));
            } else {
                long long a = rowbase + lc;
                a = a > last ? last : (a < 0 ? 0 : a);
                pix = __ldg(img + a);
            }
            const float d = pix * wv;
            const float sgn_c = colp ? fold_sign_c(lc1) : fold_sign_c(lc0);
            const float sgn_s = colp ? fold_sign_s(lc1) : fold_sign_s(lc0);
            P[v] = __fmaf_rn(d, sgn_c * whs_raw, P[v]);
            if (c1) Q[v] = __fmaf_rn(d, sgn_s * whs_raw, Q[v]);
        }
    }
}

/* STREAM: out is global memory and takes evict-first stores.  The kernel
 * writes 963 MB of CLT for a full quad frame, far more than L2 holds, and
 * later kernels read it back; retaining the stores in L2 would only evict the
 * kernel tiles and Bayer rows that neighbouring jobs of this kernel still
 * read. */
template <bool STREAM = false>
__device__ __forceinline__ void convert_finish(const float *__restrict__ kern_tab, const JobGeometry &jg, int color,
                                               int lpf_mask, float *__restrict__ out, float (*tb)[9], int l,
                                               unsigned gm, float P[8], float Q[8]);

template <bool STREAM = false>
__device__ __forceinline__ void convert_job(const Geom &g, size_t dstride,
                                            const float *__restrict__ extra_tab,
                                            const float *__restrict__ kern_tab,
                                            const float *__restrict__ img, float cx, float cy,
                                            int color, int lpf_mask, float *__restrict__ out,
                                            float (*tb)[9], int l, unsigned gm, const float *pre_ex = nullptr)
{
    const JobGeometry jg = job_geometry(g, extra_tab, cx, cy, color, pre_ex);
    /* ---- fold: lane l builds DTT row l ---- */
    float P[8], Q[8];
    fold_rows(g, dstride, img, jg, color, l, P, Q);
    convert_finish<STREAM>(kern_tab, jg, color, lpf_mask, out, tb, l, gm, P, Q);
}

/* The rest of a job after its fold: 2-D transform, CLT-domain convolution
 * with the kernel tile, residual shifts, LPF, store. */
template <bool STREAM>
__device__ __forceinline__ void convert_finish(const float *__restrict__ kern_tab, const JobGeometry &jg, int color,
                                               int lpf_mask, float *__restrict__ out, float (*tb)[9], int l,
                                               unsigned gm, float P[8], float Q[8])
{
    const size_t kidx = jg.kidx;
    const int itlx = jg.itlx, itly = jg.itly;
    const float shx = jg.shx, shy = jg.shy;
    const int c1 = (color >> 1) & 1;

    /* ---- 2-D transform: rows (registers), transpose, columns ---- */
    float cc[8], sc[8], cs[8], ss[8], t[8];
    dtt8<0>(P, t);
    group_transpose(tb, t, P, l, gm);
    dtt8<0>(P, cc); /* lane l: column l of CC */
    if (c1) {
        dtt8<1>(Q, t);
        group_transpose(tb, t, Q, l, gm);
        dtt8<0>(Q, sc); /* column l of SC */
    } else {
        /* R, B: SC[i][7-j] = +-CC[i][j] (src/TileProcessor.cuh:3459-3475) */
        const float neg1 = 1.0f - 2.0f * (float)((itlx & 1) ^ (1 ^ color));
#pragma unroll
        for (int m = 0; m < 8; m++) sc[m] = neg1 * __shfl_xor_sync(gm, cc[m], 7);
    }
    /* SS[7-i][7-j] = +-CC[i][j], CS[7-i][7-j] = +-SC[i][j] (:3486-3504) */
    const float neg2 = 1.0f - 2.0f * (float)((itlx & 1) ^ (itly & 1) ^ 1 ^ c1);
#pragma unroll
    for (int m = 0; m < 8; m++) {
        ss[m] = neg2 * __shfl_xor_sync(gm, cc[7 - m], 7);
        cs[m] = neg2 * __shfl_xor_sync(gm, sc[7 - m], 7);
    }

    /* ---- CLT-domain convolution (src/TileProcessor.cuh:2778-2827) ---- */
    const float *kr = kern_tab + kidx * 256 + l;
#pragma unroll
    for (int m = 0; m < 8; m++) {
        const float k0 = __ldg(kr + m * 8), k1 = __ldg(kr + 64 + m * 8);
        const float k2 = __ldg(kr + 128 + m * 8), k3 = __ldg(kr + 192 + m * 8);
        const float a0 = cc[m], a1 = sc[m], a2 = cs[m], a3 = ss[m];
        cc[m] = __fmaf_rn(a3, k3, __fmaf_rn(-a2, k2, __fmaf_rn(-a1, k1, a0 * k0)));
        sc[m] = __fmaf_rn(-a2, k3, __fmaf_rn(-a3, k2, __fmaf_rn(a0, k1, a1 * k0)));
        cs[m] = __fmaf_rn(-a1, k3, __fmaf_rn(a0, k2, __fmaf_rn(-a3, k1, a2 * k0)));
        ss[m] = __fmaf_rn(a0, k3, __fmaf_rn(a1, k2, __fmaf_rn(a2, k1, a3 * k0)));
    }

    /* ---- residual shift: horizontal (this lane's column), then vertical
     * (per row, angles shared across the group) (:2715-2776) ---- */
    {
        const float a = (shx * (float)(2 * l + 1)) * 0.0625f;
        float ch, sh;
        sincospif(a, &sh, &ch);
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const float x0 = cc[m], x1 = sc[m], x2 = cs[m], x3 = ss[m];
            cc[m] = x0 * ch - x1 * sh;
            sc[m] = x0 * sh + x1 * ch;
            cs[m] = x2 * ch - x3 * sh;
            ss[m] = x2 * sh + x3 * ch;
        }
    }
    {
        const float a = (shy * (float)(2 * l + 1)) * 0.0625f;
        float cvl, svl;
        sincospif(a, &svl, &cvl);
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const float cv = __shfl_sync(gm, cvl, m, 8), sv = __shfl_sync(gm, svl, m, 8);
            const float x0 = cc[m], x1 = sc[m], x2 = cs[m], x3 = ss[m];
            cc[m] = x0 * cv - x2 * sv;
            cs[m] = x0 * sv + x2 * cv;
            sc[m] = x1 * cv - x3 * sv;
            ss[m] = x1 * sv + x3 * cv;
        }
    }
    if ((lpf_mask >> color) & 1) { /* optional LPF (:3572-3593) */
#pragma unroll
        for (int m = 0; m < 8; m++) {
            const float f = __ldg(&d_lpf[color][m * 8 + l]);
            cc[m] *= f; sc[m] *= f; cs[m] *= f; ss[m] *= f;
        }
    }
#pragma unroll
    for (int m = 0; m < 8; m++) {
        if constexpr (STREAM) {
            __stcs(out + m * 8 + l, cc[m]);
            __stcs(out + 64 + m * 8 + l, sc[m]);
            __stcs(out + 128 + m * 8 + l, cs[m]);
            __stcs(out + 192 + m * 8 + l, ss[m]);
        } else {
            out[m * 8 + l] = cc[m];
            out[64 + m * 8 + l] = sc[m];
            out[128 + m * 8 + l] = cs[m];
            out[192 + m * 8 + l] = ss[m];
        }
    }
}

/* Warp w of the grid-stride loop handles tasks 4*(w/12) .. +3 for camera
 * (w%12)%4 and color (w%12)/4. */
__global__ void __launch_bounds__(256, 3) k_convert_correct_tiles(
    Geom g, size_t dstride, float *const *kernel_offsets, float *const *kernels,
    float *const *images, const tp_task *__restrict__ tasks, float *const *clt, int num_tiles,
    int lpf_mask)
{
    __shared__ float tbuf[256 / 8][8][9];
    const int l = threadIdx.x & 7;
    const int grp = threadIdx.x >> 3;
    const unsigned gm = group_mask();
    const int warps_total = gridDim.x * (blockDim.x >> 5);
    const int chunks = (num_tiles + 3) >> 2;
    /* the task fields of this group's job, read two jobs ahead so that the
     * loads overlap the jobs before it */
    auto fetch = [&](int w, int *task, int *txy, float *cx, float *cy) {
        *task = 0;
        if (w >= chunks * 12) return;
        const int chunk = w / 12, r = w - chunk * 12, cam = r & 3;
        const int n = chunk * 4 + ((threadIdx.x >> 3) & 3);
        if (n >= num_tiles) return;
        const tp_task *t = tasks + n;
        *task = __ldg(&t->task);
        *txy = __ldg(&t->txy);
        *cx = __ldg(&t->xy[cam][0]);
        *cy = __ldg(&t->xy[cam][1]);
    };
    /* its kernel tile's offsets (the kernel-tile choice of convert_job),
     * read one job ahead, and the kernel tile itself prefetched into L2
     * (lane l: bytes 128 l .. 128 l + 127 of the 1 KB tile) */
    auto fetch_extra = [&](int w, float cx, float cy, float ex[6]) {
        const int r = w % 12, color = r >> 2, cam = r & 3;
        const float step_inv = __int_as_float((127 - g.ls) << 23);
        const int ktx = min(g.KH - 1, max(0, __float2int_rn(__fmaf_rn(cx, step_inv, 1.0f))));
        const int kty = min(g.KV - 1, max(0, __float2int_rn(__fmaf_rn(cy, step_inv, 1.0f))));
        const size_t kidx = ((size_t)ktx + (size_t)kty * g.KH) * 3 + color;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(kernels[cam] + kidx * 256 + l * 32));
        const float *e = kernel_offsets[cam] + kidx * 8;
        ex[0] = __ldg(e + 0); ex[1] = __ldg(e + 1);
        ex[2] = __ldg(e + 4); ex[3] = __ldg(e + 5);
        ex[4] = __ldg(e + 6); ex[5] = __ldg(e + 7);
    };
    int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    int ntask = 0, ntxy = 0;
    float ncx = 0.0f, ncy = 0.0f, nex[6];
    fetch(w, &ntask, &ntxy, &ncx, &ncy);
    if (ntask) fetch_extra(w, ncx, ncy, nex);
    int n2task = 0, n2txy = 0;
    float n2cx = 0.0f, n2cy = 0.0f;
    fetch(w + warps_total, &n2task, &n2txy, &n2cx, &n2cy);
    for (; w < chunks * 12; w += warps_total) {
        const int chunk = w / 12, r = w - chunk * 12;
        const int color = r >> 2, cam = r & 3;
        const int task = ntask, txy = ntxy;
        const float cx = ncx, cy = ncy;
        float ex[6];
#pragma unroll
        for (int i = 0; i < 6; i++) ex[i] = nex[i];
        ntask = n2task; ntxy = n2txy; ncx = n2cx; ncy = n2cy;
        if (ntask) fetch_extra(w + warps_total, ncx, ncy, nex);
        fetch(w + 2 * warps_total, &n2task, &n2txy, &n2cx, &n2cy);
        if (!task) continue;
        const int tx = txy & 0xfff, ty = txy >> 16;
        if (tx >= g.TX || ty < 0 || ty >= g.TY) continue;
        float *out = clt[cam] + (((size_t)ty * g.TX + tx) * 3 + color) * 256;
        convert_job<true>(g, dstride, kernel_offsets[cam], kernels[cam], images[cam], cx, cy, color,
                    lpf_mask, out, tbuf[grp], l, gm, ex);
    }
}

} /* namespace tp */
