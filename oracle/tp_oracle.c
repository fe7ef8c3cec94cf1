/*
 * tp_oracle.c - FP64 CPU restatement of the reference tile processor.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA path; see tp_oracle.h).
 *
 * Each function below restates the arithmetic of one reference kernel of
 * mfkiwl/tile_processor_gpu at the level of the mathematics: 8-point
 * transforms are applied as explicit 8x8 matrices with exact FP64 constants
 * (the reference uses hand-factored butterflies with 6-digit float constants),
 * windows are evaluated from their closed forms, and every loop walks tiles,
 * quadrants and pixels directly instead of following the reference's
 * thread/shared-memory decomposition.  The references to file:line name the
 * reference code whose results each step reproduces.
 */
#include "tp_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------- */
/* constants and tables                                                       */
/* ------------------------------------------------------------------------- */

static double DCT4[8][8], DST4[8][8], DCT2[8][8], DST2[8][8];
static double HWIN[16];   /* sin(pi*(2n+1)/32): the 16-tap lapped window       */
/* window tables as used by each stage; mode 1 rounds them to 6 decimals as
 * the reference's printed tables are (HWINDOW, HWINDOW2, HWINDOW_SQ,
 * HWINDOW_SQi, src/TileProcessor.cuh:374-383) */
static double TW[16], TW2[16], TWSQ[16], TWSQI[16];
static int table_mode = 0;
static double AFADE[16][256];
static int    RIND[16];   /* window sample n -> DTT index (fold and unfold)    */
static int    tables_ready = 0;
static int    n_threads = 0;

/* Camera pairs of the correlation (src/TileProcessor.cuh:484-490). */
static const int PAIRS[6][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {0, 3}, {2, 1}};

static void init_tables(void)
{
    if (tables_ready) return;
    for (int k = 0; k < 8; k++) {
        for (int n = 0; n < 8; n++) {
            /* src/dtt8x8.cuh:621-745: orthonormal DCT-IV / DST-IV */
            DCT4[k][n] = 0.5 * cos(M_PI * (2 * k + 1) * (2 * n + 1) / 32.0);
            DST4[k][n] = 0.5 * sin(M_PI * (2 * k + 1) * (2 * n + 1) / 32.0);
            /* src/dtt8x8.cuh:382-463: DCT-II / DST-II scaled by 1/2 for every
             * k ("no 1/sqrt(2)" on the DC / Nyquist term) */
            DCT2[k][n] = 0.5 * cos(M_PI * (2 * n + 1) * k / 16.0);
            DST2[k][n] = 0.5 * sin(M_PI * (2 * n + 1) * (k + 1) / 16.0);
        }
    }
    for (int n = 0; n < 16; n++) {
        HWIN[n] = sin(M_PI * (2 * n + 1) / 32.0);
        /* fold/unfold position of window sample n (src/TileProcessor.cuh:254-305,
         * 386-395): 4..7, 7..4, 3..0, 0..3 */
        RIND[n] = (n < 4) ? n + 4 : (n < 12) ? 11 - n : n - 12;
    }
    tpo_alpha_fade(AFADE);
    for (int n = 0; n < 16; n++) {
        double v = HWIN[n];
        if (table_mode == 1) {
            TW[n] = nearbyint(v * 1e6) / 1e6;
            TW2[n] = nearbyint(0.5 * v * 1e6) / 1e6;
            TWSQ[n] = nearbyint(v * v * 1e6) / 1e6;
            TWSQI[n] = nearbyint(1e6 / (v * v)) / 1e6;
        } else {
            TW[n] = v;
            TW2[n] = 0.5 * v;
            TWSQ[n] = v * v;
            TWSQI[n] = 1.0 / (v * v);
        }
    }
    tables_ready = 1;
}

void tpo_set_table_mode(int mode)
{
    table_mode = mode ? 1 : 0;
    tables_ready = 0;
    init_tables();
}

void tpo_dtt_matrix(int kind, double out[64])
{
    init_tables();
    const double (*m)[8] = kind == 0 ? DCT4 : kind == 1 ? DST4 : kind == 2 ? DCT2 : DST2;
    for (int k = 0; k < 8; k++)
        for (int n = 0; n < 8; n++) out[k * 8 + n] = m[k][n];
}

/* Low-pass filters in the CLT domain (src/TileProcessor.cuh:421-481): the
 * separable DCT-III of the spatial kernel exp(-n^2 / (2 s)), n = 0..7,
 * normalised to 1 at DC, printed with 8 decimals.  s = 0.9 (red, blue and the
 * final correlation filter), 0.6 (green), 0.4 (mono), 0.5 (R+B correlation). */
void tpo_default_lpf(int which, float out[64])
{
    static const double sig[6] = {0.9, 0.9, 0.6, 0.4, 0.5, 0.9};
    double s = (which >= 0 && which < 6) ? sig[which] : 0.9;
    double g[8], f[8];
    for (int n = 0; n < 8; n++) g[n] = exp(-(double)(n * n) / (2.0 * s));
    for (int u = 0; u < 8; u++) {
        double acc = g[0];
        for (int n = 1; n < 8; n++) acc += 2.0 * g[n] * cos(M_PI * n * (2 * u + 1) / 16.0);
        f[u] = acc;
    }
    for (int u = 0; u < 8; u++)
        for (int v = 0; v < 8; v++) {
            double val = (f[u] / f[0]) * (f[v] / f[0]);
            out[u * 8 + v] = (float)(nearbyint(val * 1e8) / 1e8);
        }
}

/* Texture fade masks indexed by the N/E/S/W neighbour code
 * (src/TileProcessor.cuh:316-369 generator, table at :492-1005). */
void tpo_alpha_fade(double out[16][256])
{
    double fade[16];
    for (int i = 0; i < 16; i++) fade[i] = 0.5 * (1.0 - cos(M_PI * (i + 0.5) / 16.0));
    for (int m = 0; m < 16; m++) {
        for (int i = 0; i < 16; i++) {
            for (int j = 0; j < 16; j++) {
                double v;
                switch (m) {
                case 0:  v = 0.0; break;
                case 1:  v = fade[15 - i]; break;
                case 2:  v = fade[j]; break;
                case 4:  v = fade[i]; break;
                case 8:  v = fade[15 - j]; break;
                case 3:  v = (j > 15 - i) ? fade[j] : fade[15 - i]; break;
                case 6:  v = (j > i) ? fade[j] : fade[i]; break;
                case 9:  v = (j > i) ? fade[15 - i] : fade[15 - j]; break;
                case 12: v = (i > 15 - j) ? fade[i] : fade[15 - j]; break;
                default: v = 1.0; break;
                }
                out[m][i * 16 + j] = v;
            }
        }
    }
}

void tpo_set_threads(int n) { n_threads = n; }
int tpo_get_threads(void)
{
#ifdef _OPENMP
    return n_threads > 0 ? n_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

static int tiles_x(const tp_geometry *g) { return g->img_width / 8; }
static int tiles_y(const tp_geometry *g) { return g->img_height / 8; }
static int tiles_ya(const tp_geometry *g) { return (tiles_y(g) + 3) & ~3; }

/* y = M x along rows (horizontal) or columns (vertical) of an 8x8 block */
static void dtt_rows(const double (*m)[8], const double in[8][8], double out[8][8])
{
    for (int r = 0; r < 8; r++)
        for (int k = 0; k < 8; k++) {
            double a = 0.0;
            for (int n = 0; n < 8; n++) a += m[k][n] * in[r][n];
            out[r][k] = a;
        }
}
static void dtt_cols(const double (*m)[8], const double in[8][8], double out[8][8])
{
    for (int c = 0; c < 8; c++)
        for (int k = 0; k < 8; k++) {
            double a = 0.0;
            for (int n = 0; n < 8; n++) a += m[k][n] * in[n][c];
            out[k][c] = a;
        }
}

/* ------------------------------------------------------------------------- */
/* convert_correct_tiles  (src/TileProcessor.cuh:1859-1937, :3106-3635)        */
/* ------------------------------------------------------------------------- */

/* Integer corner clamp of the reference (src/TileProcessor.cuh:3188-3193,
 * :3246-3252).  `n` = image size along the axis. */
static int clamp_corner(int itl, int n, int horizontal, int mode)
{
    if (itl < 0) itl &= 1;
    if (itl >= n - 8) {
        if (mode == TP_BORDER_REFERENCE && horizontal)
            itl = itl & (1 + (n - 8 - 2)); /* `itlx & 1 +(W-10)`: C precedence */
        else
            itl = (itl & 1) + (n - 8 - 2);
    }
    return itl;
}

static int clamp_pair(int idx, int n)
{
    if (idx < 0) return idx & 1;
    if (idx >= n) return (n - 2) + (idx & 1);
    return idx;
}

/* One Bayer sample of the fold.  row_tl/col_tl: clamped corner; lr0: first
 * local row of this color phase; lr/lc: local row/col inside the 16x16 window. */
static double fetch_pixel(const tp_geometry *g, const float *img, size_t dstride,
                          int row_tl, int col_tl, int lr0, int i, int lc)
{
    const int W = g->img_width, H = g->img_height;
    const int lr = lr0 + 2 * i;
    if (col_tl >= 0 && col_tl < W - 16 && row_tl >= 0 && row_tl < H - 16)
        return img[(size_t)(row_tl + lr) * dstride + col_tl + lc];
    if (g->border_mode == TP_BORDER_CLAMP) {
        int r = clamp_pair(row_tl + lr, H), c = clamp_pair(col_tl + lc, W);
        return img[(size_t)r * dstride + c];
    }
    /* src/TileProcessor.cuh:3328-3361: columns clamped with IMG_HEIGHT/2, rows
     * with IMG_WIDTH/2; the row offset lr0 is added once. */
    int hc = H / 2 - 1, hr = W / 2 - 1;
    int cp = col_tl >> 1; if (cp < 0) cp = 0; if (cp > hc) cp = hc;
    int eff_col = (cp << 1) + (col_tl & 1);
    int rp = (row_tl >> 1) + i; if (rp < 0) rp = 0; if (rp > hr) rp = hr;
    int eff_row = (rp << 1) + (row_tl & 1);
    long long addr = (long long)(lr0 + eff_row) * (long long)dstride + eff_col + lc;
    long long last = (long long)g->image_rows * (long long)dstride - 1;
    if (addr > last) addr = last;  /* the reference reads past the image here */
    if (addr < 0) addr = 0;
    return img[addr];
}

static void convert_one(const tp_geometry *g, const float *extra_tab, const float *kern_tab,
                        const float *img, size_t dstride, const tp_task *t, int cam, int color,
                        int lpf_mask, const float *lpf, double *clt_cam, int *corner)
{
    const int KH = g->kernels_hor, KV = g->kernels_vert, ls = g->kernels_lstep;
    const int W = g->img_width, H = g->img_height, TX = tiles_x(g);
    const float cx = t->xy[cam][0], cy = t->xy[cam][1];

    /* kernel tile: lrintf(c/step + 1), clamped (src/TileProcessor.cuh:3129-3139) */
    float step_inv = 1.0f / (float)(1 << ls);
    long kx = lrintf(cx * step_inv + 1.0f), ky = lrintf(cy * step_inv + 1.0f);
    int ktx = (int)(kx < 0 ? 0 : kx > KH - 1 ? KH - 1 : kx);
    int kty = (int)(ky < 0 ? 0 : ky > KV - 1 ? KV - 1 : ky);
    float kdx = (cx - (float)(ktx << ls)) + (float)(1 << (ls - 1));
    float kdy = (cy - (float)(kty << ls)) + (float)(1 << (ls - 1));
    size_t kidx = ((size_t)ktx + (size_t)kty * KH) * 3 + color;
    const float *ex = extra_tab + kidx * 8;
    const float *kr = kern_tab + kidx * 256;

    /* fractional corner and residual shift (src/TileProcessor.cuh:3183-3255),
     * in float32 as the reference computes them */
    float px = (cx - 8.0f) - fmaf(ex[5], kdy, fmaf(ex[4], kdx, ex[0]));
    float py = (cy - 8.0f) - fmaf(ex[7], kdy, fmaf(ex[6], kdx, ex[1]));
    int itlx = clamp_corner((int)floorf(px + 0.5f), W, 1, g->border_mode);
    int itly = clamp_corner((int)floorf(py + 0.5f), H, 0, g->border_mode);
    float shx = (float)itlx - px, shy = (float)itly - py;
    if (corner) { corner[0] = ktx; corner[1] = kty; corner[2] = itlx; corner[3] = itly; }

    /* shifted windows with the fold signs embedded (:3196-3262):
     * cos branch +,+,+,+,-,...,-; sine branch (green) +x12, -x4 */
    double whc[16], whs[16], wv[16];
    const double ah = M_PI * (double)shx / 16.0, av = M_PI * (double)shy / 16.0;
    for (int n = 0; n < 16; n++) {
        /* w(n + s) = w(n) cos(pi s / 16) + w'(n) sin(pi s / 16), w' the
         * quadrature window (table mode 1 uses the 6-decimal w) */
        double wq = (n < 8) ? TW[7 - n] : -TW[n - 8];
        double sh = TW[n] * cos(ah) + wq * sin(ah);
        double sv = TW[n] * cos(av) + wq * sin(av);
        whc[n] = (n < 4) ? sh : -sh;
        whs[n] = (n < 12) ? sh : -sh;
        wv[n]  = (n < 4) ? sv : -sv;
    }

    /* Bayer fold, GR/BG mosaic with red at row 0, column 1 (:3289-3364) */
    const int c0 = color & 1, c1 = (color >> 1) & 1;
    double P[8][8], Q[8][8];
    memset(P, 0, sizeof(P));
    memset(Q, 0, sizeof(Q));
    for (int gp = 0; gp <= c1; gp++) {
        int colp = (itlx & 1) ^ (1 ^ c0 ^ c1 ^ gp);
        int rowp = (itly & 1) ^ (0 ^ c0 ^ gp);
        for (int i = 0; i < 8; i++) {
            int lr = rowp + 2 * i;
            for (int tcol = 0; tcol < 8; tcol++) {
                int lc = colp + 2 * tcol;
                double d = fetch_pixel(g, img, dstride, itly, itlx, rowp, i, lc) * wv[lr];
                P[RIND[lr]][RIND[lc]] += d * whc[lc];
                if (color == 2) Q[RIND[lr]][RIND[lc]] += d * whs[lc];
            }
        }
    }

    /* 2-D transform: rows then columns (:3408-3441) */
    double tmp[8][8], q[4][8][8];
    dtt_rows(DCT4, P, tmp);
    dtt_cols(DCT4, tmp, q[0]);
    if (color == 2) {
        dtt_rows(DST4, Q, tmp);
        dtt_cols(DCT4, tmp, q[1]);
    } else {
        /* R, B: SC from CC by mirroring columns (:3459-3475) */
        double neg = 1.0 - 2.0 * (double)((itlx & 1) ^ (1 ^ color));
        for (int i = 0; i < 8; i++)
            for (int j = 0; j < 8; j++) q[1][i][7 - j] = neg * q[0][i][j];
    }
    /* CC -> SS, SC -> CS down the anti-diagonal (:3486-3504) */
    double neg2 = 1.0 - 2.0 * (double)((itlx & 1) ^ (itly & 1) ^ (1 ^ 0 ^ c1));
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) {
            q[3][7 - i][7 - j] = neg2 * q[0][i][j];
            q[2][7 - i][7 - j] = neg2 * q[1][i][j];
        }

    /* convolution with the CLT-domain kernel (:2778-2827) */
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) {
            double a0 = q[0][i][j], a1 = q[1][i][j], a2 = q[2][i][j], a3 = q[3][i][j];
            double k0 = kr[0 * 64 + i * 8 + j], k1 = kr[1 * 64 + i * 8 + j];
            double k2 = kr[2 * 64 + i * 8 + j], k3 = kr[3 * 64 + i * 8 + j];
            q[0][i][j] = a0 * k0 - a1 * k1 - a2 * k2 + a3 * k3;
            q[1][i][j] = a1 * k0 + a0 * k1 - a3 * k2 - a2 * k3;
            q[2][i][j] = a2 * k0 - a3 * k1 + a0 * k2 - a1 * k3;
            q[3][i][j] = a3 * k0 + a2 * k1 + a1 * k2 + a0 * k3;
        }
    /* phase rotation by the residual shift: horizontal per column j, then
     * vertical per row i (:2715-2776) */
    for (int j = 0; j < 8; j++) {
        double a = M_PI * (double)shx * (2 * j + 1) / 16.0, ch = cos(a), sh = sin(a);
        for (int i = 0; i < 8; i++) {
            double x0 = q[0][i][j], x1 = q[1][i][j], x2 = q[2][i][j], x3 = q[3][i][j];
            q[0][i][j] = x0 * ch - x1 * sh; q[1][i][j] = x0 * sh + x1 * ch;
            q[2][i][j] = x2 * ch - x3 * sh; q[3][i][j] = x2 * sh + x3 * ch;
        }
    }
    for (int i = 0; i < 8; i++) {
        double a = M_PI * (double)shy * (2 * i + 1) / 16.0, ch = cos(a), sh = sin(a);
        for (int j = 0; j < 8; j++) {
            double x0 = q[0][i][j], x1 = q[1][i][j], x2 = q[2][i][j], x3 = q[3][i][j];
            q[0][i][j] = x0 * ch - x2 * sh; q[2][i][j] = x0 * sh + x2 * ch;
            q[1][i][j] = x1 * ch - x3 * sh; q[3][i][j] = x1 * sh + x3 * ch;
        }
    }
    if ((lpf_mask >> color) & 1) /* optional LPF (:3572-3593) */
        for (int k = 0; k < 4; k++)
            for (int i = 0; i < 8; i++)
                for (int j = 0; j < 8; j++) q[k][i][j] *= lpf[color * 64 + i * 8 + j];

    /* store: tile index uses (txy & 0xfff) for x (:3606) */
    int tx = t->txy & 0xfff, ty = t->txy >> 16;
    double *dst = clt_cam + (((size_t)ty * TX + tx) * 3 + color) * 256;
    for (int k = 0; k < 4; k++)
        for (int i = 0; i < 8; i++)
            for (int j = 0; j < 8; j++) dst[k * 64 + i * 8 + j] = q[k][i][j];
}

int tpo_convert_correct_tiles(const tp_geometry *g, const float *const *kernel_offsets,
                              const float *const *kernels, const float *const *images,
                              size_t dstride, const tp_task *tasks, int num_tiles,
                              int lpf_mask, const float *lpf, double *const *clt, int *corners)
{
    init_tables();
    float deflpf[4 * 64];
    if (!lpf) {
        for (int c = 0; c < 4; c++) tpo_default_lpf(c, deflpf + 64 * c);
        lpf = deflpf;
    }
    const int TX = tiles_x(g), TY = tiles_y(g);
    int done = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : done) num_threads(tpo_get_threads())
    for (int n = 0; n < num_tiles; n++) {
        const tp_task *t = tasks + n;
        if (!t->task) continue;
        int tx = t->txy & 0xfff, ty = t->txy >> 16;
        if (tx < 0 || tx >= TX || ty < 0 || ty >= TY) continue;
        for (int cam = 0; cam < 4; cam++)
            for (int color = 0; color < 3; color++) {
                convert_one(g, kernel_offsets[cam], kernels[cam], images[cam], dstride, t, cam,
                            color, lpf_mask, lpf, clt[cam],
                            corners ? corners + (((size_t)n * 4 + cam) * 3 + color) * 4 : NULL);
                done++;
            }
    }
    return done;
}

/* ------------------------------------------------------------------------- */
/* correlate2D  (src/TileProcessor.cuh:1176-1443, :2829-3008)                  */
/* ------------------------------------------------------------------------- */
int tpo_correlate2D(const tp_geometry *g, const double *const *clt, int colors,
                    double scale0, double scale1, double scale2, double fat_zero,
                    int num_corr_tiles, const int *corr_indices, size_t corr_stride,
                    int corr_radius, const float *lpf_rb_corr, const float *lpf_corr,
                    double *corrs)
{
    init_tables();
    float lrb[64], lc[64];
    if (!lpf_rb_corr) { tpo_default_lpf(4, lrb); lpf_rb_corr = lrb; }
    if (!lpf_corr) { tpo_default_lpf(5, lc); lpf_corr = lc; }
    const double scales[3] = {scale0, scale1, scale2};
    const int ntiles = tiles_x(g) * tiles_y(g);
    const int r = corr_radius, sz = 2 * r + 1;
    int done = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : done) num_threads(tpo_get_threads())
    for (int n = 0; n < num_corr_tiles; n++) {
        int code = corr_indices[n];
        int tile = code >> 8, pair = code & 0xff;
        if (pair >= 6 || tile < 0 || tile >= ntiles) continue;
        const int c1 = PAIRS[pair][0], c2 = PAIRS[pair][1];
        double acc[4][64];
        memset(acc, 0, sizeof(acc));
        for (int color = 0; color < colors; color++) {
            const double *a = clt[c1] + ((size_t)tile * 3 + color) * 256;
            const double *b = clt[c2] + ((size_t)tile * 3 + color) * 256;
            for (int e = 0; e < 64; e++) {
                double a0 = a[e], a1 = a[64 + e], a2 = a[128 + e], a3 = a[192 + e];
                double b0 = b[e], b1 = b[64 + e], b2 = b[128 + e], b3 = b[192 + e];
                double s = scales[color];
                acc[0][e] += s * ( a0 * b0 + a1 * b1 + a2 * b2 + a3 * b3);
                acc[1][e] += s * (-a1 * b0 + a0 * b1 - a3 * b2 + a2 * b3);
                acc[2][e] += s * (-a2 * b0 - a3 * b1 + a0 * b2 + a1 * b3);
                acc[3][e] += s * ( a3 * b0 - a2 * b1 - a1 * b2 + a0 * b3);
            }
            if (color == 1) /* LPF after R and B (:1263-1304) */
                for (int k = 0; k < 4; k++)
                    for (int e = 0; e < 64; e++) acc[k][e] *= lpf_rb_corr[e];
        }
        for (int e = 0; e < 64; e++) { /* amplitude normalisation (:2915-2942) */
            double s2 = fat_zero * fat_zero;
            for (int k = 0; k < 4; k++) s2 += acc[k][e] * acc[k][e];
            double sc = 1.0 / sqrt(s2);
            for (int k = 0; k < 4; k++) acc[k][e] *= sc * lpf_corr[e];
        }
        /* to the pixel domain: vertical DCT-II (q0,q1) / DST-II (q2,q3), then
         * horizontal DCT-II (q0,q2) / DST-II (q1,q3) (:1369-1388) */
        double pix[4][8][8], tmp[8][8];
        for (int k = 0; k < 4; k++) {
            dtt_cols((k >> 1) ? DST2 : DCT2, (const double (*)[8])acc[k], tmp);
            dtt_rows((k & 1) ? DST2 : DCT2, tmp, pix[k]);
        }
        /* unfold the 4 quadrants into the centred (2r+1)^2 grid (:2950-3008) */
        double *out = corrs + (size_t)n * corr_stride;
        for (int y = -r; y <= r; y++)
            for (int x = -r; x <= r; x++) {
                int i = abs(y), j = abs(x);
                double sy = y < 0 ? -1.0 : 1.0, sx = x < 0 ? -1.0 : 1.0;
                double v = pix[0][i][j];
                if (j > 0) v += sx * pix[1][i][j - 1];
                if (i > 0) v += sy * pix[2][i - 1][j];
                if (i > 0 && j > 0) v += sx * sy * pix[3][i - 1][j - 1];
                out[(r + y) * sz + (r + x)] = 0.25 * v;
            }
        done++;
    }
    return done;
}

/* ------------------------------------------------------------------------- */
/* inverse CLT of one tile (imclt / imclt8threads, :3700-4017)                 */
/* ------------------------------------------------------------------------- */
static const int SGN_C[4] = {1, -1, -1, -1}; /* idct_signs factors (:399-420) */
static const int SGN_S[4] = {1, 1, 1, -1};

static void imclt_tile(const double q[4][8][8], double out[16][16])
{
    double x[4][8][8], tmp[8][8];
    for (int k = 0; k < 4; k++) {
        /* q0: DCT both axes, q1: DST horizontal, q2: DST vertical, q3: DST both */
        dtt_rows((k & 1) ? DST4 : DCT4, q[k], tmp);
        dtt_cols((k >> 1) ? DST4 : DCT4, tmp, x[k]);
    }
    for (int rr = 0; rr < 16; rr++)
        for (int cc = 0; cc < 16; cc++) {
            int a = rr >> 2, b = cc >> 2, u = RIND[rr], v = RIND[cc];
            double d = SGN_C[a] * SGN_C[b] * x[0][u][v] + SGN_C[a] * SGN_S[b] * x[1][u][v] +
                       SGN_S[a] * SGN_C[b] * x[2][u][v] + SGN_S[a] * SGN_S[b] * x[3][u][v];
            out[rr][cc] = TW2[rr] * TW2[cc] * d;
        }
}

/* ------------------------------------------------------------------------- */
/* imclt_rbg  (src/TileProcessor.cuh:2588-2710)                                */
/* ------------------------------------------------------------------------- */
int tpo_imclt_rbg(const tp_geometry *g, const double *clt_one_cam, double *rbg, int color,
                  int v_offset, int h_offset, size_t dstride)
{
    init_tables();
    const int TX = tiles_x(g), TY = tiles_y(g);
    double *plane = rbg + dstride * (size_t)(g->img_height + 8) * color;
    const int pass = (v_offset << 1) + h_offset;
    int done = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : done) num_threads(tpo_get_threads())
    for (int ty = v_offset; ty < TY; ty += 2) {
        for (int tx = h_offset; tx < TX; tx += 2) {
            double q[4][8][8], out[16][16];
            const double *src = clt_one_cam + (((size_t)ty * TX + tx) * 3 + color) * 256;
            memcpy(q, src, sizeof(q));
            imclt_tile(q, out);
            double *top = plane + (size_t)ty * 8 * dstride + (size_t)tx * 8;
            for (int rr = 0; rr < 16; rr++)
                for (int cc = 0; cc < 16; cc++) {
                    double prev = pass ? top[rr * dstride + cc] : 0.0;
                    double v = prev + out[rr][cc];
                    if (g->debug_marks) {
                        if (tx == 0 && ty == 0) v = 100.0;
                        else if (tx == 161 && ty == 111) v *= 2.0;
                    }
                    top[rr * dstride + cc] = v;
                }
            done++;
        }
    }
    return done;
}

/* ------------------------------------------------------------------------- */
/* textures_accumulate  (src/TileProcessor.cuh:2207-2579, :4019-4665)          */
/* ------------------------------------------------------------------------- */

static void debayer_shot(int rb_mode, double min_shot, double scale_shot,
                         const double src[16][16], double dst[16][16])
{
    double t[16][16];
    for (int r = 0; r < 16; r++)      /* remove the squared window (:4028-4044) */
        for (int c = 0; c < 16; c++) t[r][c] = src[r][c] * TWSQI[r] * TWSQI[c];
    for (int r = 0; r < 16; r++)      /* 3x3 debayer of the interior (:4146-4199) */
        for (int c = 0; c < 16; c++) {
            if (r == 0 || r == 15 || c == 0 || c == 15) { dst[r][c] = t[r][c]; continue; }
            double orth = t[r - 1][c] + t[r + 1][c] + t[r][c - 1] + t[r][c + 1];
            if (rb_mode) {
                double diag = t[r - 1][c - 1] + t[r - 1][c + 1] + t[r + 1][c - 1] + t[r + 1][c + 1];
                dst[r][c] = 0.0625 * diag + 0.125 * orth + 0.25 * t[r][c];
            } else {
                dst[r][c] = 0.125 * orth + 0.5 * t[r][c];
            }
        }
    if (scale_shot > 0.0) {           /* shot-noise square root (:4080-4093) */
        double k = 1.0 / sqrt(min_shot);
        for (int r = 0; r < 16; r++)
            for (int c = 0; c < 16; c++) {
                double d = dst[r][c];
                dst[r][c] = scale_shot * ((d > min_shot) ? sqrt(d) : k * d);
            }
    }
    for (int r = 0; r < 16; r++)      /* re-apply the squared window */
        for (int c = 0; c < 16; c++) dst[r][c] *= TWSQ[r] * TWSQ[c];
}

static double rel_gap(double a, double b)
{
    double m = fmax(fabs(a), fabs(b));
    return m > 0 ? fabs(a - b) / m : 0.0;
}

/* Multi-camera fusion of one tile (tile_combine_rgba, :4202-4563).
 * D: debayered, M: plain IMCLT tiles, [cam][color][16][16].
 * out: [slices][16][16]: colors, alpha, 4 port weights, colors+1 rms. */
static void combine_rgba(int colors, const double D[4][3][16][16], const double M[4][3][16][16],
                         const float *port_offsets, double diff_sigma, const double *chw,
                         int dust_remove, int keep_weights, double out[12][16][16],
                         double *margin)
{
    const double ksigma = 1.0 / (2.0 * diff_sigma * diff_sigma);
    double pd2r[6];
    int pp[6][2], np = 0;
    for (int i = 0; i < 4; i++)
        for (int j = i + 1; j < 4; j++) {
            double dx = (double)port_offsets[2 * j] - port_offsets[2 * i];
            double dy = (double)port_offsets[2 * j + 1] - port_offsets[2 * i + 1];
            pp[np][0] = i; pp[np][1] = j;
            pd2r[np++] = ksigma / (dx * dx + dy * dy);
        }
    double (*rgba)[16][16] = out;
    double (*alpha)[16] = out[colors];
    double (*pw)[16][16] = out + colors + 1;
    double (*crms)[16][16] = out + colors + 5;
    for (int r = 0; r < 16; r++)
        for (int c = 0; c < 16; c++) {
            double gap = 1.0;
            if (keep_weights) {
                double sw = 0.0;
                for (int col = 0; col < colors; col++) {
                    double s1 = 0, s2 = 0;
                    for (int cam = 0; cam < 4; cam++) { double d = D[cam][col][r][c]; s1 += d; s2 += d * d; }
                    double mse = (4.0 * s2 - s1 * s1) / 16.0;
                    crms[col][r][c] = sqrt(mse);
                    sw += chw[col] * mse;
                }
                crms[colors][r][c] = sqrt(sw);
            }
            double wnd2 = TWSQ[r] * TWSQ[c];
            double wi = 1.0 / wnd2;
            /* Camera weights are float32 in the reference (the exponential
             * underflows to the 1e-4 floor, making weights exactly equal);
             * they are kept in float here so the best / worst camera choices
             * are the reference's.  Everything else stays FP64. */
            float w[4] = {0, 0, 0, 0};
            for (int p = 0; p < 6; p++) {
                double d = 0.0;
                for (int col = 0; col < colors; col++) {
                    double dc = (D[pp[p][0]][col][r][c] - D[pp[p][1]][col][r][c]) * wi;
                    d += chw[col] * dc * dc;
                }
                float e = (float)(exp(-pd2r[p] * d) + 1e-4);
                w[pp[p][0]] += e;
                w[pp[p][1]] += e;
            }
            int b1 = 0;
            for (int cam = 1; cam < 4; cam++) if (w[cam] > w[b1]) b1 = cam;
            int b2 = (b1 == 0) ? 1 : 0;
            for (int cam = b2 + 1; cam < 4; cam++) if (cam != b1 && w[cam] > w[b2]) b2 = cam;
            for (int cam = 0; cam < 4; cam++) {
                if (cam != b1) gap = fmin(gap, rel_gap(w[b1], w[cam]));
                if (cam != b1 && cam != b2) gap = fmin(gap, rel_gap(w[b2], w[cam]));
            }
            double w1 = (double)w[b1] / ((double)w[b1] + (double)w[b2]), w2 = 1.0 - w1;
            double avg[3];
            for (int col = 0; col < colors; col++) avg[col] = w1 * D[b1][col][r][c] + w2 * D[b2][col][r][c];
            for (int cam = 0; cam < 4; cam++) {
                double d2 = 0.0;
                for (int col = 0; col < colors; col++) {
                    double dc = (D[cam][col][r][c] - avg[col]) * wi;
                    d2 += chw[col] * dc * dc;
                }
                w[cam] = (float)(exp(-ksigma * d2) + 1e-4);
            }
            double wd[4];
            for (int cam = 0; cam < 4; cam++) wd[cam] = w[cam];
            if (dust_remove) {
                int worst = 0;
                for (int cam = 1; cam < 4; cam++) if (w[cam] < w[worst]) worst = cam;
                for (int cam = 0; cam < 4; cam++) if (cam != worst) gap = fmin(gap, rel_gap(w[worst], w[cam]));
                double wv = wd[worst];
                double a = -wv;
                for (int cam = 0; cam < 4; cam++) a += wd[cam];
                a /= 3.0;
                double scale = 1.0 + wv * (a - wv) / (a * a * 3.0);
                for (int cam = 0; cam < 4; cam++) if (cam != worst) wd[cam] *= scale;
                wd[worst] *= wv / a;
            }
            double ws = 0.0;
            for (int cam = 0; cam < 4; cam++) ws += wd[cam];
            for (int col = 0; col < colors; col++) {
                double v = 0.0;
                for (int cam = 0; cam < 4; cam++) v += (wd[cam] / ws) * M[cam][col][r][c];
                rgba[col][r][c] = v;
            }
            alpha[r][c] = wnd2 * ws / 4.0;
            for (int cam = 0; cam < 4; cam++) pw[cam][r][c] = wd[cam];
            if (margin) margin[r * 16 + c] = gap;
        }
}

/* one listed texture tile: fills out[12][16][16] */
static void texture_tile(int tile, const double *const *clt, int colors, const float *lpf,
                         double min_shot, double scale_shot, const float *port_offsets,
                         double diff_sigma, const double *chw, int dust_remove, int keep_weights,
                         double out[12][16][16], double *margin)
{
    double (*D)[3][16][16] = (double (*)[3][16][16])malloc(sizeof(double) * 4 * 3 * 256);
    double (*M)[3][16][16] = (double (*)[3][16][16])malloc(sizeof(double) * 4 * 3 * 256);
    for (int cam = 0; cam < 4; cam++)
        for (int col = 0; col < colors; col++) {
            const double *src = clt[cam] + ((size_t)tile * 3 + col) * 256;
            const float *lp = lpf + 64 * ((colors > 1) ? col : 3);
            double q[4][8][8];
            for (int k = 0; k < 4; k++)
                for (int e = 0; e < 64; e++) q[k][e >> 3][e & 7] = src[k * 64 + e] * lp[e];
            imclt_tile(q, M[cam][col]);
            if (colors > 1)
                debayer_shot(col < 2, min_shot, scale_shot, M[cam][col], D[cam][col]);
            else
                memcpy(D[cam][col], M[cam][col], sizeof(double) * 256);
        }
    combine_rgba(colors, (const double (*)[3][16][16])D, (const double (*)[3][16][16])M,
                 port_offsets, diff_sigma, chw, dust_remove, keep_weights, out, margin);
    free(D);
    free(M);
}

int tpo_textures_accumulate(const tp_geometry *g, const int *woi, const double *const *clt,
                            int num_texture_tiles, const int *texture_indices,
                            const float *port_offsets, int colors, int is_lwir,
                            double min_shot, double scale_shot, double diff_sigma,
                            double diff_threshold, double min_agree, double weight0,
                            double weight1, double weight2, int dust_remove, int keep_weights,
                            size_t texture_rbg_stride, double *texture_rbg, size_t texture_stride,
                            double *texture_tiles, const float *lpf, double *margin)
{
    (void)is_lwir; (void)diff_threshold; (void)min_agree; /* unused by the reference too */
    init_tables();
    float deflpf[4 * 64];
    if (!lpf) {
        for (int c = 0; c < 4; c++) tpo_default_lpf(c, deflpf + 64 * c);
        lpf = deflpf;
    }
    const double chw[3] = {weight0, weight1, weight2};
    const int TX = tiles_x(g), ntiles = TX * tiles_y(g);
    const int nslices_tile = (colors == 3) ? (keep_weights ? 12 : 4) : (keep_weights ? 8 : 2);
    const int nslices_img = colors + 1;
    /* tiles are computed in parallel in chunks; the overlap-add of a chunk
     * runs serially in list order (tiles of one list may overlap) */
    int done = 0;
    const int chunk = 2048;
    double (*outs)[12][16][16] = (double (*)[12][16][16])malloc(sizeof(double) * 12 * 256 * (size_t)chunk);
    const size_t slice_stride = texture_rbg_stride * (size_t)((woi ? woi[3] : 0) + 1) * 8;
    for (int n0 = 0; n0 < num_texture_tiles; n0 += chunk) {
        const int n1 = (n0 + chunk < num_texture_tiles) ? n0 + chunk : num_texture_tiles;
        int valid[2048];
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : done) num_threads(tpo_get_threads())
        for (int n = n0; n < n1; n++) {
            int code = texture_indices[n];
            int tile = code >> 8;
            valid[n - n0] = (code & (1 << 7)) && tile >= 0 && tile < ntiles;
            if (!valid[n - n0]) continue;
            texture_tile(tile, clt, colors, lpf, min_shot, scale_shot, port_offsets, diff_sigma, chw,
                         dust_remove, keep_weights, outs[n - n0], margin ? margin + (size_t)n * 256 : NULL);
            if (texture_tiles && texture_stride) {
                double *dst = texture_tiles + (size_t)n * texture_stride;
                for (int s = 0; s < nslices_tile; s++) {
                    /* colors==1 slices: Y, A, 4 weights, rms, rms_total */
                    const double *src = &outs[n - n0][s][0][0];
                    for (int e = 0; e < 256; e++) dst[s * 256 + e] = src[e];
                }
            }
            done++;
        }
        if (!(texture_rbg && texture_rbg_stride)) continue;
        for (int n = n0; n < n1; n++) {
            if (!valid[n - n0]) continue;
            int code = texture_indices[n];
            int tile = code >> 8;
            int nbr = code & 0xf;
            if (!nbr) continue;
            int tyy = tile / TX, txx = tile - tyy * TX;
            long x0 = (long)(txx - woi[0]) * 8, y0 = (long)(tyy - woi[1]) * 8;
            for (int s = 0; s < nslices_img; s++)
                for (int r = 0; r < 16; r++)
                    for (int c = 0; c < 16; c++) {
                        double v = outs[n - n0][s][r][c];
                        if (nbr != 0xf) v *= AFADE[nbr][r * 16 + c];
                        long gy = y0 + r, gx = x0 + c;
                        if (gy < 0 || gx < 0) continue;
                        texture_rbg[s * slice_stride + (size_t)gy * texture_rbg_stride + gx] += v;
                    }
        }
    }
    free(outs);
    return done;
}

/* ------------------------------------------------------------------------- */
/* texture list  (src/TileProcessor.cuh:1643-1853)                             */
/* ------------------------------------------------------------------------- */
int tpo_prepare_texture_list(const tp_geometry *g, tp_task *tasks, int num_tiles,
                             int *texture_indices, int *num_texture_tiles, int *woi,
                             int width, int height)
{
    const int TX = tiles_x(g), TY = tiles_y(g), TYA = tiles_ya(g);
    const int quarter = TX * (TYA >> 2);
    const int cap = TX * TYA;
    /* marker grid in the index buffer (clear_texture_list, :1716-1728) */
    for (int row = 0; row < height; row++)
        for (int col = 0; col <= width; col++) {
            long idx = (long)col + (long)row * TX;
            if (idx >= 0 && idx < cap) texture_indices[idx] = 0;
        }
    for (int n = 0; n < num_tiles; n++) { /* mark_texture_tiles (:1731-1747) */
        if (!(tasks[n].task & TP_TASK_TEXTURE_BITS)) continue;
        int cxy = tasks[n].txy;
        long idx = (long)(cxy & 0xffff) + (long)(cxy >> 16) * TX;
        if (idx >= 0 && idx < cap) texture_indices[idx] = 1;
    }
    woi[0] = TX; woi[1] = TY; woi[2] = 0; woi[3] = 0;
    int *newtask = (int *)malloc(sizeof(int) * (size_t)(num_tiles > 0 ? num_tiles : 1));
    for (int n = 0; n < num_tiles; n++) { /* mark_texture_neighbor_tiles (:1751-1783) */
        int task = tasks[n].task;
        newtask[n] = task;
        if (!(task & TP_TASK_TEXTURE_BITS)) continue;
        int cxy = tasks[n].txy, x = cxy & 0xffff, y = cxy >> 16;
        if (x < woi[0]) woi[0] = x;
        if (y < woi[1]) woi[1] = y;
        if (x > woi[2]) woi[2] = x;
        if (y > woi[3]) woi[3] = y;
        int d = 0;
#define MK(xx, yy) ((long)(xx) + (long)(yy) * TX)
#define AT(i) (((i) >= 0 && (i) < cap) ? texture_indices[i] : 0)
        if (y > 0 && AT(MK(x, y - 1))) d |= 1;
        if (x < TX - 1 && AT(MK(x + 1, y))) d |= 2;
        if (y < TY - 1 && AT(MK(x, y + 1))) d |= 4;
        if (x > 0 && AT(MK(x - 1, y))) d |= 8;
#undef AT
#undef MK
        newtask[n] = ((task ^ d) & TP_TASK_TEXTURE_BITS) ^ task;
    }
    for (int n = 0; n < num_tiles; n++) tasks[n].task = newtask[n];
    free(newtask);
    for (int k = 0; k < 8; k++) num_texture_tiles[k] = 0;
    for (int n = 0; n < num_tiles; n++) { /* gen_texture_list (:1785-1853) */
        int task = tasks[n].task & TP_TASK_TEXTURE_BITS;
        if (!task) continue;
        int cxy = tasks[n].txy, x = cxy & 0xffff, y = cxy >> 16;
        int border = (x == woi[0]) || (y == woi[1]) || (x == TX - 1) || (y == woi[3]);
        int head = 0, slot = 0;
        if (x & 1) { head += quarter; slot += 2; }
        if (y & 1) { head += 2 * quarter; slot += 4; }
        if (border) { head += quarter - 1; slot += 1; }
        int k = num_texture_tiles[slot]++;
        long pos = border ? (long)head - k : (long)head + k;
        if (pos >= 0 && pos < cap)
            texture_indices[pos] = task | ((x + y * TX) << 8) | (1 << 7);
    }
    woi[2] += 1 - woi[0];
    woi[3] += 1 - woi[1];
    return 0;
}

int tpo_generate_RBGA(const tp_geometry *g, tp_task *tasks, int num_tiles, int *texture_indices,
                      int *num_texture_tiles, int *woi, int width, int height,
                      const double *const *clt, const float *port_offsets, int colors,
                      int is_lwir, double min_shot, double scale_shot, double diff_sigma,
                      double diff_threshold, double min_agree, double weight0, double weight1,
                      double weight2, int dust_remove, int keep_weights,
                      size_t texture_rbga_stride, double *texture_tiles, size_t texture_rbga_rows,
                      const float *lpf)
{
    (void)keep_weights;
    tpo_prepare_texture_list(g, tasks, num_tiles, texture_indices, num_texture_tiles, woi, width,
                             height);
    const int TX = tiles_x(g), TYA = tiles_ya(g), quarter = TX * (TYA >> 2);
    /* clear_texture_rbga (:1618-1634): (w+1)*8 columns (+8 more when the
     * stride allows), (h+1)*8 rows per slice, colors+1 slices */
    size_t rows = (size_t)(woi[3] + 1) * 8 * (size_t)(colors + 1);
    size_t cols = (size_t)(woi[2] + 1) * 8 + 8;
    if (cols > texture_rbga_stride) cols = texture_rbga_stride;
    if (rows > texture_rbga_rows) rows = texture_rbga_rows;
    for (size_t rr = 0; rr < rows; rr++)
        for (size_t cc = 0; cc < cols; cc++) texture_tiles[rr * texture_rbga_stride + cc] = 0.0;
    for (int pass = 0; pass < 8; pass++) {
        int border = pass >> 2;
        int ntt = num_texture_tiles[((pass & 3) << 1) + border];
        int off = (pass & 3) * quarter + (border ? quarter - ntt : 0);
        tpo_textures_accumulate(g, woi, clt, ntt, texture_indices + off, port_offsets, colors,
                                is_lwir, min_shot, scale_shot, diff_sigma, diff_threshold,
                                min_agree, weight0, weight1, weight2, dust_remove, 0,
                                texture_rbga_stride, texture_tiles, 0, NULL, lpf, NULL);
    }
    return 0;
}

/* ---- disparity from the pair correlations (new: the reference leaves this
 * step to its Java caller; this is the method the library implements) ----
 *
 * Pair p = (i, j) of a tile correlates at its peak at rho * b_p, with
 * b_p = port_offsets[j] - port_offsets[i] and rho the residual disparity
 * (true minus task disparity).  The tile's profile is
 *   S(k) = sum over its listed pairs in pair_mask of C_p(k * b_p),
 * k = -r..r, C_p sampled bilinearly in the centred (2r+1)^2 tile; a k whose
 * sample of any contributing pair leaves the tile is not used.  rho is the
 * sub-pixel maximum of S around its first integer argmax k*:
 *   mode 0: parabola through S(k*-1), S(k*), S(k*+1);
 *   mode 1: least-squares parabola through the valid S(k*-2 .. k*+2);
 *   mode 2: centroid of S - min over k*-1 .. k*+1.
 * The sub-pixel offset is kept within [-1, 1]; a fit without a maximum gives
 * k*.  strength = the fitted peak value / number of pairs. */
static int fit_sample(const float *c, int r, double x, double y, double *out)
{
    const double fx0 = floor(x), fy0 = floor(y);
    const int ix = (int)fx0, iy = (int)fy0;
    const double fx = x - fx0, fy = y - fy0;
    const int n = 2 * r + 1;
    if (ix < -r || iy < -r || ix > r || iy > r) return 0;
    if ((fx > 0.0 && ix + 1 > r) || (fy > 0.0 && iy + 1 > r)) return 0;
    double v = (1.0 - fx) * (1.0 - fy) * c[(iy + r) * n + ix + r];
    if (fx > 0.0) v += fx * (1.0 - fy) * c[(iy + r) * n + ix + 1 + r];
    if (fy > 0.0) v += (1.0 - fx) * fy * c[(iy + 1 + r) * n + ix + r];
    if (fx > 0.0 && fy > 0.0) v += fx * fy * c[(iy + 1 + r) * n + ix + 1 + r];
    *out = v;
    return 1;
}

void tpo_fit_profile(const double *S, const int *valid, int r, int mode, double *rho, double *peak)
{
    const int n = 2 * r + 1;
    int km = -1;
    for (int k = 0; k < n; k++)
        if (valid[k] && (km < 0 || S[k] > S[km])) km = k;
    if (km < 0) { *rho = NAN; *peak = 0.0; return; }
    double off = 0.0, pk = S[km];
    if (mode == 0) {
        if (km > 0 && km < n - 1 && valid[km - 1] && valid[km + 1]) {
            const double a = S[km - 1], b = S[km], c = S[km + 1];
            const double den = a - 2.0 * b + c;
            if (den < 0.0) {
                off = 0.5 * (a - c) / den;
                if (off > 1.0) off = 1.0;
                if (off < -1.0) off = -1.0;
                pk = b - 0.25 * (a - c) * off;
            }
        }
    } else if (mode == 1) {
        double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, y0 = 0, y1 = 0, y2 = 0;
        int cnt = 0;
        for (int t = -2; t <= 2; t++) {
            const int k = km + t;
            if (k < 0 || k >= n || !valid[k]) continue;
            const double tt = t, y = S[k];
            s0 += 1; s1 += tt; s2 += tt * tt; s3 += tt * tt * tt; s4 += tt * tt * tt * tt;
            y0 += y; y1 += tt * y; y2 += tt * tt * y;
            cnt++;
        }
        if (cnt >= 3) {
            /* normal equations [s0 s1 s2; s1 s2 s3; s2 s3 s4] [a b c] = [y0 y1 y2] */
            const double det = s0 * (s2 * s4 - s3 * s3) - s1 * (s1 * s4 - s3 * s2) + s2 * (s1 * s3 - s2 * s2);
            if (det != 0.0) {
                const double a = (y0 * (s2 * s4 - s3 * s3) - s1 * (y1 * s4 - s3 * y2) + s2 * (y1 * s3 - s2 * y2)) / det;
                const double b = (s0 * (y1 * s4 - y2 * s3) - y0 * (s1 * s4 - s3 * s2) + s2 * (s1 * y2 - y1 * s2)) / det;
                const double c = (s0 * (s2 * y2 - s3 * y1) - s1 * (s1 * y2 - s3 * y0) + y0 * (s1 * s3 - s2 * s2)) / det;
                if (c < 0.0) {
                    off = -b / (2.0 * c);
                    if (off > 1.0) off = 1.0;
                    if (off < -1.0) off = -1.0;
                    pk = a + b * off + c * off * off;
                }
            }
        }
    } else {
        if (km > 0 && km < n - 1 && valid[km - 1] && valid[km + 1]) {
            const double a = S[km - 1], b = S[km], c = S[km + 1];
            const double m = fmin(a, fmin(b, c));
            const double w = (a - m) + (b - m) + (c - m);
            if (w > 0.0) off = ((c - m) - (a - m)) / w;
        }
    }
    *rho = (km - r) + off;
    *peak = pk;
}

int tpo_disparity_fit(const tp_geometry *g, const float *corrs, size_t corr_stride, int corr_radius,
                      int num_corr_tiles, const int *corr_indices, const float *port_offsets, int pair_mask,
                      int mode, double *disparity, double *strength)
{
    init_tables();
    const int r = corr_radius, n = 2 * r + 1;
    const int ntiles = tiles_x(g) * tiles_y(g);
    double bx[6], by[6];
    for (int p = 0; p < 6; p++) {
        const int i = PAIRS[p][0], j = PAIRS[p][1];
        bx[p] = (double)port_offsets[2 * j] - (double)port_offsets[2 * i];
        by[p] = (double)port_offsets[2 * j + 1] - (double)port_offsets[2 * i + 1];
    }
    int done = 0;
    for (int e = 0; e < num_corr_tiles; e++) {
        const int tile = corr_indices[e] >> 8;
        if (e > 0 && (corr_indices[e - 1] >> 8) == tile) continue; /* not the start of the tile's run */
        if (tile < 0 || tile >= ntiles) continue;
        double S[2 * TP_MAX_CORR_RADIUS + 1];
        int valid[2 * TP_MAX_CORR_RADIUS + 1];
        int npairs = 0;
        for (int k = 0; k < n; k++) { S[k] = 0.0; valid[k] = 1; }
        for (int e2 = e; e2 < num_corr_tiles && (corr_indices[e2] >> 8) == tile; e2++) {
            const int p = corr_indices[e2] & 0xff;
            if (p > 5 || !((pair_mask >> p) & 1)) continue;
            npairs++;
            for (int k = 0; k < n; k++) {
                double v;
                if (fit_sample(corrs + (size_t)e2 * corr_stride, r, (k - r) * bx[p], (k - r) * by[p], &v))
                    S[k] += v;
                else
                    valid[k] = 0;
            }
        }
        if (!npairs) continue;
        double rho, pk;
        tpo_fit_profile(S, valid, r, mode, &rho, &pk);
        disparity[tile] = rho;
        strength[tile] = pk / npairs;
        done++;
    }
    return done;
}
