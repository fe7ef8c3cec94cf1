/*
 * tp_oracle.h - FP64 CPU restatement of the reference tile processor.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA path is compared
 * against; nothing in the product links or calls it.  Only tests/,
 * __graft_entry__.smoke() and the cpu_baseline / --impl reference legs of
 * bench.py load it.
 *
 * Every function restates, in double precision and in matrix form, the
 * arithmetic of one kernel of mfkiwl/tile_processor_gpu (file:line cited at
 * each definition in tp_oracle.c).  Integer decisions that the reference takes
 * from float32 values (kernel-tile choice, integer tile corner) are taken from
 * the same float32 expressions, so task indexing is bit-exact; all other
 * arithmetic is FP64 with exact constants.  The arguments mirror the C ABI in
 * include/tp_b200.h, with host arrays in place of device pointers and double
 * outputs.
 */
#ifndef TP_ORACLE_H
#define TP_ORACLE_H
#include <stddef.h>
#include "../include/tp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Default constant tables (same generator as the library's). */
void tpo_default_lpf(int which, float out[64]);
void tpo_alpha_fade(double out[16][256]);

/* The 8-point transforms, as 8x8 matrices M[k][n] (y[k] = sum_n M[k][n] x[n]):
 * kind 0 = DCT-IV, 1 = DST-IV (orthonormal), 2 = DCT-II, 3 = DST-II
 * (both scaled by 1/2 for every k, "non-orthonormal"). */
void tpo_dtt_matrix(int kind, double out[64]);

/* convert_correct_tiles.  clt[cam] -> double[tilesy*tilesx*3*256].
 * lpf: 4x64 floats (NULL = defaults).  Returns number of (tile,cam,color)
 * jobs done.  corners (optional, may be NULL): int[num_tiles][4 cams][3 colors][4]
 * = {ktile_x, ktile_y, itlx, itly} per job, for bit-exact index checks. */
int tpo_convert_correct_tiles(const tp_geometry *g,
                              const float *const *kernel_offsets,
                              const float *const *kernels,
                              const float *const *images,
                              size_t dstride,
                              const tp_task *tasks, int num_tiles,
                              int lpf_mask, const float *lpf,
                              double *const *clt,
                              int *corners);

/* correlate2D.  lpf_rb_corr / lpf_corr: 64 floats each (NULL = defaults). */
int tpo_correlate2D(const tp_geometry *g,
                    const double *const *clt, int colors,
                    double scale0, double scale1, double scale2,
                    double fat_zero,
                    int num_corr_tiles, const int *corr_indices,
                    size_t corr_stride, int corr_radius,
                    const float *lpf_rb_corr, const float *lpf_corr,
                    double *corrs);

/* textures_accumulate.  woi: {x,y,w,h} (used with texture_rbg).
 * margin (optional): per listed tile, 256 doubles: the smallest relative gap
 * between the weights of a discrete choice (best port, second port, worst
 * port) taken at that pixel; pixels with a tiny gap may legitimately differ
 * from a float32 implementation. */
int tpo_textures_accumulate(const tp_geometry *g,
                            const int *woi,
                            const double *const *clt,
                            int num_texture_tiles, const int *texture_indices,
                            const float *port_offsets,
                            int colors, int is_lwir,
                            double min_shot, double scale_shot,
                            double diff_sigma, double diff_threshold,
                            double min_agree,
                            double weight0, double weight1, double weight2,
                            int dust_remove, int keep_weights,
                            size_t texture_rbg_stride, double *texture_rbg,
                            size_t texture_stride, double *texture_tiles,
                            const float *lpf,
                            double *margin);

/* imclt_rbg, one parity pass of one color plane. */
int tpo_imclt_rbg(const tp_geometry *g, const double *clt_one_cam, double *rbg,
                  int color, int v_offset, int h_offset, size_t dstride);

/* prepare_texture_list (the lists themselves are built in task order). */
int tpo_prepare_texture_list(const tp_geometry *g, tp_task *tasks, int num_tiles,
                             int *texture_indices, int *num_texture_tiles,
                             int *woi, int width, int height);

/* generate_RBGA: list + clear + 8 accumulation passes. */
int tpo_generate_RBGA(const tp_geometry *g, tp_task *tasks, int num_tiles,
                      int *texture_indices, int *num_texture_tiles, int *woi,
                      int width, int height,
                      const double *const *clt, const float *port_offsets,
                      int colors, int is_lwir,
                      double min_shot, double scale_shot,
                      double diff_sigma, double diff_threshold, double min_agree,
                      double weight0, double weight1, double weight2,
                      int dust_remove, int keep_weights,
                      size_t texture_rbga_stride, double *texture_tiles,
                      size_t texture_rbga_rows,
                      const float *lpf);

/* Disparity fit from the pair correlations (new: the reference leaves it
 * to its Java caller).  Entries of one tile must be adjacent in
 * corr_indices.  disparity / strength: double[tilesx * tilesy], written for
 * tiles with at least one listed pair in pair_mask (residual disparity, in
 * pixels per unit of port offset, and the fitted peak per pair).
 * mode 0: 3-point parabola, 1: 5-point least-squares parabola, 2: 3-point
 * centroid.  Returns the number of tiles fitted. */
int tpo_disparity_fit(const tp_geometry *g, const float *corrs, size_t corr_stride, int corr_radius,
                      int num_corr_tiles, const int *corr_indices, const float *port_offsets, int pair_mask,
                      int mode, double *disparity, double *strength);
/* the sub-pixel step alone, on a profile S[2r+1] with validity flags */
void tpo_fit_profile(const double *S, const int *valid, int r, int mode, double *rho, double *peak);

/* Window tables: 0 = exact (default), 1 = rounded to 6 decimals like the
 * reference's printed tables (used to find outputs sensitive to them). */
void tpo_set_table_mode(int mode);

/* Worker threads used by the tile loops (OpenMP); 0 = all. */
void tpo_set_threads(int n);
int tpo_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
