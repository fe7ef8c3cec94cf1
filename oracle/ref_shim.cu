/*
 * ref_shim.cu - host launchers for the reference kernels, rebuilt for sm_100a.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
 * the reference's own sources, read in place from the reference checkout
 * (src/dtt8x8.cuh and src/TileProcessor.cuh, included by path), into
 * oracle/_ref/libtp_ref_<W>x<H>.so, one library per frame geometry because the
 * reference fixes its geometry at compile time.  The parity tests run the
 * reference kernels through these launchers on the same inputs as the
 * B200-native library.
 *
 * The reference's dynamic-parallelism drivers (generate_RBGA,
 * prepare_texture_list) call device-side cudaDeviceSynchronize(), which CUDA 12
 * no longer has; that call is compiled as a no-op so the file builds,
 * and the drivers are never launched: the launchers below issue their child
 * kernels from the host in the same order, with host synchronisation in place
 * of the device-side one (src/TileProcessor.cuh:1446-1615, :1643-1713).
 *
 * Launch shapes follow the reference's harness (src/dtt8x8.cu:538-1002).
 */
#include <cuda_runtime.h>
#include <stdio.h>

/* The reference's sources, with device-side cudaDeviceSynchronize() (CUDA 11
 * dynamic parallelism, removed in CUDA 12) compiled as a no-op.  The paths
 * come from the Makefile. */
#define cudaDeviceSynchronize() (cudaSuccess)
#include REF_DTT_HEADER
#include REF_TP_HEADER
#undef cudaDeviceSynchronize

#define RET_CUDA(call)                                                              \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            fprintf(stderr, "ref_shim: %s: %s\n", #call, cudaGetErrorString(e_));   \
            return (int)e_;                                                         \
        }                                                                           \
    } while (0)

/* 1: synchronise the device after every launch, as the reference's harness
 * does (src/dtt8x8.cu:574-575); 0: launch back to back on the default stream
 * (the host copies that read the list counts and the window still wait), for
 * timing the kernels themselves. */
static int g_sync = 1;

#define SYNC_AFTER_LAUNCH()                          \
    do {                                             \
        if (g_sync) RET_CUDA(cudaDeviceSynchronize()); \
    } while (0)

extern "C" {

int ref_set_sync(int on)
{
    g_sync = on ? 1 : 0;
    return 0;
}

int ref_tilesx(void) { return TILESX; }
int ref_tilesy(void) { return TILESY; }
int ref_tilesya(void) { return TILESYA; }

int ref_convert_correct_tiles(float **gpu_kernel_offsets, float **gpu_kernels, float **gpu_images,
                              struct tp_task *gpu_tasks, float **gpu_clt, size_t dstride,
                              int num_tiles, int lpf_mask)
{
    dim3 threads(THREADSX, TILES_PER_BLOCK, 1);
    dim3 grid((num_tiles + TILES_PER_BLOCK - 1) / TILES_PER_BLOCK, 1);
    RET_CUDA(cudaFuncSetCacheConfig(convert_correct_tiles, cudaFuncCachePreferShared));
    convert_correct_tiles<<<grid, threads>>>(gpu_kernel_offsets, gpu_kernels, gpu_images, gpu_tasks,
                                             gpu_clt, dstride, num_tiles, lpf_mask);
    RET_CUDA(cudaGetLastError());
    SYNC_AFTER_LAUNCH();
    return 0;
}

int ref_correlate2D(float **gpu_clt, int colors, float scale0, float scale1, float scale2,
                    float fat_zero, size_t num_corr_tiles, int *gpu_corr_indices,
                    size_t corr_stride, int corr_radius, float *gpu_corrs)
{
    dim3 threads(CORR_THREADS_PER_TILE, CORR_TILES_PER_BLOCK, 1);
    dim3 grid((unsigned)((num_corr_tiles + CORR_TILES_PER_BLOCK - 1) / CORR_TILES_PER_BLOCK), 1, 1);
    correlate2D<<<grid, threads>>>(gpu_clt, colors, scale0, scale1, scale2, fat_zero,
                                   num_corr_tiles, gpu_corr_indices, corr_stride, corr_radius,
                                   gpu_corrs);
    RET_CUDA(cudaGetLastError());
    SYNC_AFTER_LAUNCH();
    return 0;
}

int ref_textures_accumulate(int *woi, float **gpu_clt, size_t num_texture_tiles,
                            int *gpu_texture_indices, float *gpu_port_offsets, int colors,
                            int is_lwir, float min_shot, float scale_shot, float diff_sigma,
                            float diff_threshold, float min_agree, float weight0, float weight1,
                            float weight2, int dust_remove, int keep_weights,
                            size_t texture_rbg_stride, float *gpu_texture_rbg,
                            size_t texture_stride, float *gpu_texture_tiles)
{
    dim3 threads(TEXTURE_THREADS_PER_TILE, NUM_CAMS, 1);
    dim3 grid((unsigned)((num_texture_tiles + TEXTURE_TILES_PER_BLOCK - 1) / TEXTURE_TILES_PER_BLOCK), 1, 1);
    if (grid.x == 0) return 0;
    textures_accumulate<<<grid, threads>>>(woi, gpu_clt, num_texture_tiles, gpu_texture_indices,
                                           gpu_port_offsets, colors, is_lwir, min_shot, scale_shot,
                                           diff_sigma, diff_threshold, min_agree, weight0, weight1,
                                           weight2, dust_remove, keep_weights, texture_rbg_stride,
                                           gpu_texture_rbg, texture_stride, gpu_texture_tiles);
    RET_CUDA(cudaGetLastError());
    SYNC_AFTER_LAUNCH();
    return 0;
}

int ref_imclt_rbg(float *gpu_clt, float *gpu_rbg, int color, int v_offset, int h_offset,
                  size_t dstride)
{
    int tilesy_half = (TILESY + (v_offset ^ 1)) >> 1;
    int tilesx_half = (TILESX + (h_offset ^ 1)) >> 1;
    int tiles_in_pass = tilesy_half * tilesx_half;
    dim3 threads(IMCLT_THREADS_PER_TILE, IMCLT_TILES_PER_BLOCK, 1);
    dim3 grid((tiles_in_pass + IMCLT_TILES_PER_BLOCK - 1) / IMCLT_TILES_PER_BLOCK, 1, 1);
    imclt_rbg<<<grid, threads>>>(gpu_clt, gpu_rbg, color, v_offset, h_offset, dstride);
    RET_CUDA(cudaGetLastError());
    SYNC_AFTER_LAUNCH();
    return 0;
}

/* prepare_texture_list with the child kernels launched from the host
 * (src/TileProcessor.cuh:1643-1713). */
int ref_prepare_texture_list(struct tp_task *gpu_tasks, int num_tiles, int *gpu_texture_indices,
                             int *gpu_num_texture_tiles, int *gpu_woi, int width, int height)
{
    const int nthr = 1 << THREADS_DYNAMIC_BITS;
    dim3 threads0(nthr, 1, 1);
    dim3 blocks0((width + nthr - 1) >> THREADS_DYNAMIC_BITS, height, 1);
    clear_texture_list<<<blocks0, threads0>>>(gpu_texture_indices, width, height);
    RET_CUDA(cudaGetLastError());
    SYNC_AFTER_LAUNCH();
    dim3 threads(nthr, 1, 1);
    dim3 blocks((num_tiles + nthr - 1) >> THREADS_DYNAMIC_BITS, 1, 1);
    if (blocks.x) {
        mark_texture_tiles<<<blocks, threads>>>(gpu_tasks, num_tiles, gpu_texture_indices);
        RET_CUDA(cudaGetLastError());
    }
    SYNC_AFTER_LAUNCH();
    int woi0[4] = {TILESX, TILESY, 0, 0};
    RET_CUDA(cudaMemcpy(gpu_woi, woi0, sizeof(woi0), cudaMemcpyHostToDevice));
    if (blocks.x) {
        mark_texture_neighbor_tiles<<<blocks, threads>>>(gpu_tasks, num_tiles, gpu_texture_indices,
                                                         gpu_woi);
        RET_CUDA(cudaGetLastError());
    }
    SYNC_AFTER_LAUNCH();
    RET_CUDA(cudaMemset(gpu_num_texture_tiles, 0, 8 * sizeof(int)));
    if (blocks.x) {
        gen_texture_list<<<blocks, threads>>>(gpu_tasks, num_tiles, gpu_texture_indices,
                                              gpu_num_texture_tiles, gpu_woi);
        RET_CUDA(cudaGetLastError());
    }
    SYNC_AFTER_LAUNCH();
    int woi[4];
    RET_CUDA(cudaMemcpy(woi, gpu_woi, sizeof(woi), cudaMemcpyDeviceToHost));
    woi[2] += 1 - woi[0];
    woi[3] += 1 - woi[1];
    RET_CUDA(cudaMemcpy(gpu_woi, woi, sizeof(woi), cudaMemcpyHostToDevice));
    return 0;
}

/* generate_RBGA with host-launched children (src/TileProcessor.cuh:1446-1615). */
int ref_generate_RBGA(struct tp_task *gpu_tasks, int num_tiles, int *gpu_texture_indices,
                      int *gpu_num_texture_tiles, int *gpu_woi, int width, int height,
                      float **gpu_clt, float *gpu_port_offsets, int colors, int is_lwir,
                      float min_shot, float scale_shot, float diff_sigma, float diff_threshold,
                      float min_agree, float weight0, float weight1, float weight2,
                      int dust_remove, int keep_weights, size_t texture_rbga_stride,
                      float *gpu_texture_tiles)
{
    (void)keep_weights;
    int rc = ref_prepare_texture_list(gpu_tasks, num_tiles, gpu_texture_indices,
                                      gpu_num_texture_tiles, gpu_woi, width, height);
    if (rc) return rc;
    int woi[4], ntt8[8];
    RET_CUDA(cudaMemcpy(woi, gpu_woi, sizeof(woi), cudaMemcpyDeviceToHost));
    RET_CUDA(cudaMemcpy(ntt8, gpu_num_texture_tiles, sizeof(ntt8), cudaMemcpyDeviceToHost));
    int texture_width = (woi[2] + 1) * DTT_SIZE;
    int texture_tiles_height = (woi[3] + 1) * DTT_SIZE;
    int texture_slices = colors + 1;
    const int nthr = 1 << THREADS_DYNAMIC_BITS;
    dim3 threads2(nthr, 1, 1);
    int blocks_x = (texture_width + (1 << (THREADS_DYNAMIC_BITS + DTT_SIZE_LOG2)) - 1) >>
                   (THREADS_DYNAMIC_BITS + DTT_SIZE_LOG2);
    dim3 blocks2(blocks_x, texture_tiles_height * texture_slices, 1);
    clear_texture_rbga<<<blocks2, threads2>>>(texture_width, texture_tiles_height * texture_slices,
                                              texture_rbga_stride, gpu_texture_tiles);
    RET_CUDA(cudaGetLastError());
    SYNC_AFTER_LAUNCH();
    for (int pass = 0; pass < 8; pass++) {
        dim3 threads_texture(TEXTURE_THREADS_PER_TILE, NUM_CAMS, 1);
        int border_tile = pass >> 2;
        int ntt = ntt8[((pass & 3) << 1) + border_tile];
        int ti_offset = (pass & 3) * (TILESX * (TILESYA >> 2));
        if (border_tile) ti_offset += TILESX * (TILESYA >> 2) - ntt;
        if (ntt <= 0) continue;
        dim3 grid_texture((ntt + TEXTURE_TILES_PER_BLOCK - 1) / TEXTURE_TILES_PER_BLOCK, 1, 1);
        textures_accumulate<<<grid_texture, threads_texture>>>(
            gpu_woi, gpu_clt, ntt, gpu_texture_indices + ti_offset, gpu_port_offsets, colors,
            is_lwir, min_shot, scale_shot, diff_sigma, diff_threshold, min_agree, weight0, weight1,
            weight2, dust_remove, 0, texture_rbga_stride, gpu_texture_tiles, 0, gpu_texture_tiles);
        RET_CUDA(cudaGetLastError());
        SYNC_AFTER_LAUNCH();
    }
    return 0;
}

} /* extern "C" */
