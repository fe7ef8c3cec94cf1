/*
 * tp_frame.cuh - one frame through the whole hot path in one kernel per tile
 * parity: forward CLT with aberration correction, the tile's camera-pair
 * correlations and its texture, with the tile's CLT kept in shared memory.
 *
 * This has no single counterpart in the reference, which runs the three
 * stages as separate kernels through a 963 MB CLT buffer in device memory
 * (convert_correct_tiles, correlate2D, textures_accumulate via generate_RBGA:
 * src/TileProcessor.cuh:1859-1937, :1176-1443, :1446-1615).  The per-stage
 * arithmetic is the same device code as the drop-in kernels.
 *
 * One 128-thread block per tile (grid-stride over the task list):
 *   warps 0-2 (12 groups, one colour per warp) run the 12 forward jobs into
 *   shared memory; after one barrier, warp 3 runs the tile's pair
 *   correlations (4 groups, 2 rounds) while warps 0-2 invert and debayer the
 *   12 (camera, colour) tiles; after a second barrier all 128 threads fuse the
 *   cameras and add the faded RGBA tile into the image.
 * The frame is processed in four launches, one per 2x2 tile parity, so the
 * tiles of one launch never overlap in the RGBA image: the read-modify-write
 * needs no atomics and each pixel accumulates in a fixed order.
 */
#pragma once
#include "tp_common.cuh"
#include "tp_convert.cuh"
#include "tp_correlate.cuh"
#include "tp_texture.cuh"

namespace tp {

struct FrameParams {
    int lpf_mask;
    int corr_colors;
    float s0, s1, s2, fat_zero;
    int corr_radius;
    size_t corr_stride;
    TextureParams tex; /* colors == 3, keep_weights == 0 */
};

/* dynamic shared memory of k_frame, in floats */
constexpr int kFrameSmemFloats = 12 * kCltJob + 12 * kJob + 12 * kJob + 12 * kTB4 + 4 * kCorrBuf + 16 + 2 * kFac;
constexpr size_t kFrameSmemBytes = sizeof(float) * kFrameSmemFloats;

__global__ void __launch_bounds__(128, 3) k_frame(
    Geom g, size_t dstride, float *const *kernel_offsets, float *const *kernels, float *const *images,
    const tp_task *__restrict__ tasks, int num_tiles, int parity, FrameParams p, float *__restrict__ corrs,
    const float *__restrict__ port_offsets, const int *__restrict__ woi, size_t rgba_stride,
    float *__restrict__ rgba, float *const *clt_out)
{
    extern __shared__ __align__(16) float smem[];
    float *s_clt = smem;                      /* the tile's CLT, job = camera * 3 + colour */
    float *s_m = s_clt + 12 * kCltJob;        /* inverse-CLT tiles M                        */
    float *s_t = s_m + 12 * kJob;             /* un-windowed tiles T, then the RGBA slices  */
    float *s_x = s_t + 12 * kJob;             /* transposes, then the debayered tiles D     */
    float *s_corr = s_x + 12 * kTB4;          /* warp 3's correlation buffers               */
    float *s_hsq = s_corr + 4 * kCorrBuf;
    float *s_tfac = s_hsq + 16, *s_mfac = s_tfac + kFac;

    const int tid = threadIdx.x;
    const int l = tid & 7, grp = tid >> 3;
    const unsigned gm = group_mask();
    fill_unfold_factors(s_tfac, s_mfac, tid, 128);
    if (tid < 16) {
        const float s = c_hwin[tid];
        s_hsq[tid] = s * s;
    }
    const int wx0 = woi[0], wy0 = woi[1], wh = woi[3];
    const size_t slice_stride = rgba_stride * (size_t)(wh + 1) * 8;
    const float ksigma = (float)(1.0 / (2.0 * (double)p.tex.diff_sigma * (double)p.tex.diff_sigma));
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
    const float chw[3] = {p.tex.w0, p.tex.w1, p.tex.w2};
    __syncthreads();

    for (int n = blockIdx.x; n < num_tiles; n += gridDim.x) {
        const tp_task *t = tasks + n;
        const int task = t->task;
        const int txy = t->txy;
        const int tx = txy & 0xffff, ty = txy >> 16;
        if (!task || tx >= g.TX || ty < 0 || ty >= g.TY) continue;
        if (((tx & 1) | ((ty & 1) << 1)) != parity) continue;

        /* ---- forward CLT: warp = colour, group = camera ---- */
        if (grp < 12) {
            const int color = grp >> 2, cam = grp & 3;
            convert_job(g, dstride, kernel_offsets[cam], kernels[cam], images[cam], t->xy[cam][0], t->xy[cam][1],
                        color, p.lpf_mask, s_clt + (cam * 3 + color) * kCltJob,
                        reinterpret_cast<float(*)[9]>(s_x + grp * kTB4), l, gm);
        }
        __syncthreads();
        if (clt_out) {
            const size_t base = ((size_t)ty * g.TX + tx) * 3;
            for (int e = tid; e < 12 * 256; e += 128) {
                const int job = e >> 8, cam = job / 3, color = job - cam * 3;
                clt_out[cam][(base + color) * 256 + (e & 255)] = s_clt[job * kCltJob + (e & 255)];
            }
        }
        const int pairs = (task >> TP_TASK_CORR_BITS) & 0x3f;
        const int nbr = task & TP_TASK_TEXTURE_BITS;

        /* ---- correlation on warp 3, texture stages 1-2 on warps 0-2 ---- */
        if (grp >= 12) {
            for (int pair = grp - 12; pair < 6; pair += 4) {
                if (!((pairs >> pair) & 1)) continue;
                corr_job(s_clt + c_pairs[pair][0] * 3 * kCltJob, s_clt + c_pairs[pair][1] * 3 * kCltJob, kCltJob,
                         p.corr_colors, p.s0, p.s1, p.s2, p.fat_zero, p.corr_radius, s_corr + (grp - 12) * kCorrBuf,
                         corrs + ((size_t)n * 6 + pair) * p.corr_stride, l, gm);
            }
        } else if (nbr) {
            const int cam = grp / 3, color = grp - cam * 3;
            float *mj = s_m + grp * kJob, *tj = s_t + grp * kJob, *xj = s_x + grp * kTB4;
            imclt_unfold_job(s_clt + (cam * 3 + color) * kCltJob, d_lpf[color], xj, mj, tj, s_tfac, s_mfac, l, gm);
            debayer_job(tj, xj, color < 2, p.tex.min_shot, p.tex.scale_shot, l, gm);
        }
        if (nbr) {
            __syncthreads();
            /* ---- fuse the cameras; slices to s_t ---- */
#pragma unroll 1
            for (int px = tid; px < 256; px += 128) {
                const int r = px >> 4, c = px & 15;
                const float wnd2 = s_hsq[sym8(r)] * s_hsq[sym8(c)];
                float o[12];
                combine_pixel<3>(s_x, kTB4, s_m, kJob, 1.0f, JT(r, c), pd2r, ksigma, chw, wnd2, __frcp_rn(wnd2),
                                 p.tex.dust_remove, 0, o);
#pragma unroll
                for (int sl = 0; sl < 4; sl++) s_t[sl * kJob + JT(r, c)] = o[sl];
            }
            __syncthreads();
            /* ---- fade by the neighbour mask and add into the RGBA image ---- */
            const long long x0 = (long long)(tx - wx0) * 8, y0 = (long long)(ty - wy0) * 8;
            for (int e = tid; e < 4 * 256; e += 128) {
                const int s = e >> 8, r = (e >> 4) & 15, c = e & 15;
                float v = s_t[s * kJob + JT(r, c)];
                if (nbr != TP_TASK_TEXTURE_BITS) v *= __ldg(&d_alpha_fade[nbr][r * 16 + c]);
                const long long gy = y0 + r, gx = x0 + c;
                if (gy < 0 || gx < 0) continue;
                float *pdst = rgba + (size_t)s * slice_stride + (size_t)gy * rgba_stride + (size_t)gx;
                *pdst += v;
            }
        }
        __syncthreads();
    }
}

} /* namespace tp */
