/*
 * tp_frame.cuh - one frame through the whole hot path with the CLT kept on
 * chip: forward CLT with aberration correction, the tile's camera-pair
 * correlations and its texture, one tile at a time per block.
 *
 * This has no single counterpart in the reference, which runs the three
 * stages as separate kernels through a 963 MB CLT buffer in device memory
 * (convert_correct_tiles, correlate2D, textures_accumulate via generate_RBGA:
 * src/TileProcessor.cuh:1859-1937, :1176-1443, :1446-1615).  The per-stage
 * arithmetic is the same device code as the drop-in kernels, so the CLT and
 * the correlations are bit-identical to theirs.
 *
 * One 96-thread block (12 groups of 8 lanes) per tile, grid-stride over the
 * task list, seven blocks per SM (27.6 KB of shared memory each, the same
 * budget as the texture kernel):
 *   1. forward CLT: group = (colour, camera) job, CLT into shared memory;
 *   2. correlations: groups 0-5, one camera pair each, from shared memory;
 *   3. texture: group = (camera, colour) job, inverse CLT into the
 *      un-windowed tile T in place of the job's CLT, debayer into D;
 *   4. fusion of the four cameras at the block's 256 pixels, faded by the
 *      neighbour mask and added into the overlapped RGBA image.
 * Idle groups in one phase leave their issue slots to the other six blocks
 * of the SM, which are in other phases.
 *
 * The frame runs as four launches, one per 2x2 tile parity, so the tiles of
 * one launch never overlap in the RGBA image: the read-modify-write needs no
 * atomics and every pixel accumulates in a fixed order.  Each launch is a
 * programmatic dependent of the one before: its blocks convert, correlate
 * and texture their first tile while the previous launch drains, and wait
 * for it only before their first RGBA update.
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

constexpr int kFrameThreads = 96;
constexpr int kFrameBlocksPerSm = 7;
/* dynamic shared memory of k_frame, in floats: per job its CLT, then T in
 * place (kJob floats); per group the transpose buffer, the correlation
 * buffers of groups 0-5 (kCorrBuf each) and then the debayered tile D */
constexpr int kFrameSmemFloats = 12 * kJob + 12 * kTB4;
static_assert(6 * kCorrBuf <= 12 * kTB4, "correlation buffers overlay the transpose buffers");
static_assert(kJob >= 256 && kJob % 4 == 0, "a job holds its 256 CLT floats, 16-byte aligned");
constexpr size_t kFrameSmemBytes = sizeof(float) * kFrameSmemFloats;

__global__ void __launch_bounds__(kFrameThreads, kFrameBlocksPerSm) k_frame(
    Geom g, size_t dstride, float *const *kernel_offsets, float *const *kernels, float *const *images,
    const tp_task *__restrict__ tasks, int num_tiles, int parity, FrameParams p, float *__restrict__ corrs,
    const float *__restrict__ port_offsets, const int *__restrict__ woi, size_t rgba_stride,
    float *__restrict__ rgba, float *const *clt_out)
{
    extern __shared__ __align__(16) float smem[];
    float *s_clt = smem;            /* job CLT, job = camera * 3 + colour, then T */
    float *s_x = s_clt + 12 * kJob; /* transposes, correlation buffers, then D    */
    __shared__ float s_pd2r[6], s_chw[3], s_chws[3];

    const int tid = threadIdx.x;
    const int l = tid & 7, grp = tid >> 3;
    const unsigned gm = group_mask();
    /* 1 / (2 sigma^2) times log2(e), as combine_pixel takes it */
    const float ksigma = (float)(1.0 / (2.0 * (double)p.tex.diff_sigma * (double)p.tex.diff_sigma)) * kLog2e;
    if (tid == 0) {
        int k = 0;
        for (int i = 0; i < 4; i++)
            for (int j = i + 1; j < 4; j++) {
                const float dx = port_offsets[2 * j] - port_offsets[2 * i];
                const float dy = port_offsets[2 * j + 1] - port_offsets[2 * i + 1];
                s_pd2r[k++] = ksigma / (dx * dx + dy * dy);
            }
        s_chw[0] = p.tex.w0; s_chw[1] = p.tex.w1; s_chw[2] = p.tex.w2;
        /* D without the window and the shot scale (debayer_job<false>): the
         * distance factors carry the shot scale */
        const float dsc = p.tex.scale_shot > 0.0f ? p.tex.scale_shot : 1.0f;
        for (int c = 0; c < 3; c++) s_chws[c] = sqrtf(s_chw[c]) * dsc;
    }
    /* the next parity launch may be scheduled on the SM slots this grid frees */
    grid_dependents_launch();
    bool waited = false;
    int wx0 = 0, wy0 = 0, wh = 0;
    size_t slice_stride = 0;
    __syncthreads();

    /* this tile's task in this pass */
    auto in_pass = [&](int m) -> bool {
        if (m >= num_tiles) return false;
        const tp_task *c = tasks + m;
        const int ctask = c->task, cxy = c->txy;
        const int cx = cxy & 0xffff, cy = cxy >> 16;
        return ctask && cx < g.TX && cy >= 0 && cy < g.TY && ((cx & 1) | ((cy & 1) << 1)) == parity;
    };
    /* Group (colour, camera) converts the same job of every tile; the inputs
     * of its job in the block's next tile are fetched while the block works
     * on the current one, by asynchronous copies into s_pf[group] (0-5: the
     * kernel tile's offsets 0, 1, 4, 5, 6, 7, the pre_ex order of
     * convert_job; 6-7: the tile centre): the centre after the forward
     * transform, the offsets (and the kernel tile itself into L2) after the
     * correlations, the window's Bayer rows into L2 before the fusion. */
    __shared__ __align__(16) float s_pf[12][8];
    const int color_c = grp >> 2, cam_c = grp & 3;
    int pf_n = -1; /* the tile whose inputs s_pf holds */
    const float step_inv = __int_as_float((127 - g.ls) << 23);
    auto kernel_tile = [&](float cx, float cy) -> size_t {
        const int ktx = min(g.KH - 1, max(0, __float2int_rn(__fmaf_rn(cx, step_inv, 1.0f))));
        const int kty = min(g.KV - 1, max(0, __float2int_rn(__fmaf_rn(cy, step_inv, 1.0f))));
        return ((size_t)ktx + (size_t)kty * g.KH) * 3 + color_c;
    };
    /* this thread's copies landed and the group's visible to all its lanes */
    auto pf_sync = [&]() {
        cp_async_wait_all();
        __syncwarp(gm);
    };
    auto fetch_offsets = [&]() {
        pf_sync();
        if (pf_n < 0) return;
        const size_t kidx = kernel_tile(s_pf[grp][6], s_pf[grp][7]);
        asm volatile("prefetch.global.L2 [%0];" ::"l"(kernels[cam_c] + kidx * 256 + l * 32));
        if (l < 6) cp_async4(&s_pf[grp][l], kernel_offsets[cam_c] + kidx * 8 + (l < 2 ? l : l + 2));
        cp_async_commit();
    };
    /* lane l: rows l and l + 8 of the window, both ends, at the corner the
     * offsets give before the centre correction (a hint: addresses are kept
     * inside the image) */
    auto prefetch_window = [&]() {
        pf_sync();
        if (pf_n < 0) return;
        const float px = s_pf[grp][6] - 8.0f - s_pf[grp][0], py = s_pf[grp][7] - 8.0f - s_pf[grp][1];
        const int x0 = min(max(__float2int_rd(px + 0.5f), 0), g.W - 16);
        const int y0 = min(max(__float2int_rd(py + 0.5f), 0), g.H - 16);
        const float *img_c = images[cam_c];
        const long long img_last = (long long)g.image_rows * (long long)dstride - 1;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const long long a = (long long)(y0 + l + 8 * h) * (long long)dstride + x0;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(img_c + min(max(a, 0LL), img_last)));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(img_c + min(max(a + 15, 0LL), img_last)));
        }
    };

    for (int n = blockIdx.x; n < num_tiles; n += gridDim.x) {
        if (!in_pass(n)) continue;
        const tp_task *t = tasks + n;
        const int task = t->task;
        const int txy = t->txy;
        const int tx = txy & 0xffff, ty = txy >> 16;

        /* ---- 1. forward CLT: warp = colour, group = camera ---- */
        {
            float cx, cy, ex[6];
            if (pf_n == n) {
                cx = s_pf[grp][6]; cy = s_pf[grp][7];
#pragma unroll
                for (int i = 0; i < 6; i++) ex[i] = s_pf[grp][i];
            } else {
                cx = t->xy[cam_c][0]; cy = t->xy[cam_c][1];
                const float *e = kernel_offsets[cam_c] + kernel_tile(cx, cy) * 8;
                ex[0] = __ldg(e + 0); ex[1] = __ldg(e + 1); ex[2] = __ldg(e + 4);
                ex[3] = __ldg(e + 5); ex[4] = __ldg(e + 6); ex[5] = __ldg(e + 7);
            }
            convert_job(g, dstride, kernel_offsets[cam_c], kernels[cam_c], images[cam_c], cx, cy, color_c, p.lpf_mask,
                        s_clt + (cam_c * 3 + color_c) * kJob, reinterpret_cast<float(*)[9]>(s_x + grp * kTB4), l,
                        gm, ex);
        }
        /* the block's next tile in this pass: lane i of every warp tests the
         * tile i + 1 strides on */
        {
            const long long cand = n + (long long)((tid & 31) + 1) * gridDim.x;
            const unsigned m = __ballot_sync(0xffffffffu, cand < num_tiles && in_pass((int)cand));
            pf_n = m ? n + __ffs(m) * (int)gridDim.x : -1;
            /* every lane of the group has read s_pf (before the transposes'
             * first __syncwarp in convert_job) */
            if (pf_n >= 0 && l >= 6) cp_async4(&s_pf[grp][l], &tasks[pf_n].xy[cam_c][l - 6]);
            cp_async_commit();
        }
        __syncthreads();
        if (clt_out) {
            const size_t base = ((size_t)ty * g.TX + tx) * 3;
            for (int e = tid; e < 12 * 256; e += kFrameThreads) {
                const int job = e >> 8, cam = job / 3, color = job - cam * 3;
                clt_out[cam][(base + color) * 256 + (e & 255)] = s_clt[job * kJob + (e & 255)];
            }
        }
        const int pairs = (task >> TP_TASK_CORR_BITS) & 0x3f;
        const int nbr = task & TP_TASK_TEXTURE_BITS;

        /* ---- 2. correlations: group = pair ---- */
        if (grp < 6 && ((pairs >> grp) & 1))
            corr_job<4>(s_clt + c_pairs[grp][0] * 3 * kJob, s_clt + c_pairs[grp][1] * 3 * kJob, kJob, p.corr_colors,
                        p.s0, p.s1, p.s2, p.fat_zero, p.corr_radius, s_x + grp * kCorrBuf,
                        corrs + ((size_t)n * 6 + grp) * p.corr_stride, l, gm);
        /* the convert above has read s_pf: its next contents may be copied in */
        fetch_offsets();
        if (nbr) {
            __syncthreads(); /* the correlations have read the CLT and freed s_x */
            /* ---- 3. inverse CLT to T (in place), debayer to D: group = job ---- */
            {
                const int color = grp % 3;
                float *cj = s_clt + grp * kJob, *xj = s_x + grp * kTB4;
                imclt_unfold_job<false>(cj, d_lpf[color], xj, cj, l, gm);
                debayer_job<false>(cj, xj, color < 2, p.tex.min_shot, p.tex.scale_shot, l, gm);
            }
            __syncthreads();
            prefetch_window();
            /* ---- 4. fuse the cameras and add the faded tile into the RGBA image ---- */
            if (!waited) {
                /* the previous parity launch (or the RGBA clear) writes the image */
                grid_dependency_wait();
                waited = true;
                wx0 = woi[0]; wy0 = woi[1]; wh = woi[3];
                slice_stride = rgba_stride * (size_t)(wh + 1) * 8;
            }
            const int gy0 = (ty - wy0) * 8, gx0 = (tx - wx0) * 8;
#pragma unroll 1
            for (int px = tid; px < 256; px += kFrameThreads) {
                const int r = px >> 4, c = px & 15;
                const float wnd2 = __ldg(&d_tex_wnd2[px]), wi = __ldg(&d_tex_wi[px]);
                /* the pixel's RGBA values, loaded before the fusion covers their latency */
                const int gy = gy0 + r, gx = gx0 + c;
                float *b = (gy < 0 || gx < 0) ? nullptr : rgba + (size_t)gy * rgba_stride + (size_t)gx;
                float old[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                if (b) {
#pragma unroll
                    for (int sl = 0; sl < 4; sl++) old[sl] = b[(size_t)sl * slice_stride];
                }
                float o[12];
                combine_pixel<3, false>(s_x, kTB4, s_clt, kJob, wnd2, JTS(kJS, r, c), s_pd2r, ksigma, s_chw, s_chws, wnd2,
                                        wi, p.tex.dust_remove, 0, o);
                if (!b) continue;
                const float f = (nbr != TP_TASK_TEXTURE_BITS) ? __ldg(&d_alpha_fade[nbr][px]) : 1.0f;
#pragma unroll
                for (int sl = 0; sl < 4; sl++) {
                    const float v = (nbr != TP_TASK_TEXTURE_BITS) ? o[sl] * f : o[sl];
                    b[(size_t)sl * slice_stride] = old[sl] + v;
                }
            }
        }
        if (!nbr) prefetch_window();
        __syncthreads(); /* the tile's buffers free for the next one */
    }
}

} /* namespace tp */
