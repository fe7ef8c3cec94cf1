/*
 * tp_common.cuh - shared device code of the B200 tile processor.
 *
 * Work decomposition used by every kernel: one 8x8 transform job (one tile,
 * camera and color) is owned by a group of 8 consecutive lanes of a warp.
 * Lane l of the group holds one row or one column of each 8x8 quadrant in
 * registers, so the 8-point transforms along the held direction are
 * butterflies in registers (dct4_fast, dct2_fast); the other direction goes
 * through one 8x9 shared-memory
 * transpose per quadrant, padded so that both the row writes and the column
 * reads are bank-conflict free.  Groups never wait on each other: the only
 * synchronisation is __syncwarp on the group's 8-lane mask, so a block has no
 * block-wide barrier and groups of a warp may take different paths.
 */
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/tp_b200.h"
#include "tp_tables.inc"

namespace tp {

/* ---- constant tables (generated by gen_tables.py) -------------------------- */
__device__ __constant__ float c_hwin[16] = TP_HWIN_INIT;
__device__ __constant__ float c_hwinc[16] = TP_HWINC_INIT;
/* Tables that lanes index by their own row / column live in global memory
 * and are read through the read-only data cache: the lanes of a warp then
 * fetch distinct words in one pass, where the constant cache would serialise
 * them.  Runtime-settable low-pass filters: lpf_data[0..3], lpf_rb_corr,
 * lpf_corr. */
__device__ __align__(16) float d_lpf[6][64] = TP_LPF_DEFAULT_INIT;
__device__ float d_alpha_fade[16][256] = TP_ALPHA_FADE_INIT;
__device__ float d_hwin[16] = TP_HWIN_INIT;
__device__ float d_hwinc[16] = TP_HWINC_INIT;
/* camera pairs (src/TileProcessor.cuh:484-490) */
__device__ __constant__ int c_pairs[6][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {0, 3}, {2, 1}};

/* Geometry as kernels see it. */
struct Geom {
    int W, H;        /* image size                                  */
    int TX, TY, TYA; /* tiles                                       */
    int KH, KV, ls;  /* kernel table grid and log2 step             */
    int image_rows;  /* rows allocated per source image             */
    int border_mode;
    int debug_marks;
};

/* Per-group buffer for four 8x9 quadrant transposes, padded to 296 floats
 * (296 % 32 == 8) so that the four groups of a warp hit distinct banks. */
constexpr int kTB4 = 4 * 72 + 8;
#define TBI(q, r, c) ((q) * 72 + (r) * 9 + (c))

__device__ __forceinline__ unsigned group_mask() { return 0xffu << (threadIdx.x & 24); }

/* One (camera, colour) CLT tile staged in shared memory: 256 coefficients
 * padded to 264 floats (264 % 32 == 8, 16-byte multiple), so the four groups
 * of a warp reading column l of their own job hit distinct banks. */
constexpr int kCltJob = 264;

/* Asynchronous global -> shared copies (LDGSTS).  Completion is awaited with
 * cp_async_wait_all() by the issuing thread; other threads see the data after
 * a following block barrier. */
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4(void *sdst, const void *gsrc)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

/* Programmatic dependent launch.  A kernel launched with programmatic stream
 * serialisation may start while the launch before it on the stream is still
 * running: grid_dependency_wait() blocks the calling thread until that grid
 * has completed and its memory operations are visible (a no-op for an
 * ordinary launch), and grid_dependents_launch() lets such a dependent grid
 * be scheduled once every block of this grid has issued it. */
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_launch() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

/* 8-point DCT-IV (SINE false) or DST-IV (SINE true) with the tables' scale,
 * y[k] = 0.5 sum_n x[n] cos|sin(pi (2k+1)(2n+1) / 32), through a 4-point
 * complex transform: with a_m = x[2m], b_m = x[7-2m] (swapped for the sine,
 * as DST-IV x = (-1)^k DCT-IV of x reversed), z_m = (a_m - i b_m)
 * e^{i pi m / 8}, Z_p = sum_m z_m i^{mp} and Y_p = 0.5 e^{i pi (4p+1) / 32}
 * Z_p: y[2p] = Re Y_p, y[7-2p] = Im Y_p (negated for the sine).  44
 * operations against the 64 multiply-adds of the matrix product. */
template <bool SINE>
__host__ __device__ __forceinline__ void dct4_fast(const float x[8], float y[8])
{
    constexpr float pre[4][2] = TP_DCT4_PRE_INIT;
    constexpr float post[4][2] = TP_DCT4_POST_INIT;
    float zr[4], zi[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const float a = SINE ? x[7 - 2 * m] : x[2 * m];
        const float b = SINE ? x[2 * m] : x[7 - 2 * m];
        if (m == 0) {
            zr[0] = a;
            zi[0] = -b;
        } else {
            zr[m] = fmaf(a, pre[m][0], b * pre[m][1]);
            zi[m] = fmaf(a, pre[m][1], -(b * pre[m][0]));
        }
    }
    const float s02r = zr[0] + zr[2], s02i = zi[0] + zi[2], d02r = zr[0] - zr[2], d02i = zi[0] - zi[2];
    const float s13r = zr[1] + zr[3], s13i = zi[1] + zi[3], d13r = zr[1] - zr[3], d13i = zi[1] - zi[3];
    const float Zr[4] = {s02r + s13r, d02r - d13i, s02r - s13r, d02r + d13i};
    const float Zi[4] = {s02i + s13i, d02i + d13r, s02i - s13i, d02i - d13r};
#pragma unroll
    for (int p = 0; p < 4; p++) {
        const float yr = fmaf(Zr[p], post[p][0], -(Zi[p] * post[p][1]));
        const float yi = fmaf(Zr[p], post[p][1], Zi[p] * post[p][0]);
        y[2 * p] = yr;
        y[7 - 2 * p] = SINE ? -yi : yi;
    }
}

/* 8-point DCT-II (SINE false) or DST-II (SINE true) with the tables' scale,
 * y[k] = 0.5 sum_n x[n] cos(pi (2n+1) k / 16) | sin(pi (2n+1) (k+1) / 16):
 * the even outputs are the 4-point DCT-II of u_n = x_n + x_{7-n}, the odd
 * ones the 4-point DCT-IV of v_n = x_n - x_{7-n} (through a 2-point complex
 * transform, as in dct4_fast); the DST-II is the DCT-II of (-1)^n x_n with
 * the outputs in reverse order.  36 operations against 64. */
template <bool SINE>
__host__ __device__ __forceinline__ void dct2_fast(const float xin[8], float y[8])
{
    constexpr float K[8] = TP_DCT2_FAST_INIT;
    float x[8];
#pragma unroll
    for (int n = 0; n < 8; n++) x[n] = (SINE && (n & 1)) ? -xin[n] : xin[n];
    const float u0 = x[0] + x[7], u1 = x[1] + x[6], u2 = x[2] + x[5], u3 = x[3] + x[4];
    const float v0 = x[0] - x[7], v1 = x[1] - x[6], v2 = x[2] - x[5], v3 = x[3] - x[4];
    const float w0 = u0 + u3, w1 = u1 + u2, d0 = u0 - u3, d1 = u1 - u2;
    float r[8];
    r[0] = 0.5f * (w0 + w1);
    r[4] = K[0] * (w0 - w1);
    r[2] = fmaf(d0, K[1], d1 * K[2]);
    r[6] = fmaf(d0, K[2], -(d1 * K[1]));
    /* 4-point DCT-IV of v: z0 = v0 - i v3, z1 = (v2 - i v1) e^{i pi / 4} */
    const float z1r = K[3] * (v2 + v1), z1i = K[3] * (v2 - v1);
    const float p0r = v0 + z1r, p0i = z1i - v3; /* Z_0 = z0 + z1 */
    const float p1r = v0 - z1r, p1i = -v3 - z1i; /* Z_1 = z0 - z1 */
    r[1] = fmaf(p0r, K[4], -(p0i * K[5]));
    r[7] = fmaf(p0r, K[5], p0i * K[4]);
    r[5] = fmaf(p1r, K[6], -(p1i * K[7]));
    r[3] = fmaf(p1r, K[7], p1i * K[6]);
#pragma unroll
    for (int k = 0; k < 8; k++) y[k] = SINE ? r[7 - k] : r[k];
}

/* y[k] = sum_n M[k][n] x[n] for the four 8-point transforms of the tables:
 * DCT-IV / DST-IV (KIND 0 / 1) through dct4_fast, DCT-II / DST-II (KIND 2 /
 * 3) through dct2_fast */
template <int KIND>
__device__ __forceinline__ void dtt8(const float x[8], float y[8])
{
    if constexpr (KIND == 0 || KIND == 1)
        dct4_fast<KIND == 1>(x, y);
    else
        dct2_fast<KIND == 3>(x, y);
}

/* 8x8 transpose inside an 8-lane group through an 8x9 buffer: lane l
 * contributes row l (in[0..7]) and receives column l (out[0..7]). */
__device__ __forceinline__ void group_transpose(float (*buf)[9], const float in[8], float out[8], int l,
                                                unsigned gm)
{
#pragma unroll
    for (int k = 0; k < 8; k++) buf[l][k] = in[k];
    __syncwarp(gm);
#pragma unroll
    for (int k = 0; k < 8; k++) out[k] = buf[k][l];
    __syncwarp(gm);
}

/* window sample n -> DTT index (4..7, 7..4, 3..0, 0..3) and back: the two
 * samples that fold onto index u have opposite parity; return the one with
 * parity p. */
__device__ __forceinline__ int fold_sample(int u, int p)
{
    int a = (u >= 4) ? u - 4 : 11 - u;
    int b = (u >= 4) ? 11 - u : 12 + u;
    return ((a & 1) == p) ? a : b;
}

/* sign of the cosine / sine fold branch for window sample n */
__device__ __forceinline__ float fold_sign_c(int n) { return n < 4 ? 1.0f : -1.0f; }
__device__ __forceinline__ float fold_sign_s(int n) { return n < 12 ? 1.0f : -1.0f; }

/* window value w(n + s) = sin(pi (2 (n + s) + 1) / 32) from (cos, sin)(pi s / 16);
 * n uniform across the warp */
__device__ __forceinline__ float shifted_window(int n, float cs, float sn)
{
    return __fmaf_rn(c_hwin[n], cs, c_hwinc[n] * sn);
}
/* the same with a lane-dependent n */
__device__ __forceinline__ float shifted_window_lane(int n, float cs, float sn)
{
    return __fmaf_rn(__ldg(&d_hwin[n]), cs, __ldg(&d_hwinc[n]) * sn);
}

} /* namespace tp */
