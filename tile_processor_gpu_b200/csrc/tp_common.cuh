/*
 * tp_common.cuh - shared device code of the B200 tile processor.
 *
 * Work decomposition used by every kernel: one 8x8 transform job (one tile,
 * camera and color) is owned by a group of 8 consecutive lanes of a warp.
 * Lane l of the group holds one row or one column of each 8x8 quadrant in
 * registers, so the 8-point transforms along the held direction are plain
 * register matrix-vector products (the DTT matrices are __constant__ operands
 * of the FMAs); the other direction goes through one 8x9 shared-memory
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
__device__ __constant__ float c_dct4[8][8] = TP_DCT4_INIT;
__device__ __constant__ float c_dst4[8][8] = TP_DST4_INIT;
__device__ __constant__ float c_dct2[8][8] = TP_DCT2_INIT;
__device__ __constant__ float c_dst2[8][8] = TP_DST2_INIT;
__device__ __constant__ float c_hwin[16] = TP_HWIN_INIT;
__device__ __constant__ float c_hwinc[16] = TP_HWINC_INIT;
__device__ __constant__ int c_rind[16] = TP_RIND_INIT;
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

/* y[k] = sum_n M[k][n] x[n] with M a constant table */
template <int KIND>
__device__ __forceinline__ void dtt8(const float x[8], float y[8])
{
#pragma unroll
    for (int k = 0; k < 8; k++) {
        float a = 0.0f;
#pragma unroll
        for (int n = 0; n < 8; n++) {
            float m = KIND == 0 ? c_dct4[k][n] : KIND == 1 ? c_dst4[k][n] : KIND == 2 ? c_dct2[k][n] : c_dst2[k][n];
            a = __fmaf_rn(m, x[n], a);
        }
        y[k] = a;
    }
}

/* Same with the matrix chosen at run time (group-uniform). */
__device__ __forceinline__ void dtt8_sel(int sine, int dtt2, const float x[8], float y[8])
{
    if (dtt2) {
        if (sine) dtt8<3>(x, y); else dtt8<2>(x, y);
    } else {
        if (sine) dtt8<1>(x, y); else dtt8<0>(x, y);
    }
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
