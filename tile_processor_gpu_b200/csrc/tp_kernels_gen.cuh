/*
 * tp_kernels_gen.cuh - CLT aberration-kernel tables from spatial kernels.
 *
 * The reference loads its kernel tables from files written by its Java
 * caller (src/dtt8x8.cu:228-238, 357-376), which is not part of it; this is
 * the generator the library defines.  A spatial kernel h[m][n] (m vertical,
 * n horizontal, taps -7..7) becomes the four CLT quadrants that
 * convert_correct_tiles multiplies in (the layout of one [4][8][8] table
 * entry, CC, SC, CS, SS):
 *   K_q[u][v] = sum_mn h[m][n] A_q(u, m) B_q(v, n),
 *   A = cos(pi m (2u+1) / 16) for CC, SC and sin(...) for CS, SS (vertical),
 *   B = cos(pi n (2v+1) / 16) for CC, CS and sin(...) for SC, SS (horizontal),
 * i.e. every tap as the CLT-domain shift by (n, m).  A unit tap at the centre
 * gives the identity kernel (CC = 1, others 0).  The CLT-domain product equals
 * the spatial convolution only approximately (each tap rotates the phase
 * without moving the window): on interior pixels of the inverse transform the
 * error is 1.5e-4 of the signal for a Gaussian of sigma 0.3 px, 0.5% at
 * 0.5 px, 4% at 1 px.
 *
 * One block per kernel: 120 threads form the 2 x 8 x 15 vertical partial
 * sums (double), then 256 threads the outputs.
 */
#pragma once
#include "tp_common.cuh"

namespace tp {

constexpr int kGenTaps = 15; /* taps -7..7 */

__global__ void __launch_bounds__(256) k_psf_to_clt(const float *__restrict__ psf, long long n,
                                                    float *__restrict__ out)
{
    __shared__ double s_h[kGenTaps * kGenTaps];
    __shared__ double s_t[2][8][kGenTaps]; /* [vertical cos|sin][u][n] */
    __shared__ double s_cs[2][8][kGenTaps]; /* cos, sin of pi m (2u+1) / 16 */
    const int tid = threadIdx.x;
    for (int i = tid; i < 8 * kGenTaps; i += blockDim.x) {
        const int u = i / kGenTaps, m = i - u * kGenTaps - 7;
        double s, c;
        sincospi((double)(m * (2 * u + 1)) / 16.0, &s, &c);
        s_cs[0][u][m + 7] = c;
        s_cs[1][u][m + 7] = s;
    }
    for (long long k = blockIdx.x; k < n; k += gridDim.x) {
        __syncthreads();
        const float *h = psf + (size_t)k * kGenTaps * kGenTaps;
        for (int i = tid; i < kGenTaps * kGenTaps; i += blockDim.x) s_h[i] = (double)h[i];
        __syncthreads();
        if (tid < 2 * 8 * kGenTaps) {
            const int t = tid / (8 * kGenTaps), r = tid - t * 8 * kGenTaps;
            const int u = r / kGenTaps, nn = r - u * kGenTaps;
            double acc = 0.0;
            for (int m = 0; m < kGenTaps; m++) acc = fma(s_cs[t][u][m], s_h[m * kGenTaps + nn], acc);
            s_t[t][u][nn] = acc;
        }
        __syncthreads();
        {
            const int q = tid >> 6, u = (tid >> 3) & 7, v = tid & 7;
            const int vert = q >> 1, hor = q & 1; /* CC 0,0  SC 0,1  CS 1,0  SS 1,1 */
            double acc = 0.0;
            for (int nn = 0; nn < kGenTaps; nn++) acc = fma(s_t[vert][u][nn], s_cs[hor][v][nn], acc);
            out[(size_t)k * 256 + tid] = (float)acc;
        }
    }
}

} /* namespace tp */
