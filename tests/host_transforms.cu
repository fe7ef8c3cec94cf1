#include <cmath>
#include <cstdio>
#include <random>
// Host check of the library's 8-point transforms (tp_common.cuh dct2_fast,
// dct4_fast) against the closed forms in double precision; built and run by
// tests/test_transforms.py.
#include "tp_common.cuh"
int main() {
    std::mt19937 g(2);
    std::normal_distribution<float> nd(0.f, 1.f);
    double wc = 0, ws = 0, w4c = 0, w4s = 0;
    for (int t = 0; t < 100000; t++) {
        float x[8], a[8], b[8], c[8], d[8];
        for (int i = 0; i < 8; i++) x[i] = nd(g) * (t % 5 == 0 ? 1e4f : 1.f);
        tp::dct2_fast<false>(x, a); tp::dct2_fast<true>(x, b);
        tp::dct4_fast<false>(x, c); tp::dct4_fast<true>(x, d);
        double amax = 0;
        for (int i = 0; i < 8; i++) amax = fmax(amax, fabs((double)x[i]));
        for (int k = 0; k < 8; k++) {
            double r2c = 0, r2s = 0, r4c = 0, r4s = 0;
            for (int n = 0; n < 8; n++) {
                r2c += 0.5 * cos(M_PI * (2 * n + 1) * k / 16.0) * x[n];
                r2s += 0.5 * sin(M_PI * (2 * n + 1) * (k + 1) / 16.0) * x[n];
                r4c += 0.5 * cos(M_PI * (2 * k + 1) * (2 * n + 1) / 32.0) * x[n];
                r4s += 0.5 * sin(M_PI * (2 * k + 1) * (2 * n + 1) / 32.0) * x[n];
            }
            wc = fmax(wc, fabs(a[k] - r2c) / amax); ws = fmax(ws, fabs(b[k] - r2s) / amax);
            w4c = fmax(w4c, fabs(c[k] - r4c) / amax); w4s = fmax(w4s, fabs(d[k] - r4s) / amax);
        }
    }
    printf("max |err| / max|x|: DCT-II %.3g DST-II %.3g DCT-IV %.3g DST-IV %.3g\n", wc, ws, w4c, w4s);
    return (wc < 1e-6 && ws < 1e-6 && w4c < 1e-6 && w4s < 1e-6) ? 0 : 1;
}
