"""Generate tp_tables.inc: the constant tables of the CUDA kernels.

Run from this directory: ``python gen_tables.py`` (the build does not run it;
the generated file is committed).  Every table is computed here from its
closed form, in double precision, and printed as a correctly rounded float:

* ``TP_DCT4 / TP_DST4``   orthonormal 8-point DCT-IV / DST-IV, M[k][n] =
  0.5 cos|sin(pi (2k+1)(2n+1) / 32) -- the transforms of the reference's
  dctiv_nodiverg / dstiv_nodiverg (src/dtt8x8.cuh:621-745);
* ``TP_DCT2 / TP_DST2``   DCT-II / DST-II scaled by 1/2 for every k, the
  reference's dttii_shared_mem_nonortho (src/dtt8x8.cuh:382-463);
* ``TP_DCT4_PRE / TP_DCT4_POST``  the twiddles of the 8-point DCT-IV through
  a 4-point complex transform: (cos, sin)(pi m / 8), m = 0..3, and
  0.5 (cos, sin)(pi (4p+1) / 32), p = 0..3 (tp_common.cuh dct4_fast);
* ``TP_DCT2_FAST``         the constants of the 8-point DCT-II split into a
  4-point DCT-II and a 4-point DCT-IV: 0.5 cos(pi/4), 0.5 cos(pi/8),
  0.5 cos(3 pi/8), cos(pi/4), 0.5 (cos, sin)(pi/16), 0.5 (cos, sin)(5 pi/16)
  (tp_common.cuh dct2_fast);
* ``TP_TEX_TFAC / TP_TEX_MFAC / TP_TEX_WND2 / TP_TEX_WI``  per-pixel factors
  of the texture kernel, computed from the float TP_HWIN values in float32
  arithmetic in the device's operation order (so they equal what the kernel
  would compute): tfac[r][c] = (0.25 / w[c]) / w[r], mfac[r][c] = (0.5 w[r])
  (0.5 w[c]) ([16][17], column 16 zero), wnd2 = w[r]^2 w[c]^2 and
  wi = 1 / wnd2 ([256]);
* ``TP_HWIN / TP_HWINC``  sin / cos (pi (2n+1) / 32), n = 0..15: the 16-tap
  lapped window and its quadrature (HWINDOW, src/TileProcessor.cuh:374-383);
* ``TP_RIND``             window sample -> DTT index of the fold / unfold
  (fold_indx2, imclt_indx9: src/TileProcessor.cuh:386-395);
* ``TP_LPF_DEFAULT``      the default low-pass filters (lpf_data[4],
  lpf_rb_corr, lpf_corr; src/TileProcessor.cuh:421-481): separable DCT-III of
  exp(-n^2 / (2 s)) normalised to 1 at DC and rounded to 8 decimals, with
  s = 0.9, 0.9, 0.6, 0.4, 0.5, 0.9;
* ``TP_ALPHA_FADE``       texture fade masks by neighbour code
  (alphaFade, generator at src/TileProcessor.cuh:316-369).
"""
import math
import os


def f32(x):
    return "%.9ef" % x


def dtt(kind):
    m = []
    for k in range(8):
        row = []
        for n in range(8):
            if kind == 0:
                v = 0.5 * math.cos(math.pi * (2 * k + 1) * (2 * n + 1) / 32.0)
            elif kind == 1:
                v = 0.5 * math.sin(math.pi * (2 * k + 1) * (2 * n + 1) / 32.0)
            elif kind == 2:
                v = 0.5 * math.cos(math.pi * (2 * n + 1) * k / 16.0)
            else:
                v = 0.5 * math.sin(math.pi * (2 * n + 1) * (k + 1) / 16.0)
            row.append(v)
        m.append(row)
    return m


def default_lpf(which):
    s = [0.9, 0.9, 0.6, 0.4, 0.5, 0.9][which]
    g = [math.exp(-(n * n) / (2.0 * s)) for n in range(8)]
    f = []
    for u in range(8):
        acc = g[0] + sum(2.0 * g[n] * math.cos(math.pi * n * (2 * u + 1) / 16.0) for n in range(1, 8))
        f.append(acc)
    out = []
    for u in range(8):
        for v in range(8):
            val = (f[u] / f[0]) * (f[v] / f[0])
            out.append(round(val * 1e8) / 1e8)
    return out


def alpha_fade():
    fade = [0.5 * (1.0 - math.cos(math.pi * (i + 0.5) / 16.0)) for i in range(16)]
    out = []
    for m in range(16):
        t = []
        for i in range(16):
            for j in range(16):
                if m == 0:
                    v = 0.0
                elif m == 1:
                    v = fade[15 - i]
                elif m == 2:
                    v = fade[j]
                elif m == 4:
                    v = fade[i]
                elif m == 8:
                    v = fade[15 - j]
                elif m == 3:
                    v = fade[j] if j > 15 - i else fade[15 - i]
                elif m == 6:
                    v = fade[j] if j > i else fade[i]
                elif m == 9:
                    v = fade[15 - i] if j > i else fade[15 - j]
                elif m == 12:
                    v = fade[i] if i > 15 - j else fade[15 - j]
                else:
                    v = 1.0
                t.append(v)
        out.append(t)
    return out


def texture_factors(hw):
    """The texture kernel's per-pixel tables in float32, operation by operation."""
    import numpy as np
    f = np.float32
    w = [f(float(f32(v)[:-1])) for v in hw]  # the float the compiler makes of each printed literal
    tfac = [[f(0.0)] * 17 for _ in range(16)]
    mfac = [[f(0.0)] * 17 for _ in range(16)]
    for r in range(16):
        for c in range(16):
            tfac[r][c] = (f(0.25) / w[c]) / w[r]
            mfac[r][c] = (f(0.5) * w[r]) * (f(0.5) * w[c])
    hsq = [w[i] * w[i] for i in range(16)]
    sym8 = lambda i: (i ^ 15) if (i & 8) else i
    wnd2 = [hsq[sym8(px >> 4)] * hsq[sym8(px & 15)] for px in range(256)]
    wi = [f(1.0) / v for v in wnd2]
    lines = []
    for name, vals in (("TP_TEX_TFAC", [v for row in tfac for v in row]), ("TP_TEX_MFAC", [v for row in mfac for v in row]),
                       ("TP_TEX_WND2", wnd2), ("TP_TEX_WI", wi)):
        lines.append("#define %s_INIT {" % name + ", ".join("%.9ef" % float(v) for v in vals) + "}")
    return lines


def rind(n):
    return n + 4 if n < 4 else (11 - n if n < 12 else n - 12)


def fmt_matrix(name, m):
    lines = ["#define %s_INIT { \\" % name]
    for row in m:
        lines.append("    {" + ", ".join(f32(v) for v in row) + "}, \\")
    lines.append("}")
    return "\n".join(lines)


def main():
    out = ["/* Generated by gen_tables.py -- do not edit. */", "#pragma once", ""]
    names = ["TP_DCT4", "TP_DST4", "TP_DCT2", "TP_DST2"]
    for kind, name in enumerate(names):
        out.append(fmt_matrix(name, dtt(kind)))
    pre = [[math.cos(math.pi * m / 8.0), math.sin(math.pi * m / 8.0)] for m in range(4)]
    post = [[0.5 * math.cos(math.pi * (4 * p + 1) / 32.0), 0.5 * math.sin(math.pi * (4 * p + 1) / 32.0)]
            for p in range(4)]
    out.append(fmt_matrix("TP_DCT4_PRE", pre))
    out.append(fmt_matrix("TP_DCT4_POST", post))
    q = math.pi
    d2 = [0.5 * math.cos(q / 4), 0.5 * math.cos(q / 8), 0.5 * math.cos(3 * q / 8), math.cos(q / 4),
          0.5 * math.cos(q / 16), 0.5 * math.sin(q / 16), 0.5 * math.cos(5 * q / 16), 0.5 * math.sin(5 * q / 16)]
    out.append("#define TP_DCT2_FAST_INIT {" + ", ".join(f32(v) for v in d2) + "}")
    hw = [math.sin(math.pi * (2 * n + 1) / 32.0) for n in range(16)]
    out.extend(texture_factors(hw))
    hwc = [math.cos(math.pi * (2 * n + 1) / 32.0) for n in range(16)]
    out.append("#define TP_HWIN_INIT {" + ", ".join(f32(v) for v in hw) + "}")
    out.append("#define TP_HWINC_INIT {" + ", ".join(f32(v) for v in hwc) + "}")
    out.append("#define TP_RIND_INIT {" + ", ".join(str(rind(n)) for n in range(16)) + "}")
    lp = [default_lpf(w) for w in range(6)]
    out.append("#define TP_LPF_DEFAULT_INIT { \\")
    for w in range(6):
        out.append("    {" + ", ".join(f32(v) for v in lp[w]) + "}, \\")
    out.append("}")
    af = alpha_fade()
    out.append("#define TP_ALPHA_FADE_INIT { \\")
    for m in range(16):
        out.append("    {" + ", ".join(f32(v) for v in af[m]) + "}, \\")
    out.append("}")
    out.append("")
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "tp_tables.inc"), "w") as fh:
        fh.write("\n".join(out))


if __name__ == "__main__":
    main()
