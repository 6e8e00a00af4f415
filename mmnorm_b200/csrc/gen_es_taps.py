"""Writes es_taps.cuh: the eight tap weights of the exponential-of-semicircle interpolation
kernel used by the position pass (bp_pos_nufft.cu) as degree-8 polynomials in the
fractional grid offset s in [0, 1).

Kernel: phi(z) = exp(beta (sqrt(1 - (2z/W)^2) - 1)) for |z| < W/2, W = 8, beta = 2.3 W.
Tap i sits at z = s + W/2 - 1 - i.  Each tap is a least-squares fit on 4001 points of
[0, 1]; the fit error is below 2e-8 (phi(0) = 1), the FP32 Horner evaluation's rounding
about 1e-7.  Run:  python mmnorm_b200/csrc/gen_es_taps.py
"""
import os

import numpy as np

W = 8
BETA = 2.30 * W
DEG = 8


def es(z):
    t = 2.0 * z / W
    q = 1.0 - t * t
    return np.where(q > 0, np.exp(BETA * (np.sqrt(np.clip(q, 0.0, None)) - 1.0)), 0.0)


def fit():
    s = np.linspace(0.0, 1.0, 4001)
    coefs, worst = [], 0.0
    for i in range(W):
        y = es(s + W / 2 - 1 - i)
        c = np.polynomial.Polynomial.fit(s, y, DEG, domain=[0, 1], window=[0, 1]).coef
        worst = max(worst, float(np.abs(np.polynomial.polynomial.polyval(s, c) - y).max()))
        coefs.append(c.astype(np.float32))
    return coefs, worst


def main():
    coefs, worst = fit()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "es_taps.cuh")
    lines = [
        "// es_taps.cuh -- generated by gen_es_taps.py; do not edit.",
        "// Tap weights of the exponential-of-semicircle kernel (W = %d, beta = 2.3 W) as" % W,
        "// degree-%d polynomials in the fractional grid offset s: weight_i(s) =" % DEG,
        "// sum_n kEsTap[i][n] s^n, tap i at z = s + W/2 - 1 - i.  Fit error %.1e." % worst,
        "#pragma once",
        "",
        "namespace mmn {",
        "",
        "constexpr int kEsDeg = %d;" % DEG,
        "__constant__ float kEsTap[%d][%d] = {" % (W, DEG + 1),
    ]
    for c in coefs:
        lines.append("    {" + ", ".join("%.9ef" % float(v) for v in c) + "},")
    lines += ["};", "", "}  // namespace mmn", ""]
    with open(out, "w") as f:
        f.write("\n".join(lines))
    print("wrote", out, "fit error %.2e" % worst)


if __name__ == "__main__":
    main()
