"""Writes es_taps.cuh: the tap weights of the exponential-of-semicircle interpolation kernel
used by the position pass (bp_nufft.cu), as polynomials in the fractional grid offset.

Kernel: phi(z) = exp(beta (sqrt(1 - (2z/W)^2) - 1)) for |z| < W/2, W = 8, beta = 2.3 W --
the "exponential of semicircle" kernel of Barnett, Magland and af Klinteberg (SIAM J. Sci.
Comput. 41, 2019) with their width and shape for ~1e-7 at 2x oversampling.
Tap i (0..7) sits at z = s + W/2 - 1 - i for the fractional offset s in [0, 1).  With
t = s - 1/2, tap i is P_i(t) = phi(t + W/2 - 1/2 - i) and, phi being even, tap W-1-i is
P_i(-t).  So only P_0..P_3 are fitted (degree 8, least squares on 4001 points of
[-1/2, 1/2]) and stored as even and odd parts:  P_i(t) = E_i(t^2) + t O_i(t^2), which gives
both taps of a mirror pair from one E and one O.  Fit error below 2e-8 (phi(0) = 1); the
FP32 evaluation's rounding is about 1e-7.  Run:  python mmnorm_b200/csrc/gen_es_taps.py
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
    t = np.linspace(-0.5, 0.5, 4001)
    even, odd, worst = [], [], 0.0
    for i in range(W // 2):
        c = np.polynomial.Polynomial.fit(t, es(t + W / 2 - 0.5 - i), DEG,
                                         domain=[-0.5, 0.5], window=[-0.5, 0.5]).coef
        c = np.concatenate([c, np.zeros(DEG + 1 - len(c))])
        for sign, tap in ((1.0, i), (-1.0, W - 1 - i)):
            y = es(sign * t + W / 2 - 0.5 - i) if sign > 0 else es(t + W / 2 - 0.5 - tap)
            worst = max(worst, float(np.abs(np.polynomial.polynomial.polyval(sign * t, c)
                                            - y).max()))
        even.append(c[0::2].astype(np.float32))
        odd.append(c[1::2].astype(np.float32))
    return even, odd, worst


def main():
    even, odd, worst = fit()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "es_taps.cuh")
    ne, no = len(even[0]), len(odd[0])
    lines = [
        "// es_taps.cuh -- generated by gen_es_taps.py; do not edit.",
        "// Exponential-of-semicircle kernel (W = %d, beta = 2.3 W): with t = s - 1/2 for the" % W,
        "// fractional grid offset s, tap i (0..%d) weighs P_i(t) and tap %d-i weighs P_i(-t)," % (W // 2 - 1, W - 1),
        "// P_i(t) = sum_n kEsEven[i][n] t^(2n) + t sum_n kEsOdd[i][n] t^(2n).  Fit error %.1e." % worst,
        "#pragma once",
        "",
        "namespace mmn {",
        "",
        "constexpr int kEsEvenTerms = %d, kEsOddTerms = %d;" % (ne, no),
        "__constant__ float kEsEven[%d][%d] = {" % (W // 2, ne),
    ]
    lines += ["    {" + ", ".join("%.9ef" % float(v) for v in c) + "}," for c in even]
    lines += ["};", "__constant__ float kEsOdd[%d][%d] = {" % (W // 2, no)]
    lines += ["    {" + ", ".join("%.9ef" % float(v) for v in c) + "}," for c in odd]
    lines += ["};", "", "}  // namespace mmn", ""]
    with open(out, "w") as f:
        f.write("\n".join(lines))
    print("wrote", out, "fit error %.2e" % worst)


if __name__ == "__main__":
    main()
