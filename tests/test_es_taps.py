"""The interpolation kernel's tap polynomials (mmnorm_b200/csrc/es_taps.cuh, used by the
interpolation forms of the forward and adjoint): the committed header is what
gen_es_taps.py writes, and its FP32 Horner evaluation -- the order the kernels use,
mirror taps from one even and one odd part -- stays within 2e-7 of the exact
exponential-of-semicircle kernel on all 8 taps.  With the grid's 1/phihat deconvolution
this is what keeps the interpolated sums at the FP32 chains' ~1e-7 level.  CPU only."""
import importlib.util
import os
import re

import numpy as np

from conftest import ROOT

CSRC = os.path.join(ROOT, "mmnorm_b200", "csrc")


def _header_arrays():
    src = open(os.path.join(CSRC, "es_taps.cuh")).read()

    def arr(name):
        i = src.index("float " + name + "[")
        body = src[i:src.index("};", i)]
        rows = re.findall(r"\{([^{}]*)\}", body + "}")
        return np.array([[float(v.strip().rstrip("f")) for v in r.split(",") if v.strip()]
                         for r in rows[:4]], np.float32)

    return arr("kEsEven"), arr("kEsOdd")


def _gen_module():
    spec = importlib.util.spec_from_file_location("gen_es_taps",
                                                  os.path.join(CSRC, "gen_es_taps.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_header_is_the_generator_output():
    gen = _gen_module()
    even, odd, worst = gen.fit()
    E, O = _header_arrays()
    assert worst < 2e-8
    np.testing.assert_array_equal(E, np.array(even, np.float32))
    np.testing.assert_array_equal(O, np.array(odd, np.float32))


def test_fp32_tap_evaluation_matches_the_kernel():
    gen = _gen_module()
    E, O = _header_arrays()
    s = np.linspace(0.0, 1.0, 20001, dtype=np.float32)
    t = (s - np.float32(0.5)).astype(np.float32)
    t2 = (t * t).astype(np.float32)
    worst = 0.0
    total = np.zeros(s.shape, np.float64)
    for i in range(4):
        e = np.full_like(t, E[i][-1])
        for c in E[i][-2::-1]:
            e = (e * t2 + c).astype(np.float32)
        o = np.full_like(t, O[i][-1])
        for c in O[i][-2::-1]:
            o = (o * t2 + c).astype(np.float32)
        for tap, w in ((i, (t * o + e).astype(np.float32)),
                       (gen.W - 1 - i, (-t * o + e).astype(np.float32))):
            exact = gen.es(s.astype(np.float64) + gen.W / 2 - 1 - tap)
            worst = max(worst, float(np.abs(w - exact).max()))
            total += w
    assert worst < 2e-7
    # the 8 taps' weights sum to the periodised kernel: flat in s (partition of unity
    # up to the kernel's aliasing), which is what makes the gather exact for constants
    assert float(total.max() - total.min()) < 1e-5 * float(total.mean())
