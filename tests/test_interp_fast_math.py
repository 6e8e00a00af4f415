"""The arithmetic of the interpolated mode's fast form (csrc/bp_interp.cu fast_bin and
fast_phasor), restated operation by operation in float32 NumPy (IEEE single precision,
round to nearest, as the device executes these non-contracted operations):

  * fast_bin must give floor(RN(path / fsp) / 2) -- the reference's range bin,
    imaging_gpu.cu:100 -- for every path it does not hand to the division itself;
  * fast_phasor's wrapped turn count must be within 1e-7 turns of path/lambda (FP64).
CPU only."""
import numpy as np

F32 = np.float32
M = F32(12582912.0)  # 1.5 * 2^23


def fast_bin_np(path, fsp):
    """Returns (bin, took_fast_path) for float32 arrays."""
    half_inv = F32(0.5) * (F32(1.0) / F32(fsp))
    h = (path * half_inv).astype(F32)
    hm = (h + M).astype(F32)
    r = (hm - M).astype(F32)
    above = (r > h).astype(np.int32)
    fr = (h - (r - above.astype(F32))).astype(F32)
    tol = (np.maximum(h, F32(1.0)) * F32(1.2e-6)).astype(F32)
    fast = ~((fr < tol) | (fr > F32(1.0) - tol))
    b = hm.view(np.int32) - np.array(M, F32).view(np.int32) - above
    return b, fast


def ref_bin_np(path, fsp):
    q = (path / F32(fsp)).astype(F32)          # correctly rounded FP32 quotient
    return np.floor((q / F32(2)).astype(F32)).astype(np.int32)


def test_fast_bin_matches_the_reference_quotient():
    rng = np.random.default_rng(0)
    for fsp in (F32(2.3437500e-3), F32(0.0146484375), F32(7.3e-4), F32(1.0 / 3.0) * F32(1e-2)):
        path = rng.uniform(0.0, float(fsp) * 4096, 2_000_000).astype(F32)
        # paths on and around the bin edges 2k*fsp, a few ulps either side
        k = rng.integers(0, 2048, 200_000)
        edge = (F32(2) * k.astype(F32) * fsp).astype(F32)
        ulps = rng.integers(-6, 7, edge.size).astype(np.int32)
        near = (edge.view(np.int32) + ulps).view(F32)
        near = near[(near >= 0) & np.isfinite(near)]
        for p in (path, near):
            b, fast = fast_bin_np(p, fsp)
            ref = ref_bin_np(p, fsp)
            assert np.array_equal(b[fast], ref[fast]), (fsp, int((b[fast] != ref[fast]).sum()))
        # the division fallback is rare on uniformly spread paths
        _, fast = fast_bin_np(path, fsp)
        assert (~fast).mean() < 5e-3


def _fma32(a, b, c):
    """float32 fma via float64 (a*b is exact in float64; one final rounding)."""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F32)


def test_fast_phasor_turns_within_1e7():
    rng = np.random.default_rng(1)
    for wl in (F32(2.99792458e8 / 77e9), F32(2.99792458e8 / 60e9), F32(0.0123)):
        inv = 1.0 / float(wl)
        hi = F32(inv)
        lo = F32(inv - float(hi))
        path = rng.uniform(0.0, 3.0, 1_000_000).astype(F32)
        q = (path * hi).astype(F32)
        e = _fma32(path, np.full_like(path, hi), -q)
        n = ((q + M).astype(F32) - M).astype(F32)
        f = ((q - n).astype(F32) + _fma32(path, np.full_like(path, lo), e)).astype(F32)
        exact = path.astype(np.float64) / float(wl)
        err = np.abs(((f.astype(np.float64) - (exact - n.astype(np.float64))) + 0.5) % 1.0 - 0.5)
        assert err.max() < 1e-7, err.max()
        # |f| exceeds 0.5 by at most the product's rounding error (half an ulp of path/lambda)
        assert np.abs(f).max() <= 0.5 + 1e-4
