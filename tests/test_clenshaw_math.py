"""CPU checks of the forward kernel's second-order block sum (no GPU).

The kernel sums a block of L samples, h = sum_t m_t z^t with z = e^{i phi}, through the
backward three-term recurrence b_t = m_t + 2 cos(phi) b_{t+1} - b_{t+2} and
h = b_0 - conj(z) b_1.  These tests restate that in NumPy: exactly in FP64 (the identity),
and with FP32 rounding after every operation in the kernel's order (FADD for
m_t - b_{t+2}, FMA for the rest), to pin the error statements the kernel's selector
relies on: inside |cos phi| <= 0.98 the FP32 recurrence stays within a few 1e-6 of the
block sum for L = 32 and 64 and within a small factor of the first-order Horner form, and
toward phi = 0 it degrades (which is why the kernel falls back to Horner there)."""
import numpy as np
import pytest

F32 = np.float32
COS_LIMIT = 0.98  # the kernel's kClenMaxCos


def _fma(a, b, c):
    # one FP32 rounding of a*b + c (the product of two FP32 values is exact in FP64)
    return (a.astype(np.float64) * b + c).astype(F32)


def clenshaw_fp64(m, phi):
    """h = sum_t m_t e^{i phi t} by the backward recurrence, complex128."""
    L = m.shape[-1]
    c2 = 2 * np.cos(phi)
    b1 = np.zeros(m.shape[:-1], np.complex128)
    b2 = np.zeros_like(b1)
    for t in range(L - 1, -1, -1):
        b1, b2 = m[..., t] + c2 * b1 - b2, b1
    return b1 - np.exp(-1j * phi) * b2


def clenshaw_fp32(m, phi):
    """The kernel's FP32 arithmetic: c2 = 2 zr, b_{L-1} = m_{L-1},
    b_{L-2} = fma(c2, b_{L-1}, m_{L-2}), then d = m_t - b_{t+2}, b_t = fma(c2, b_{t+1}, d),
    and h_re = fma(-zr, b1_re, fma(-zi, b1_im, b0_re)), h_im = fma(-zr, b1_im,
    fma(zi, b1_re, b0_im)) with (zr, zi) = FP32 (cos phi, sin phi)."""
    L = m.shape[-1]
    mr, mi = m.real.astype(F32), m.imag.astype(F32)
    zr, zi = np.cos(phi).astype(F32), np.sin(phi).astype(F32)
    c2 = (F32(2) * zr).astype(F32)
    b2r, b2i = mr[..., L - 1].copy(), mi[..., L - 1].copy()
    b1r, b1i = _fma(c2, b2r, mr[..., L - 2]), _fma(c2, b2i, mi[..., L - 2])
    for t in range(L - 3, -1, -1):
        dr = (mr[..., t] - b2r).astype(F32)
        di = (mi[..., t] - b2i).astype(F32)
        b2r, b2i = b1r, b1i
        b1r, b1i = _fma(c2, b1r, dr), _fma(c2, b1i, di)
    hr = _fma(-zr, b2r, _fma(-zi, b2i, b1r))
    hi = _fma(-zr, b2i, _fma(zi, b2r, b1i))
    return hr.astype(np.float64) + 1j * hi.astype(np.float64)


def horner_fp32(m, phi):
    """First-order Horner h <- h z + m_t in FP32 (the fallback form)."""
    L = m.shape[-1]
    mr, mi = m.real.astype(F32), m.imag.astype(F32)
    zr, zi = np.cos(phi).astype(F32), np.sin(phi).astype(F32)
    hr, hi = mr[..., L - 1].copy(), mi[..., L - 1].copy()
    for t in range(L - 2, -1, -1):
        u, w = _fma(hr, zr, mr[..., t]), _fma(hr, zi, mi[..., t])
        hr, hi = _fma(-hi, zi, u), _fma(hi, zr, w)
    return hr.astype(np.float64) + 1j * hi.astype(np.float64)


def _case(rng, n, L, phi0, coherent):
    phi = phi0 * (1 + 0.01 * rng.standard_normal(n))
    m = rng.standard_normal((n, L)) + 1j * rng.standard_normal((n, L))
    if coherent:  # a row dominated by one scatterer at the voxel's own range
        m = m * 0.05 + np.exp(-1j * np.outer(phi, np.arange(L)))
    m = m.astype(np.complex64).astype(np.complex128)
    exact = (m * np.exp(1j * np.outer(phi, np.arange(L)))).sum(1)
    return m, phi, exact


@pytest.mark.parametrize("L", [32, 64])
def test_recurrence_identity_fp64(L):
    rng = np.random.default_rng(L)
    for phi0 in (-2.5, -0.3, 0.05, 0.21, 1.0, 3.0):
        m, phi, exact = _case(rng, 256, L, phi0, False)
        h = clenshaw_fp64(m, phi)
        assert np.max(np.abs(h - exact)) < 1e-10 * np.max(np.abs(exact)), phi0


@pytest.mark.parametrize("L", [32, 64])
@pytest.mark.parametrize("coherent", [False, True])
def test_fp32_error_inside_the_selector_range(L, coherent):
    """|cos phi| <= 0.98, random rows and rows dominated by one scatterer focused on the
    voxel: RMS error relative to the RMS block sum within 2.5e-6 (L = 32) / 4e-6 (L = 64),
    and at most 6x the first-order Horner form's (about 4.7x at the selector's edge,
    phi = 0.21; below 1x for phi near 1 and beyond)."""
    rng = np.random.default_rng(100 + L + coherent)
    for phi0 in (0.21, 0.3, 0.45, 1.0, 2.0, -2.9):
        assert abs(np.cos(phi0)) <= COS_LIMIT
        m, phi, exact = _case(rng, 20000, L, phi0, coherent)
        scale = np.sqrt((np.abs(exact) ** 2).mean())
        ec = np.sqrt((np.abs(clenshaw_fp32(m, phi) - exact) ** 2).mean()) / scale
        eh = np.sqrt((np.abs(horner_fp32(m, phi) - exact) ** 2).mean()) / scale
        assert ec < (2.5e-6 if L == 32 else 4e-6), (phi0, ec)
        assert ec < 6 * eh, (phi0, ec, eh)


def test_fp32_error_grows_toward_zero_angle():
    """Toward phi = 0 the FP32 recurrence loses accuracy (rounding errors amplified up to
    min(t + 1, 1/sin phi), FP32 c2 = 2 cos phi resolving phi coarsely), while Horner does
    not: the reason the kernel runs those blocks in the Horner form."""
    rng = np.random.default_rng(7)
    errs = []
    for phi0 in (0.005, 0.21):
        m, phi, exact = _case(rng, 20000, 32, phi0, False)
        scale = np.sqrt((np.abs(m) ** 2).sum(1).mean())
        ec = np.sqrt((np.abs(clenshaw_fp32(m, phi) - exact) ** 2).mean()) / scale
        eh = np.sqrt((np.abs(horner_fp32(m, phi) - exact) ** 2).mean()) / scale
        errs.append((ec, eh))
    (ec0, eh0), (ec1, _) = errs
    assert np.cos(0.005) > COS_LIMIT  # outside the selector's range
    assert ec0 > 3 * ec1 and ec0 > 10 * eh0
