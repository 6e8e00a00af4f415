"""The interpolation forms' mathematics (bp_nufft.cu) restated in numpy, CPU only: the
1/phihat midpoint quadrature, the extended grid rows (cell k = (jj - W/2 + 1) mod N), the
cell index and fraction of N (u mod 1), the type-2 gather (forward, position pass) and the
type-1 spread with its per-antenna output transform (measurement pass).  The gather and
the spread must reproduce the exact discrete-time Fourier sums to ~1e-7, and be exact
transposes of each other -- which is what makes the interpolation-form measurement pass
the adjoint of the interpolation-form forward."""
import numpy as np
import pytest

W = 8
BETA = 2.30 * W
QUAD = 256


def es(z):
    t = 2.0 * z / W
    q = 1.0 - t * t
    return np.where(q > 0, np.exp(BETA * (np.sqrt(np.clip(q, 0.0, None)) - 1.0)), 0.0)


def tables(F):
    N, J0 = 2 * F, F // 2
    h = 0.5 * W / QUAD
    z = (np.arange(QUAD) + 0.5) * h
    xi = (np.arange(F) - J0) / N
    sc = 1.0 / (2 * h * (es(z)[None, :] * np.cos(2 * np.pi * np.outer(xi, z))).sum(1))
    tw = np.exp(-2j * np.pi * np.arange(N) / N)
    return N, J0, sc, tw


def cells(u, N):
    """Cell index and fraction of N (u mod 1), as the kernels form them, with the clamp."""
    x = (u - np.floor(u)) * N
    ix = np.floor(x).astype(np.int64)
    s = x - ix
    lo, hi = ix < 0, ix >= N
    return np.where(lo, 0, np.where(hi, N - 1, ix)), np.where(lo, 0.0, np.where(hi, 1.0, s))


def weights(s):
    return es(s[:, None] + W / 2 - 1 - np.arange(W)[None, :])  # [P, W]


def gather(m, u):
    """type-2: M(u) = sum_j' m[J0+j'] e^{-2 pi i j' u} from the extended grid row."""
    F = m.size
    N, J0, sc, tw = tables(F)
    jp = np.arange(F) - J0
    G = np.array([(m * sc * tw[(jp * k) % N]).sum() for k in range(N)])
    row = np.array([G[(jj - (W // 2 - 1)) % N] for jj in range(N + W - 1)])
    ix, s = cells(u, N)
    return (weights(s) * row[ix[:, None] + np.arange(W)[None, :]]).sum(1)


def spread(h, u, F):
    """type-1: H(j') = sum_v h_v e^{2 pi i j' u_v} via the extended row and the fold."""
    N, J0, sc, tw = tables(F)
    mrow = N + 16
    row = np.zeros(mrow, complex)
    ix, s = cells(u, N)
    np.add.at(row, ix[:, None] + np.arange(W)[None, :], h[:, None] * weights(s))
    S = np.zeros(N, complex)
    for k in range(N):
        S[k] = row[np.arange((k + W // 2 - 1) % N, mrow, N)].sum()
    jp = np.arange(F) - J0
    return np.array([sc[j] * (S * np.conj(tw[(jp[j] * np.arange(N)) % N])).sum()
                     for j in range(F)])


@pytest.mark.parametrize("F", [1, 3, 40, 129])
def test_gather_and_spread_reproduce_the_fourier_sums(F):
    rng = np.random.default_rng(F)
    J0 = F // 2
    jp = np.arange(F) - J0
    m = rng.standard_normal(F) + 1j * rng.standard_normal(F)
    u = np.concatenate([rng.uniform(0.0, 3.0, 300), [0.0, 1.0, 2.5, 1 - 1e-16]])
    exact = np.exp(-2j * np.pi * np.outer(u, jp)) @ m
    got = gather(m, u)
    assert np.linalg.norm(got - exact) / np.linalg.norm(exact) < 5e-7
    h = rng.standard_normal(u.size) + 1j * rng.standard_normal(u.size)
    exact_t = np.exp(2j * np.pi * np.outer(jp, u)) @ h
    got_t = spread(h, u, F)
    assert np.linalg.norm(got_t - exact_t) / np.linalg.norm(exact_t) < 5e-7


def test_spread_is_the_transpose_of_the_gather():
    rng = np.random.default_rng(1)
    F = 24
    m = rng.standard_normal(F) + 1j * rng.standard_normal(F)
    u = rng.uniform(0.0, 2.0, 50)
    h = rng.standard_normal(50) + 1j * rng.standard_normal(50)
    lhs = np.vdot(h, gather(m, u))       # <h, A m>
    rhs = np.vdot(spread(h, u, F), m)    # <A^H h, m>
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
