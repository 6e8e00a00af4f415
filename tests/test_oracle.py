"""The oracle itself: pinned to the reference's own C++ imager through the golden
fixtures, cross-checked against the numpy restatement, and its adjoint against finite
differences.  CPU only."""
import numpy as np
import pytest

from conftest import load_golden
from mmnorm_b200 import scenes

GOLDEN = ["full_r1", "full_r2_ti", "interp_r1", "cfg0_sub12"]


def _golden_rows(g):
    """Reference imager layout [A][S][R] -> virtual antennas [A*R] (TX repeated per RX)."""
    meas = g["meas"]
    A, S, R = meas.shape
    ant = np.repeat(g["ant"], R, axis=0)
    rows = np.transpose(meas, (0, 2, 1)).reshape(A * R, S)
    return ant, rows, A


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_matches_reference_imager(oracle, name):
    """The reference imager (imaging.cpp) computes its phase in float32 (imaging.cpp:111),
    so it sits ~4e-5 from the FP64 oracle; 2e-4 bounds that with margin."""
    g = load_golden(name)
    ant, rows, A = _golden_rows(g)
    vox = oracle._grid_vox(g["x"], g["y"], g["z"])
    if bool(g["interp"]):
        img, _ = oracle.interp(vox, ant, g["rxo"], rows, float(g["wavelength"]), float(g["fsp"]),
                               bool(g["ti"]), dist_mode=1)
    else:
        img, _ = oracle.full(vox, ant, g["rxo"], rows, float(g["wavelength"]),
                             float(g["slope"]), bool(g["ti"]), vote=False)
    ref = g["ref_image"].ravel()
    assert np.linalg.norm(ref) > 0
    assert oracle.rel_l2(ref, img / A) < 2e-4


def test_oracle_restatement_semantics_match_reference_imager(oracle):
    """ref_image_cuda (the reference wrapper's /A^2 normalisation) times A equals the
    reference imager's /A output."""
    g = load_golden("full_r2_ti")
    A = g["ant"].shape[0]
    wl = 2.99792458e8 / float(g["f_lo"])
    img = oracle.ref_image_cuda(g["x"], g["y"], g["z"], g["ant"], g["meas"], g["rxo"],
                                float(g["slope"]), wl, 4e9, g["meas"].shape[1], use_4_rx=True,
                                is_ti_radar=True, return_phase_centers=False)
    assert oracle.rel_l2(g["ref_image"].ravel(), img.ravel() * A) < 2e-4


def test_c_oracle_matches_numpy_restatement(oracle):
    sc = scenes.sphere_scene(seed=7, n_ap=6, nf=20, n_vox=4, n_pts=15)
    vox = sc.voxel_centres()
    rxo = np.array([[0.0, -0.004, 0.001]], np.float32)
    I, W = oracle.full(vox, sc.antenna_locs, rxo, sc.meas, sc.wavelength, sc.slope, True)
    In, Wn = oracle.full_np(vox, sc.antenna_locs, rxo, sc.meas, sc.wavelength, sc.slope, True)
    assert oracle.rel_l2(I, In) < 1e-11
    assert oracle.rel_l2(W, Wn) < 1e-11


def test_oracle_phase_modes_agree(oracle):
    sc = scenes.sphere_scene(seed=8, n_ap=8, nf=100, n_vox=4, n_pts=15)
    vox = sc.voxel_centres()
    rxo = np.zeros((1, 3), np.float32)
    I0, W0 = oracle.full(vox, sc.antenna_locs, rxo, sc.meas, sc.wavelength, sc.slope,
                         phase_mode=0)
    I1, W1 = oracle.full(vox, sc.antenna_locs, rxo, sc.meas, sc.wavelength, sc.slope,
                         phase_mode=1)
    assert oracle.rel_l2(I1, I0) < 1e-11
    assert oracle.rel_l2(W1, W0) < 1e-11


def test_oracle_adjoint_matches_finite_differences(oracle):
    """orc_full_backward vs central differences of a real loss of (I, W)."""
    rng = np.random.default_rng(0)
    sc = scenes.sphere_scene(seed=9, n_ap=4, nf=12, n_vox=3, n_pts=10)
    vox = sc.voxel_centres()
    rxo = np.array([[0.0, -0.003, 0.0]], np.float32)
    nv = vox.shape[0]
    gI = rng.standard_normal(nv) + 1j * rng.standard_normal(nv)
    gW = rng.standard_normal((nv, 3)) + 1j * rng.standard_normal((nv, 3))

    def loss(meas, ant):
        I, W = oracle.full(vox, ant, rxo, meas, sc.wavelength, sc.slope)
        return float(np.sum(np.real(np.conj(gI) * I)) + np.sum(np.real(np.conj(gW) * W)))

    gm, gp = oracle.full_backward(vox, sc.antenna_locs, rxo, sc.meas, sc.wavelength, sc.slope,
                                  gI, gW)
    # measurement gradient: the loss is linear in meas, so the check is exact-ish
    m = sc.meas.astype(np.complex128)
    for (i, j) in [(0, 0), (3, 5), (15, 11)]:
        for unit, comp in ((1.0, np.real), (1j, np.imag)):
            e = np.zeros_like(m)
            e[i, j] = unit
            # loss is evaluated on complex64 inputs; use exact linearity instead of FD
            d = loss((m + e).astype(np.complex64), sc.antenna_locs) - \
                loss((m - e).astype(np.complex64), sc.antenna_locs)
            assert abs(d / 2 - comp(gm[i, j])) < 1e-6 * max(1.0, abs(comp(gm[i, j])))
    # position gradient: FD in FP64 needs FP64 positions; the oracle takes float32, so use
    # h = 1e-4 m (exactly representable steps are not needed for a 1e-3 relative check)
    h = 2.0 ** -14
    for i in (0, 7):
        for k in range(3):
            a1 = sc.antenna_locs.astype(np.float64).copy()
            a2 = a1.copy()
            a1[i, k] += h
            a2[i, k] -= h
            fd = (loss(sc.meas, a1.astype(np.float32)) - loss(sc.meas, a2.astype(np.float32))) \
                / (np.float32(a1[i, k]) - np.float32(a2[i, k]))
            assert abs(fd - gp[i, k]) <= 2e-3 * np.abs(gp).max()


def test_normals_epilogue_restatement(oracle):
    rng = np.random.default_rng(1)
    I = rng.standard_normal(50) + 1j * rng.standard_normal(50)
    W = rng.standard_normal((50, 3)) + 1j * rng.standard_normal((50, 3))
    unit, mask, raw = oracle.normals_from_vote(I, W, 0.3)
    assert mask.sum() > 0 and (~mask).sum() > 0
    assert np.all(np.isnan(unit[~mask]))
    np.testing.assert_allclose(np.linalg.norm(unit[mask], axis=1), 1.0, rtol=1e-12)
    # raw equals the reference's per-antenna form when W = sum c_i u_i with one antenna
    c = rng.standard_normal() + 1j * rng.standard_normal()
    u = rng.standard_normal(3)
    raw1 = np.real(c * np.conj(I[0])) / abs(I[0]) * u
    _, _, r = oracle.normals_from_vote(I[:1], (c * u)[None, :], 0.0)
    np.testing.assert_allclose(r[0], raw1, rtol=1e-12)


def test_numpy_restatement_in_fp32_tracks_fp64():
    """The FP32 NumPy variant (bench's FP32 CPU baseline) computes the same formula in
    single precision: complex64 outputs within the FP32 phase error of the FP64 form."""
    from mmnorm_b200 import scenes
    from oracle import oracle as O
    sc = scenes.sphere_scene(seed=1, n_ap=6, nf=16, n_vox=3, n_pts=10)
    args = (sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas, sc.wavelength,
            sc.slope)
    I64, W64 = O.full_np(*args)
    I32, W32 = O.full_np(*args, precision="f32")
    assert I32.dtype == np.complex64 and I64.dtype == np.complex128
    assert O.rel_l2(I32, I64) < 1e-3 and O.rel_l2(W32, W64) < 1e-3
