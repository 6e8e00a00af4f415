"""The drop-in wrappers (same signatures as the reference's image_cuda /
normal_estimates_cuda) against the oracle's restatement of the reference wrappers and
against the reference imager's golden outputs."""
import numpy as np
import pytest

from conftest import load_golden
from mmnorm_b200 import pipeline, py_image_gpu, py_sn_est_gpu, scenes

pytestmark = pytest.mark.gpu


def _radar(sc, R=1, seed=0):
    """(A, S, R) radar data: RX k sees the scene scaled by a per-RX complex gain."""
    rng = np.random.default_rng(seed)
    g = (rng.standard_normal(R) + 1j * rng.standard_normal(R)).astype(np.complex64)
    return (sc.meas[:, :, None] * g[None, None, :]).astype(np.complex64)


def _rx_offsets(R):
    wl = scenes.C / 77e9
    return np.array([[0.0, -0.005 - wl / 2 * (R - 1 - k), 0.0] for k in range(R)])


@pytest.mark.parametrize("R,use_4_rx,ti", [(1, False, False), (4, True, True)])
def test_image_cuda_full_mode(cuda_dev, oracle, R, use_4_rx, ti):
    sc = scenes.sphere_scene(seed=11, n_ap=8, nf=24, n_vox=6, n_pts=20)
    data = _radar(sc, R)
    if not use_4_rx:
        data = data[:, :, 0]
    rxo = _rx_offsets(R)
    ant = sc.antenna_locs.astype(np.float64)
    args = (sc.x_locs, sc.y_locs, sc.z_locs, ant, data, rxo, sc.slope, sc.wavelength,
            sc.f_hi - sc.f_lo, sc.num_freqs)
    img, centres = py_image_gpu.image_cuda(*args, use_4_rx=use_4_rx, is_ti_radar=ti)
    ref, ref_c = oracle.ref_image_cuda(*args, use_4_rx=use_4_rx, is_ti_radar=ti)
    assert img.dtype == np.complex64 and img.shape == sc.grid_shape
    assert oracle.rel_l2(img, ref) < 2e-5
    np.testing.assert_array_equal(centres, ref_c)
    # the same contract with the sums by interpolation (precision="nufft")
    img_n, centres_n = py_image_gpu.image_cuda(*args, use_4_rx=use_4_rx, is_ti_radar=ti,
                                               precision="nufft")
    assert img_n.dtype == np.complex64 and img_n.shape == sc.grid_shape
    assert oracle.rel_l2(img_n, ref) < 2e-5
    np.testing.assert_array_equal(centres_n, ref_c)


@pytest.mark.parametrize("R,use_4_rx,ti", [(1, False, False), (4, True, True)])
def test_interp_mode_image_and_normals(cuda_dev, oracle, R, use_4_rx, ti):
    sc = scenes.sphere_scene(seed=12, n_ap=8, nf=64, n_vox=6, n_pts=20, sign=+1)
    data = _radar(sc, R)
    nb = 512
    pad = np.zeros((data.shape[0], nb, R), np.complex64)
    pad[:, :64, :] = data
    fft = np.fft.fft(pad, axis=1)
    if not use_4_rx:
        fft = fft[:, :, 0]
    rxo = _rx_offsets(R)
    ant = sc.antenna_locs.astype(np.float64)
    args = (sc.x_locs, sc.y_locs, sc.z_locs, ant, fft, rxo, sc.slope, sc.wavelength,
            sc.f_hi - sc.f_lo, 64)
    img, centres = py_image_gpu.image_cuda(*args, use_4_rx=use_4_rx, is_ti_radar=ti,
                                           use_interpolated_processing=True)
    ref, ref_c = oracle.ref_image_cuda(*args, use_4_rx=use_4_rx, is_ti_radar=ti,
                                       use_interpolated_processing=True, dist_mode=1)
    assert oracle.rel_l2(img, ref) < 5e-4
    np.testing.assert_array_equal(centres, ref_c)
    nrm = py_sn_est_gpu.normal_estimates_cuda(img, *args, use_4_rx=use_4_rx, is_ti_radar=ti)
    nref = oracle.ref_normal_estimates_cuda(img, *args, use_4_rx=use_4_rx, is_ti_radar=ti,
                                            dist_mode=1)
    assert nrm.dtype == np.float64 and nrm.shape == sc.grid_shape + (3,)
    np.testing.assert_array_equal(np.isnan(nrm), np.isnan(nref))
    ok = ~np.isnan(nref[..., 0])
    assert ok.sum() > 0
    assert oracle.rel_l2(nrm[ok], nref[ok]) < 5e-4


@pytest.mark.parametrize("name", ["full_r1", "full_r2_ti", "interp_r1", "cfg0_sub12"])
def test_dropin_matches_reference_imager_golden(cuda_dev, oracle, name):
    """image_cuda on the fixture inputs vs the reference C++ imager's output (/TX count);
    the imager's FP32 phase bounds the agreement (~5e-5)."""
    g = load_golden(name)
    meas = g["meas"]
    A, S, R = meas.shape
    interp = bool(g["interp"])
    wl = float(g["wavelength"])
    bandwidth = float(g["slope"]) * (S - 1)
    num_samples = S
    if interp:
        # fft_spacing = 3e8/(2B)*num_samples/S must equal the fixture's spacing
        num_samples = 64
        bandwidth = 3e8 / (2 * float(g["fsp"])) * num_samples / S
    img = py_image_gpu.image_cuda(g["x"], g["y"], g["z"], g["ant"].astype(np.float64), meas,
                                  g["rxo"], float(g["slope"]), wl, bandwidth, num_samples,
                                  use_4_rx=True, is_ti_radar=bool(g["ti"]),
                                  use_interpolated_processing=interp,
                                  return_phase_centers=False)
    scale = A if not interp else 1  # full mode divides by A twice, the imager once
    assert oracle.rel_l2(img * scale, g["ref_image"]) < 2e-4


def test_full_mode_normals_and_pipeline(cuda_dev, oracle):
    sc = scenes.sphere_scene(seed=13, n_ap=16, nf=32, n_vox=8, n_pts=40, sign=+1)
    data = sc.meas[:, :, None]
    rxo = np.zeros((1, 3))
    args = (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), data, rxo,
            sc.slope, sc.wavelength, sc.f_hi - sc.f_lo, sc.num_freqs)
    img, _ = py_image_gpu.image_cuda(*args, use_4_rx=True)
    raw = py_sn_est_gpu.normal_estimates_cuda(img, *args, use_4_rx=True,
                                              use_interpolated_processing=False)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, rxo, sc.meas, sc.wavelength,
                         sc.slope)
    mask = np.abs(img) > np.abs(img).max() * 0.05
    np.testing.assert_array_equal(~np.isnan(raw[..., 0]), mask)
    sel = mask.ravel()
    ang = oracle.angle_deg(raw.reshape(-1, 3)[sel],
                           np.real(np.conj(Io[sel])[:, None] * Wo[sel]))
    assert np.median(ang) < 0.05
    s2, unit, centres = pipeline.surface_normals(*args, use_4_rx=True)
    np.testing.assert_array_equal(s2, img)
    np.testing.assert_allclose(np.linalg.norm(unit.reshape(-1, 3)[sel], axis=1), 1, rtol=1e-6)
    assert np.all(np.isnan(unit.reshape(-1, 3)[~sel]))


def test_interp_antenna_groups(cuda_dev, oracle, monkeypatch):
    """Interpolated mode processes at most MAX_NUM_ANT virtual antennas per group and sums
    per-group means (py_image_gpu.py:337-362); exercised with a small group size."""
    import oracle.oracle as O
    sc = scenes.sphere_scene(seed=14, n_ap=6, nf=64, n_vox=5, n_pts=20, sign=+1)
    pad = np.zeros((36, 512, 1), np.complex64)
    pad[:, :64, 0] = sc.meas
    fft = np.fft.fft(pad, axis=1)
    args = (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), fft,
            np.zeros((1, 3)), sc.slope, sc.wavelength, sc.f_hi - sc.f_lo, 64)
    monkeypatch.setattr(py_image_gpu, "MAX_NUM_ANT", 10)
    img, c = py_image_gpu.image_cuda(*args, use_4_rx=True, use_interpolated_processing=True)
    # oracle: four groups of 10,10,10,6 antennas, per-group mean, summed
    ref = 0
    for g0 in range(0, 36, 10):
        part = O.ref_image_cuda(sc.x_locs, sc.y_locs, sc.z_locs,
                                sc.antenna_locs[g0:g0 + 10].astype(np.float64),
                                fft[g0:g0 + 10], np.zeros((1, 3)), sc.slope, sc.wavelength,
                                sc.f_hi - sc.f_lo, 64, use_4_rx=True,
                                use_interpolated_processing=True, return_phase_centers=False,
                                dist_mode=1)
        ref = ref + part
    assert oracle.rel_l2(img, ref) < 5e-4
    assert c.shape == (36, 3)
