"""Device-resident imaging + normal stage (mmnorm_b200.stage1) against the oracle's
restatement of the reference wrappers: the range FFT against numpy's, the full matched
filter and the interpolated mode (several antenna groups) images and unit normals, and
the normal_data.npz file against the one GenericLoader.save_surface_normals writes."""
import os

import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu


def _case(seed=3, R=3, n_ap=8, nf=48, n_vox=10):
    sc = scenes.sphere_scene(seed=seed, n_ap=n_ap, nf=nf, n_vox=n_vox, spacing=4e-3, n_pts=40)
    rng = np.random.default_rng(seed)
    # (A, S, R) raw samples: the scene's response with a per-RX phase, TI-style RX offsets
    data = (sc.meas[:, :, None] * np.exp(1j * rng.uniform(0, 6.28, (1, 1, R)))).astype(np.complex64)
    rxo = np.array([[0.0, -0.005 - 0.0019 * k, 0.0] for k in range(R)], np.float64)
    bandwidth = sc.slope * (nf - 1)
    return sc, data, rxo, bandwidth


def _angle(a, b):
    a = a / np.linalg.norm(a, axis=-1, keepdims=True)
    b = b / np.linalg.norm(b, axis=-1, keepdims=True)
    return np.degrees(np.arccos(np.clip((a * b).sum(-1), -1, 1)))


def test_range_fft_matches_numpy(cuda_dev):
    import torch
    from mmnorm_b200 import stage1
    rng = np.random.default_rng(0)
    x = (rng.standard_normal((37, 300, 4)) + 1j * rng.standard_normal((37, 300, 4))).astype(np.complex64)
    pad = np.zeros((37, 4096, 4), np.complex64)
    pad[:, :300] = x
    ref = np.fft.fft(pad, axis=1)
    got = stage1.range_fft(torch.as_tensor(x, device=cuda_dev)).cpu().numpy()
    assert got.dtype == np.complex64 and got.shape == (37, 4096, 4)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6
    with pytest.raises(ValueError):
        stage1.range_fft(torch.zeros((2, 5000, 1), dtype=torch.complex64, device=cuda_dev))


def test_full_mode_matches_oracle(cuda_dev, oracle):
    from mmnorm_b200 import stage1
    sc, data, rxo, bw = _case()
    img, (x, y, z), nrm, cl, meas = stage1.generate_mmwave_surface_normals(
        sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), data, rxo,
        sc.slope, sc.wavelength, bw, data.shape[1], is_ti_radar=True,
        use_interpolated_processing=False)
    ref_img, ref_cl = oracle.ref_image_cuda(sc.x_locs, sc.y_locs, sc.z_locs,
                                            sc.antenna_locs.astype(np.float64), data, rxo,
                                            sc.slope, sc.wavelength, bw, data.shape[1],
                                            use_4_rx=True, is_ti_radar=True)
    assert img.dtype == np.complex64 and img.shape == ref_img.shape
    assert oracle.rel_l2(img, ref_img) <= 2e-5
    np.testing.assert_allclose(cl, ref_cl, rtol=0, atol=1e-9)
    # normals: the oracle's vote on the same virtual antennas
    rxo_f, rows, locs_rep = oracle.ref_prep(data, rxo, sc.antenna_locs, True)
    Io, Wo = oracle.full(oracle._grid_vox(sc.x_locs, sc.y_locs, sc.z_locs), locs_rep, rxo_f,
                         rows, float(np.float32(sc.wavelength)), float(np.float32(sc.slope)),
                         is_ti=True)
    unit_o, mask_o, _ = oracle.normals_from_vote(Io, Wo, 0.05)
    mask = ~np.isnan(nrm[..., 0]).ravel()
    mag = np.abs(Io)
    border = np.abs(mag - 0.05 * mag.max()) <= 1e-4 * mag.max()
    assert np.all((mask == mask_o) | border)
    both = mask & mask_o
    assert nrm.dtype == np.float64
    assert np.median(_angle(nrm.reshape(-1, 3)[both], unit_o[both])) < 0.01


def test_interpolated_mode_groups_match_dropin_and_oracle(cuda_dev, oracle, monkeypatch):
    """Against the numpy-in drop-in (the reference-exact kernels on numpy's FFT) the only
    difference is the FFT's precision; against the oracle, FP32 ranges that land on the
    other side of a bin boundary add a little more (the drop-in tests allow 5e-4)."""
    from mmnorm_b200 import py_image_gpu, py_sn_est_gpu, stage1
    sc, data, rxo, bw = _case(seed=4, R=2, n_ap=6, nf=64)
    A = sc.antenna_locs.shape[0]
    group = 2 * 10                           # virtual antennas per group: 4 groups of TX
    monkeypatch.setattr(stage1, "MAX_NUM_ANT", group)
    monkeypatch.setattr(py_image_gpu, "MAX_NUM_ANT", group)
    monkeypatch.setattr(py_sn_est_gpu, "MAX_NUM_ANT", group)
    img, _, nrm, cl, _ = stage1.generate_mmwave_surface_normals(
        sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), data, rxo,
        sc.slope, sc.wavelength, bw, data.shape[1], is_ti_radar=False,
        use_interpolated_processing=True)
    pad = np.zeros((A, 4096, 2), np.complex64)
    pad[:, :data.shape[1]] = data
    fft = np.fft.fft(pad, axis=1)
    args = (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), fft, rxo,
            sc.slope, sc.wavelength, bw, data.shape[1])
    d_img, d_cl = py_image_gpu.image_cuda(*args, use_4_rx=True, use_interpolated_processing=True)
    assert oracle.rel_l2(img, d_img) <= 1e-5
    np.testing.assert_allclose(cl, d_cl, rtol=0, atol=1e-9)
    d_n = py_sn_est_gpu.normal_estimates_cuda(d_img, *args, use_4_rx=True)
    d_unit = d_n / np.linalg.norm(d_n, axis=-1, keepdims=True)
    m_d = ~np.isnan(d_unit[..., 0])
    m = ~np.isnan(nrm[..., 0])
    mag = np.abs(d_img)
    border = np.abs(mag - 0.05 * mag.max()) <= 1e-4 * mag.max()
    assert np.all((m == m_d) | border)
    both = m & m_d
    assert np.median(_angle(nrm[both], d_unit[both])) < 1e-3

    ref_img, ref_cl = oracle.ref_image_cuda(*args, use_4_rx=True,
                                            use_interpolated_processing=True,
                                            max_num_ant=group, dist_mode=1)
    assert np.abs(ref_img).max() > 0
    assert oracle.rel_l2(img, ref_img) <= 1e-3
    np.testing.assert_allclose(cl, ref_cl, rtol=0, atol=1e-9)
    ref_n = oracle.ref_normal_estimates_cuda(ref_img, *args, use_4_rx=True, max_num_ant=group,
                                             dist_mode=1)
    ref_unit = ref_n / np.linalg.norm(ref_n, axis=-1, keepdims=True)
    both = m & ~np.isnan(ref_unit[..., 0])
    assert np.median(_angle(nrm[both], ref_unit[both])) < 0.05


def test_normal_data_file_matches_loader_format(cuda_dev, tmp_path):
    from mmnorm_b200 import stage1
    sc, data, rxo, bw = _case(seed=5, R=1, n_ap=6, nf=32, n_vox=6)
    res = stage1.generate_mmwave_surface_normals(
        sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), data, rxo,
        sc.slope, sc.wavelength, bw, data.shape[1], is_ti_radar=True,
        use_interpolated_processing=True)
    img, (x, y, z), nrm, cl, meas = res
    ours = os.path.join(tmp_path, "ours.npz")
    stage1.save_surface_normals(ours, img, x, y, z, antenna_locs=cl, channels=meas, normals=nrm)
    # the file GenericLoader.save_surface_normals writes for the same arrays
    theirs = os.path.join(tmp_path, "theirs.npz")
    np.savez_compressed(theirs, sum_img=img, x_locs=x, y_locs=y, z_locs=z,
                        antenna_locs=np.array(cl), channels=meas, normals=nrm)
    assert open(ours, "rb").read() == open(theirs, "rb").read()
    s_img, (lx, ly, lz), l_ant, l_ch, l_n = stage1.load_surface_normals(ours)
    np.testing.assert_array_equal(s_img, img)
    np.testing.assert_array_equal(l_n, nrm)
    np.testing.assert_array_equal(l_ant, cl)
    np.testing.assert_array_equal(l_ch, meas)


def test_interpolated_mode_fast_form(cuda_dev, oracle):
    """precision="fast" in the stage-1 driver: the fast form of interpolated mode against
    the reference-exact kernels on the same device FFT (same bins; the phasor differs by
    ~5e-7 per term)."""
    from mmnorm_b200 import stage1
    sc, data, rxo, bw = _case(seed=5, R=2, n_ap=6, nf=64)
    args = (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), data, rxo,
            sc.slope, sc.wavelength, bw, data.shape[1])
    img_e, _, nrm_e, _, _ = stage1.generate_mmwave_surface_normals(
        *args, is_ti_radar=True, use_interpolated_processing=True)
    img_f, _, nrm_f, _, _ = stage1.generate_mmwave_surface_normals(
        *args, is_ti_radar=True, use_interpolated_processing=True, precision="fast")
    assert oracle.rel_l2(img_f, img_e) <= 2e-6
    m = ~np.isnan(nrm_e[..., 0])
    assert m.sum() > 0
    np.testing.assert_array_equal(~np.isnan(nrm_f[..., 0]), m)
    assert np.median(_angle(nrm_f[m], nrm_e[m])) < 1e-4
