"""Host-side logic of the drop-in wrappers against the oracle's restatement of the
reference wrappers, and the synthetic scene generator.  CPU only except the normal
epilogue, which runs on the device."""
import numpy as np
import pytest

from mmnorm_b200 import py_image_gpu, py_sn_est_gpu, scenes


def test_prep_inputs_matches_reference_layout(oracle):
    rng = np.random.default_rng(0)
    A, S, R = 5, 7, 4
    data = rng.standard_normal((A, S, R)) + 1j * rng.standard_normal((A, S, R))
    ant = rng.standard_normal((A, 3))
    rxo = rng.standard_normal((R, 3))
    rxo1, meas, ant_rep = py_image_gpu.prep_inputs(data, rxo, ant, True)
    rows = py_image_gpu._rows(meas, S, len(ant_rep))
    rxo2, rows2, ant2 = oracle.ref_prep(data, rxo, ant, True)
    np.testing.assert_array_equal(ant_rep, ant2)
    np.testing.assert_array_equal(rows, rows2.astype(np.complex64))
    # virtual antenna i = TX i//R with RX i%R; its row is data[i//R, :, i%R]
    for i in range(A * R):
        np.testing.assert_array_equal(rows[i], data[i // R, :, i % R].astype(np.complex64))


def test_sn_prep_inputs_layout_matches_image_prep():
    rng = np.random.default_rng(1)
    A, S, R = 3, 4, 2
    data = rng.standard_normal((A, S, R)) + 1j * rng.standard_normal((A, S, R))
    ant = rng.standard_normal((A, 3))
    rxo = rng.standard_normal((R, 3))
    a1, m1, l1 = py_image_gpu.prep_inputs(data, rxo, ant, True)
    a2, m2, l2 = py_sn_est_gpu.prep_inputs(data, rxo, ant, True)
    np.testing.assert_array_equal(np.asarray(m1).reshape(-1), np.asarray(m2).reshape(-1))
    np.testing.assert_array_equal(l1, l2)
    np.testing.assert_array_equal(np.asarray(a1).reshape(-1), np.asarray(a2).reshape(-1))


def test_rows_rejects_short_measurements():
    import pytest
    with pytest.raises(ValueError):
        py_image_gpu._rows(np.zeros(10, np.complex64), 4, 3)


def test_phase_centres_match_reference_formula():
    rng = np.random.default_rng(2)
    locs_rep = rng.standard_normal((8, 3))
    rxo = rng.standard_normal((4, 3))
    c = py_image_gpu._centres(locs_rep, rxo)
    np.testing.assert_allclose(c, locs_rep + np.tile(rxo, (2, 1)) / 2, rtol=0, atol=1e-15)


def test_mask_coordinates_follow_reference_meshgrid_order():
    rng = np.random.default_rng(3)
    img = rng.standard_normal((4, 5, 6)) + 1j * rng.standard_normal((4, 5, 6))
    filt, coords = py_sn_est_gpu._mask_and_coords(img, 0.5)
    m1, m2, m3 = np.meshgrid(np.arange(5), np.arange(4), np.arange(6))   # py_sn_est_gpu.py:327
    full = np.concatenate((m2[..., None], m1[..., None], m3[..., None]), axis=-1)
    np.testing.assert_array_equal(coords, full[filt])


@pytest.mark.gpu
def test_raw_normals_from_vote_matches_oracle(cuda_dev, oracle):
    """The drop-in's normal epilogue (formed on the device, masked on the host in the
    image's dtype) against the oracle's restatement of py_sn_est_gpu.py:326-376."""
    rng = np.random.default_rng(4)
    shape = (3, 4, 5)
    V = 60
    I = (rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64)
    W = (rng.standard_normal((3, V)) + 1j * rng.standard_normal((3, V))).astype(np.complex64)
    for image in (I, I.astype(np.complex128)):
        out = py_sn_est_gpu.raw_normals_from_vote(image.reshape(shape), W.reshape((3,) + shape),
                                                  0.2)
        unit, mask, raw = oracle.normals_from_vote(I.astype(np.complex128),
                                                   W.T.astype(np.complex128), 0.2)
        got = out.reshape(V, 3)
        assert out.dtype == np.float64
        assert np.array_equal(np.isnan(got[:, 0]), ~mask)
        err = np.linalg.norm(got[mask] - raw[mask], axis=1)
        assert np.all(err <= 2e-6 * np.linalg.norm(raw[mask], axis=1))
        out_u = py_sn_est_gpu.raw_normals_from_vote(image.reshape(shape),
                                                    W.reshape((3,) + shape), 0.2, unit=True)
        np.testing.assert_allclose(out_u.reshape(V, 3)[mask], unit[mask], atol=2e-6)


def test_scene_configs_have_baseline_shapes():
    sc = scenes.sphere_scene(seed=0, n_ap=8, nf=16, n_vox=5, n_pts=10)
    assert sc.meas.shape == (64, 16) and sc.meas.dtype == np.complex64
    assert sc.grid_shape == (5, 5, 5)
    # frequency mapping f_j = 77 GHz + j*4 GHz/(F-1)
    assert abs(sc.slope - 4e9 / 15) < 1e-3 and abs(sc.wavelength - scenes.C / 77e9) < 1e-15
    ap = scenes.planar_aperture(32, 3e-3)
    assert ap.shape == (1024, 3) and np.allclose(ap[:, :2].mean(0), 0, atol=1e-9)
    assert np.isclose(ap[:, 0].max() - ap[:, 0].min(), 31 * 3e-3)
    x, y, z = scenes.voxel_axes(48, 4e-3, (0, 0, 0.4))
    assert np.isclose(z.mean(), 0.4, atol=1e-6) and np.isclose(x[1] - x[0], 4e-3)


def test_scene_snr_and_determinism():
    a = scenes.sphere_scene(seed=5, n_ap=6, nf=8, n_vox=3, n_pts=20, snr_db=20)
    b = scenes.sphere_scene(seed=5, n_ap=6, nf=8, n_vox=3, n_pts=20, snr_db=20)
    np.testing.assert_array_equal(a.meas, b.meas)
    clean = scenes.synthesize(a.antenna_locs, a.points, a.rho,
                              77e9 + np.arange(8) * 4e9 / 7, sign=-1)
    noise = a.meas - clean
    snr = 10 * np.log10(np.mean(np.abs(clean) ** 2) / np.mean(np.abs(noise) ** 2))
    assert abs(snr - 20) < 1.5


def test_union_surface_points_are_on_the_boundary():
    rng = np.random.default_rng(0)
    c = np.array([0, 0, 0.45])
    p = scenes.box_cylinder_union_surface(rng, 2000, (0.12, 0.08, 0.04), 0.04, 0.08, c)
    assert p.shape == (2000, 3)
    q = p - c
    in_box = np.all(np.abs(q) < np.array([0.06, 0.04, 0.02]) * (1 - 1e-6), axis=1)
    in_cyl = (q[:, 0] ** 2 + q[:, 1] ** 2 < 0.04 ** 2 * (1 - 1e-6)) & \
             (np.abs(q[:, 2]) < 0.04 * (1 - 1e-6))
    assert not np.any(in_box & in_cyl)


def test_lazy_conjugate_views_are_refused_or_resolved():
    """The kernels read raw memory; torch's lazy conj/neg views must never reach them."""
    import pytest
    import torch
    from mmnorm_b200 import ops
    z = torch.tensor([1 + 2j, 3 - 1j], dtype=torch.complex64)
    zc = z.conj()
    assert zc.is_conj()
    with pytest.raises(ValueError):
        ops._need(zc, "meas", torch.complex64, z.device)
    r = ops._plain(zc)
    assert not r.is_conj() and torch.equal(r, torch.conj_physical(z))
    ops._need(r, "meas", torch.complex64, z.device)
