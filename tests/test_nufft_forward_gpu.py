"""The forward in interpolation form (mmn_backproject_nufft, ops.backproject mode="nufft"):
the mixed form's per-(voxel, antenna) sample sum by an 8-tap gather from each antenna's
2x oversampled grid.  Parity with the FP64 oracle at the mixed form's tolerance and with
the mixed form itself, over the forward suite's edge cases."""
import numpy as np
import pytest

from mmnorm_b200 import scenes
from test_forward_gpu import TOL_MIXED, _t, run_ops, small_scene

pytestmark = pytest.mark.gpu


def test_tiny_grid_matches_oracle_and_mixed(cuda_dev, oracle):
    sc = small_scene()
    I, W = run_ops(cuda_dev, sc, "nufft")
    Im, Wm = run_ops(cuda_dev, sc, "mixed")
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    assert oracle.rel_l2(I, Io) < TOL_MIXED and oracle.rel_l2(W, Wo) < TOL_MIXED
    assert oracle.rel_l2(I, Im) < 1e-5 and oracle.rel_l2(W, Wm) < 1e-5


@pytest.mark.parametrize("nf", [1, 3, 31, 100])
def test_sample_counts(cuda_dev, oracle, nf):
    sc = small_scene(seed=4, nf=max(nf, 2))
    meas = sc.meas[:, :nf]
    I, W = run_ops(cuda_dev, sc, "nufft", meas=meas)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), meas,
                         sc.wavelength, sc.slope)
    assert oracle.rel_l2(I, Io) < TOL_MIXED
    assert oracle.rel_l2(W, Wo) < TOL_MIXED


def test_multi_rx_offsets_ti_and_position_offsets(cuda_dev, oracle):
    sc = small_scene(seed=5)
    rng = np.random.default_rng(5)
    rxo = np.array([[0, -0.005, 0], [0, -0.007, 0.001], [0.002, 0, 0]], np.float32)
    A = sc.antenna_locs.shape[0]
    ant = np.repeat(sc.antenna_locs, 3, axis=0)[: A + 7]
    meas = (rng.standard_normal((ant.shape[0], 16)) +
            1j * rng.standard_normal((ant.shape[0], 16))).astype(np.complex64)
    I, W = run_ops(cuda_dev, sc, "nufft", rxo=rxo, ti=True, meas=meas, ant=ant)
    Io, Wo = oracle.full(sc.voxel_centres(), ant, rxo, meas, sc.wavelength, sc.slope,
                         is_ti=True)
    assert oracle.rel_l2(I, Io) < TOL_MIXED and oracle.rel_l2(W, Wo) < TOL_MIXED
    pos = rng.normal(0, 5e-4, sc.antenna_locs.shape)
    I, W = run_ops(cuda_dev, sc, "nufft", pos=pos)
    Im, Wm = run_ops(cuda_dev, sc, "mixed", pos=pos)
    assert oracle.rel_l2(I, Im) < 1e-5 and oracle.rel_l2(W, Wm) < 1e-5


def test_antenna_split_path_and_repeatability(cuda_dev, oracle):
    """Few voxels and many antennas: the antenna range is split across CTAs and the
    partial sums are reduced in split order -- bitwise repeatable."""
    sc = scenes.sphere_scene(seed=7, n_ap=48, nf=32, n_vox=6, n_pts=20)
    I1, W1 = run_ops(cuda_dev, sc, "nufft")
    I2, W2 = run_ops(cuda_dev, sc, "nufft")
    assert np.array_equal(I1, I2) and np.array_equal(W1, W2)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    assert oracle.rel_l2(I1, Io) < TOL_MIXED and oracle.rel_l2(W1, Wo) < TOL_MIXED


def test_sample_count_limit(cuda_dev):
    from mmnorm_b200 import _lib, ops
    sc = small_scene(seed=9, nf=2)
    meas = np.zeros((sc.antenna_locs.shape[0], 1600), np.complex64)
    with pytest.raises(_lib.MmnError):
        ops.backproject(_t(sc.x_locs, cuda_dev), _t(sc.y_locs, cuda_dev),
                        _t(sc.z_locs, cuda_dev), _t(sc.antenna_locs, cuda_dev),
                        _t(np.zeros((1, 3), np.float32), cuda_dev), _t(meas, cuda_dev),
                        sc.wavelength, sc.slope, mode="nufft")
