"""The second-order (Clenshaw) variants of the fused forward against the FP64 oracle.

A warp runs an antenna's block sums in the second-order form only when every lane's
per-sample rotation angle theta = 2 pi d slope / c (wrapped) keeps |cos theta| <= 0.98;
otherwise that antenna's blocks take the first-order Horner form.  These cases put the
per-sample angle on both sides of that threshold (some warps in each form, and warps
that switch from antenna to antenna), entirely below it (every block in the Horner form),
and well inside the second-order range, for every mixed_clen* variant."""
import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu

TOL = 2e-5  # the mixed form's bound in the forward tests


def _clen_variants():
    from mmnorm_b200 import ops
    return [v["name"] for v in ops.variants("mixed") if "clen" in v["name"]]


def _run(dev, sc, name, meas=None):
    import torch
    from mmnorm_b200 import ops
    names = [v["name"] for v in ops.variants("mixed")]
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    meas = sc.meas if meas is None else meas
    ops.set_variant("mixed", names.index(name))
    try:
        img, vote = ops.backproject(t(sc.x_locs), t(sc.y_locs), t(sc.z_locs),
                                    t(sc.antenna_locs), t(np.zeros((1, 3), np.float32)),
                                    t(meas.astype(np.complex64)), sc.wavelength, sc.slope,
                                    mode="mixed")
        torch.cuda.synchronize()
    finally:
        ops.set_variant("mixed", 0)
    return img.cpu().numpy().ravel(), vote.cpu().numpy().reshape(3, -1).T


def _theta(sc):
    """Per-sample rotation angle of every (voxel, antenna) pair, wrapped to [0, pi]."""
    v = sc.voxel_centres().astype(np.float64)
    a = sc.antenna_locs.astype(np.float64)
    d = 2 * np.sqrt(((v[:, None, :] - a[None, :, :]) ** 2).sum(-1))
    th = 2 * np.pi * d * sc.slope / 2.99792458e8
    return np.abs(np.angle(np.exp(1j * th)))


def test_variants_exist(cuda_dev):
    assert len(_clen_variants()) >= 2


def test_angle_straddles_the_threshold(cuda_dev, oracle):
    # 256 samples over 77-81 GHz: theta = 0.2 at a round trip of ~0.61 m; voxels at
    # 0.28-0.32 m put theta on both sides of it
    sc = scenes.sphere_scene(seed=50, n_ap=8, pitch=3e-3, nf=256, n_vox=8, spacing=4e-3,
                             n_pts=30, radius=0.01, centre=(0.0, 0.0, 0.3))
    th = _theta(sc)
    frac = float(np.mean(np.cos(th) > 0.98))
    assert 0.1 < frac < 0.9, frac  # both forms are exercised
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    for name in _clen_variants():
        I, W = _run(cuda_dev, sc, name)
        assert oracle.rel_l2(I, Io) < TOL, name
        assert oracle.rel_l2(W, Wo) < TOL, name


def test_small_angle_runs_the_first_order_form(cuda_dev, oracle):
    # 1024 samples: theta ~ 0.03 rad everywhere, every block in the Horner form
    sc = scenes.sphere_scene(seed=51, n_ap=6, pitch=3e-3, nf=1024, n_vox=5, spacing=4e-3,
                             n_pts=20, radius=0.01, centre=(0.0, 0.0, 0.25))
    assert float(np.mean(np.cos(_theta(sc)) > 0.98)) == 1.0
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    for name in _clen_variants():
        I, W = _run(cuda_dev, sc, name)
        assert oracle.rel_l2(I, Io) < TOL, name
        assert oracle.rel_l2(W, Wo) < TOL, name


@pytest.mark.parametrize("nf", [2, 63, 64, 65, 130])
def test_second_order_range_and_padding(cuda_dev, oracle, nf):
    """Sample counts around the 32- and 64-sample blocks: whole blocks, then a last block
    over the row's remaining valid samples (the zeros padding rows to 32 are skipped)."""
    sc = scenes.sphere_scene(seed=52 + nf, n_ap=8, pitch=3e-3, nf=nf, n_vox=6, n_pts=20)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    for name in _clen_variants():
        I, W = _run(cuda_dev, sc, name)
        assert oracle.rel_l2(I, Io) < TOL, (name, nf)
        assert oracle.rel_l2(W, Wo) < TOL, (name, nf)


def test_bit_reproducible(cuda_dev):
    sc = scenes.sphere_scene(seed=60, n_ap=10, nf=96, n_vox=8, n_pts=20)
    for name in _clen_variants():
        a = _run(cuda_dev, sc, name)
        b = _run(cuda_dev, sc, name)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), name
