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
    """The forward stages one antenna's (G.re, G.im) grid row of 2F + 7 cells of 8 bytes
    per stage at least: F = 3200 does not fit a 48 KB stage."""
    from mmnorm_b200 import _lib, ops
    sc = small_scene(seed=9, nf=2)
    meas = np.zeros((sc.antenna_locs.shape[0], 3200), np.complex64)
    with pytest.raises(_lib.MmnError):
        ops.backproject(_t(sc.x_locs, cuda_dev), _t(sc.y_locs, cuda_dev),
                        _t(sc.z_locs, cuda_dev), _t(sc.antenna_locs, cuda_dev),
                        _t(np.zeros((1, 3), np.float32), cuda_dev), _t(meas, cuda_dev),
                        sc.wavelength, sc.slope, mode="nufft")


def test_torch_operator_and_autograd(cuda_dev):
    """torch.ops.mmnorm.backproject and backproject_differentiable take mode "nufft"; the
    gradients (the same adjoint kernels) agree with mode "mixed" to the forms' distance."""
    import torch
    import mmnorm_b200.torch_ops  # noqa: F401
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=11, n_ap=8, nf=40, n_vox=8, n_pts=20)
    t = lambda a: _t(a, cuda_dev)
    args = (t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs),
            t(np.zeros((1, 3), np.float32)))
    i0, v0 = ops.backproject(*args, t(sc.meas), sc.wavelength, sc.slope, mode="nufft")
    i1, v1 = torch.ops.mmnorm.backproject(*args, t(sc.meas), sc.wavelength, sc.slope, "nufft",
                                          0.0, False, None)
    assert torch.equal(i0, i1) and torch.equal(v0, v1)
    grads = {}
    for mode in ("mixed", "nufft"):
        meas = t(sc.meas).requires_grad_(True)
        pos = torch.zeros_like(args[3]).requires_grad_(True)
        img, vote = ops.backproject_differentiable(*args, meas, sc.wavelength, sc.slope,
                                                   pos_offsets=pos, mode=mode)
        ((img.abs() ** 2).sum() * 1e-6 + (vote.real ** 2).sum() * 1e-9).backward()
        grads[mode] = (meas.grad.clone(), pos.grad.clone())
    rel = lambda a, b: float((a - b).norm() / b.norm())
    assert rel(grads["nufft"][0], grads["mixed"][0]) < 1e-4
    assert rel(grads["nufft"][1], grads["mixed"][1]) < 1e-4


def test_near_the_sample_limit_forward_and_adjoint(cuda_dev, oracle):
    """F = 1500: one antenna's grid row (3007 cells, 48 KB) fills a stage on its own, the
    measurement spread's rows need opt-in shared memory (~113 KB per CTA), and the output
    transform's 3000-cell grid sits just under 48 KB -- forward and both gradient passes
    against the oracle."""
    import torch
    from mmnorm_b200 import ops
    nf = 1500
    sc = scenes.sphere_scene(seed=12, n_ap=4, nf=nf, n_vox=5, n_pts=10)
    rxo = np.array([[0.0, -0.004, 0.001]], np.float32)
    I, W = run_ops(cuda_dev, sc, "nufft", rxo=rxo)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, rxo, sc.meas, sc.wavelength,
                         sc.slope)
    assert oracle.rel_l2(I, Io) < TOL_MIXED and oracle.rel_l2(W, Wo) < TOL_MIXED
    rng = np.random.default_rng(12)
    V = sc.num_voxels
    gI = (rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64)
    gW = (rng.standard_normal((3, V)) + 1j * rng.standard_normal((3, V))).astype(np.complex64)
    args = [_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs, rxo,
                                      sc.meas)]
    gm, gp = ops.backproject_backward(*args, sc.wavelength, sc.slope, _t(gI, cuda_dev),
                                      _t(gW, cuda_dev))
    torch.cuda.synchronize()
    gm_o, gp_o = oracle.full_backward(sc.voxel_centres(), sc.antenna_locs, rxo, sc.meas,
                                      sc.wavelength, sc.slope, gI.astype(np.complex128),
                                      gW.T.astype(np.complex128))
    assert oracle.rel_l2(gm.cpu().numpy().astype(np.complex128), gm_o) < 2e-5
    assert oracle.rel_l2(gp.cpu().numpy().astype(np.float64), gp_o) < 2e-4


def test_forward_near_its_sample_limit(cuda_dev, oracle):
    """F = 3000: one forward grid row (6007 cells of 8 bytes, 47 KB) fills a stage."""
    nf = 3000
    sc = scenes.sphere_scene(seed=13, n_ap=3, nf=nf, n_vox=4, n_pts=8)
    I, W = run_ops(cuda_dev, sc, "nufft")
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    assert oracle.rel_l2(I, Io) < TOL_MIXED and oracle.rel_l2(W, Wo) < TOL_MIXED
