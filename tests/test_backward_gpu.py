"""Backward (adjoint) of the fused backprojection + vote: gradients with respect to the
complex measurements and to per-antenna position offsets, against
  * the FP64 C oracle's adjoint for given upstream gradients,
  * a dense FP64 torch autograd model on a 16^3 grid x 16x16 aperture (config 3's check)
    with the loss L2(|I| - target) + cosine loss of the normals vs the analytic sphere,
  * FP64 central finite differences (h = 1e-6 m) at 64 random position entries and at
    64 random measurement entries,
  * the adjoint (dot-product) identity <gI, I(m)> = <dL/dm, m> at a larger size."""
import math

import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu
C = 2.99792458e8


def _t(a, dev):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), device=dev)


def dense_fp64(x, y, z, ant, rxo, meas, wl, slope, pos, ti=False, chunk=128):
    """Dense FP64 torch model of the fused forward: I [V], W [3, V] (complex128),
    differentiable with respect to meas (complex128 [A, F]) and pos (float64 [A, 3])."""
    import torch
    X, Y, Zz = torch.meshgrid(x.double(), y.double(), z.double(), indexing="ij")
    vox = torch.stack([X.reshape(-1), Y.reshape(-1), Zz.reshape(-1)], dim=1)
    A, F = meas.shape
    o = rxo.double()[torch.arange(A, device=ant.device) % rxo.shape[0]]
    tx = ant.double() + pos
    rx = tx + o
    virt = tx + o / 2
    kap = 2 * math.pi * (1.0 / wl + torch.arange(F, device=ant.device, dtype=torch.float64)
                         * slope / C)
    Is, Ws = [], []
    for v0 in range(0, vox.shape[0], chunk):
        vv = vox[v0:v0 + chunk]
        d = (vv[:, None] - tx[None]).norm(dim=2) + (vv[:, None] - rx[None]).norm(dim=2)
        if ti:
            d = d + 0.15
        p = torch.exp(-1j * d[..., None] * kap)
        c = (p * meas[None]).sum(-1)
        Is.append(c.sum(1))
        Ws.append(torch.einsum("va,vak->kv", c, (virt[None] - vv[:, None]).to(c.dtype)))
    return torch.cat(Is), torch.cat(Ws, dim=1)


def loss_fn(I, W, target, n_true, mask):
    """L2 between |I| and the target plus the mean cosine loss of the unit normals
    against the analytic sphere normals on the masked voxels (config 3)."""
    import torch
    I = I.to(torch.complex128)
    W = W.to(torch.complex128).reshape(3, -1)
    l_img = ((I.abs() - target) ** 2).sum() / (target ** 2).sum()
    mag = I.abs()
    raw = (I.conj()[None] * W).real / mag[None]
    n = raw / raw.norm(dim=0, keepdim=True)
    l_nrm = (1 - (n[:, mask] * n_true[:, mask]).sum(0)).mean()
    return l_img + l_nrm


def _problem(dev, n_ap=16, n_vox=16, nf=128, seed=0):
    import torch
    sc = scenes.sphere_scene(seed=seed, n_ap=n_ap, pitch=3e-3, nf=nf, n_vox=n_vox,
                             spacing=3e-3 * 64 / n_vox, sign=+1)
    rng = np.random.default_rng(seed + 100)
    pos = rng.normal(0, 5e-4, sc.antenna_locs.shape).astype(np.float32)
    t = {k: _t(v, dev) for k, v in dict(x=sc.x_locs, y=sc.y_locs, z=sc.z_locs,
                                         ant=sc.antenna_locs,
                                         rxo=np.zeros((1, 3), np.float32), meas=sc.meas,
                                         pos=pos).items()}
    # seeded target image and analytic normals
    centre = np.array(sc.sphere[0])
    vox = sc.voxel_centres().astype(np.float64)
    nt = vox - centre
    nt /= np.linalg.norm(nt, axis=1, keepdims=True)
    # the vote points from the surface toward the aperture: the visible cap's outward normal
    return sc, t, rng, torch.as_tensor(nt.T.copy(), device=dev)


@pytest.fixture(params=["interp", "horner"])
def pos_form(request):
    from mmnorm_b200 import ops
    ops.set_position_pass(request.param)
    yield request.param
    ops.set_position_pass("interp")


@pytest.fixture(params=["horner", "interp"])
def meas_form(request):
    from mmnorm_b200 import ops
    ops.set_measurement_pass(request.param)
    yield request.param
    ops.set_measurement_pass("interp")


def test_adjoint_matches_oracle(cuda_dev, oracle, pos_form, meas_form):
    import torch
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=41, n_ap=6, nf=40, n_vox=5, n_pts=10)
    rng = np.random.default_rng(41)
    rxo = np.array([[0.0, -0.004, 0.001]], np.float32)
    V = sc.num_voxels
    gI = (rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64)
    gW = (rng.standard_normal((3, V)) + 1j * rng.standard_normal((3, V))).astype(np.complex64)
    args = [_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs, rxo,
                                      sc.meas)]
    gm, gp = ops.backproject_backward(*args, sc.wavelength, sc.slope, _t(gI, cuda_dev),
                                      _t(gW, cuda_dev), is_ti_radar=True)
    torch.cuda.synchronize()
    gm_o, gp_o = oracle.full_backward(sc.voxel_centres(), sc.antenna_locs, rxo, sc.meas,
                                      sc.wavelength, sc.slope, gI.astype(np.complex128),
                                      gW.T.astype(np.complex128), is_ti=True)
    assert oracle.rel_l2(gm.cpu().numpy(), gm_o) < 2e-5
    assert oracle.rel_l2(gp.cpu().numpy(), gp_o) < 2e-4


def test_gradients_vs_dense_fp64_and_finite_differences(cuda_dev, pos_form, meas_form):
    import torch
    from mmnorm_b200 import ops
    sc, t, rng, n_true = _problem(cuda_dev)
    V = sc.num_voxels
    # mask and target from an FP64 evaluation at the starting point (held fixed)
    with torch.no_grad():
        I0, _ = dense_fp64(t["x"], t["y"], t["z"], t["ant"], t["rxo"],
                           t["meas"].to(torch.complex128), sc.wavelength, sc.slope,
                           t["pos"].double())
        mag = I0.abs()
        mask = mag > 0.05 * mag.max()
        target = mag * torch.as_tensor(rng.uniform(0.8, 1.2, V), device=cuda_dev)
    assert int(mask.sum()) > 20

    # ours: complex64 measurements, float32 offsets, library forward + adjoint
    meas = t["meas"].clone().requires_grad_(True)
    pos = t["pos"].clone().requires_grad_(True)
    I, W = ops.backproject_differentiable(t["x"], t["y"], t["z"], t["ant"], t["rxo"], meas,
                                          sc.wavelength, sc.slope, pos_offsets=pos)
    loss_fn(I.reshape(-1), W, target, n_true, mask).backward()
    gm, gp = meas.grad.to(torch.complex128), pos.grad.double()

    # dense FP64 autograd
    meas64 = t["meas"].to(torch.complex128).requires_grad_(True)
    pos64 = t["pos"].double().requires_grad_(True)

    def L64(m, p_):
        I_, W_ = dense_fp64(t["x"], t["y"], t["z"], t["ant"], t["rxo"], m, sc.wavelength,
                            sc.slope, p_)
        return loss_fn(I_, W_, target, n_true, mask)

    L64(meas64, pos64).backward()
    rel = lambda a, b: float((a - b).norm() / b.norm())
    assert rel(gm, meas64.grad) < 1e-3
    assert rel(gp, pos64.grad) < 1e-3

    # FP64 central finite differences, h = 1e-6 m, 64 random position entries
    h = 1e-6
    A = pos.shape[0]
    sel = rng.choice(A * 3, 64, replace=False)
    fd, ad = [], []
    with torch.no_grad():
        for s in sel:
            a, k = divmod(int(s), 3)
            e = torch.zeros_like(pos64)
            e[a, k] = h
            fd.append((L64(meas64, pos64 + e) - L64(meas64, pos64 - e)).item() / (2 * h))
            ad.append(gp[a, k].item())
    fd, ad = np.array(fd), np.array(ad)
    assert np.linalg.norm(ad - fd) / np.linalg.norm(fd) < 2e-3
    # and 64 random measurement entries (real and imaginary parts)
    hm = 1e-3 * float(t["meas"].abs().mean())
    selm = rng.choice(meas.numel(), 64, replace=False)
    fdm, adm = [], []
    with torch.no_grad():
        for s in selm:
            a, j = divmod(int(s), meas.shape[1])
            for unit, part in ((1.0, "re"), (1j, "im")):
                e = torch.zeros_like(meas64)
                e[a, j] = unit * hm
                fdm.append((L64(meas64 + e, pos64) - L64(meas64 - e, pos64)).item() / (2 * hm))
                g = gm[a, j]
                adm.append(g.real.item() if part == "re" else g.imag.item())
    fdm, adm = np.array(fdm), np.array(adm)
    assert np.linalg.norm(adm - fdm) / np.linalg.norm(fdm) < 2e-3


def test_adjoint_dot_product_identity(cuda_dev, meas_form):
    """I is linear in the measurements, so for any gI: Re<gI, I(m)> = Re<dL/dm, m>."""
    import torch
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=43, n_ap=32, nf=64, n_vox=24, n_pts=50)
    rng = np.random.default_rng(43)
    V = sc.num_voxels
    gI = torch.as_tensor((rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64),
                         device=cuda_dev)
    args = [_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs,
                                      np.zeros((1, 3), np.float32), sc.meas)]
    I, _ = ops.backproject(*args, sc.wavelength, sc.slope, want_vote=False)
    gm, _ = ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, None, want_pos=False)
    lhs = (gI.conj().to(torch.complex128) * I.reshape(-1).to(torch.complex128)).sum().real
    rhs = (gm.conj().to(torch.complex128) * args[5].to(torch.complex128)).sum().real
    assert abs(float(lhs - rhs)) <= 2e-5 * abs(float(lhs))


def test_image_only_position_gradient(cuda_dev, oracle, pos_form, meas_form):
    """Without a vote term the position pass skips the vote terms (Horner form: one chain
    per voxel-antenna, voxel pairs in the FFMA2 halves); it must agree with the oracle's
    adjoint and with the full kernel given an all-zero vote gradient."""
    import torch
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=44, n_ap=10, nf=72, n_vox=9, n_pts=20)
    rng = np.random.default_rng(44)
    rxo = np.array([[0.0, -0.004, 0.001]], np.float32)
    V = sc.num_voxels
    gI = (rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64)
    args = [_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs, rxo,
                                      sc.meas)]
    gm1, gp1 = ops.backproject_backward(*args, sc.wavelength, sc.slope, _t(gI, cuda_dev), None,
                                        is_ti_radar=True)
    zeros = torch.zeros((3, V), dtype=torch.complex64, device=cuda_dev)
    gm2, gp2 = ops.backproject_backward(*args, sc.wavelength, sc.slope, _t(gI, cuda_dev), zeros,
                                        is_ti_radar=True)
    torch.cuda.synchronize()
    _, gp_o = oracle.full_backward(sc.voxel_centres(), sc.antenna_locs, rxo, sc.meas,
                                   sc.wavelength, sc.slope, gI.astype(np.complex128),
                                   np.zeros((V, 3), np.complex128), is_ti=True)
    assert oracle.rel_l2(gp1.cpu().numpy(), gp_o) < 2e-4
    assert oracle.rel_l2(gp1.cpu().numpy(), gp2.cpu().numpy().astype(np.float64)) < 1e-5
    assert torch.equal(gm1, gm2)
    # autograd: a loss on the image only reaches the image-only path and the same gradients
    meas = args[5].clone().requires_grad_(True)
    pos = torch.zeros_like(args[3]).requires_grad_(True)
    I, W = ops.backproject_differentiable(*args[:5], meas, sc.wavelength, sc.slope,
                                          pos_offsets=pos, is_ti_radar=True)
    (I.reshape(-1).conj() * _t(gI, cuda_dev)).real.sum().backward()
    assert oracle.rel_l2(pos.grad.cpu().numpy().astype(np.float64),
                         gp1.cpu().numpy().astype(np.float64)) < 1e-6


@pytest.mark.parametrize("nf", [1, 3, 40, 129])
def test_interpolation_form_matches_horner_form(cuda_dev, oracle, nf):
    """The position pass's two forms on the same problem, over sample counts down to one
    (grid of 2 cells, narrower than the 8-cell kernel: taps wrap around the grid several
    times) and odd counts (J0 = F/2 rounds down); both against the oracle."""
    import torch
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=45 + nf, n_ap=7, nf=max(nf, 2), n_vox=7, n_pts=12)
    meas = np.ascontiguousarray(sc.meas[:, :nf])
    rng = np.random.default_rng(45)
    rxo = np.array([[0.0, -0.004, 0.001]], np.float32)
    V = sc.num_voxels
    gI = (rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64)
    gW = (rng.standard_normal((3, V)) + 1j * rng.standard_normal((3, V))).astype(np.complex64)
    args = [_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs, rxo,
                                      meas)]
    out = {}
    try:
        for form in ("interp", "horner"):
            ops.set_position_pass(form)
            out[form] = ops.backproject_backward(*args, sc.wavelength, sc.slope,
                                                 _t(gI, cuda_dev), _t(gW, cuda_dev),
                                                 want_meas=False)[1]
    finally:
        ops.set_position_pass("interp")
    torch.cuda.synchronize()
    _, gp_o = oracle.full_backward(sc.voxel_centres(), sc.antenna_locs, rxo, meas,
                                   sc.wavelength, sc.slope, gI.astype(np.complex128),
                                   gW.T.astype(np.complex128))
    a, b = (out[f].cpu().numpy().astype(np.float64) for f in ("interp", "horner"))
    assert oracle.rel_l2(a, gp_o) < 2e-4 and oracle.rel_l2(b, gp_o) < 2e-4
    assert oracle.rel_l2(a, b) < 2e-5


def test_position_variants_agree(cuda_dev, oracle):
    """Every launch shape of the interpolation form gives the oracle's position gradient
    (voxel-to-thread mapping and summation order differ, the values only by rounding)."""
    import torch
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=47, n_ap=12, nf=48, n_vox=11, n_pts=16)
    rng = np.random.default_rng(47)
    rxo = np.array([[0.0, -0.004, 0.001]], np.float32)
    V = sc.num_voxels
    gI = (rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64)
    gW = (rng.standard_normal((3, V)) + 1j * rng.standard_normal((3, V))).astype(np.complex64)
    args = [_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs, rxo,
                                      sc.meas)]
    _, gp_o = oracle.full_backward(sc.voxel_centres(), sc.antenna_locs, rxo, sc.meas,
                                   sc.wavelength, sc.slope, gI.astype(np.complex128),
                                   gW.T.astype(np.complex128))
    names = ops.position_variants()
    assert len(names) >= 2
    outs = []
    try:
        for i in range(len(names)):
            ops.set_position_variant(i)
            for g in (_t(gW, cuda_dev), None):
                gp = ops.backproject_backward(*args, sc.wavelength, sc.slope, _t(gI, cuda_dev),
                                              g, want_meas=False)[1]
                outs.append((i, g is None, gp.cpu().numpy().astype(np.float64)))
    finally:
        ops.set_position_variant(0)
    _, gp_img = oracle.full_backward(sc.voxel_centres(), sc.antenna_locs, rxo, sc.meas,
                                     sc.wavelength, sc.slope, gI.astype(np.complex128),
                                     np.zeros((V, 3), np.complex128))
    for i, img, gp in outs:
        assert oracle.rel_l2(gp, gp_img if img else gp_o) < 2e-4, (names[i], img)
    with pytest.raises(Exception):
        ops.set_position_variant(len(names))


@pytest.mark.parametrize("nf", [1, 3, 40, 129])
@pytest.mark.parametrize("spacing", [None, 0.04])
def test_interpolation_measurement_pass(cuda_dev, oracle, nf, spacing):
    """The measurement gradient's interpolation form against the voxel-sum form and the
    oracle, over sample counts down to one and on a sparse grid (4 cm voxel pitch: a warp's
    32 voxels spread over ~80 grid cells, so its window reduction takes many rounds)."""
    import torch
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=60 + nf, n_ap=7, nf=max(nf, 2), n_vox=7, n_pts=12)
    meas = np.ascontiguousarray(sc.meas[:, :nf])
    x, y, z = sc.x_locs, sc.y_locs, sc.z_locs
    if spacing is not None:
        x = (x.mean() + spacing * (np.arange(5) - 2)).astype(np.float32)
        y = (y.mean() + spacing * (np.arange(4) - 1.5)).astype(np.float32)
        z = (z.mean() + spacing * (np.arange(40) - 19.5)).astype(np.float32)
    rng = np.random.default_rng(60)
    rxo = np.array([[0.0, -0.004, 0.001]], np.float32)
    V = len(x) * len(y) * len(z)
    gI = (rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64)
    gW = (rng.standard_normal((3, V)) + 1j * rng.standard_normal((3, V))).astype(np.complex64)
    args = [_t(a, cuda_dev) for a in (x, y, z, sc.antenna_locs, rxo, meas)]
    out = {}
    try:
        for form in ("interp", "horner"):
            ops.set_measurement_pass(form)
            out[form] = ops.backproject_backward(*args, sc.wavelength, sc.slope,
                                                 _t(gI, cuda_dev), _t(gW, cuda_dev),
                                                 want_pos=False)[0]
        ops.set_measurement_pass("interp")
        again = ops.backproject_backward(*args, sc.wavelength, sc.slope, _t(gI, cuda_dev),
                                         _t(gW, cuda_dev), want_pos=False)[0]
    finally:
        ops.set_measurement_pass("interp")
    torch.cuda.synchronize()
    assert torch.equal(out["interp"], again)  # no atomics: bitwise repeatable
    vox = np.stack(np.meshgrid(x, y, z, indexing="ij"), -1).reshape(-1, 3)
    gm_o, _ = oracle.full_backward(vox, sc.antenna_locs, rxo, meas, sc.wavelength, sc.slope,
                                   gI.astype(np.complex128), gW.T.astype(np.complex128))
    a, b = (out[f].cpu().numpy().astype(np.complex128) for f in ("interp", "horner"))
    assert oracle.rel_l2(b, gm_o) < 2e-5
    assert oracle.rel_l2(a, gm_o) < 2e-5


def test_position_autotuner(cuda_dev):
    """autotune.tune_position times every launch shape, selects the fastest, and the
    selection gives the gradient of that shape."""
    import torch
    from mmnorm_b200 import autotune, ops
    sc = scenes.sphere_scene(seed=48, n_ap=16, nf=64, n_vox=16, n_pts=20)
    rng = np.random.default_rng(48)
    V = sc.num_voxels
    gI = _t((rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64),
            cuda_dev)
    args = [_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs,
                                      np.zeros((1, 3), np.float32), sc.meas)]
    try:
        res = autotune.tune_position(*args, sc.wavelength, sc.slope, gI)
        assert set(res["times_ms"]) == {str(i) for i in range(len(ops.position_variants()))}
        gp = ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, None,
                                      want_meas=False)[1]
        ops.set_position_variant(res["best"])
        gp2 = ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, None,
                                       want_meas=False)[1]
        torch.cuda.synchronize()
        assert torch.equal(gp, gp2)
    finally:
        ops.set_position_variant(0)


def test_position_autotuner_keeps_the_callers_selection_without_apply(cuda_dev):
    from mmnorm_b200 import autotune, ops
    sc = scenes.sphere_scene(seed=49, n_ap=16, nf=96, n_vox=16, n_pts=20)
    rng = np.random.default_rng(49)
    V = sc.num_voxels
    gI = _t((rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64),
            cuda_dev)
    args = [_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs,
                                      np.zeros((1, 3), np.float32), sc.meas)]
    mine = len(ops.position_variants()) - 1
    ops.set_position_variant(mine)
    try:
        autotune.tune_position(*args, sc.wavelength, sc.slope, gI, apply=False)
        assert ops.current_position_variant() == mine
    finally:
        ops.set_position_variant(0)
