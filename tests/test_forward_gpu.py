"""Parity of the fused forward kernels (through the C ABI via mmnorm_b200.ops) with the
FP64 oracle, on seeded inputs small enough for the oracle, plus edge cases."""
import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu

# Tolerances (relative L2 against the FP64 oracle).  The mixed form's error budget is
# the FP32 Horner recurrence within a 32-sample block plus FP32 accumulation; the
# plain form carries FP32 range and phase (~1e-4 rad at ~1.5e3 rad of phase).
TOL_MIXED = 2e-5
TOL_PLAIN = 6e-4


def _t(a, dev, dtype=None):
    import torch
    a = np.ascontiguousarray(a)
    return torch.as_tensor(a, device=dev) if dtype is None else \
        torch.as_tensor(a, device=dev, dtype=dtype)


def run_ops(dev, sc, mode="mixed", rxo=None, ti=False, pos=None, meas=None, ant=None,
            vote=True):
    import torch
    from mmnorm_b200 import ops
    rxo = np.zeros((1, 3), np.float32) if rxo is None else np.asarray(rxo, np.float32)
    meas = sc.meas if meas is None else meas
    ant = sc.antenna_locs if ant is None else ant
    img, w = ops.backproject(
        _t(sc.x_locs, dev), _t(sc.y_locs, dev), _t(sc.z_locs, dev),
        _t(np.asarray(ant, np.float32), dev), _t(rxo, dev),
        _t(np.asarray(meas, np.complex64), dev), sc.wavelength, sc.slope, mode=mode,
        is_ti_radar=ti, pos_offsets=None if pos is None else _t(pos.astype(np.float32), dev),
        want_vote=vote)
    torch.cuda.synchronize()
    I = img.cpu().numpy().ravel()
    W = w.cpu().numpy().reshape(3, -1).T if vote else None
    return I, W


def small_scene(seed=3, n_ap=8, nf=16, n_vox=6):
    return scenes.sphere_scene(seed=seed, n_ap=n_ap, nf=nf, n_vox=n_vox, n_pts=20)


@pytest.mark.parametrize("mode,tol", [("mixed", TOL_MIXED), ("plain", TOL_PLAIN)])
def test_tiny_full_grid(cuda_dev, oracle, mode, tol):
    sc = small_scene()
    I, W = run_ops(cuda_dev, sc, mode)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    assert oracle.rel_l2(I, Io) < tol
    assert oracle.rel_l2(W, Wo) < tol


@pytest.mark.parametrize("nf", [1, 31, 45, 64, 100])
def test_sample_counts_not_multiple_of_block(cuda_dev, oracle, nf):
    sc = small_scene(seed=4, nf=max(nf, 2))
    meas = sc.meas[:, :nf]
    I, W = run_ops(cuda_dev, sc, "mixed", meas=meas)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), meas,
                         sc.wavelength, sc.slope)
    assert oracle.rel_l2(I, Io) < TOL_MIXED
    assert oracle.rel_l2(W, Wo) < TOL_MIXED


def test_multi_rx_offsets_and_ti(cuda_dev, oracle):
    sc = small_scene(seed=5)
    rng = np.random.default_rng(5)
    rxo = np.array([[0, -0.005, 0], [0, -0.007, 0.001], [0.002, 0, 0]], np.float32)
    A = sc.antenna_locs.shape[0]
    ant = np.repeat(sc.antenna_locs, 3, axis=0)[: A + 7]  # A+7: ragged, not a multiple of R
    meas = (rng.standard_normal((ant.shape[0], 16)) +
            1j * rng.standard_normal((ant.shape[0], 16))).astype(np.complex64)
    for mode, tol in (("mixed", TOL_MIXED), ("plain", TOL_PLAIN)):
        I, W = run_ops(cuda_dev, sc, mode, rxo=rxo, ti=True, meas=meas, ant=ant)
        Io, Wo = oracle.full(sc.voxel_centres(), ant, rxo, meas, sc.wavelength, sc.slope,
                             is_ti=True)
        assert oracle.rel_l2(I, Io) < tol, mode
        assert oracle.rel_l2(W, Wo) < tol, mode


def test_per_antenna_position_offsets(cuda_dev, oracle):
    sc = small_scene(seed=6)
    rng = np.random.default_rng(6)
    pos = rng.normal(0, 5e-4, sc.antenna_locs.shape)
    I, W = run_ops(cuda_dev, sc, "mixed", pos=pos)
    moved = (sc.antenna_locs.astype(np.float64) + pos.astype(np.float32)).astype(np.float32)
    Io, Wo = oracle.full(sc.voxel_centres(), moved, np.zeros((1, 3)), sc.meas, sc.wavelength,
                         sc.slope)
    # float32 rounding of (position + offset) in the oracle input: <= 1.2e-8 m
    assert oracle.rel_l2(I, Io) < 1e-4
    assert oracle.rel_l2(W, Wo) < 1e-4


def test_antenna_split_path(cuda_dev, oracle):
    """Few voxels and many antennas: the planner splits the antenna range across CTAs and
    reduces the partial sums in split order."""
    from mmnorm_b200 import ops
    import torch
    sc = scenes.sphere_scene(seed=7, n_ap=48, nf=32, n_vox=6, n_pts=20)
    p = ops.make_problem(*(_t(a, cuda_dev) for a in (sc.x_locs, sc.y_locs, sc.z_locs,
                                                     sc.antenna_locs,
                                                     np.zeros((1, 3), np.float32),
                                                     sc.meas)), sc.wavelength, sc.slope)
    info = ops.plan_info(p, "mixed")
    assert info["splits"] > 1, info
    I, W = run_ops(cuda_dev, sc, "mixed")
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope, phase_mode=1)
    assert oracle.rel_l2(I, Io) < TOL_MIXED
    assert oracle.rel_l2(W, Wo) < TOL_MIXED


def test_ragged_grid_and_single_antenna(cuda_dev, oracle):
    sc = scenes.sphere_scene(seed=8, n_ap=1, nf=33, n_vox=1, n_pts=5)
    sc.x_locs = np.linspace(-0.05, 0.05, 7).astype(np.float32)
    sc.y_locs = np.linspace(-0.04, 0.04, 3).astype(np.float32)
    sc.z_locs = np.linspace(0.35, 0.45, 11).astype(np.float32)
    I, W = run_ops(cuda_dev, sc, "mixed")
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    assert I.shape == (7 * 3 * 11,)
    assert oracle.rel_l2(I, Io) < TOL_MIXED


def test_zero_antennas_gives_zero_image(cuda_dev):
    sc = small_scene()
    I, W = run_ops(cuda_dev, sc, "mixed", meas=np.zeros((0, 16), np.complex64),
                   ant=np.zeros((0, 3), np.float32))
    assert np.all(I == 0) and np.all(W == 0)


def test_deterministic_and_status_clean(cuda_dev):
    import torch
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=9, n_ap=24, nf=64, n_vox=10, n_pts=20)
    a = run_ops(cuda_dev, sc, "mixed")
    b = run_ops(cuda_dev, sc, "mixed")
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    args = [_t(v, cuda_dev) for v in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs,
                                      np.zeros((1, 3), np.float32), sc.meas)]
    p = ops.make_problem(*args, sc.wavelength, sc.slope)
    ws = torch.empty(ops.workspace_bytes(p), dtype=torch.uint8, device=cuda_dev)
    ops.backproject(*args, sc.wavelength, sc.slope, workspace=ws)
    assert ops.read_status(ws) == 0


@pytest.mark.parametrize("idx", list(range(40)))
def test_every_mixed_variant(cuda_dev, oracle, idx):
    from mmnorm_b200 import ops
    n = len(ops.variants("mixed"))
    if idx >= n:
        pytest.skip("no variant %d" % idx)
    ops.set_variant("mixed", idx)
    try:
        sc = small_scene(seed=10, n_vox=9)
        I, W = run_ops(cuda_dev, sc, "mixed")
    finally:
        ops.set_variant("mixed", 0)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    assert oracle.rel_l2(I, Io) < TOL_MIXED
    assert oracle.rel_l2(W, Wo) < TOL_MIXED


def test_config0_subset_and_normals(cuda_dev, oracle):
    """Config 0 (32x32 aperture, F=64, 48^3 voxels) on the GPU, checked against the FP64
    oracle on a seeded random 4096-voxel subset: image/vote error and the normal angle
    (mask from the GPU image's own maximum)."""
    import torch
    from mmnorm_b200 import ops
    sc = scenes.config0()
    I, W = run_ops(cuda_dev, sc, "mixed")
    rng = np.random.default_rng(0)
    idx = np.sort(rng.choice(sc.num_voxels, 4096, replace=False))
    Io, Wo = oracle.full(sc.voxel_centres(idx), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope, phase_mode=1)
    assert oracle.rel_l2(I[idx], Io) < TOL_MIXED
    assert oracle.rel_l2(W[idx], Wo) < TOL_MIXED
    img_t = torch.as_tensor(I.reshape(sc.grid_shape), device=cuda_dev)
    w_t = torch.as_tensor(np.ascontiguousarray(W.T).reshape((3,) + sc.grid_shape),
                          device=cuda_dev)
    n, mask = ops.surface_normals(img_t, w_t, 0.05)
    n = n.cpu().numpy().reshape(-1, 3)
    mask = mask.cpu().numpy().ravel()
    mag = np.abs(I.astype(np.complex128))
    thr = mag.max() * 0.05
    differ = mask != (mag > thr)
    # |I| is formed in FP32 on the device: only voxels within rounding of the threshold
    # may land on the other side
    assert np.all(np.abs(mag[differ] - thr) <= 1e-6 * thr)
    sel = idx[mask[idx]]
    assert sel.size > 10
    _, _, raw_o = oracle.normals_from_vote(Io, Wo, 0.0)
    pos = np.searchsorted(idx, sel)
    ang = oracle.angle_deg(n[sel], raw_o[pos])
    assert np.median(ang) < 0.5
    assert np.all(np.isnan(n[~mask]))


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_every_plain_variant(cuda_dev, oracle, idx):
    from mmnorm_b200 import ops
    if idx >= len(ops.variants("plain")):
        pytest.skip("no variant %d" % idx)
    ops.set_variant("plain", idx)
    try:
        sc = small_scene(seed=15, n_vox=7)
        I, W = run_ops(cuda_dev, sc, "plain")
    finally:
        ops.set_variant("plain", 0)
    Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), sc.meas,
                         sc.wavelength, sc.slope)
    assert oracle.rel_l2(I, Io) < TOL_PLAIN
    assert oracle.rel_l2(W, Wo) < TOL_PLAIN


@pytest.mark.parametrize("n_ap", [12, 7])
def test_pair_and_scalar_mixed_forms_agree_bitwise(cuda_dev, n_ap):
    """FFMA2 computes each half with a single rounding, exactly like FFMA, and every form
    accumulates a voxel's antennas in antenna order: the voxel-pair, antenna-pair and
    scalar mixed kernels produce identical bits (n_ap=7: an odd antenna count, padded
    with a zero antenna by the antenna-pair form)."""
    from mmnorm_b200 import ops
    names = [v["name"] for v in ops.variants("mixed")]
    groups = [("mixed_ffma_t4_n128", "mixed_ffma2_t4_n128", "mixed_antpair_t2_n256",
               "mixed_antpair_t1_n256"),
              ("mixed_ffma2_fx_t2_n256", "mixed_ffma2_fx_t4_n128", "mixed_antpair_fx_t2_n256",
               "mixed_antpair_fx_t1_n256"),
              ("mixed_ffma2_fx2_t2_n256", "mixed_ffma2_fx2_t2_n128_s24", "mixed_antpair_fx2_t2_n256",
               "mixed_antpair_fx2_t1_n256")]
    sc = scenes.sphere_scene(seed=16, n_ap=n_ap, nf=64, n_vox=11, n_pts=20)
    for group in groups:
        out = []
        for name in group:
            ops.set_variant("mixed", names.index(name))
            try:
                out.append(run_ops(cuda_dev, sc, "mixed"))
            finally:
                ops.set_variant("mixed", 0)
        for o in out[1:]:
            assert np.array_equal(out[0][0], o[0])
            assert np.array_equal(out[0][1], o[1])


def test_autotuner_selects_a_variant(cuda_dev):
    import torch
    from mmnorm_b200 import autotune, ops
    sc = scenes.sphere_scene(seed=17, n_ap=16, nf=64, n_vox=16, n_pts=20)
    args = [_t(v, cuda_dev) for v in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs,
                                      np.zeros((1, 3), np.float32), sc.meas)]
    res = autotune.tune(*args, sc.wavelength, sc.slope, mode="mixed", max_antennas=64)
    try:
        assert res["best"] in range(len(ops.variants("mixed")))
        assert len(res["times_ms"]) == len(ops.variants("mixed"))
    finally:
        ops.set_variant("mixed", 0)


def test_autotuner_restricted_to_accurate_forms(cuda_dev):
    from mmnorm_b200 import autotune, ops
    sc = scenes.sphere_scene(seed=18, n_ap=16, nf=64, n_vox=16, n_pts=20)
    args = [_t(v, cuda_dev) for v in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs,
                                      np.zeros((1, 3), np.float32), sc.meas)]
    names = [v["name"] for v in ops.variants("mixed")]
    res = autotune.tune(*args, sc.wavelength, sc.slope, mode="mixed", max_antennas=64,
                        candidates=autotune.ACCURATE_FORMS)
    try:
        timed = {names[int(i)] for i in res["times_ms"]}
        assert timed and all(n.startswith(autotune.ACCURATE_FORMS) for n in timed)
        assert names[res["best"]].startswith(autotune.ACCURATE_FORMS)
        assert ops.current_variant("mixed") == res["best"]
    finally:
        ops.set_variant("mixed", 0)


def test_autotuner_keeps_the_callers_selection_without_apply(cuda_dev):
    """tune(apply=False) times the variants and leaves the caller's selection in place; the
    same call with apply (answered from the cache) selects the winner."""
    from mmnorm_b200 import autotune, ops
    sc = scenes.sphere_scene(seed=19, n_ap=16, nf=96, n_vox=16, n_pts=20)
    args = [_t(v, cuda_dev) for v in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs,
                                      np.zeros((1, 3), np.float32), sc.meas)]
    mine = len(ops.variants("mixed")) - 1
    ops.set_variant("mixed", mine)
    try:
        res = autotune.tune(*args, sc.wavelength, sc.slope, mode="mixed", max_antennas=64,
                            apply=False)
        assert ops.current_variant("mixed") == mine
        again = autotune.tune(*args, sc.wavelength, sc.slope, mode="mixed", max_antennas=64)
        assert again["best"] == res["best"] and ops.current_variant("mixed") == res["best"]
    finally:
        ops.set_variant("mixed", 0)

@pytest.mark.parametrize("idx", list(range(40)))
def test_every_mixed_variant_edge_cases(cuda_dev, oracle, idx):
    """Each mixed variant on F = 1, 33 and 100 (not multiples of the 32-sample block), on
    several RX offsets with the TI offset and a ragged antenna count, and with per-antenna
    position offsets, against the FP64 oracle."""
    from mmnorm_b200 import ops
    n = len(ops.variants("mixed"))
    if idx >= n:
        pytest.skip("no variant %d" % idx)
    rng = np.random.default_rng(30 + idx)
    ops.set_variant("mixed", idx)
    try:
        for nf in (1, 33, 100):
            sc = small_scene(seed=40 + nf, nf=max(nf, 2), n_vox=7)
            meas = sc.meas[:, :nf]
            I, W = run_ops(cuda_dev, sc, "mixed", meas=meas)
            Io, Wo = oracle.full(sc.voxel_centres(), sc.antenna_locs, np.zeros((1, 3)), meas,
                                 sc.wavelength, sc.slope)
            assert oracle.rel_l2(I, Io) < TOL_MIXED, nf
            assert oracle.rel_l2(W, Wo) < TOL_MIXED, nf
        sc = small_scene(seed=5)
        rxo = np.array([[0, -0.005, 0], [0, -0.007, 0.001], [0.002, 0, 0]], np.float32)
        A = sc.antenna_locs.shape[0]
        ant = np.repeat(sc.antenna_locs, 3, axis=0)[: A + 7]
        meas = (rng.standard_normal((ant.shape[0], 40)) +
                1j * rng.standard_normal((ant.shape[0], 40))).astype(np.complex64)
        I, W = run_ops(cuda_dev, sc, "mixed", rxo=rxo, ti=True, meas=meas, ant=ant)
        Io, Wo = oracle.full(sc.voxel_centres(), ant, rxo, meas, sc.wavelength, sc.slope,
                             is_ti=True)
        assert oracle.rel_l2(I, Io) < TOL_MIXED
        assert oracle.rel_l2(W, Wo) < TOL_MIXED
        pos = rng.normal(0, 5e-4, sc.antenna_locs.shape)
        I, W = run_ops(cuda_dev, sc, "mixed", pos=pos)
        moved = (sc.antenna_locs.astype(np.float64) + pos.astype(np.float32)).astype(np.float32)
        Io, Wo = oracle.full(sc.voxel_centres(), moved, np.zeros((1, 3)), sc.meas,
                             sc.wavelength, sc.slope)
        assert oracle.rel_l2(I, Io) < 1e-4
        assert oracle.rel_l2(W, Wo) < 1e-4
    finally:
        ops.set_variant("mixed", 0)


def test_plan_reports_its_launches(cuda_dev):
    """mmn_plan_launches: the default (second-order) form reads 16-byte aligned rows of a
    multiple of 32 samples in place (antenna records + forward kernel), and stages rows of
    any other length (one more launch), plus the split reduction when the plan splits."""
    import torch
    from mmnorm_b200 import ops
    ops.set_variant("mixed", 0)
    for nf, want in ((64, 2), (50, 3)):
        sc = small_scene(seed=70, nf=nf, n_vox=16)
        args = [_t(v, cuda_dev) for v in (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs,
                                          np.zeros((1, 3), np.float32), sc.meas)]
        p = ops.make_problem(*args, sc.wavelength, sc.slope)
        info = ops.plan_info(p, "mixed")
        assert info["launches"] == want + (1 if info["splits"] > 1 else 0), (nf, info)


@pytest.mark.parametrize("idx", [0, 1])
def test_rows_off_a_16_byte_boundary_are_staged(cuda_dev, idx):
    """Sample rows that start 8 bytes past a 16-byte boundary (a view one sample into a
    buffer) cannot be read in place by the bulk copies: the plan stages them (one more
    launch) and the result is bit-identical to the same rows from an aligned buffer."""
    import torch
    from mmnorm_b200 import ops
    ops.set_variant("mixed", idx)
    try:
        sc = small_scene(seed=71, nf=64, n_vox=16)
        A, F = sc.meas.shape
        axes = [_t(v, cuda_dev) for v in (sc.x_locs, sc.y_locs, sc.z_locs)]
        ant, rxo = _t(sc.antenna_locs, cuda_dev), _t(np.zeros((1, 3), np.float32), cuda_dev)
        aligned = _t(sc.meas, cuda_dev)
        buf = torch.zeros(A * F + 1, dtype=torch.complex64, device=cuda_dev)
        buf[1:].copy_(aligned.reshape(-1))
        shifted = buf[1:].view(A, F)
        assert aligned.data_ptr() % 16 == 0 and shifted.data_ptr() % 16 == 8
        plans = [ops.plan_info(ops.make_problem(*axes, ant, rxo, m, sc.wavelength, sc.slope),
                               "mixed") for m in (aligned, shifted)]
        staged = [pl["launches"] - (1 if pl["splits"] > 1 else 0) for pl in plans]
        if ops.variants("mixed")[idx]["name"].startswith("mixed_clen64eo_"):
            assert staged == [2, 3], plans  # the default form reads aligned rows in place
        outs = [ops.backproject(*axes, ant, rxo, m, sc.wavelength, sc.slope, mode="mixed")
                for m in (aligned, shifted)]
        torch.cuda.synchronize()
        assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    finally:
        ops.set_variant("mixed", 0)
