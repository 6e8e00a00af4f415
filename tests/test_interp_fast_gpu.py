"""Fast form of the interpolated mode (MMN_MODE_INTERP_FAST, mmn_cuda_image with
use_interpolated_processing == 2, mmn_cuda_sn_est_fast) against the reference's own
kernels (cuda_image / cuda_sn_est compiled from its sources), against this library's
bit-exact interpolated kernels, and against the FP64 oracle.

The fast form gathers the same range bin as the reference (same FP32 path length, same
floor of the FP32 quotient) and forms the phasor from the wrapped FP32 turn count with the
hardware sine/cosine: about 5e-7 relative per term.  The tolerance is 2e-6 relative L2 on
these small cases, where one pair gathering a neighbouring bin would move the result by
~1e-3; 1e-5 at the full-size workload."""
import ctypes

import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu

TOL = 2e-6
TOL_WORKLOAD = 1e-5

FORMS = ["packed", "scalar"]


@pytest.fixture
def fast_form(request):
    from mmnorm_b200 import ops
    ops.set_interp_fast_form(request.param)
    yield request.param
    ops.set_interp_fast_form("packed")


def _rel(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _setup(dev, nf=64, nb=512, R=1, seed=41, n_vox=10, n_ap=12, ti=True, grid=None):
    import torch
    sc = scenes.sphere_scene(seed=seed, n_ap=n_ap, nf=nf, n_vox=n_vox, n_pts=30, sign=+1)
    if grid is not None:  # a ragged grid around the same centre
        sp = float(sc.x_locs[1] - sc.x_locs[0])
        cx, cy, cz = (float(np.mean(a)) for a in (sc.x_locs, sc.y_locs, sc.z_locs))
        sc.x_locs, sc.y_locs, sc.z_locs = (
            (c + (np.arange(n) - (n - 1) / 2) * sp).astype(np.float32)
            for c, n in zip((cx, cy, cz), grid))
    rng = np.random.default_rng(seed)
    A = sc.antenna_locs.shape[0]
    rxo = np.array([[0, -0.005 - 0.0019 * k, 0] for k in range(R)], np.float32)
    ant = np.repeat(sc.antenna_locs, R, axis=0)
    pad = np.zeros((A * R, nb), np.complex64)
    for k in range(R):
        pad[k::R, :nf] = sc.meas * np.complex64(np.exp(1j * rng.uniform(0, 6.28)))
    fft = np.fft.fft(pad, axis=1).astype(np.complex64)
    fsp = np.float32(3e8 / (2 * (sc.f_hi - sc.f_lo)) * nf / nb)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    return dict(sc=sc, x=t(sc.x_locs), y=t(sc.y_locs), z=t(sc.z_locs), ant=t(ant),
                rxo=t(rxo), fft=t(fft), fft_np=fft, ant_np=ant, rxo_np=rxo, A=A * R, R=R,
                nb=nb, fsp=fsp, ti=int(ti), wl=np.float32(sc.wavelength),
                slope=np.float32(sc.slope))


def _backproject(d, mode):
    import torch
    from mmnorm_b200 import ops
    img, vote = ops.backproject(d["x"], d["y"], d["z"], d["ant"], d["rxo"], d["fft"],
                                float(d["wl"]), float(d["slope"]), mode=mode,
                                fft_spacing=float(d["fsp"]), is_ti_radar=bool(d["ti"]))
    torch.cuda.synchronize()
    return img.cpu().numpy().ravel(), vote.cpu().numpy().reshape(3, -1)


def _cuda_image(d, flag, start=0, count=-1, dev=None):
    """mmn_cuda_image (SoA inputs, reference argument list) with the given interp flag."""
    import torch
    from mmnorm_b200 import _lib, ops
    nx, ny, nz = len(d["sc"].x_locs), len(d["sc"].y_locs), len(d["sc"].z_locs)
    V = nx * ny * nz
    dev = d["x"].device
    out_r = torch.full((V,), 7.0, device=dev)
    out_i = torch.full((V,), 7.0, device=dev)
    mr = d["fft"].real.contiguous().reshape(-1)
    mi = d["fft"].imag.contiguous().reshape(-1)
    ws = torch.empty(256, dtype=torch.uint8, device=dev)
    vp = ops._vp
    rc = _lib.load().mmn_cuda_image(
        vp(out_r), vp(out_i), vp(d["x"]), vp(d["y"]), vp(d["z"]), vp(d["ant"]), vp(mr),
        vp(mi), vp(d["rxo"]), float(d["slope"]), float(d["wl"]), float(d["fsp"]), nx, ny, nz,
        d["A"], d["R"], d["nb"], start, d["ti"], flag, count, vp(ws), 256, ops._stream(dev))
    _lib.check(rc, "mmn_cuda_image")
    torch.cuda.synchronize()
    return out_r.cpu().numpy() + 1j * out_i.cpu().numpy()


@pytest.mark.parametrize("fast_form", FORMS, indirect=True)
@pytest.mark.parametrize("R,ti", [(1, False), (4, True)])
def test_fast_image_vs_reference_kernel(cuda_dev, R, ti, fast_form):
    import torch
    from oracle import ref_cuda
    if not ref_cuda.available():
        pytest.skip("reference cubins not built (python oracle/build.py)")
    d = _setup(cuda_dev, R=R, ti=ti)
    sc = d["sc"]
    nx, ny, nz = sc.grid_shape
    V = nx * ny * nz
    p_r = torch.zeros(V, device=cuda_dev)
    p_i = torch.zeros(V, device=cuda_dev)
    mr = d["fft"].real.contiguous().reshape(-1)
    mi = d["fft"].imag.contiguous().reshape(-1)
    ref_cuda.cuda_image(p_r, p_i, d["x"], d["y"], d["z"], d["ant"].reshape(-1), mr, mi,
                        d["rxo"].reshape(-1), d["slope"], d["wl"], d["fsp"], nx, ny, nz,
                        d["A"], d["R"], d["nb"], d["ti"], 1)
    torch.cuda.synchronize()
    ref = p_r.cpu().numpy() + 1j * p_i.cpu().numpy()
    fast = _cuda_image(d, 2)
    exact = _cuda_image(d, 1)
    np.testing.assert_array_equal(exact, ref)
    assert np.abs(ref).max() > 0
    assert _rel(fast, ref) < TOL


@pytest.mark.parametrize("fast_form", FORMS, indirect=True)
@pytest.mark.parametrize("R", [1, 4])
def test_fast_sn_est_vs_reference_kernel(cuda_dev, R, fast_form):
    import torch
    from mmnorm_b200 import _lib, ops
    from oracle import ref_cuda
    if not ref_cuda.available():
        pytest.skip("reference cubins not built (python oracle/build.py)")
    d = _setup(cuda_dev, R=R)
    sc = d["sc"]
    nx, ny, nz = sc.grid_shape
    img = _cuda_image(d, 1).reshape(sc.grid_shape)
    coords = np.argwhere(np.abs(img) > np.abs(img).max() * 0.05).astype(np.int32)
    nv = coords.shape[0]
    assert nv > 0
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    vx, vy, vz = (t(coords[:, k]) for k in range(3))
    img_r = t(img.real.astype(np.float32).ravel())
    img_i = t(img.imag.astype(np.float32).ravel())
    mr = d["fft"].real.contiguous().reshape(-1)
    mi = d["fft"].imag.contiguous().reshape(-1)
    ant, rxo = d["ant"].reshape(-1), d["rxo"].reshape(-1)
    ref = [torch.zeros(nv, device=cuda_dev) for _ in range(3)]
    ref_cuda.cuda_sn_est(*ref, vx, vy, vz, img_r, img_i, d["x"], d["y"], d["z"], ant, mr, mi,
                         rxo, d["slope"], d["wl"], d["fsp"], nx, ny, nz, d["A"], d["R"], nv,
                         d["nb"], d["ti"])
    fast = [torch.zeros(nv, device=cuda_dev) for _ in range(3)]
    ws = torch.empty(256, dtype=torch.uint8, device=cuda_dev)
    vp = ops._vp
    rc = _lib.load().mmn_cuda_sn_est_fast(
        vp(fast[0]), vp(fast[1]), vp(fast[2]), vp(vx), vp(vy), vp(vz), vp(img_r), vp(img_i),
        vp(d["x"]), vp(d["y"]), vp(d["z"]), vp(ant), vp(mr), vp(mi), vp(rxo),
        float(d["slope"]), float(d["wl"]), float(d["fsp"]), nx, ny, nz, d["A"], d["R"], nv,
        d["nb"], 0, d["ti"], -1, vp(ws), 256, ops._stream(cuda_dev))
    _lib.check(rc, "mmn_cuda_sn_est_fast")
    torch.cuda.synchronize()
    r = np.stack([a.cpu().numpy() for a in ref], 1)
    f = np.stack([a.cpu().numpy() for a in fast], 1)
    assert np.abs(r).max() > 0
    assert _rel(f, r) < TOL


@pytest.mark.parametrize("fast_form", FORMS, indirect=True)
@pytest.mark.parametrize("R,ti,grid,n_ap", [(1, False, None, 12), (2, True, (7, 9, 11), 18),
                                            (1, True, (5, 3, 37), 17)])
def test_fast_native_path_image_and_vote(cuda_dev, oracle, R, ti, grid, n_ap, fast_form):
    """Ragged grids (voxel counts not a multiple of the 512 voxels of a CTA), antenna counts
    across the 256-antenna staging chunk (18^2 * 2 = 648, 17^2 = 289), several RX offsets
    and the TI offset: fused image and vote vs the bit-exact kernel and the FP64 oracle,
    for every form of the fast image pass."""
    d = _setup(cuda_dev, R=R, ti=ti, grid=grid, n_ap=n_ap)
    img_f, vote_f = _backproject(d, "interp_fast")
    img_e, vote_e = _backproject(d, "interp")
    assert _rel(img_f, img_e) < TOL
    assert _rel(vote_f, vote_e) < TOL
    # against the FP64 oracle (the reference's FP32 path, FP64 phasor and sums) the bit-exact
    # form carries the reference's FP32 accumulation error (~4e-5 here); the fast form may
    # add no more than its phasor error to it
    sc = d["sc"]
    Io, Wo = oracle.interp(sc.voxel_centres(), d["ant_np"], d["rxo_np"], d["fft_np"],
                           float(d["wl"]), float(d["fsp"]), is_ti=bool(ti), dist_mode=1,
                           vote=True)
    assert _rel(img_e, Io) < 5e-4
    assert _rel(img_f, Io) < _rel(img_e, Io) + TOL
    assert _rel(vote_f, Wo.T) < _rel(vote_e, Wo.T) + TOL


def test_fast_out_of_range_and_launch_extent(cuda_dev):
    """A range-FFT so short that most (voxel, antenna) pairs fall beyond fft_spacing*bins
    (skipped, as imaging_gpu.cu:92-94 does), and launches over a voxel sub-range
    (start_ind, voxel_count) that leave the rest of the output untouched."""
    d = _setup(cuda_dev, nb=128, nf=64)
    d["fsp"] = np.float32(d["fsp"] * 0.75)  # max range 0.75x: the far pairs drop out
    fast = _cuda_image(d, 2)
    exact = _cuda_image(d, 1)
    assert np.abs(exact).max() > 0
    assert _rel(fast, exact) < TOL
    V = fast.size
    s, n = 123, 517
    part = _cuda_image(d, 2, start=s, count=n)
    np.testing.assert_array_equal(part[s:s + n], fast[s:s + n])
    assert np.all(part[:s] == 7 + 7j) and np.all(part[s + n:] == 7 + 7j)
    assert V > s + n


def test_fast_empty_aperture(cuda_dev):
    import torch
    from mmnorm_b200 import ops
    d = _setup(cuda_dev)
    img, vote = ops.backproject(d["x"], d["y"], d["z"], d["ant"][:0], d["rxo"], d["fft"][:0],
                                float(d["wl"]), float(d["slope"]), mode="interp_fast",
                                fft_spacing=float(d["fsp"]))
    torch.cuda.synchronize()
    assert float(img.abs().max()) == 0 and float(vote.abs().max()) == 0


def test_fast_rejects_too_many_bins(cuda_dev):
    from mmnorm_b200 import _lib, ops
    d = _setup(cuda_dev)
    p = ops.make_problem(d["x"], d["y"], d["z"], d["ant"], d["rxo"], d["fft"], float(d["wl"]),
                         float(d["slope"]), float(d["fsp"]))
    p.num_samples = (1 << 22) + 1
    lib = _lib.load()
    assert lib.mmn_workspace_bytes(ctypes.byref(p), _lib.MODE_INTERP_FAST, 1) == 0


def test_fast_dropin_wrappers(cuda_dev):
    """image_cuda / normal_estimates_cuda with precision='fast' against the same calls
    with the reference's arithmetic (several RX, TI offset)."""
    from mmnorm_b200 import pipeline, py_image_gpu, py_sn_est_gpu
    sc = scenes.sphere_scene(seed=42, n_ap=10, nf=64, n_vox=8, n_pts=25, sign=+1)
    R = 4
    rng = np.random.default_rng(42)
    g = (rng.standard_normal(R) + 1j * rng.standard_normal(R)).astype(np.complex64)
    data = sc.meas[:, :, None] * g[None, None, :]
    pad = np.zeros((data.shape[0], 512, R), np.complex64)
    pad[:, :64, :] = data
    fft = np.fft.fft(pad, axis=1)
    wl = scenes.C / 77e9
    rxo = np.array([[0.0, -0.005 - wl / 2 * (R - 1 - k), 0.0] for k in range(R)])
    args = (sc.x_locs, sc.y_locs, sc.z_locs, sc.antenna_locs.astype(np.float64), fft, rxo,
            sc.slope, sc.wavelength, sc.f_hi - sc.f_lo, 64)
    kw = dict(use_4_rx=True, is_ti_radar=True, use_interpolated_processing=True)
    img_e, c_e = py_image_gpu.image_cuda(*args, **kw)
    img_f, c_f = py_image_gpu.image_cuda(*args, **kw, precision="fast")
    np.testing.assert_array_equal(c_f, c_e)
    assert _rel(img_f, img_e) < TOL
    n_e = py_sn_est_gpu.normal_estimates_cuda(img_e, *args, use_4_rx=True, is_ti_radar=True)
    n_f = py_sn_est_gpu.normal_estimates_cuda(img_e, *args, use_4_rx=True, is_ti_radar=True,
                                              precision="fast")
    np.testing.assert_array_equal(np.isnan(n_f), np.isnan(n_e))
    ok = ~np.isnan(n_e[..., 0])
    assert ok.sum() > 0
    assert _rel(n_f[ok], n_e[ok]) < TOL
    s2, unit, _ = pipeline.surface_normals(*args, use_4_rx=True, is_ti_radar=True,
                                           use_interpolated_processing=True, precision="fast")
    np.testing.assert_array_equal(s2, img_f)
    assert np.all(np.isnan(unit[~ok]))
    np.testing.assert_allclose(np.linalg.norm(unit[ok], axis=-1), 1, rtol=1e-6)


@pytest.mark.parametrize("fast_form", FORMS, indirect=True)
def test_fast_at_the_full_workload(cuda_dev, fast_form):
    """128^3 voxels, 128x128 antennas, a 4096-bin range FFT of the 256-sample workload:
    fast image and vote within 1e-5 of the bit-exact kernel, for every form of the fast
    image pass (a squared range one ulp off the reference's moves the phase by ~1e-4 rad,
    so a form whose FMA contraction order differs from the reference's fails here: the
    order fma(dz, dz, fma(dy, dy, dx*dx)) measured 2.5e-4)."""
    import torch
    from mmnorm_b200 import ops
    sc = scenes.config1(sign=-1, device=cuda_dev)
    A, F = sc.meas.shape
    nb = 4096
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    pad = torch.zeros((A, nb), dtype=torch.complex64, device=cuda_dev)
    pad[:, :F] = t(sc.meas)
    fft = torch.fft.fft(pad, dim=1)
    del pad
    fsp = float(np.float32(3e8 / (2 * (sc.f_hi - sc.f_lo)) * F / nb))
    args = (t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs),
            t(np.zeros((1, 3), np.float32)), fft, sc.wavelength, sc.slope)
    img_f, vote_f = ops.backproject(*args, mode="interp_fast", fft_spacing=fsp)
    img_e, vote_e = ops.backproject(*args, mode="interp", fft_spacing=fsp)
    rel = lambda a, b: float((a.to(torch.complex128) - b.to(torch.complex128)).norm() /
                             b.to(torch.complex128).norm())
    e_img, e_vote = rel(img_f, img_e), rel(vote_f, vote_e)
    print("fast (%s) vs bit-exact at the workload: image %.2e vote %.2e"
          % (fast_form, e_img, e_vote))
    assert e_img < TOL_WORKLOAD and e_vote < TOL_WORKLOAD


def test_fast_form_through_torch_operator(cuda_dev):
    import torch
    import mmnorm_b200.torch_ops  # noqa: F401
    d = _setup(cuda_dev, R=2)
    i0, v0 = _backproject(d, "interp_fast")
    i1, v1 = torch.ops.mmnorm.backproject(d["x"], d["y"], d["z"], d["ant"], d["rxo"], d["fft"],
                                          float(d["wl"]), float(d["slope"]), "interp_fast",
                                          float(d["fsp"]), bool(d["ti"]), None)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(i1.cpu().numpy().ravel(), i0)
    np.testing.assert_array_equal(v1.cpu().numpy().reshape(3, -1), v0)
