"""Against the reference's OWN CUDA kernels (cuda_image, cuda_sn_est), compiled from its
sources for sm_100a (oracle/build.py) and launched with the reference's argument list and
launch shape (oracle/ref_cuda.py).

Interpolated mode keeps the reference's arithmetic expression for expression, so the
image and the normal vote must match BIT FOR BIT.  The full matched filter differs by
design (FP64 range here, FP32 range in the reference), so it is compared with a
tolerance and both are measured against the FP64 oracle."""
import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_cuda():
    from oracle import ref_cuda as R
    if not R.available():
        pytest.skip("reference cubins not built (python oracle/build.py)")
    return R


def _setup(dev, nf=64, nb=512, R=1, seed=21, n_vox=10, n_ap=12, ti=True):
    import torch
    sc = scenes.sphere_scene(seed=seed, n_ap=n_ap, nf=nf, n_vox=n_vox, n_pts=30, sign=+1)
    rng = np.random.default_rng(seed)
    A = sc.antenna_locs.shape[0]
    rxo = np.array([[0, -0.005 - 0.0019 * k, 0] for k in range(R)], np.float32)
    ant = np.repeat(sc.antenna_locs, R, axis=0)
    pad = np.zeros((A * R, nb), np.complex64)
    for k in range(R):
        pad[k::R, :nf] = sc.meas * np.complex64(np.exp(1j * rng.uniform(0, 6.28)))
    fft = np.fft.fft(pad, axis=1).astype(np.complex64)
    fsp = np.float32(3e8 / (2 * (sc.f_hi - sc.f_lo)) * nf / nb)
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), device=dev, dtype=dt)
    d = dict(sc=sc, x=t(sc.x_locs), y=t(sc.y_locs), z=t(sc.z_locs), ant=t(ant.reshape(-1)),
             rxo=t(rxo.reshape(-1)), mr=t(fft.real.reshape(-1)), mi=t(fft.imag.reshape(-1)),
             fft=fft, ant_np=ant, rxo_np=rxo, A=A * R, R=R, nb=nb, fsp=fsp, ti=int(ti),
             wl=np.float32(sc.wavelength), slope=np.float32(sc.slope))
    return d


def _mmn_cuda_image(d, interp, dev):
    import torch
    from mmnorm_b200 import _lib, ops
    sc = d["sc"]
    nx, ny, nz = sc.grid_shape
    V = nx * ny * nz
    out_r = torch.zeros(V, device=dev)
    out_i = torch.zeros(V, device=dev)
    S = d["nb"] if interp else d["S"]
    lib = _lib.load()
    ws_n = lib.mmn_cuda_image_workspace_bytes_for(nx, ny, nz, d["A"], S, 0, -1, int(interp))
    ws = torch.empty(max(ws_n, 256), dtype=torch.uint8, device=dev)
    vp = ops._vp
    rc = lib.mmn_cuda_image(vp(out_r), vp(out_i), vp(d["x"]), vp(d["y"]), vp(d["z"]),
                            vp(d["ant"]), vp(d["mr"]), vp(d["mi"]), vp(d["rxo"]),
                            float(d["slope"]), float(d["wl"]), float(d["fsp"]), nx, ny, nz,
                            d["A"], d["R"], S, 0, d["ti"], int(interp), -1, vp(ws),
                            ws.numel(), ops._stream(dev))
    _lib.check(rc, "mmn_cuda_image")
    torch.cuda.synchronize()
    return out_r.cpu().numpy(), out_i.cpu().numpy()


def _ref_cuda_image(ref_cuda, d, interp, dev):
    import torch
    sc = d["sc"]
    nx, ny, nz = sc.grid_shape
    V = nx * ny * nz
    p_r = torch.zeros(V, device=dev)
    p_i = torch.zeros(V, device=dev)
    S = d["nb"] if interp else d["S"]
    ref_cuda.cuda_image(p_r, p_i, d["x"], d["y"], d["z"], d["ant"], d["mr"], d["mi"], d["rxo"],
                        d["slope"], d["wl"], d["fsp"], nx, ny, nz, d["A"], d["R"], S, d["ti"],
                        int(interp))
    torch.cuda.synchronize()
    return p_r.cpu().numpy(), p_i.cpu().numpy()


@pytest.mark.parametrize("R", [1, 4])
def test_interp_image_bit_exact_vs_reference_kernel(cuda_dev, ref_cuda, R):
    d = _setup(cuda_dev, R=R)
    ours = _mmn_cuda_image(d, True, cuda_dev)
    ref = _ref_cuda_image(ref_cuda, d, True, cuda_dev)
    assert np.abs(ref[0]).max() > 0
    np.testing.assert_array_equal(ours[0], ref[0])
    np.testing.assert_array_equal(ours[1], ref[1])


def test_native_interp_path_bit_exact_vs_reference_kernel(cuda_dev, ref_cuda):
    import torch
    from mmnorm_b200 import ops
    d = _setup(cuda_dev, R=2)
    ref = _ref_cuda_image(ref_cuda, d, True, cuda_dev)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    img, _ = ops.backproject(d["x"], d["y"], d["z"], t(d["ant_np"]), t(d["rxo_np"]),
                             t(d["fft"]), float(d["wl"]), float(d["slope"]), mode="interp",
                             fft_spacing=float(d["fsp"]), is_ti_radar=bool(d["ti"]))
    img = img.cpu().numpy().ravel()
    np.testing.assert_array_equal(img.real, ref[0])
    np.testing.assert_array_equal(img.imag, ref[1])


@pytest.mark.parametrize("R", [1, 4])
def test_sn_est_bit_exact_vs_reference_kernel(cuda_dev, ref_cuda, R):
    import torch
    from mmnorm_b200 import _lib, ops
    d = _setup(cuda_dev, R=R)
    sc = d["sc"]
    nx, ny, nz = sc.grid_shape
    pr, pi = _ref_cuda_image(ref_cuda, d, True, cuda_dev)
    img = (pr + 1j * pi).reshape(sc.grid_shape)
    filt = np.abs(img) > np.abs(img).max() * 0.05
    coords = np.argwhere(filt).astype(np.int32)
    nv = coords.shape[0]
    assert nv > 0
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev,
                                                   dtype=dt)
    vx, vy, vz = (t(coords[:, k], torch.int32) for k in range(3))
    img_r, img_i = t(pr), t(pi)
    outs = []
    for which in ("ref", "ours"):
        n = [torch.zeros(nv, device=cuda_dev) for _ in range(3)]
        if which == "ref":
            ref_cuda.cuda_sn_est(*n, vx, vy, vz, img_r, img_i, d["x"], d["y"], d["z"], d["ant"],
                                 d["mr"], d["mi"], d["rxo"], d["slope"], d["wl"], d["fsp"], nx,
                                 ny, nz, d["A"], d["R"], nv, d["nb"], d["ti"])
        else:
            vp = ops._vp
            ws = torch.empty(256, dtype=torch.uint8, device=cuda_dev)
            rc = _lib.load().mmn_cuda_sn_est(
                vp(n[0]), vp(n[1]), vp(n[2]), vp(vx), vp(vy), vp(vz), vp(img_r), vp(img_i),
                vp(d["x"]), vp(d["y"]), vp(d["z"]), vp(d["ant"]), vp(d["mr"]), vp(d["mi"]),
                vp(d["rxo"]), float(d["slope"]), float(d["wl"]), float(d["fsp"]), nx, ny, nz,
                d["A"], d["R"], nv, d["nb"], 0, d["ti"], -1, vp(ws), 256,
                ops._stream(cuda_dev))
            _lib.check(rc, "mmn_cuda_sn_est")
        torch.cuda.synchronize()
        outs.append([a.cpu().numpy() for a in n])
    for k in range(3):
        np.testing.assert_array_equal(outs[1][k], outs[0][k])


def test_full_mode_vs_reference_kernel(cuda_dev, ref_cuda, oracle):
    """Full matched filter: the reference kernel (FP32 range, FP64 phase and sin/cos) and
    the mixed kernel (FP64 range and wrap, FP32 recurrence) agree; against the FP64
    oracle the mixed kernel is the more accurate of the two."""
    import torch
    d = _setup(cuda_dev, nf=64, R=1, ti=False)
    sc = d["sc"]
    d["S"] = 64
    m = sc.meas
    d["mr"] = torch.as_tensor(np.ascontiguousarray(m.real.reshape(-1)), device=cuda_dev)
    d["mi"] = torch.as_tensor(np.ascontiguousarray(m.imag.reshape(-1)), device=cuda_dev)
    d["A"] = m.shape[0]
    d["ant"] = torch.as_tensor(sc.antenna_locs.reshape(-1), device=cuda_dev)
    ref = _ref_cuda_image(ref_cuda, d, False, cuda_dev)
    ours = _mmn_cuda_image(d, False, cuda_dev)
    ref_c = ref[0] + 1j * ref[1]
    ours_c = ours[0] + 1j * ours[1]
    Io, _ = oracle.full(sc.voxel_centres(), sc.antenna_locs, d["rxo_np"], m,
                        float(d["wl"]), float(d["slope"]), vote=False)
    e_ours = oracle.rel_l2(ours_c, Io)
    e_ref = oracle.rel_l2(ref_c, Io)
    assert e_ours < 2e-5
    assert e_ref < 5e-4
    assert oracle.rel_l2(ours_c, ref_c) < e_ref + 2e-5
