"""mmn_backproject_noalloc: the backprojection entry point for callers that cannot
allocate device memory where they image (hosts that own the whole device pool and forbid
allocation after start-up, plugin hosts that pass only raw device pointers, real-time
loops that must not block on the allocator).  It must give the same image and vote as
mmn_backproject, call after call, report a clean status word after a normal call, and
refuse problems whose scratch would not fit its built-in 16 MiB array.

This file is collected last on purpose: the entry point's first call on a device
performs its one-time set-up, and the test must pass both in a fresh process and after
every other test has run."""
import ctypes

import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu

TOL = 2e-5  # the mixed form's tolerance used throughout the forward tests


def _tensors(dev, sc, meas=None, ant=None):
    import torch
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    meas = sc.meas if meas is None else meas
    ant = sc.antenna_locs if ant is None else ant
    return [t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(ant),
            t(np.zeros((1, 3), np.float32)), t(meas)]


def _noalloc(args, sc, mode, dev):
    import torch
    from mmnorm_b200 import _lib, ops
    p = ops.make_problem(*args, sc.wavelength, sc.slope, fft_spacing=getattr(sc, "fsp", 0.0))
    V = p.num_x * p.num_y * p.num_z
    image = torch.empty(V, dtype=torch.complex64, device=dev)
    vote = torch.empty((3, V), dtype=torch.complex64, device=dev)
    rc = _lib.load().mmn_backproject_noalloc(ctypes.byref(p), _lib.MODES[mode], ops._vp(image),
                                             ops._vp(vote), ops._stream(dev))
    return rc, image, vote


def _rel(a, b):
    a = a.cpu().numpy().ravel()
    b = b.cpu().numpy().ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("mode", ["mixed", "plain"])
def test_noalloc_matches_backproject_twice(cuda_dev, mode):
    import torch
    from mmnorm_b200 import _lib, ops
    sc = scenes.config0()  # 32x32 aperture, 64 frequencies, 48^3 voxels
    args = _tensors(cuda_dev, sc)
    ref_img, ref_vote = ops.backproject(*args, sc.wavelength, sc.slope, mode=mode)
    firsts = None
    for call in range(2):
        rc, img, vote = _noalloc(args, sc, mode, cuda_dev)
        assert rc == _lib.MMN_OK
        torch.cuda.synchronize()
        assert _rel(img, ref_img) < TOL, call
        assert _rel(vote, ref_vote) < TOL, call
        if firsts is None:
            firsts = (img.clone(), vote.clone())
        else:  # the shared scratch keeps no state that changes a later call's result
            assert torch.equal(img, firsts[0]) and torch.equal(vote, firsts[1])


def test_noalloc_interpolated_mode(cuda_dev):
    import torch
    from mmnorm_b200 import _lib, ops
    sc = scenes.sphere_scene(seed=31, n_ap=12, nf=64, n_vox=10, n_pts=30, sign=+1)
    pad = np.zeros((sc.meas.shape[0], 512), np.complex64)
    pad[:, :64] = sc.meas
    fft = np.fft.fft(pad, axis=1).astype(np.complex64)
    sc.fsp = float(np.float32(3e8 / (2 * (sc.f_hi - sc.f_lo)) * 64 / 512))
    args = _tensors(cuda_dev, sc, meas=fft)
    ref_img, ref_vote = ops.backproject(*args, sc.wavelength, sc.slope, mode="interp",
                                        fft_spacing=sc.fsp)
    for _ in range(2):
        rc, img, vote = _noalloc(args, sc, "interp", cuda_dev)
        assert rc == _lib.MMN_OK
        torch.cuda.synchronize()
        assert torch.equal(img, ref_img.reshape(-1))
        assert torch.equal(vote, ref_vote.reshape(3, -1))


def test_noalloc_rejects_problems_beyond_its_scratch(cuda_dev):
    from mmnorm_b200 import _lib
    sc = scenes.sphere_scene(seed=32, n_ap=4, nf=16, n_vox=4, n_pts=5)
    # 250 samples are not a whole number of blocks, so every kernel form stages padded
    # rows: at least 16384 x 256 x 8 bytes = 32 MiB > 16 MiB
    A, F = 16384, 250
    meas = np.zeros((A, F), np.complex64)
    ant = np.zeros((A, 3), np.float32)
    ant[:, 2] = -0.1
    args = _tensors(cuda_dev, sc, meas=meas, ant=ant)
    rc, _, _ = _noalloc(args, sc, "mixed", cuda_dev)
    assert rc == _lib.MMN_ERR_TOO_LARGE


def test_noalloc_status_word_reads_ok_after_a_call(cuda_dev):
    import torch
    from mmnorm_b200 import _lib, ops
    sc = scenes.sphere_scene(seed=33, n_ap=8, nf=32, n_vox=8, n_pts=20)
    args = _tensors(cuda_dev, sc)
    rc, _, _ = _noalloc(args, sc, "mixed", cuda_dev)
    assert rc == _lib.MMN_OK
    status = ctypes.c_int32(-1)
    assert _lib.load().mmn_noalloc_read_status(ctypes.byref(status),
                                               ops._stream(cuda_dev)) == _lib.MMN_OK
    assert status.value == _lib.MMN_OK
    torch.cuda.synchronize()


def test_noalloc_just_under_its_scratch_limit(cuda_dev):
    """The default kernel form stages (re, im) rows padded to 32 samples when the sample
    count is not a multiple of 32: 7940 antennas x 250 samples take 256 + 64*7940 +
    8*7940*256 = 16,769,536 of the array's 16,777,216 bytes."""
    import torch
    from mmnorm_b200 import _lib, ops
    ops.set_variant("mixed", 0)  # the default form, whose scratch the sizes above assume
    sc = scenes.sphere_scene(seed=34, n_ap=4, nf=250, n_vox=8, n_pts=20)
    A, F = 7940, 250
    rng = np.random.default_rng(34)
    meas = (rng.standard_normal((A, F)) + 1j * rng.standard_normal((A, F))).astype(np.complex64)
    g = np.arange(A)
    ant = np.stack([(g % 80 - 40) * 2e-3, (g // 80 - 50) * 2e-3, np.zeros(A)], 1)
    args = _tensors(cuda_dev, sc, meas=meas, ant=ant.astype(np.float32))
    ref_img, ref_vote = ops.backproject(*args, sc.wavelength, sc.slope, mode="mixed")
    for _ in range(2):
        rc, img, vote = _noalloc(args, sc, "mixed", cuda_dev)
        assert rc == _lib.MMN_OK
        torch.cuda.synchronize()
        assert _rel(img, ref_img) < TOL
        assert _rel(vote, ref_vote) < TOL


def test_noalloc_records_into_a_cuda_graph(cuda_dev):
    """The advertised real-time use: one warm call, then the call recorded into a CUDA graph
    and replayed.  Each replay reads the inputs as they are at replay time and gives the
    direct call's result bit for bit."""
    import torch
    from mmnorm_b200 import _lib, ops
    sc = scenes.sphere_scene(seed=35, n_ap=16, nf=64, n_vox=12, n_pts=30)
    args = _tensors(cuda_dev, sc)
    lib = _lib.load()
    p = ops.make_problem(*args, sc.wavelength, sc.slope)
    V = p.num_x * p.num_y * p.num_z
    image = torch.empty(V, dtype=torch.complex64, device=cuda_dev)
    vote = torch.empty((3, V), dtype=torch.complex64, device=cuda_dev)

    def call():
        return lib.mmn_backproject_noalloc(ctypes.byref(p), _lib.MODES["mixed"], ops._vp(image),
                                           ops._vp(vote), ops._stream(cuda_dev))

    assert call() == _lib.MMN_OK  # warm: the context's scratch address is looked up here
    torch.cuda.synchronize()
    direct = (image.clone(), vote.clone())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        rc = call()
    assert rc == _lib.MMN_OK
    image.zero_()
    vote.zero_()
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(image, direct[0]) and torch.equal(vote, direct[1])

    rng = np.random.default_rng(35)
    new = (rng.standard_normal(sc.meas.shape)
           + 1j * rng.standard_normal(sc.meas.shape)).astype(np.complex64)
    args[5].copy_(torch.as_tensor(new, device=cuda_dev))
    graph.replay()
    torch.cuda.synchronize()
    replayed = (image.clone(), vote.clone())
    assert call() == _lib.MMN_OK
    torch.cuda.synchronize()
    assert torch.equal(replayed[0], image) and torch.equal(replayed[1], vote)
    assert not torch.equal(replayed[0], direct[0])
    status = ctypes.c_int32(-1)
    assert lib.mmn_noalloc_read_status(ctypes.byref(status), ops._stream(cuda_dev)) == _lib.MMN_OK
    assert status.value == _lib.MMN_OK
    del graph
