"""The C-ABI library loads and exports every entry point include/mmnorm_b200.h declares;
argument validation paths that need no device return the documented codes.  CPU only:
no compute call is made."""
import ctypes
import os
import re

from conftest import ROOT


def _declared():
    txt = open(os.path.join(ROOT, "include", "mmnorm_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mmn_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = _declared()
    for must in ("mmn_backproject", "mmn_normals", "mmn_cuda_image", "mmn_cuda_sn_est",
                 "mmn_workspace_bytes", "mmn_read_status"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from mmnorm_b200 import _lib
    h = _lib.load()
    for name in _declared():
        assert hasattr(h, name), name
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert set(_declared()) <= bound, set(_declared()) - bound


def test_version_and_validation_without_device():
    from mmnorm_b200 import _lib
    h = _lib.load()
    assert h.mmn_version().startswith(b"mmnorm_b200")
    assert h.mmn_backproject(None, 0, None, None, None, 0, None) == _lib.MMN_ERR_NULL_POINTER
    p = _lib.MmnProblem()
    p.num_x = 0
    assert h.mmn_workspace_bytes(ctypes.byref(p), 0, 1) == 0
    p.num_x = p.num_y = p.num_z = 4
    p.num_rx = 1
    p.num_samples = 8
    p.wavelength = 3.9e-3
    assert h.mmn_backproject(ctypes.byref(p), 9, None, None, None, 0, None) == \
        _lib.MMN_ERR_INVALID_ARGUMENT
    assert h.mmn_backproject(ctypes.byref(p), 0, None, None, None, 0, None) == \
        _lib.MMN_ERR_NULL_POINTER
    assert h.mmn_normals(0, None, None, 0.05, None, None, None, None, 0, None) == \
        _lib.MMN_ERR_INVALID_ARGUMENT
    # the no-alloc status accessor checks its output pointer before touching a device
    assert h.mmn_noalloc_read_status(None, None) == _lib.MMN_ERR_NULL_POINTER
    assert h.mmn_set_variant(7, 0) == _lib.MMN_ERR_INVALID_ARGUMENT
    assert h.mmn_get_variant(7) == _lib.MMN_ERR_INVALID_ARGUMENT
    assert h.mmn_plan_launches(ctypes.byref(p), 0, None) == _lib.MMN_ERR_NULL_POINTER
    n = h.mmn_num_variants(_lib.MODE_MIXED)
    assert h.mmn_set_variant(_lib.MODE_MIXED, n - 1) == _lib.MMN_OK
    assert h.mmn_get_variant(_lib.MODE_MIXED) == n - 1
    assert h.mmn_set_variant(_lib.MODE_MIXED, 0) == _lib.MMN_OK
    assert h.mmn_get_variant(_lib.MODE_MIXED) == 0
    assert h.mmn_num_variants(_lib.MODE_MIXED) >= 1
    assert h.mmn_num_variants(_lib.MODE_PLAIN) >= 1



def test_misaligned_arrays_are_refused_without_device():
    """A float array off a 4-byte boundary or a complex64 array off an 8-byte boundary is
    refused with MMN_ERR_INVALID_ARGUMENT before any device call (the kernels load a sample
    as one 8-byte word).  The addresses are never dereferenced."""
    from mmnorm_b200 import _lib
    h = _lib.load()
    INV = _lib.MMN_ERR_INVALID_ARGUMENT

    def problem(**off):
        p = _lib.MmnProblem()
        p.num_x = p.num_y = p.num_z = 4
        p.num_antennas, p.num_rx, p.num_samples = 8, 1, 64
        p.wavelength, p.slope, p.fft_spacing = 3.9e-3, 1.6e7, 2e-3
        base = 1 << 20
        for k, name in enumerate(("x_locs", "y_locs", "z_locs", "antenna_locs",
                                  "rx_offsets", "meas")):
            setattr(p, name, base + (k << 12) + off.get(name, 0))
        return p

    fake = lambda a: ctypes.c_void_p(a)
    img, vote, ws = fake(1 << 24), fake(1 << 25), fake(1 << 26)
    for bad in ({"meas": 4}, {"x_locs": 2}, {"antenna_locs": 1}, {"rx_offsets": 2}):
        p = problem(**bad)
        for mode in (_lib.MODE_MIXED, _lib.MODES["interp"]):
            assert h.mmn_backproject(ctypes.byref(p), mode, img, vote, ws, 1 << 30, None) == INV
            assert h.mmn_workspace_bytes(ctypes.byref(p), mode, 1) == 0
        assert h.mmn_backproject_noalloc(ctypes.byref(p), _lib.MODE_MIXED, img, vote,
                                         None) == INV
        assert h.mmn_backproject_nufft(ctypes.byref(p), img, vote, ws, 1 << 30, None) == INV
        n = ctypes.c_int32(-1)
        assert h.mmn_plan_launches(ctypes.byref(p), _lib.MODE_MIXED, ctypes.byref(n)) == INV
    p = problem()
    p.pos_offsets = (1 << 21) + 2
    assert h.mmn_backproject(ctypes.byref(p), _lib.MODE_MIXED, img, vote, ws, 1 << 30,
                             None) == INV
    p = problem()  # every input aligned: the outputs are checked next
    assert h.mmn_backproject(ctypes.byref(p), _lib.MODE_MIXED, fake((1 << 24) + 4), vote, ws,
                             1 << 30, None) == INV
    assert h.mmn_backproject(ctypes.byref(p), _lib.MODE_MIXED, img, fake((1 << 25) + 4), ws,
                             1 << 30, None) == INV
    assert h.mmn_backproject_noalloc(ctypes.byref(p), _lib.MODE_MIXED, fake((1 << 24) + 4),
                                     vote, None) == INV
    assert h.mmn_backproject_backward(ctypes.byref(p), fake((1 << 24) + 4), None,
                                      fake(1 << 27), None, ws, 1 << 30, None) == INV
    assert h.mmn_backproject_backward(ctypes.byref(p), img, None, fake((1 << 27) + 4), None,
                                      ws, 1 << 30, None) == INV
    assert h.mmn_image_max_abs(64, fake((1 << 24) + 4), fake(1 << 27), None) == INV
    assert h.mmn_normals(64, img, fake((1 << 25) + 4), 0.05, fake(1 << 27), None, None, ws,
                         1 << 20, None) == INV
    # the reference-signature kernels' float and int arrays: 4-byte words
    arr = [fake((1 << 20) + (k << 12)) for k in range(16)]
    odd = fake((1 << 28) + 2)
    for slot in (0, 6, 8):  # p_xyz_r, meas_r, rx_offsets
        a = list(arr[:9])
        a[slot] = odd
        assert h.mmn_cuda_image(*a, 1.6e7, 3.9e-3, 2e-3, 4, 4, 4, 8, 1, 64, 0, 0, 1, -1, ws,
                                1 << 20, None) == INV
    for slot in (0, 3, 11):  # normals_x, valid_idx_x, antenna_locs
        a = list(arr[:15])
        a[slot] = odd
        assert h.mmn_cuda_sn_est(*a, 1.6e7, 3.9e-3, 2e-3, 4, 4, 4, 8, 1, 10, 64, 0, 0, -1,
                                 ws, 1 << 20, None) == INV


def test_interpolation_form_and_probe_validation_without_device():
    """Argument checks of the interpolation-form entry points, the pass selectors and the
    wait probe, all answered before any device call."""
    from mmnorm_b200 import _lib
    h = _lib.load()
    assert h.mmn_set_position_pass(2) == _lib.MMN_ERR_INVALID_ARGUMENT
    assert h.mmn_set_measurement_pass(-1) == _lib.MMN_ERR_INVALID_ARGUMENT
    assert h.mmn_set_position_pass(0) == _lib.MMN_OK  # the defaults, set again
    assert h.mmn_set_measurement_pass(0) == _lib.MMN_OK
    n = h.mmn_num_position_variants()
    assert n >= 2
    assert h.mmn_set_position_variant(n - 1) == _lib.MMN_OK
    assert h.mmn_get_position_variant() == n - 1
    assert h.mmn_set_position_variant(0) == _lib.MMN_OK
    assert h.mmn_get_position_variant() == 0
    assert h.mmn_position_variant_name(0).startswith(b"interp_")
    assert h.mmn_position_variant_name(n) is None
    assert h.mmn_set_position_variant(n) == _lib.MMN_ERR_INVALID_ARGUMENT
    assert h.mmn_backproject_nufft(None, None, None, None, 0, None) == _lib.MMN_ERR_NULL_POINTER
    assert h.mmn_backproject_nufft_workspace_bytes(None) == 0
    p = _lib.MmnProblem()
    p.num_x = p.num_y = p.num_z = 4
    p.num_rx = 1
    p.num_samples = 8
    p.wavelength = 3.9e-3
    assert h.mmn_backproject_nufft(ctypes.byref(p), None, None, None, 0, None) == \
        _lib.MMN_ERR_NULL_POINTER  # no grid axes
    assert h.mmn_wait_timeout_probe(100, 0, None, None) == _lib.MMN_ERR_NULL_POINTER
    dummy = ctypes.c_void_p(256)  # never dereferenced: the limit check comes first
    assert h.mmn_wait_timeout_probe(20000000, 0, dummy, None) == \
        _lib.MMN_ERR_INVALID_ARGUMENT


def test_interpolated_fast_form_validation_without_device():
    """The fast interpolated form's selector and entry points check their arguments before
    any device call: bad form, bad mode, missing fft_spacing, too many bins, null output."""
    from mmnorm_b200 import _lib
    h = _lib.load()
    assert h.mmn_set_interp_fast_form(2) == _lib.MMN_ERR_INVALID_ARGUMENT
    assert h.mmn_set_interp_fast_form(-1) == _lib.MMN_ERR_INVALID_ARGUMENT
    assert h.mmn_set_interp_fast_form(1) == _lib.MMN_OK
    assert h.mmn_set_interp_fast_form(0) == _lib.MMN_OK  # the default, set again
    p = _lib.MmnProblem()
    p.num_x = p.num_y = p.num_z = 4
    p.num_rx = 1
    p.num_samples = 4096
    p.wavelength = 3.9e-3
    dummy = ctypes.c_void_p(256)
    p.x_locs = p.y_locs = p.z_locs = dummy
    # interpolated modes need a positive fft_spacing
    assert h.mmn_workspace_bytes(ctypes.byref(p), _lib.MODE_INTERP_FAST, 1) == 0
    p.fft_spacing = 2.3e-3
    assert h.mmn_workspace_bytes(ctypes.byref(p), _lib.MODE_INTERP_FAST, 1) == 256
    p.num_samples = (1 << 22) + 1  # beyond the fast form's rounding-constant bins
    assert h.mmn_workspace_bytes(ctypes.byref(p), _lib.MODE_INTERP_FAST, 1) == 0
    assert h.mmn_backproject(ctypes.byref(p), _lib.MODE_INTERP_FAST, None, None, None, 0,
                             None) == _lib.MMN_ERR_TOO_LARGE
    assert h.mmn_backproject(ctypes.byref(p), 4, None, None, None, 0, None) == \
        _lib.MMN_ERR_INVALID_ARGUMENT
    args = [None] * 15 + [0.0, 3.9e-3, 2.3e-3, 4, 4, 4, 16, 1, 8, 64, 0, 0, -1, None, 0, None]
    assert h.mmn_cuda_sn_est_fast(*args) == _lib.MMN_ERR_NULL_POINTER


def test_library_is_sm100a_only_build():
    """The build recipe targets exactly sm_100a."""
    from mmnorm_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_autotuner_refuses_candidates_that_match_no_variant():
    """Checked before any device work, so CPU tensors suffice."""
    import pytest
    import torch
    from mmnorm_b200 import autotune
    z = torch.zeros(4)
    with pytest.raises(ValueError):
        autotune.tune(z, z, z, torch.zeros(2, 3), torch.zeros(1, 3),
                      torch.zeros(2, 8, dtype=torch.complex64), 3.9e-3, 1.6e7,
                      candidates=("no_such_form_",))
