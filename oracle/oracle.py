"""CPU oracle for mmNorm's backprojection + normal vote.  TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` import this module, and only as the checker (or as the timed CPU
baseline).  The product package never imports it.

Layers:
  * ctypes bindings to the FP64 C restatement (``bp_oracle.c``);
  * a pure-numpy FP64 restatement of the same formulas for tiny cases (used to
    cross-check the C code);
  * a restatement of the reference's host-side wrapper semantics
    (src/data_processing/cuda/py_image_gpu.py:237-366 and
    src/data_processing/cuda/py_sn_est_gpu.py:267-424): input re-layout for several
    RX antennas, the /A and /A^2 normalisations, the interpolated-mode chunking into
    groups of at most 4096*32 virtual antennas, the 5 %-of-max voxel mask, the NaN
    scatter, and the virtual phase centres.

Parity status: pinned.  The C restatement is checked against the reference's own
C++ imager (compiled from src/data_processing/cpp/imaging.cpp by oracle/build.py, run
by oracle/ref_imager.py) through the committed fixtures in tests/golden/, and on the
GPU against the reference's own CUDA kernels (oracle/ref_cuda.py).
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
C = 2.99792458e8

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "_build", "libbp_oracle.so")
        if not os.path.exists(path):
            from oracle import build as _b  # noqa: WPS433
            _b.build_oracle()
        L = ctypes.CDLL(path)
        f32 = ctypes.POINTER(ctypes.c_float)
        f64 = ctypes.POINTER(ctypes.c_double)
        i64, i32, d = ctypes.c_int64, ctypes.c_int32, ctypes.c_double
        L.orc_full.argtypes = [i64, f32, f32, f32, i64, i32, f32, f32, i32, f32, d, d,
                               i32, i32, f64, f64]
        L.orc_interp.argtypes = [i64, f32, f32, f32, i64, i32, f32, f32, i32, f32, d, d,
                                 i32, i32, f64, f64]
        L.orc_sn_interp.argtypes = [i64, f32, f32, f32, f32, f32, i64, i32, f32, f32,
                                    i32, f32, d, d, i32, i32, f64]
        L.orc_full_backward.argtypes = [i64, f32, f32, f32, i64, i32, f32, f32, i32, f32,
                                        d, d, i32, f64, f64, f64, f64]
        for fn in (L.orc_full, L.orc_interp, L.orc_sn_interp, L.orc_full_backward):
            fn.restype = None
        _lib = L
    return _lib


def _f32(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _cplx_f32(m):
    m = np.ascontiguousarray(np.asarray(m).astype(np.complex64))
    return m, m.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _vox(vox):
    vox = np.asarray(vox, dtype=np.float32)
    x, px = _f32(vox[:, 0])
    y, py = _f32(vox[:, 1])
    z, pz = _f32(vox[:, 2])
    return (x, y, z), (px, py, pz)


# --------------------------------------------------------------------------- kernels
def full(vox, ant, rx_offsets, meas, wavelength, slope, is_ti=False, phase_mode=0,
         vote=True):
    """FP64 full matched-filter image (complex128 [nv]) and vote (complex128 [nv,3])."""
    keep, (px, py, pz) = _vox(vox)
    nv = keep[0].shape[0]
    a, pa = _f32(ant)
    o, po = _f32(np.asarray(rx_offsets).reshape(-1, 3))
    m, pm = _cplx_f32(meas)
    na, ns = m.shape
    img = np.zeros((nv, 2))
    _, pimg = _f64(img)
    w = np.zeros((nv, 6)) if vote else None
    pw = w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if vote else None
    lib().orc_full(nv, px, py, pz, na, o.shape[0], pa, po, ns, pm, float(wavelength),
                   float(slope), int(bool(is_ti)), int(phase_mode), pimg, pw)
    I = img[:, 0] + 1j * img[:, 1]
    if not vote:
        return I, None
    return I, w[:, 0::2] + 1j * w[:, 1::2]


def interp(vox, ant, rx_offsets, meas_fft, wavelength, fft_spacing, is_ti=False,
           dist_mode=0, vote=False):
    """Interpolated-mode image (complex128 [nv]) and optional fused vote."""
    keep, (px, py, pz) = _vox(vox)
    nv = keep[0].shape[0]
    a, pa = _f32(ant)
    o, po = _f32(np.asarray(rx_offsets).reshape(-1, 3))
    m, pm = _cplx_f32(meas_fft)
    na, nb = m.shape
    img = np.zeros((nv, 2))
    _, pimg = _f64(img)
    w = np.zeros((nv, 6)) if vote else None
    pw = w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if vote else None
    lib().orc_interp(nv, px, py, pz, na, o.shape[0], pa, po, nb, pm, float(wavelength),
                     float(fft_spacing), int(bool(is_ti)), int(dist_mode), pimg, pw)
    I = img[:, 0] + 1j * img[:, 1]
    return (I, (w[:, 0::2] + 1j * w[:, 1::2]) if vote else None)


def sn_interp(vox, image_vals, ant, rx_offsets, meas_fft, wavelength, fft_spacing,
              is_ti=False, dist_mode=0):
    """Reference normal vote (un-normalised) for listed voxels, float64 [nv, 3]."""
    keep, (px, py, pz) = _vox(vox)
    nv = keep[0].shape[0]
    ir, pir = _f32(np.real(image_vals))
    ii, pii = _f32(np.imag(image_vals))
    a, pa = _f32(ant)
    o, po = _f32(np.asarray(rx_offsets).reshape(-1, 3))
    m, pm = _cplx_f32(meas_fft)
    na, nb = m.shape
    out = np.zeros((nv, 3))
    _, pout = _f64(out)
    lib().orc_sn_interp(nv, px, py, pz, pir, pii, na, o.shape[0], pa, po, nb, pm,
                        float(wavelength), float(fft_spacing), int(bool(is_ti)),
                        int(dist_mode), pout)
    return out


def full_backward(vox, ant, rx_offsets, meas, wavelength, slope, gI, gW, is_ti=False):
    """Adjoint of ``full``: (grad_meas complex128 [na, ns], grad_pos float64 [na, 3])."""
    keep, (px, py, pz) = _vox(vox)
    nv = keep[0].shape[0]
    a, pa = _f32(ant)
    o, po = _f32(np.asarray(rx_offsets).reshape(-1, 3))
    m, pm = _cplx_f32(meas)
    na, ns = m.shape
    gi = np.stack([np.real(gI), np.imag(gI)], axis=1)
    gw = np.stack([np.real(gW), np.imag(gW)], axis=2).reshape(nv, 6)
    gi, pgi = _f64(gi)
    gw, pgw = _f64(gw)
    gm = np.zeros((na, ns, 2))
    _, pgm = _f64(gm)
    gp = np.zeros((na, 3))
    _, pgp = _f64(gp)
    lib().orc_full_backward(nv, px, py, pz, na, o.shape[0], pa, po, ns, pm,
                            float(wavelength), float(slope), int(bool(is_ti)), pgi, pgw,
                            pgm, pgp)
    return gm[..., 0] + 1j * gm[..., 1], gp


# ----------------------------------------------------------- numpy restatement (tiny)
def full_np(vox, ant, rx_offsets, meas, wavelength, slope, is_ti=False, precision="f64"):
    """Pure-numpy full matched-filter image and vote; O(nv*na*ns) memory-light.
    precision "f64" (default): every step in FP64 on float32-rounded inputs; "f32": the
    same formula with every array in float32 / complex64 (range, phase, exponential and
    sums), the straightforward single-precision CPU version."""
    fdt, cdt = (np.float64, np.complex128) if precision == "f64" else (np.float32, np.complex64)
    vox = np.asarray(vox, dtype=np.float32).astype(fdt)
    ant = np.asarray(ant, dtype=np.float32).astype(fdt)
    rxo = np.asarray(rx_offsets, dtype=np.float32).reshape(-1, 3).astype(fdt)
    meas = np.asarray(meas).astype(np.complex64).astype(cdt)
    na, ns = meas.shape
    o = rxo[np.arange(na) % rxo.shape[0]]
    k = (2 * math.pi * (1.0 / wavelength + np.arange(ns) * slope / C)).astype(fdt)
    diff = vox[:, None, :] - ant[None, :, :]                                # [nv, na, 3]
    d = np.linalg.norm(diff, axis=2) + np.linalg.norm(diff - o[None], axis=2)
    if is_ti:
        d = d + fdt(0.15)
    c = np.einsum("vaf,af->va", np.exp(cdt(-1j) * (d[:, :, None] * k[None, None, :])), meas)
    u = (ant + o / 2)[None, :, :] - vox[:, None, :]
    return c.sum(axis=1), np.einsum("va,vak->vk", c, u)


# ------------------------------------------------------------- epilogue restatement
def normals_from_vote(img, vote, filter_percent=0.05):
    """Unit normals (float64 [nv,3], NaN outside the mask) and the mask.

    mask: |I| > filter_percent * max|I|  (src/data_processing/cuda/py_sn_est_gpu.py:326)
    raw normal: Re(conj(I) * W) / |I|    (surface_normal_est.cu:138-144, summed form)
    unit: n / |n|                        (src/data_processing/image_processor.py:396)
    """
    mag = np.abs(img)
    mask = mag > mag.max() * filter_percent
    raw = np.real(np.conj(img)[:, None] * vote) / np.where(mag > 0, mag, 1)[:, None]
    unit = raw / np.linalg.norm(raw, axis=1, keepdims=True)
    unit[~mask] = np.nan
    return unit, mask, raw


def angle_deg(a, b):
    """Angle in degrees between rows of a and b (unit or not)."""
    a = a / np.linalg.norm(a, axis=1, keepdims=True)
    b = b / np.linalg.norm(b, axis=1, keepdims=True)
    return np.degrees(np.arccos(np.clip(np.sum(a * b, axis=1), -1.0, 1.0)))


def rel_l2(x, ref):
    return float(np.linalg.norm(np.asarray(x) - ref) / np.linalg.norm(ref))


# ------------------------------------------- reference host-wrapper semantics (numpy)
def _grid_vox(x_locs, y_locs, z_locs):
    X, Y, Z = np.meshgrid(np.asarray(x_locs, np.float32), np.asarray(y_locs, np.float32),
                          np.asarray(z_locs, np.float32), indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def ref_prep(radar_data, rx_offsets, antenna_locs, use_4_rx):
    """py_image_gpu._prep_inputs (py_image_gpu.py:219-235): [A*R, S] measurements with
    the TX location repeated per RX when use_4_rx."""
    radar_data = np.asarray(radar_data)
    antenna_locs = np.asarray(antenna_locs)
    S = radar_data.shape[1]
    if use_4_rx:
        radar_data = np.transpose(radar_data, (0, 2, 1))
        antenna_locs = np.repeat(antenna_locs, radar_data.shape[1], axis=0)
    # the kernel reads row i*S.. for i < len(antenna_locs) only (imaging_gpu.cu:100,110)
    meas = radar_data.reshape(-1).reshape(-1, S)[: antenna_locs.shape[0]]
    return np.asarray(rx_offsets).reshape(-1, 3), meas, antenna_locs


def ref_image_cuda(x_locs, y_locs, z_locs, antenna_locs, radar_data, rx_offsets, slope,
                   wavelength, bandwidth, num_samples, use_4_rx=False, is_ti_radar=False,
                   use_interpolated_processing=False, return_phase_centers=True,
                   dist_mode=0, max_num_ant=4096 * 32):
    """Restatement of py_image_gpu.image_cuda (py_image_gpu.py:308-366) over the FP64
    oracle kernels.  Returns the complex128 image [NX,NY,NZ] (and phase centres)."""
    vox = _grid_vox(x_locs, y_locs, z_locs)
    shape = (len(x_locs), len(y_locs), len(z_locs))
    rx_offsets = np.asarray(rx_offsets)

    def run(locs, data):
        norm = np.asarray(locs).shape[0]
        S = np.asarray(data).shape[1]
        rxo, meas, locs_rep = ref_prep(data, rx_offsets, locs, use_4_rx)
        fsp = float(np.float32(3e8 / (2 * bandwidth) * num_samples / S))
        wl = float(np.float32(wavelength))
        sl = float(np.float32(slope))
        if use_interpolated_processing:
            img, _ = interp(vox, locs_rep, rxo, meas, wl, fsp, is_ti_radar, dist_mode)
        else:
            img, _ = full(vox, locs_rep, rxo, meas, wl, sl, is_ti_radar, vote=False)
        return img.reshape(shape) / norm, locs_rep

    def centres(locs_rep):
        rep = np.tile(rx_offsets, reps=(len(locs_rep) // len(rx_offsets), 1))
        return (locs_rep + (locs_rep + rep)) / 2

    if not use_interpolated_processing:
        img, locs_rep = run(antenna_locs, radar_data)
        img = img / np.asarray(antenna_locs).shape[0]
        cl = centres(locs_rep)
    else:
        num_rx = len(rx_offsets)
        groups = math.ceil(np.asarray(antenna_locs).shape[0] * num_rx / max_num_ant)
        img, cl = None, None
        for i in range(groups):
            sl_ = slice(i * max_num_ant // num_rx, (i + 1) * max_num_ant // num_rx)
            part, locs_rep = run(np.asarray(antenna_locs)[sl_], np.asarray(radar_data)[sl_])
            c = centres(locs_rep)
            img = part if img is None else img + part
            cl = c if cl is None else np.concatenate((cl, c), axis=0)
    return (img, cl) if return_phase_centers else img


def ref_normal_estimates_cuda(sum_image, x_locs, y_locs, z_locs, antenna_locs,
                              radar_data, rx_offset, slope, wavelength, bandwidth,
                              num_samples, use_4_rx=False, is_ti_radar=False,
                              initial_filter_percent=0.05, dist_mode=0,
                              max_num_ant=4096 * 32):
    """Restatement of py_sn_est_gpu.normal_estimates_cuda (interpolated mode,
    py_sn_est_gpu.py:291-424): float64 [NX,NY,NZ,3], NaN outside the mask, not unit."""
    sum_image = np.asarray(sum_image)
    shape = sum_image.shape
    filt = np.abs(sum_image) > np.max(np.abs(sum_image)) * initial_filter_percent
    vox_all = _grid_vox(x_locs, y_locs, z_locs)
    flat = np.flatnonzero(filt.ravel())
    vox = vox_all[flat]
    vals = sum_image.ravel()[flat].astype(np.complex64)
    rx_offset = np.asarray(rx_offset)
    num_rx = len(rx_offset)
    groups = math.ceil(np.asarray(antenna_locs).shape[0] * num_rx / max_num_ant)
    total = None
    for g in range(groups):
        sl_ = slice(g * max_num_ant // num_rx, (g + 1) * max_num_ant // num_rx)
        data = np.asarray(radar_data)[sl_]
        S = data.shape[1]
        rxo, meas, locs_rep = ref_prep(data, rx_offset, np.asarray(antenna_locs)[sl_],
                                       use_4_rx)
        fsp = float(np.float32(3e8 / (2 * bandwidth) * num_samples / S))
        n = sn_interp(vox, vals, locs_rep, rxo, meas, float(np.float32(wavelength)), fsp,
                      is_ti_radar, dist_mode)
        out = np.full(shape + (3,), np.nan)
        out[filt] = n
        total = out if total is None else total + out
    return total
