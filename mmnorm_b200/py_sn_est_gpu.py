"""Drop-in for src/data_processing/cuda/py_sn_est_gpu.py (the reference's surface-normal
wrapper).  ``normal_estimates_cuda`` keeps the reference signature and return contract:
float64 [NX, NY, NZ, 3], NaN outside |I| > initial_filter_percent * max|I|
(py_sn_est_gpu.py:326,374-376), NOT unit-normalised (the caller normalises,
image_processor.py:396), summed over groups of at most 4096*32 virtual antennas
(py_sn_est_gpu.py:408-422).

Interpolated mode runs the reference's vote arithmetic on the valid voxels through the
``mmn_cuda_sn_est`` entry point.  The reference raises for the full matched filter
(py_sn_est_gpu.py:404-405); here that mode is supported: the vote vector W comes from
the fused mixed-precision backprojection and the normal is Re(conj(I) W)/|I|, which is
the reference's sum_i Re(c_i conj(I))/|I| * u_i with c_i the full per-frequency sum.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib, ops
from .py_image_gpu import MAX_NUM_ANT, _device, run_cuda_image


def prep_inputs(radar_data, rx_offset, antenna_locs, use_4_rx):
    """py_sn_est_gpu._prep_inputs (py_sn_est_gpu.py:267-288)."""
    if not use_4_rx:
        rx_offset = np.array([rx_offset])
        radar_data = np.array(radar_data).flatten()
    else:
        radar_data = np.transpose(radar_data, (0, 2, 1))
        rx_offset = np.array(rx_offset).flatten()
        antenna_locs = np.repeat(antenna_locs, radar_data.shape[1], axis=0)
    return rx_offset, radar_data, antenna_locs


def _mask(sum_image, initial_filter_percent):
    """|I| > initial_filter_percent * max|I| (py_sn_est_gpu.py:326)."""
    mag = np.abs(sum_image)
    return mag > (np.max(mag) * initial_filter_percent)


def _mask_and_coords(sum_image, initial_filter_percent):
    filter_idx = _mask(sum_image, initial_filter_percent)
    coords = np.argwhere(filter_idx)  # C order == the reference's meshgrid order
    return filter_idx, coords


def sn_est_cuda(sum_image, x_locs, y_locs, z_locs, antenna_locs, radar_data, rx_offset, slope,
                wavelength, bandwidth, num_samples, use_4_rx=False, is_ti_radar=False,
                initial_filter_percent=0.05, precision="exact"):
    """py_sn_est_gpu._sn_est_cuda (py_sn_est_gpu.py:291-379) for one antenna group;
    ``precision="fast"`` runs the fast form of the vote (mmn_cuda_sn_est_fast)."""
    dev = _device()
    samples_per_meas = radar_data.shape[1]
    rx_offset_flat, measurements, antenna_locs = prep_inputs(radar_data, rx_offset,
                                                             antenna_locs, use_4_rx)
    measurements = np.asarray(measurements).reshape(-1)
    num_ant = len(antenna_locs)
    need = num_ant * samples_per_meas
    if measurements.size < need:
        raise ValueError("radar_data holds %d samples, the antenna list needs %d"
                         % (measurements.size, need))
    # one host-to-device copy of the complex samples; the float32 real / imaginary planes
    # the kernel reads are split on the device
    meas_dev = torch.as_tensor(np.ascontiguousarray(measurements[:need]).astype(
        np.complex64, copy=False), device=dev)
    sum_image = np.asarray(sum_image)
    filter_idx, coords = _mask_and_coords(sum_image, initial_filter_percent)
    num_x, num_y, num_z = len(x_locs), len(y_locs), len(z_locs)
    nvalid = coords.shape[0]
    all_normals = np.zeros((num_x, num_y, num_z, 3))
    all_normals[:] = np.nan
    if nvalid == 0:
        return all_normals
    fft_spacing = np.float32(3e8 / (2 * bandwidth) * num_samples / (radar_data.shape[1]))
    t32 = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a, dtype=np.float32)),
                                    device=dev)
    ti32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)
    keep = dict(
        vx=ti32(coords[:, 0]), vy=ti32(coords[:, 1]), vz=ti32(coords[:, 2]),
        ir=t32(np.real(sum_image).reshape(-1)), ii=t32(np.imag(sum_image).reshape(-1)),
        x=t32(x_locs), y=t32(y_locs), z=t32(z_locs),
        ant=t32(np.asarray(antenna_locs).reshape(-1)), mr=meas_dev.real.contiguous(),
        mi=meas_dev.imag.contiguous(),
        rxo=t32(np.asarray(rx_offset_flat).reshape(-1)),
        nx=torch.zeros(nvalid, dtype=torch.float32, device=dev),
        ny=torch.zeros(nvalid, dtype=torch.float32, device=dev),
        nz=torch.zeros(nvalid, dtype=torch.float32, device=dev))
    del meas_dev
    ws_bytes = max(256, _lib.load().mmn_cuda_sn_est_workspace_bytes(num_ant, samples_per_meas))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    vp = ops._vp
    entry = _lib.load().mmn_cuda_sn_est_fast if precision == "fast" else \
        _lib.load().mmn_cuda_sn_est
    rc = entry(
        vp(keep["nx"]), vp(keep["ny"]), vp(keep["nz"]), vp(keep["vx"]), vp(keep["vy"]),
        vp(keep["vz"]), vp(keep["ir"]), vp(keep["ii"]), vp(keep["x"]), vp(keep["y"]),
        vp(keep["z"]), vp(keep["ant"]), vp(keep["mr"]), vp(keep["mi"]), vp(keep["rxo"]),
        float(np.float32(slope)), float(np.float32(wavelength)), float(fft_spacing), num_x,
        num_y, num_z, num_ant, len(rx_offset), nvalid, samples_per_meas, 0,
        int(bool(is_ti_radar)), -1, vp(ws), ws_bytes, ops._stream(dev))
    _lib.check(rc, "mmn_cuda_sn_est")
    normals = torch.stack([keep["nx"], keep["ny"], keep["nz"]], dim=1).cpu().numpy()
    all_normals[filter_idx] = normals
    return all_normals


def raw_normals_from_vote(sum_image, vote, initial_filter_percent=0.05, unit=False):
    """Reference-layout normals (float64, NaN outside the mask) from the fused vote:
    n = Re(conj(I) W)/|I| with I the given image cast to float32 as the reference passes it
    to the kernel (py_sn_est_gpu.py:236-237); ``unit`` also divides by |n| (the caller's
    step at image_processor.py:396).  ``vote`` is the complex64 [3, ...] vote, preferably
    still on the device.  The normals are formed on the GPU and come back as one float32
    [V, 3] array; the mask |I| > initial_filter_percent * max|I| is taken on the host in
    the image's own dtype, exactly as py_sn_est_gpu.py:326 does."""
    sum_image = np.asarray(sum_image)
    filter_idx = _mask(sum_image, initial_filter_percent)
    dev = _device()
    V = sum_image.size
    img = torch.as_tensor(np.ascontiguousarray(sum_image.reshape(-1), dtype=np.complex64),
                          device=dev)
    w = vote if torch.is_tensor(vote) else torch.as_tensor(np.ascontiguousarray(vote), device=dev)
    w = w.to(dev).reshape(3, V)
    # filter 0: every voxel with |I| > 0 gets its normal; the host mask then decides
    normals, _, raw = ops.surface_normals(img, w, 0.0, want_raw=True)
    src = normals if unit else raw
    out = src.cpu().numpy().astype(np.float64).reshape(sum_image.shape + (3,))
    out[~filter_idx] = np.nan
    return out


def normal_estimates_cuda(sum_image, x_locs, y_locs, z_locs, antenna_locs, radar_data,
                          rx_offset, slope, wavelength, bandwidth, num_samples, use_4_rx=False,
                          is_ti_radar=False, initial_filter_percent=0.05,
                          use_interpolated_processing=True, precision="mixed"):
    """mmWave surface-normal estimates; same contract as the reference
    (py_sn_est_gpu.py:382-424), plus the full matched filter.  ``precision``: for the full
    matched filter 'mixed' (default), 'plain' or 'nufft'; for interpolated mode 'fast'
    selects the fast form (the reference's bins, hardware sine/cosine phasor, ~5e-7 from
    the reference arithmetic), anything else the reference's arithmetic bit for bit."""
    if not use_interpolated_processing:
        _, _, _, vote = run_cuda_image(x_locs, y_locs, z_locs, antenna_locs, radar_data,
                                       rx_offset, slope, wavelength, bandwidth, num_samples,
                                       use_4_rx, is_ti_radar, False, precision, want_vote=True,
                                       vote_on_device=True)
        return raw_normals_from_vote(sum_image, vote, initial_filter_percent)
    num_rx = len(rx_offset)
    groups = math.ceil(antenna_locs.shape[0] * num_rx / MAX_NUM_ANT)
    normals = None
    for i in range(groups):
        sl = slice(i * MAX_NUM_ANT // num_rx, (i + 1) * MAX_NUM_ANT // num_rx)
        part = sn_est_cuda(sum_image, x_locs, y_locs, z_locs, antenna_locs[sl], radar_data[sl],
                           rx_offset, slope, wavelength, bandwidth, num_samples, use_4_rx,
                           is_ti_radar, initial_filter_percent, precision)
        normals = part if normals is None else normals + part
    return normals
