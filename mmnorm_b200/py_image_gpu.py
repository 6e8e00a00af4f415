"""Drop-in for src/data_processing/cuda/py_image_gpu.py (the reference's SAR imaging
wrapper).  ``image_cuda`` keeps the reference signature, argument meaning, return
types and normalisation quirks:

* full matched filter (``use_interpolated_processing=False``): the raw sum is
  divided by the TX count twice (py_image_gpu.py:302 and :330);
* interpolated mode: antennas are processed in groups of at most 4096*32 virtual
  antennas and the per-group means are summed (py_image_gpu.py:337-362);
* the image is complex64 (float32 sums combined as ``r + 1j*i``, py_image_gpu.py:301);
* the virtual phase centres ``(tx + (tx + o))/2`` are returned in the caller's dtype
  (py_image_gpu.py:332-336,351-355).

What differs is underneath: one call on the current CUDA device through the sm_100a
library (no per-call JIT, no host threads per GPU, no host-side sum of partial images),
and the full matched filter runs the mixed-precision kernel (FP64 range and phase
wrap, FP32 rotation recurrence) instead of one FP64 sin/cos pair per sample.
``precision='plain'`` selects the FP32 sincos-per-sample kernel instead, and
``precision='nufft'`` the same sums by 8-tap interpolation from per-antenna oversampled
grids (~2e-6 from the mixed form, faster for F above ~100; F up to ~1500).  In
interpolated mode the default is the reference's arithmetic bit for bit, and
``precision='fast'`` the fast form: the same range bins, the phasor from the wrapped
FP32 turn count and the hardware sine/cosine (~5e-7 per term from the reference's).
"""
from __future__ import annotations

import copy
import math

import numpy as np
import torch

from . import ops

MAX_NUM_ANT = 4096 * 32  # virtual antennas per group (py_image_gpu.py:339)


def _device():
    if not torch.cuda.is_available():
        raise RuntimeError("mmnorm_b200 needs a CUDA device")
    return torch.device("cuda", torch.cuda.current_device())


def prep_inputs(radar_data, rx_offset, antenna_locs, use_4_rx):
    """py_image_gpu._prep_inputs (py_image_gpu.py:219-235): reorder to (meas, rx, sample)
    and repeat each TX location once per RX antenna when ``use_4_rx``."""
    if use_4_rx:
        radar_data = np.transpose(radar_data, (0, 2, 1))
        antenna_locs = np.repeat(antenna_locs, radar_data.shape[1], axis=0)
    rx_offset = np.array(rx_offset)
    measurements = radar_data.reshape((-1))
    return rx_offset, measurements, antenna_locs


def _rows(measurements, samples_per_meas, num_ant):
    """[num_ant, S] complex64 rows as the kernel indexes them (i*S + j,
    imaging_gpu.cu:100,110)."""
    need = num_ant * samples_per_meas
    if measurements.size < need:
        raise ValueError("radar_data holds %d samples, the antenna list needs %d"
                         % (measurements.size, need))
    # no copy when the caller's samples are already contiguous complex64 (numpy >= 2 keeps
    # complex64 through np.fft, so the range-FFT bins of interpolated mode arrive that way)
    return np.ascontiguousarray(measurements[:need].astype(np.complex64, copy=False)).reshape(
        num_ant, samples_per_meas)


def run_cuda_image(x_locs, y_locs, z_locs, antenna_locs, radar_data, rx_offset, slope,
                   wavelength, bandwidth, num_samples, use_4_rx=False, is_ti_radar=False,
                   use_interpolated_processing=False, precision="mixed", want_vote=False,
                   vote_on_device=False):
    """py_image_gpu._run_cuda_image (py_image_gpu.py:237-305): one device pass.

    Returns (image complex64 [NX,NY,NZ] divided once by the TX count, norm_factor,
    repeated antenna locations, vote complex64 [3,NX,NY,NZ] (raw, or None); a device
    tensor with ``vote_on_device``)."""
    dev = _device()
    norm_factor = antenna_locs.shape[0]
    samples_per_meas = radar_data.shape[1]
    rx_offset_flat, measurements, antenna_locs = prep_inputs(radar_data, rx_offset,
                                                             antenna_locs, use_4_rx)
    num_ant = len(antenna_locs)
    rows = _rows(measurements, samples_per_meas, num_ant)
    fft_spacing = np.float32(3e8 / (2 * bandwidth) * num_samples / (radar_data.shape[1]))
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a, dtype=np.float32)),
                                    device=dev)
    if use_interpolated_processing:
        mode = "interp_fast" if precision == "fast" else "interp"
    else:
        mode = precision
    image, vote = ops.backproject(
        f32(x_locs), f32(y_locs), f32(z_locs), f32(np.asarray(antenna_locs).reshape(-1, 3)),
        f32(np.asarray(rx_offset_flat).reshape(-1, 3)), torch.as_tensor(rows, device=dev),
        float(np.float32(wavelength)), float(np.float32(slope)), mode=mode,
        fft_spacing=float(fft_spacing), is_ti_radar=bool(is_ti_radar), want_vote=want_vote)
    p_xyz = image.cpu().numpy()
    p_xyz /= norm_factor
    if vote is not None and not vote_on_device:
        vote = vote.cpu().numpy()
    return p_xyz, norm_factor, antenna_locs, vote


def _centres(locs_rep, rx_offsets):
    rx_locs = copy.deepcopy(locs_rep)
    rx_offsets = np.array(rx_offsets)
    rx_offset_rep = np.tile(rx_offsets, reps=(len(locs_rep) // len(rx_offsets), 1))
    rx_locs += rx_offset_rep
    return (locs_rep + rx_locs) / 2


def image_cuda(x_locs, y_locs, z_locs, antenna_locs, radar_data, rx_offsets, slope, wavelength,
               bandwidth, num_samples, use_4_rx=False, is_ti_radar=False,
               use_interpolated_processing=False, return_phase_centers=True,
               precision="mixed"):
    """SAR image on the GPU; same contract as the reference (py_image_gpu.py:308-366)."""
    sum_image = None
    center_locs = None
    if not use_interpolated_processing:
        sum_image, norm_factor, locs_rep, _ = run_cuda_image(
            x_locs, y_locs, z_locs, antenna_locs, radar_data, rx_offsets, slope, wavelength,
            bandwidth, num_samples, use_4_rx, is_ti_radar, False, precision)
        sum_image /= norm_factor
        center_locs = _centres(locs_rep, rx_offsets)
    else:
        num_rx = len(rx_offsets)
        groups = math.ceil(antenna_locs.shape[0] * num_rx / MAX_NUM_ANT)
        for i in range(groups):
            sl = slice(i * MAX_NUM_ANT // num_rx, (i + 1) * MAX_NUM_ANT // num_rx)
            image_subset, _, locs_rep, _ = run_cuda_image(
                x_locs, y_locs, z_locs, antenna_locs[sl], radar_data[sl], rx_offsets, slope,
                wavelength, bandwidth, num_samples, use_4_rx, is_ti_radar, True, precision)
            if return_phase_centers:
                center_locs_subset = _centres(locs_rep, rx_offsets)
            if i == 0:
                sum_image = image_subset
                if return_phase_centers:
                    center_locs = center_locs_subset
            else:
                sum_image += image_subset
                if return_phase_centers:
                    center_locs = np.concatenate((center_locs, center_locs_subset), axis=0)
    if return_phase_centers:
        return sum_image, center_locs
    return sum_image
