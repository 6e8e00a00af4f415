"""The reference's interpolated-mode imaging tail run with its own CUDA kernels:
ImageProcessor.interpolate_measurements (image_processor.py:22-35) and the host steps of
py_image_gpu.image_cuda / py_sn_est_gpu.normal_estimates_cuda around cuda_image and
cuda_sn_est (launched by ref_cuda with pycuda's per-call transfer pattern), then the unit
normalisation of image_processor.py:396.  TEST INFRASTRUCTURE AND MEASUREMENT ONLY: the
parity tests compare the drop-in against it, and bench.py times it as the reference side.
"""
from __future__ import annotations

import numpy as np

from . import ref_cuda


def range_fft_host(radar, nbins):
    """ImageProcessor.interpolate_measurements (image_processor.py:22-35): zero-pad the
    samples to nbins and FFT along the sample axis with numpy."""
    A, S, R = radar.shape
    pad = np.zeros((A, nbins, R), dtype=np.complex64)
    pad[:, :S, :] = radar
    return np.fft.fft(pad, axis=1)


def reference_dropin_calls(x, y, z, locs, bins, rxo, slope, wavelength, bandwidth, S,
                           is_ti=0):
    """image_processor.py:390-396 with the reference's own CUDA kernels: image_cuda's host
    steps (py_image_gpu.py:219-235, 258-302, 339-362: use_4_rx re-layout, one group of
    <= 131072 virtual antennas, per-group mean) around cuda_image with pycuda's per-call
    transfers, normal_estimates_cuda's (py_sn_est_gpu.py:308-376: mask at 5 % of max|I|,
    meshgrid voxel lists, NaN scatter) around cuda_sn_est, and the unit normalisation.
    Host numpy in and out."""
    A, nbins, R = bins.shape
    assert A * R <= 4096 * 32  # one antenna group, as at this workload
    rows = np.transpose(bins, (0, 2, 1)).reshape(-1, nbins)  # use_4_rx re-layout
    ant = np.repeat(locs, R, axis=0).astype(np.float32)
    mr, mi = np.ascontiguousarray(rows.real), np.ascontiguousarray(rows.imag)
    fsp = np.float32(3e8 / (2 * bandwidth) * S / nbins)
    nx, ny, nz = len(x), len(y), len(z)
    p_r, p_i = ref_cuda.cuda_image_in_out(x, y, z, ant.ravel(), mr, mi, rxo.ravel(), slope,
                                          wavelength, fsp, A * R, R, nbins, is_ti, 1)
    image = (p_r.astype(np.float64) + 1j * p_i.astype(np.float64)).reshape(nx, ny, nz) / A
    filt = np.abs(image) > np.max(np.abs(image)) * 0.05
    m1, m2, m3 = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz))
    coords = np.concatenate((m2[..., None], m1[..., None], m3[..., None]), axis=-1)[filt]
    n = ref_cuda.cuda_sn_est_in_out(coords[:, 0], coords[:, 1], coords[:, 2],
                                    np.real(image).ravel(), np.imag(image).ravel(), x, y, z,
                                    ant.ravel(), mr, mi, rxo.ravel(), slope, wavelength, fsp,
                                    A * R, R, nbins, is_ti)
    normals = np.full((nx, ny, nz, 3), np.nan)
    normals[filt] = np.stack(n, axis=1)
    normals /= np.linalg.norm(normals, axis=-1)[..., np.newaxis].repeat(3, axis=-1)
    return image, normals


def reference_full_image(x, y, z, locs, radar, rxo, slope, wavelength, bandwidth, S,
                         is_ti=0):
    """py_image_gpu.image_cuda in full matched-filter mode (py_image_gpu.py:308-336) with
    the reference's cuda_image: use_4_rx re-layout, the kernel's full branch, the division
    by the TX count in _run_cuda_image (:302) and again in image_cuda (:330), and the
    virtual phase centres (:332-336).  Host numpy in and out."""
    A, _, R = radar.shape
    rows = np.transpose(radar, (0, 2, 1)).reshape(-1, S)
    ant = np.repeat(locs, R, axis=0).astype(np.float32)
    mr, mi = np.ascontiguousarray(rows.real), np.ascontiguousarray(rows.imag)
    fsp = np.float32(3e8 / (2 * bandwidth) * S / S)
    nx, ny, nz = len(x), len(y), len(z)
    p_r, p_i = ref_cuda.cuda_image_in_out(x, y, z, ant.ravel(), mr, mi, rxo.ravel(), slope,
                                          wavelength, fsp, A * R, R, S, is_ti, 0)
    image = (p_r.astype(np.float64) + 1j * p_i.astype(np.float64)).reshape(nx, ny, nz) / A
    image = image / A
    rep = np.tile(rxo, reps=(len(ant) // len(rxo), 1))
    centres = (ant + (ant + rep)) / 2
    return image, centres
