"""Device-resident imaging + surface-normal stage: the tail of
``ImageProcessor.generate_mmwave_surface_normals`` (src/data_processing/image_processor.py:
380-398) and the ``normal_data.npz`` file it feeds (src/utils/generic_loader.py:357-411),
with every array step on the GPU.

Reference order of operations, kept here:

  1. interpolated mode: zero-pad the samples to 4096 and FFT along the sample axis
     (``interpolate_measurements``, image_processor.py:22-35) -- here ``torch.fft`` on the
     device, complex64, instead of numpy on the host in complex128;
  2. the image (``image_cuda``, image_processor.py:390): full matched filter divided by
     the TX count twice (py_image_gpu.py:302,330); interpolated mode in groups of at most
     4096*32 virtual antennas, summing the per-group means (py_image_gpu.py:337-362);
  3. the normals (``normal_estimates_cuda``, image_processor.py:393): the vote
     Re(conj(I) c_i)/|I| (virtual antenna - voxel) summed over all antennas, NaN outside
     |I| > 5 % max|I| (py_sn_est_gpu.py:326,374-376) -- here the vote comes out of the
     imaging pass itself (one pass instead of two) and the per-group vote sums add up to
     the reference's sum of per-group normals;
  4. unit normalisation (image_processor.py:396).

Inputs are uploaded once, outputs read back once; the intermediate FFT, image, vote,
mask and normals never leave the GPU.
"""
from __future__ import annotations

import numpy as np
import torch

from . import ops

FFT_SIZE = 4096                # image_processor.py:22
MAX_NUM_ANT = 4096 * 32        # virtual antennas per interpolated-mode group (py_image_gpu.py:339)


def _dev_tensor(a, dtype, device):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), device=device).to(dtype).contiguous()


def range_fft(radar_data, fft_size=FFT_SIZE):
    """(A, S, R) complex -> (A, fft_size, R) complex64: the samples zero-padded to
    ``fft_size`` and transformed along the sample axis (image_processor.py:22-35)."""
    if radar_data.dim() != 3:
        raise ValueError("radar_data must be (num meas, num samples, num rx)")
    if radar_data.shape[1] > fft_size:
        raise ValueError("%d samples do not fit an FFT of %d" % (radar_data.shape[1], fft_size))
    return torch.fft.fft(radar_data.to(torch.complex64), n=fft_size, dim=1)


def virtual_rows(radar_data):
    """(A, S, R) -> [A*R, S] rows, virtual antenna i = TX i // R with RX i % R (the
    reference's (meas, rx, sample) order, py_image_gpu.py:219-235)."""
    A, S, R = radar_data.shape
    return radar_data.permute(0, 2, 1).reshape(A * R, S).contiguous()


def image_and_normals(x_locs, y_locs, z_locs, antenna_locs, radar_data, rx_offsets, slope,
                      wavelength, bandwidth, num_samples, *, is_ti_radar=False,
                      use_interpolated_processing=False, initial_filter_percent=0.05,
                      precision="mixed", fft_size=FFT_SIZE, device=None):
    """Image and unit normals for the already-correlated aperture, all on the GPU.

    ``radar_data``: (A, S, R) complex raw samples (the FFT is applied here in
    interpolated mode); ``antenna_locs``: (A, 3) TX positions; ``rx_offsets``: (R, 3).
    ``num_samples`` is the chirp's sample count (the range-bin spacing uses it,
    py_image_gpu.py:270).  ``precision``: the full matched filter's form ("mixed", "plain",
    "nufft"); in interpolated mode "fast" selects the fast form (the reference's range
    bins, hardware sine/cosine phasor) and anything else the reference's arithmetic.
    Returns device tensors:

      sum_image    complex64 [NX, NY, NZ], normalised as image_cuda does
      normals      float32 [NX, NY, NZ, 3] unit vectors, NaN outside the mask
      mask         bool [NX, NY, NZ]
      center_locs  float64 [A*R, 3] virtual phase centres (tx + (tx + o)) / 2
    """
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    f32 = torch.float32
    x, y, z = (_dev_tensor(a, f32, dev) for a in (x_locs, y_locs, z_locs))
    ant64 = _dev_tensor(antenna_locs, torch.float64, dev).reshape(-1, 3)
    rxo64 = _dev_tensor(rx_offsets, torch.float64, dev).reshape(-1, 3)
    data = _dev_tensor(radar_data, torch.complex64, dev)
    A, R = ant64.shape[0], rxo64.shape[0]
    if data.dim() != 3 or data.shape[0] != A or data.shape[2] != R:
        raise ValueError("radar_data must be (%d, S, %d), got %s" % (A, R, tuple(data.shape)))
    rxo = rxo64.to(f32)
    wl, sl = float(np.float32(wavelength)), float(np.float32(slope))

    if use_interpolated_processing:
        data = range_fft(data, fft_size)
        spacing = float(np.float32(3e8 / (2 * bandwidth) * num_samples / data.shape[1]))
        image = vote = None
        groups = -(-A * R // MAX_NUM_ANT)
        for g in range(groups):
            # the reference's group bounds (py_image_gpu.py:340-341)
            a0, a1 = g * MAX_NUM_ANT // R, min(A, (g + 1) * MAX_NUM_ANT // R)
            rows = virtual_rows(data[a0:a1])
            locs = ant64[a0:a1].to(f32).repeat_interleave(R, dim=0).contiguous()
            img_g, vote_g = ops.backproject(x, y, z, locs, rxo, rows, wl, sl,
                                            mode="interp_fast" if precision == "fast"
                                            else "interp",
                                            fft_spacing=spacing, is_ti_radar=is_ti_radar)
            img_g /= (a1 - a0)
            image = img_g if image is None else image.add_(img_g)
            vote = vote_g if vote is None else vote.add_(vote_g)
    else:
        rows = virtual_rows(data)
        locs = ant64.to(f32).repeat_interleave(R, dim=0).contiguous()
        image, vote = ops.backproject(x, y, z, locs, rxo, rows, wl, sl, mode=precision,
                                      is_ti_radar=is_ti_radar)
        image /= A
        image /= A

    mx = ops.image_max_abs(image)
    normals, mask = ops.surface_normals_from_max(image, vote, mx, initial_filter_percent)
    rep = ant64.repeat_interleave(R, dim=0)
    centres = (rep + (rep + rxo64.repeat(A, 1))) / 2
    return {"sum_image": image, "normals": normals, "mask": mask, "center_locs": centres}


def generate_mmwave_surface_normals(x_locs, y_locs, z_locs, all_locs, radar_data_clip,
                                    rx_offsets, slope, wavelength, bandwidth,
                                    samples_per_chirp, *, is_ti_radar=True,
                                    use_interpolated_processing=True, all_meas=None,
                                    precision="mixed"):
    """The reference's return tuple (image_processor.py:398) for correlated inputs:
    (sum_image complex64 [NX,NY,NZ], (x_locs, y_locs, z_locs), normals float64 unit /
    NaN [NX,NY,NZ,3], center_locs float64 [A*R,3], all_meas)."""
    res = image_and_normals(x_locs, y_locs, z_locs, all_locs, radar_data_clip, rx_offsets,
                            slope, wavelength, bandwidth, samples_per_chirp,
                            is_ti_radar=is_ti_radar,
                            use_interpolated_processing=use_interpolated_processing,
                            precision=precision)
    sum_image = res["sum_image"].cpu().numpy()
    normals = res["normals"].to(torch.float64).cpu().numpy()
    centres = res["center_locs"].cpu().numpy()
    meas = all_meas if all_meas is not None else np.asarray(radar_data_clip)
    return sum_image, (x_locs, y_locs, z_locs), normals, centres, meas


def save_surface_normals(path, image, x_locs, y_locs, z_locs, antenna_locs=None, channels=None,
                         normals=None):
    """``normal_data.npz`` exactly as GenericLoader.save_surface_normals writes it
    (generic_loader.py:377-381): the same keys in the same order, compressed."""
    np.savez_compressed(path, sum_img=image, x_locs=x_locs, y_locs=y_locs, z_locs=z_locs,
                        antenna_locs=np.array(antenna_locs), channels=channels, normals=normals)


def load_surface_normals(path):
    """GenericLoader.load_surface_normals (generic_loader.py:403-411): (sum_img,
    (x_locs, y_locs, z_locs), antenna_locs, channels, normals)."""
    d = np.load(path, allow_pickle=True)
    return (d["sum_img"], (d["x_locs"], d["y_locs"], d["z_locs"]), d["antenna_locs"],
            d["channels"], d["normals"])
