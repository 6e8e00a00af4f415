"""One-call replacement of the imaging + normal-estimation step of
``ImageProcessor.generate_mmwave_surface_normals``
(src/data_processing/image_processor.py:383-396):

    sum_image, center_locs = image_cuda(...)            # :390
    normals = normal_estimates_cuda(sum_image, ...)      # :393
    normals /= ||normals||                               # :396

For the full matched filter this is ONE fused device pass (image and vote together),
where the reference runs two kernels, and the unit normals are formed on the device
from the vote, which never leaves it.  For interpolated mode it runs the reference's
two-pass arithmetic (image, then the vote on the valid voxels), or with
``precision="fast"`` the fast form of both passes.  The outputs are the
same objects the reference produces: complex64 image normalised as image_cuda does,
float64 unit normals with NaN outside the mask, and the virtual phase centres.
"""
from __future__ import annotations

import numpy as np

from . import py_image_gpu, py_sn_est_gpu


def surface_normals(x_locs, y_locs, z_locs, antenna_locs, measurement_data, rx_offsets, slope,
                    wavelength, bandwidth, num_samples, use_4_rx=True, is_ti_radar=False,
                    use_interpolated_processing=False, initial_filter_percent=0.05,
                    precision="mixed"):
    """Returns (sum_image, unit normals float64 [NX,NY,NZ,3], center_locs)."""
    if use_interpolated_processing:
        sum_image, center_locs = py_image_gpu.image_cuda(
            x_locs, y_locs, z_locs, antenna_locs, measurement_data, rx_offsets, slope,
            wavelength, bandwidth, num_samples, use_4_rx=use_4_rx, is_ti_radar=is_ti_radar,
            use_interpolated_processing=True, precision=precision)
        normals = py_sn_est_gpu.normal_estimates_cuda(
            sum_image, x_locs, y_locs, z_locs, antenna_locs, measurement_data, rx_offsets,
            slope, wavelength, bandwidth, num_samples, use_4_rx=use_4_rx,
            is_ti_radar=is_ti_radar, initial_filter_percent=initial_filter_percent,
            use_interpolated_processing=True, precision=precision)
    else:
        image, norm_factor, locs_rep, vote = py_image_gpu.run_cuda_image(
            x_locs, y_locs, z_locs, antenna_locs, measurement_data, rx_offsets, slope,
            wavelength, bandwidth, num_samples, use_4_rx, is_ti_radar, False, precision,
            want_vote=True, vote_on_device=True)
        sum_image = image
        sum_image /= norm_factor
        center_locs = py_image_gpu._centres(locs_rep, rx_offsets)
        # unit normals formed on the device from the vote that never left it
        normals = py_sn_est_gpu.raw_normals_from_vote(sum_image, vote, initial_filter_percent,
                                                      unit=True)
        return sum_image, normals, center_locs
    with np.errstate(invalid="ignore", divide="ignore"):
        normals /= np.linalg.norm(normals, axis=-1)[..., np.newaxis].repeat(3, axis=-1)
    return sum_image, normals, center_locs
