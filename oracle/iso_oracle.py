"""Restatement of the reference's isosurface channel simulation with the reference's own
ray-marching extension.  TEST INFRASTRUCTURE: only the tests use it, as the checker of
mmnorm_b200.isosurface.

* ``ref_ray_matching``: the reference extension (src/data_processing/cpp/ray_tracing.cpp +
  src/data_processing/cuda/ray_tracing_kernel.cu), built unmodified by oracle/build.py
  into oracle/_ref/raytrace/ and loaded here;
* ``simulate_channels``: _simulate_channels (src/data_processing/isosurface_optimization.py:
  116-208) step by step in torch -- the extension's rough hits, the trilinear refinement of
  _compute_intersection_pos (:66-92), FP64 round trips, and sum(exp(1j 2 pi d / lambda));
* ``dense_dft_loss``: loss_fn (:211-246) with its dense DFT written out in FP64 (the
  reference builds the DFT matrix in complex64, whose twiddles at k*n ~ 2.6e5 carry
  ~1e-2 rad errors; the FP64 form is the exact transform its FFT replacement must match).
"""
from __future__ import annotations

import importlib.machinery
import importlib.util
import math
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
_ext = None


def available():
    return os.path.exists(os.path.join(HERE, "_ref", "raytrace", "ray_tracing_ref.so"))


def ref_ray_matching():
    global _ext
    if _ext is None:
        path = os.path.join(HERE, "_ref", "raytrace", "ray_tracing_ref.so")
        loader = importlib.machinery.ExtensionFileLoader("ray_tracing_ref", path)
        spec = importlib.util.spec_from_loader("ray_tracing_ref", loader)
        _ext = importlib.util.module_from_spec(spec)
        loader.exec_module(_ext)
    return _ext.ray_matching


def march(grid_subset, width, height, width_fov, height_fov, bounding_box, rx_loc, rx_dir):
    """The extension's (rough hit, voxel index, direction), each [W, H, 3]."""
    rm = ref_ray_matching()
    w_h_3 = torch.zeros(width, height, 3).cuda()
    w_h = torch.zeros(width, height).cuda()
    bx0, by0, bz0, bx1, by1, bz1 = bounding_box
    gx, gy, gz = grid_subset.shape
    return rm(w_h_3, w_h, grid_subset.contiguous(), width, height, width_fov, height_fov,
              bx0, by0, bz0, bx1, by1, bz1, gx, gy, gz, float(rx_loc[0]), float(rx_loc[1]),
              float(rx_loc[2]), float(rx_dir[0]), float(rx_dir[1]), float(rx_dir[2]))


def simulate_channels(bounding_box, voxel_size, width, height, width_fov, height_fov, grid,
                      rx_loc, rx_dir, wavelengths, taus, is_real_data):
    """grid: float32 CUDA [NX, NY, NZ, C]; taus: per component (already clipped);
    rx_loc float64 [3]; wavelengths float64 [K].  Returns complex64 [K]."""
    dev = grid.device
    lower = torch.tensor([bounding_box[0], bounding_box[1], bounding_box[2]],
                         dtype=torch.float32, device=dev)
    rx_pos_rep = rx_loc.to(dev).repeat(width, height, 1)
    combined = torch.zeros(wavelengths.shape, dtype=torch.complex64, device=dev)
    for c in range(grid.shape[-1]):
        grid_subset = grid[:, :, :, c] - taus[c]
        rough, vindex, direction = march(grid_subset, width, height, width_fov, height_fov,
                                         bounding_box, rx_loc, rx_dir)
        x = vindex[:, :, 0].long()
        y = vindex[:, :, 1].long()
        z = vindex[:, :, 2].long()
        x[x == -1] = 0
        y[y == -1] = 0
        z[z == -1] = 0
        mask = (vindex[:, :, 0] != -1).float()
        if torch.sum(mask) == 0:
            continue
        vmin = lower + vindex * voxel_size
        tx = (rough[:, :, 0] - vmin[:, :, 0]) / voxel_size
        c01 = (1 - tx) * grid_subset[x, y, z] + tx * grid_subset[x + 1, y, z]
        c23 = (1 - tx) * grid_subset[x, y + 1, z] + tx * grid_subset[x + 1, y + 1, z]
        c45 = (1 - tx) * grid_subset[x, y, z + 1] + tx * grid_subset[x + 1, y, z + 1]
        c67 = (1 - tx) * grid_subset[x, y + 1, z + 1] + tx * grid_subset[x + 1, y + 1, z + 1]
        ty = (rough[:, :, 1] - vmin[:, :, 1]) / voxel_size
        c0 = (1 - ty) * c01 + ty * c23
        c1 = (1 - ty) * c45 + ty * c67
        tz = (rough[:, :, 2] - vmin[:, :, 2]) / voxel_size
        sdf_value = (1 - tz) * c0 + tz * c1
        pos = (rough + direction * sdf_value.view(width, height, 1).repeat(1, 1, 3)) \
            + (1 - mask.view(width, height, 1).repeat(1, 1, 3))
        pos = pos * mask.repeat(3, 1, 1).permute(1, 2, 0)
        dist = torch.norm(rx_pos_rep - pos, p=2, dim=2) * 2
        if is_real_data:
            dist = dist + 0.15
        valid = mask == 1
        vd = dist[valid][:, None].repeat(1, wavelengths.shape[0])
        wl = wavelengths[None, :].repeat(vd.shape[0], 1)
        combined += torch.sum(torch.exp(1j * 2 * torch.pi * vd / wl), axis=0)
    return combined


def dense_dft_loss(output_ch, target_ch, is_real_data, fft_size, min_idx, max_idx, max_idx_real):
    def dft(x):
        n = torch.arange(fft_size, dtype=torch.float64, device=x.device)
        xr = torch.zeros(fft_size, dtype=torch.complex128, device=x.device)
        xr[:x.shape[-1]] = x.to(torch.complex128)
        mat = torch.exp(-2j * math.pi * n[:, None] * n[None, :] / fft_size)
        return mat @ xr
    o, g = dft(output_ch), dft(target_ch)
    if is_real_data:
        g[max_idx_real:] = 0
    o, g = o[min_idx:max_idx], g[min_idx:max_idx]
    o, g = o / torch.linalg.norm(o), g / torch.linalg.norm(g)
    return torch.sum(torch.abs(torch.abs(o) - torch.abs(g)))
