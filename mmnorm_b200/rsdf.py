"""Connected components and the relative signed distance field (RSDF) of the normal field
on the GPU: the steps of ``compute_rsdf`` (src/data_processing/sdf.py:258-296) after the
binary-image separation, with the reference's function contracts.

    labeled, valid_labels = find_connected_components(all_normals, x_locs)      # sdf.py:94
    rsdf = construct_rsdf_components(all_normals, coords_full, labeled,
                                     valid_labels, x_locs)                       # sdf.py:122

The components are found by the library's union-find kernels (6-connectivity, like
``cc3d.connected_components(mask, connectivity=6)``) and every component's breadth-first
integration runs on the GPU in the reference's queue order, so the RSDF values equal the
reference's Python search bit for bit.  Label numbering: the reference adds 1 to cc3d's
labels (background 1, components 2..); here components are numbered 2.. in the order of
their first voxel in C (x-major) order.  cc3d is not available to pin its own numbering;
the RSDF and the set of valid components do not depend on it.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .ops import _stream, _vp


def _device():
    if not torch.cuda.is_available():
        raise RuntimeError("mmnorm_b200 needs a CUDA device")
    return torch.device("cuda", torch.cuda.current_device())


def component_roots(mask):
    """Device connected components of a bool/uint8 CUDA tensor [NX, NY, NZ]:
    (root int32 [NX,NY,NZ] = smallest flat index of the component or -1, count int32 [V]
    = component size at the root index)."""
    dev = mask.device
    nx, ny, nz = mask.shape
    m = mask.to(torch.uint8).contiguous()
    root = torch.empty((nx, ny, nz), dtype=torch.int32, device=dev)
    count = torch.empty(nx * ny * nz, dtype=torch.int32, device=dev)
    lib = _lib.load()
    nbytes = lib.mmn_components_workspace_bytes(nx * ny * nz)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    _lib.check(lib.mmn_components(nx, ny, nz, _vp(m), _vp(root), _vp(count), _vp(ws), nbytes,
                                  _stream(dev)), "mmn_components")
    return root, count


def _valid_labels(areas, x_locs):
    """The reference's size filter (sdf.py:106-119) on areas indexed by label - 1."""
    dx = x_locs[1] - x_locs[0]
    labels = np.arange(1, len(areas) + 1)
    size, size_z = int(0.03 / dx), int(0.04 / dx)
    valid = labels[areas > size ** 2 * size_z]
    if len(valid) == 0:
        size, size_z = int(0.015 / dx), int(0.02 / dx)
        valid = labels[areas > size ** 2 * size_z]
    return valid


def find_connected_components(all_normals, x_locs, _roots=None):
    """(labeled int64 [NX,NY,NZ]: 1 background, 2.. components; valid_labels)."""
    dev = _device()
    if _roots is None:
        normals = torch.as_tensor(np.asarray(all_normals), device=dev)
        root, count = component_roots(~torch.isnan(normals[..., 0]))
    else:
        root, count = _roots
    roots = torch.nonzero(count > 0).flatten()            # ascending: first-voxel order
    lut = torch.zeros(count.numel(), dtype=torch.int64, device=dev)
    lut[roots] = torch.arange(2, roots.numel() + 2, device=dev)
    flat = root.reshape(-1).long()
    labeled = torch.where(flat >= 0, lut[flat.clamp_min(0)], torch.ones_like(flat))
    # areas of labels 1 .. max+1, as ndimage.sum(mask, labeled, arange(1, max + 2))
    areas = np.zeros(roots.numel() + 2, np.float64)
    areas[1:roots.numel() + 1] = count[roots].cpu().numpy()
    valid = _valid_labels(areas, np.asarray(x_locs))
    return labeled.reshape(root.shape).cpu().numpy(), valid


def _seed(all_normals, coords_full, labeled, component_num):
    """The reference's start voxel (sdf.py:187-193): the component voxel nearest the mean
    of its coordinates, first in C order among ties -- computed with the same numpy calls so
    the choice is identical."""
    idxs = np.argwhere(np.logical_and(labeled == component_num, ~np.isnan(all_normals[:, :, :, 0])))
    idxs_mask = np.logical_and(labeled == component_num, ~np.isnan(all_normals[:, :, :, 0]))
    coords_sel = coords_full[idxs_mask, :]
    mean_coord = np.mean(coords_sel, axis=0)[None, :]
    dists = np.linalg.norm((coords_sel - mean_coord), axis=1)
    return idxs[np.argmin(dists)]


def _seed_from_voxels(flat, shape, axes):
    """_seed for a component given its voxels' flat indices in ascending (C) order: the same
    coordinate rows, in the same order and dtype, as coords_full[labeled == component], so
    numpy's mean, norms and argmin -- and the chosen voxel -- are the same."""
    ny, nz = shape[1], shape[2]
    ii, rem = np.divmod(flat, ny * nz)
    jj, kk = np.divmod(rem, nz)
    x, y, z = axes
    coords_sel = np.stack([x[ii], y[jj], z[kk]], axis=1)
    mean_coord = np.mean(coords_sel, axis=0)[None, :]
    dists = np.linalg.norm((coords_sel - mean_coord), axis=1)
    return int(flat[np.argmin(dists)])


def coordinate_grid(x_locs, y_locs, z_locs):
    """coords_full of sdf.py:285-287 (the concatenated meshgrid): [NX,NY,NZ,3] with
    coords[i, j, k] = (x[i], y[j], z[k]), in the meshgrid's dtype, filled by broadcasting."""
    x, y, z = np.asarray(x_locs), np.asarray(y_locs), np.asarray(z_locs)
    out = np.empty((len(x), len(y), len(z), 3), dtype=np.result_type(y, x, z))
    out[..., 0] = x[:, None, None]
    out[..., 1] = y[None, :, None]
    out[..., 2] = z[None, None, :]
    return out


def construct_rsdf_components(all_normals, coords_full, labeled, valid_labels, x_locs,
                              _roots=None, _normals=None, _axes=None):
    """float64 [NX,NY,NZ]: RSDF on the valid components, NaN elsewhere (sdf.py:122-224)."""
    dev = _device()
    all_normals = np.asarray(all_normals)
    nx, ny, nz = all_normals.shape[:3]
    normals = _normals if _normals is not None else torch.as_tensor(
        np.ascontiguousarray(all_normals, dtype=np.float64), device=dev)
    if _roots is None:
        root, count = component_roots(~torch.isnan(normals[..., 0]))
    else:
        root, count = _roots
    root = root.contiguous()
    rsdf = torch.full((nx, ny, nz), float("nan"), dtype=torch.float64, device=dev)
    lib = _lib.load()
    nbytes = lib.mmn_rsdf_workspace_bytes(nx, ny, nz)
    if nbytes == 0:
        raise _lib.MmnError(_lib.MMN_ERR_INVALID_ARGUMENT, "mmn_rsdf_workspace_bytes")
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    dx = float(x_locs[1] - x_locs[0])
    # with the library's own labels (the roots in ascending order are labels 2, 3, ...),
    # each component's voxels come from the device and its seed from them alone
    own = _roots is not None and _axes is not None
    roots_sorted = torch.nonzero(count > 0).flatten().cpu().numpy() if own else None
    root_flat = root.reshape(-1)
    root_host = None
    for component_num in valid_labels:
        if own:
            comp_root = int(roots_sorted[component_num - 2])
            flat = torch.nonzero(root_flat == comp_root).flatten().cpu().numpy()
            seed = _seed_from_voxels(flat, (nx, ny, nz), _axes)
        else:
            i0, j0, k0 = _seed(all_normals, coords_full, labeled, component_num)
            if root_host is None:
                root_host = root.cpu().numpy()
            comp_root = int(root_host[i0, j0, k0])
            seed = int((i0 * ny + j0) * nz + k0)
        count_v = ctypes.c_int64(0)
        _lib.check(lib.mmn_rsdf_component(nx, ny, nz, _vp(normals), _vp(root), comp_root, seed,
                                          dx, _vp(rsdf), ctypes.byref(count_v), _vp(ws), nbytes,
                                          _stream(dev)), "mmn_rsdf_component")
    return rsdf.cpu().numpy()


def compute_rsdf(all_normals, x_locs, y_locs, z_locs):
    """Steps 2-3 of compute_rsdf (sdf.py:285-289) on normals already masked by the binary
    image and normalised: (rsdf, labeled, valid_labels, coords_full)."""
    coords_full = coordinate_grid(x_locs, y_locs, z_locs)
    dev = _device()
    normals = torch.as_tensor(np.ascontiguousarray(all_normals, dtype=np.float64), device=dev)
    roots = component_roots(~torch.isnan(normals[..., 0]))
    labeled, valid = find_connected_components(all_normals, x_locs, _roots=roots)
    axes = (np.asarray(x_locs), np.asarray(y_locs), np.asarray(z_locs))
    rsdf = construct_rsdf_components(all_normals, coords_full, labeled, valid, x_locs,
                                     _roots=roots, _normals=normals, _axes=axes)
    return rsdf, labeled, valid, coords_full
