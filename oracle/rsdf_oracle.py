"""CPU restatement of the RSDF steps of src/data_processing/sdf.py.  TEST INFRASTRUCTURE:
only the tests use it, as the checker of mmnorm_b200.rsdf.

* components: scipy.ndimage.label with the 6-neighbour cross (the partition
  cc3d.connected_components(mask, connectivity=6) produces, sdf.py:98), renumbered so that
  components are 2.. in order of their first voxel in C order, background 1 (sdf.py:98 adds
  1 to cc3d's labels);
* valid components: the size filter of sdf.py:101-119;
* RSDF: the sequential FIFO breadth-first search of sdf.py:173-222 -- seed at the component
  voxel nearest the mean coordinate, neighbours tried in the order -x, +y, +x, -y, +z, -z,
  a voxel is marked and valued when it is enqueued: value = parent value +
  numpy.dot(step * dx, normal[voxel]).

Parity note: cc3d is not installed here, so the label numbering (not the RSDF) is unpinned.
"""
from __future__ import annotations

from collections import deque

import numpy as np
from scipy import ndimage

STEPS = ((-1, 0, 0), (0, 1, 0), (1, 0, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))


def components(all_normals):
    mask = ~np.isnan(all_normals[..., 0])
    structure = ndimage.generate_binary_structure(3, 1)
    lab, n = ndimage.label(mask, structure=structure)
    # renumber by first voxel in C order
    first = {}
    flat = lab.ravel()
    for idx in np.flatnonzero(flat):
        first.setdefault(flat[idx], idx)
    order = sorted(first, key=first.get)
    remap = np.ones(n + 1, np.int64)
    for k, old in enumerate(order):
        remap[old] = k + 2
    return remap[lab], mask


def valid_labels(labeled, mask, x_locs):
    areas = np.array(ndimage.sum(mask, labeled, np.arange(1, labeled.max() + 2)))
    dx = x_locs[1] - x_locs[0]
    labels = np.arange(1, labeled.max() + 2)
    size, size_z = int(0.03 / dx), int(0.04 / dx)
    valid = labels[areas > size ** 2 * size_z]
    if len(valid) == 0:
        size, size_z = int(0.015 / dx), int(0.02 / dx)
        valid = labels[areas > size ** 2 * size_z]
    return valid


def rsdf(all_normals, coords_full, labeled, valid, x_locs):
    out = np.full(all_normals.shape[:-1], np.nan)
    dx = x_locs[1] - x_locs[0]
    seen = np.zeros(labeled.shape, bool)
    shape = labeled.shape
    has_normal = ~np.isnan(all_normals[..., 0])
    for comp in valid:
        members = np.logical_and(labeled == comp, has_normal)
        idxs = np.argwhere(members)
        sel = coords_full[members, :]
        centre = np.mean(sel, axis=0)[None, :]
        start = tuple(idxs[np.argmin(np.linalg.norm(sel - centre, axis=1))])
        out[start] = 0
        seen[start] = True
        todo = deque([start])
        while todo:
            cell = todo.popleft()
            base = out[cell]
            for step in STEPS:
                nb = (cell[0] + step[0], cell[1] + step[1], cell[2] + step[2])
                if not all(0 <= nb[k] < shape[k] for k in range(3)):
                    continue
                if seen[nb] or not has_normal[nb] or labeled[nb] != comp:
                    continue
                seen[nb] = True
                todo.append(nb)
                out[nb] = base + np.dot(np.array(step) * dx, all_normals[nb])
    return out


def coords(x_locs, y_locs, z_locs):
    m1, m2, m3 = np.meshgrid(y_locs, x_locs, z_locs)
    return np.concatenate((m2[..., None], m1[..., None], m3[..., None]), axis=-1)
