"""Multi-GPU imaging: one process per GPU (torch.distributed, NCCL over NVLink), the
voxel grid or the aperture split across ranks.

Two decompositions of the fused backprojection + vote + normal epilogue:

* ``"slabs"`` (default): rank r images the x-planes [x0, x1) of the grid against every
  antenna.  Voxels are independent outputs, so the data path has no exchange; the one
  collective is an all-reduce (MAX) of a single float, because the normal mask compares
  |I| with 5 % of the maximum over the WHOLE grid (src/data_processing/cuda/
  py_sn_est_gpu.py:326).  The reference splits the voxel range over GPUs the same way
  (``start_ind``, src/data_processing/cuda/py_image_gpu.py:187,273) but then sums the
  per-GPU output arrays of the full grid; here every rank owns only its slab.
* ``"antennas"``: rank r sums over its share of the TX positions for the whole grid; the
  image and the vote (8 floats per voxel) are all-reduced (SUM) before the epilogue.  For
  grids too small to give every GPU a slab of useful size.

The adjoint (``backproject_backward``, trajectory calibration on several GPUs) splits the
same ways: with ``"slabs"`` every rank's slab contributes to every measurement and
antenna-offset gradient, so the partial gradients are all-reduced (SUM) -- the data
path's one exchange, A (F + 3) values; with ``"antennas"`` a rank owns its antennas' rows
of both gradients and the rows are all-gathered.

The compute is reached through a backend object (``CudaBackend``: this library's
kernels).  Every rank issues the same collectives in the same order, including ranks
whose slab is empty.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def split_bounds(n: int, world: int, rank: int, unit: int = 1):
    """[start, stop) of rank's share when n items (in groups of ``unit``) are split as
    evenly as possible; the first n_groups % world ranks take one group more."""
    if n % unit:
        raise ValueError("%d items do not split into groups of %d" % (n, unit))
    groups = n // unit
    base, extra = divmod(groups, world)
    g0 = rank * base + min(rank, extra)
    g1 = g0 + base + (1 if rank < extra else 0)
    return g0 * unit, g1 * unit


class CudaBackend:
    """The library's kernels (ops.*) on the rank's current CUDA device."""

    def backproject(self, x, y, z, ant, rxo, meas, wavelength, slope, **kw):
        from . import ops
        return ops.backproject(x, y, z, ant, rxo, meas, wavelength, slope, **kw)

    def max_abs(self, image):
        from . import ops
        return ops.image_max_abs(image)

    def normals_from_max(self, image, vote, max_abs, filter_percent):
        from . import ops
        return ops.surface_normals_from_max(image, vote, max_abs, filter_percent)

    def backward(self, x, y, z, ant, rxo, meas, wavelength, slope, grad_image, grad_vote,
                 **kw):
        from . import ops
        return ops.backproject_backward(x, y, z, ant, rxo, meas, wavelength, slope,
                                        grad_image, grad_vote, **kw)


def _world(group):
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(group), dist.get_rank(group)
    return 1, 0


def _as_real(t):
    return torch.view_as_real(t) if t.is_complex() else t


def _all_reduce(t, op, group):
    dist.all_reduce(_as_real(t), op=op, group=group)
    return t


def _gather_slabs(local, counts, group):
    """all_gather of x-slabs with different plane counts: pad every slab to the largest,
    gather, then cut each back.  ``local`` is [planes, ...]."""
    rest = tuple(local.shape[1:])
    pmax = max(counts)
    buf = torch.zeros((pmax,) + rest, dtype=local.dtype, device=local.device)
    if local.shape[0]:
        buf[:local.shape[0]] = local
    parts = [torch.empty_like(buf) for _ in counts]
    dist.all_gather([_as_real(p) for p in parts], _as_real(buf), group=group)
    return torch.cat([p[:c] for p, c in zip(parts, counts)], dim=0)


def surface_normals(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope,
                    *, decomposition="slabs", filter_percent=0.05, gather=False, group=None,
                    backend=None, **kw):
    """Sharded image + unit normals.  Every rank passes the full inputs (grid axes,
    antennas, measurements) and receives its own part:

      {"x_range": (x0, x1), "image": complex64 [x1-x0, NY, NZ], "vote": [3, ...],
       "normals": float32 [..., 3] (NaN outside the mask), "mask": bool, "max_abs": [1]}

    For ``"antennas"`` every rank receives the whole grid (x_range = (0, NX)).  With
    ``gather=True`` the slabs are all-gathered so every rank holds the whole grid too.
    ``kw`` is passed to the backend's backproject (mode, is_ti_radar, fft_spacing, ...).
    """
    be = backend if backend is not None else CudaBackend()
    world, rank = _world(group)
    nx, ny, nz = x_locs.numel(), y_locs.numel(), z_locs.numel()
    R = rx_offsets.shape[0]

    if decomposition == "slabs":
        x0, x1 = split_bounds(nx, world, rank)
        if x1 > x0:
            image, vote = be.backproject(x_locs[x0:x1].contiguous(), y_locs, z_locs,
                                         antenna_locs, rx_offsets, meas, wavelength, slope, **kw)
            mx = be.max_abs(image)
        else:
            image = torch.zeros((0, ny, nz), dtype=torch.complex64, device=meas.device)
            vote = torch.zeros((3, 0, ny, nz), dtype=torch.complex64, device=meas.device)
            mx = torch.zeros(1, dtype=torch.float32, device=meas.device)
        if world > 1:
            _all_reduce(mx, dist.ReduceOp.MAX, group)
    elif decomposition == "antennas":
        A = antenna_locs.shape[0]
        a0, a1 = split_bounds(A, world, rank, unit=R)
        x0, x1 = 0, nx
        if a1 > a0:
            image, vote = be.backproject(x_locs, y_locs, z_locs,
                                         antenna_locs[a0:a1].contiguous(), rx_offsets,
                                         meas[a0:a1].contiguous(), wavelength, slope, **kw)
        else:
            image = torch.zeros((nx, ny, nz), dtype=torch.complex64, device=meas.device)
            vote = torch.zeros((3, nx, ny, nz), dtype=torch.complex64, device=meas.device)
        if world > 1:
            _all_reduce(image, dist.ReduceOp.SUM, group)
            _all_reduce(vote, dist.ReduceOp.SUM, group)
        mx = be.max_abs(image)
    else:
        raise ValueError("decomposition must be 'slabs' or 'antennas'")

    if image.numel():
        normals, mask = be.normals_from_max(image, vote, mx, filter_percent)
    else:
        normals = torch.zeros((0, ny, nz, 3), dtype=torch.float32, device=meas.device)
        mask = torch.zeros((0, ny, nz), dtype=torch.bool, device=meas.device)

    if gather and decomposition == "slabs" and world > 1:
        counts = [b - a for a, b in (split_bounds(nx, world, r) for r in range(world))]
        image = _gather_slabs(image, counts, group)
        vote = _gather_slabs(vote.transpose(0, 1).contiguous(), counts, group) \
            .transpose(0, 1).contiguous()
        normals = _gather_slabs(normals, counts, group)
        mask = _gather_slabs(mask.to(torch.uint8), counts, group).bool()
        x0, x1 = 0, nx
    return {"x_range": (x0, x1), "image": image, "vote": vote, "normals": normals,
            "mask": mask, "max_abs": mx}


def backproject_backward(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength,
                         slope, grad_image, grad_vote, *, decomposition="slabs", group=None,
                         backend=None, **kw):
    """Sharded adjoint of the fused backprojection + vote.  Every rank passes the full
    inputs and the upstream gradients of the WHOLE grid (``grad_image`` complex64
    [NX, NY, NZ]; ``grad_vote`` [3, NX, NY, NZ] or None) and receives the full gradients
    ``(grad_meas complex64 [A, F], grad_pos float32 [A, 3])``.  ``kw`` goes to the backend
    (``is_ti_radar``, ``pos_offsets`` [A, 3])."""
    be = backend if backend is not None else CudaBackend()
    world, rank = _world(group)
    nx = x_locs.numel()
    A, F = meas.shape
    R = rx_offsets.shape[0]
    dev = meas.device

    if decomposition == "slabs":
        x0, x1 = split_bounds(nx, world, rank)
        if x1 > x0:
            gv = grad_vote[:, x0:x1].contiguous() if grad_vote is not None else None
            gm, gp = be.backward(x_locs[x0:x1].contiguous(), y_locs, z_locs, antenna_locs,
                                 rx_offsets, meas, wavelength, slope,
                                 grad_image[x0:x1].contiguous(), gv, **kw)
        else:
            gm = torch.zeros((A, F), dtype=torch.complex64, device=dev)
            gp = torch.zeros((A, 3), dtype=torch.float32, device=dev)
        if world > 1:
            _all_reduce(gm, dist.ReduceOp.SUM, group)
            _all_reduce(gp, dist.ReduceOp.SUM, group)
        return gm, gp
    if decomposition == "antennas":
        a0, a1 = split_bounds(A, world, rank, unit=R)
        pos = kw.pop("pos_offsets", None)
        if a1 > a0:
            gm, gp = be.backward(x_locs, y_locs, z_locs, antenna_locs[a0:a1].contiguous(),
                                 rx_offsets, meas[a0:a1].contiguous(), wavelength, slope,
                                 grad_image, grad_vote,
                                 pos_offsets=None if pos is None else pos[a0:a1].contiguous(),
                                 **kw)
        else:
            gm = torch.zeros((0, F), dtype=torch.complex64, device=dev)
            gp = torch.zeros((0, 3), dtype=torch.float32, device=dev)
        if world > 1:
            counts = [b - a for a, b in (split_bounds(A, world, r, unit=R) for r in range(world))]
            gm = _gather_slabs(gm, counts, group)
            gp = _gather_slabs(gp, counts, group)
        return gm, gp
    raise ValueError("decomposition must be 'slabs' or 'antennas'")
