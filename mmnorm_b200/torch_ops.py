"""The library's entry points as PyTorch operators (``torch.ops.mmnorm.*``), for callers
that hold tensors inside larger torch programs: schema-checked, stream-ordered on the
current stream, with fake (meta) implementations for shape propagation and the adjoint
kernels registered as the autograd formula of ``backproject``.

    import mmnorm_b200.torch_ops
    image, vote = torch.ops.mmnorm.backproject(x, y, z, ant, rxo, meas, wl, slope,
                                               "mixed", 0.0, False, None)
    image, vote, normals, mask = torch.ops.mmnorm.backproject_normals(..., 0.05)

Each operator calls the same C ABI as ``mmnorm_b200.ops``; nothing here computes.
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import torch
from torch import Tensor

from . import ops

_MODES = ("mixed", "plain", "interp", "interp_fast", "nufft")


@torch.library.custom_op("mmnorm::backproject", mutates_args=())
def backproject(x_locs: Tensor, y_locs: Tensor, z_locs: Tensor, antenna_locs: Tensor,
                rx_offsets: Tensor, meas: Tensor, wavelength: float, slope: float,
                mode: str, fft_spacing: float, is_ti_radar: bool,
                pos_offsets: Optional[Tensor]) -> Tuple[Tensor, Tensor]:
    """Fused backprojection + vote: image complex64 [NX,NY,NZ], vote [3,NX,NY,NZ]."""
    if mode not in _MODES:
        raise ValueError("mode must be one of %s" % (_MODES,))
    return ops.backproject(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength,
                           slope, mode=mode, fft_spacing=fft_spacing, is_ti_radar=is_ti_radar,
                           pos_offsets=pos_offsets)


@backproject.register_fake
def _(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope, mode,
      fft_spacing, is_ti_radar, pos_offsets):
    shp = (x_locs.shape[0], y_locs.shape[0], z_locs.shape[0])
    return (meas.new_empty(shp, dtype=torch.complex64),
            meas.new_empty((3,) + shp, dtype=torch.complex64))


@torch.library.custom_op("mmnorm::backproject_backward", mutates_args=())
def backproject_backward(x_locs: Tensor, y_locs: Tensor, z_locs: Tensor, antenna_locs: Tensor,
                         rx_offsets: Tensor, meas: Tensor, wavelength: float, slope: float,
                         is_ti_radar: bool, pos_offsets: Optional[Tensor],
                         grad_image: Tensor, grad_vote: Optional[Tensor]) -> Tuple[Tensor, Tensor]:
    """Adjoint of the mixed form: (dL/dmeas complex64 [A,F], dL/dpos float32 [A,3])."""
    return ops.backproject_backward(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas,
                                    wavelength, slope, grad_image, grad_vote,
                                    is_ti_radar=is_ti_radar, pos_offsets=pos_offsets)


@backproject_backward.register_fake
def _(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope, is_ti_radar,
      pos_offsets, grad_image, grad_vote):
    return (meas.new_empty(meas.shape, dtype=torch.complex64),
            meas.new_empty((meas.shape[0], 3), dtype=torch.float32))


def _setup_context(ctx, inputs, output):
    (x, y, z, ant, rxo, meas, wl, sl, mode, fsp, ti, pos) = inputs
    ctx.set_materialize_grads(False)
    if mode not in ("mixed", "nufft") and (ctx.needs_input_grad[5] or ctx.needs_input_grad[11]):
        raise NotImplementedError("gradients are implemented for modes 'mixed' and 'nufft'")
    ctx.save_for_backward(x, y, z, ant, rxo, meas, pos)
    ctx.consts = (wl, sl, ti)


def _backward(ctx, grad_image, grad_vote):
    x, y, z, ant, rxo, meas, pos = ctx.saved_tensors
    wl, sl, ti = ctx.consts
    if grad_image is None and grad_vote is None:
        return (None,) * 12
    V = x.shape[0] * y.shape[0] * z.shape[0]
    gI = grad_image if grad_image is not None else torch.zeros(
        (V,), dtype=torch.complex64, device=meas.device)
    gW = grad_vote.contiguous() if grad_vote is not None else None   # no vote term
    gm, gp = torch.ops.mmnorm.backproject_backward(x, y, z, ant, rxo, meas, wl, sl, ti, pos,
                                                   gI.contiguous(), gW)
    return (None, None, None, None, None, gm, None, None, None, None, None,
            gp if pos is not None else None)


backproject.register_autograd(_backward, setup_context=_setup_context)


@torch.library.custom_op("mmnorm::backproject_normals", mutates_args=())
def backproject_normals(x_locs: Tensor, y_locs: Tensor, z_locs: Tensor, antenna_locs: Tensor,
                        rx_offsets: Tensor, meas: Tensor, wavelength: float, slope: float,
                        mode: str, fft_spacing: float, is_ti_radar: bool,
                        filter_percent: float) -> Tuple[Tensor, Tensor, Tensor, Tensor]:
    """Image, vote, unit normals float32 [NX,NY,NZ,3] (NaN outside the mask), mask."""
    image, vote = ops.backproject(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas,
                                  wavelength, slope, mode=mode, fft_spacing=fft_spacing,
                                  is_ti_radar=is_ti_radar)
    normals, mask = ops.surface_normals(image, vote, filter_percent)
    return image, vote, normals, mask


@backproject_normals.register_fake
def _(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope, mode,
      fft_spacing, is_ti_radar, filter_percent):
    shp = (x_locs.shape[0], y_locs.shape[0], z_locs.shape[0])
    return (meas.new_empty(shp, dtype=torch.complex64),
            meas.new_empty((3,) + shp, dtype=torch.complex64),
            meas.new_empty(shp + (3,), dtype=torch.float32),
            meas.new_empty(shp, dtype=torch.bool))


@torch.library.custom_op("mmnorm::backproject_batched", mutates_args=())
def backproject_batched(x_locs: List[Tensor], y_locs: List[Tensor], z_locs: List[Tensor],
                        antenna_locs: List[Tensor], rx_offsets: List[Tensor], meas: List[Tensor],
                        wavelength: List[float], slope: List[float], is_ti_radar: List[bool],
                        items_per_slot: int) -> Tuple[List[Tensor], List[Tensor]]:
    """Many objects in one persistent launch (mixed form): images and votes per object."""
    objs = [dict(x_locs=x_locs[o], y_locs=y_locs[o], z_locs=z_locs[o],
                 antenna_locs=antenna_locs[o], rx_offsets=rx_offsets[o], meas=meas[o],
                 wavelength=wavelength[o], slope=slope[o], is_ti_radar=is_ti_radar[o])
            for o in range(len(meas))]
    plan = ops.BatchPlan(objs, items_per_slot=items_per_slot)
    plan.run()
    res = plan.results()
    return [r[0] for r in res], [r[1] for r in res]


@backproject_batched.register_fake
def _(x_locs, y_locs, z_locs, antenna_locs, rx_offsets, meas, wavelength, slope, is_ti_radar,
      items_per_slot):
    imgs, votes = [], []
    for o in range(len(meas)):
        shp = (x_locs[o].shape[0], y_locs[o].shape[0], z_locs[o].shape[0])
        imgs.append(meas[o].new_empty(shp, dtype=torch.complex64))
        votes.append(meas[o].new_empty((3,) + shp, dtype=torch.complex64))
    return imgs, votes
