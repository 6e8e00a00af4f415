"""Isosurface channel simulation and the isosurface-offset search on the GPU
(src/data_processing/isosurface_optimization.py).

    scene = make_scene(sdf, bounding_box, voxel_size, wavelengths, width, height,
                       width_fov, height_fov, is_real_data)
    ch = simulate_channels_batch(scene, taus, rx_locs, rx_dirs)      # [T, A, K] complex64

``simulate_channels`` keeps the signature of ``_simulate_channels`` (:116); the library's
``mmn_iso_channels`` marches every ray of every (offset set, antenna) pair through every
RSDF component and sums the channel of the hits in one launch.  ``channel_loss`` is
``loss_fn`` (:211) with the dense DFT replaced by an FFT; ``search_taus`` is the offset
grid search of the reference's main loop (:448-508) over all offset sets and antennas in
batched launches; ``filter_channels``, ``select_tau`` and ``final_point_cloud`` are the
host-side steps (:248, :301, :372).
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .ops import _stream, _vp

UNDEF_VAL = -50          # isosurface_optimization.py:27
SPEED_OF_LIGHT = 2.99792458e8


class IsoScene:
    """Device-resident grids and ray/frequency parameters of one object."""

    def __init__(self, grids, bounding_box, voxel_size, wavelengths, width, height, width_fov,
                 height_fov, is_real_data):
        self.grids = grids                        # float32 [C, NX, NY, NZ], contiguous
        s = _lib.MmnIsoScene()
        s.grids = grids.data_ptr()
        s.num_comp, s.res_x, s.res_y, s.res_z = grids.shape
        for k in range(6):
            s.bbox[k] = float(np.float32(bounding_box[k]))
        s.voxel_size = float(np.float32(voxel_size))
        for k in range(3):
            s.lower[k] = float(np.float32(bounding_box[k]))
        s.width, s.height = int(width), int(height)
        s.width_fov, s.height_fov = float(width_fov), float(height_fov)
        s.range_offset = 0.15 if is_real_data else 0.0   # TI radar offset (:200)
        inv = 1.0 / np.asarray(wavelengths, np.float64)   # f_k / c
        K = inv.size
        df = (inv[-1] - inv[0]) / (K - 1) if K > 1 else 0.0
        if K > 1 and np.max(np.abs(inv - (inv[0] + np.arange(K) * df))) > 1e-9 * inv[0]:
            raise ValueError("wavelengths must come from uniformly spaced frequencies")
        s.f0_over_c, s.df_over_c, s.num_wl = float(inv[0]), float(df), int(K)
        self.scene = s
        self.num_comp = s.num_comp
        self.num_wl = K


def make_scene(sdf, bounding_box, voxel_size, wavelengths, width, height, width_fov, height_fov,
               is_real_data, device=None):
    """``sdf``: [NX, NY, NZ, C] RSDF per component with UNDEF_VAL outside it (the layout
    _read_sdf_file builds, :73-80)."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    g = torch.as_tensor(sdf).to(device=dev, dtype=torch.float32)
    if g.dim() == 3:
        g = g[..., None]
    grids = g.permute(3, 0, 1, 2).contiguous()
    return IsoScene(grids, bounding_box, voxel_size, wavelengths, width, height, width_fov,
                    height_fov, is_real_data)


def simulate_channels_batch(scene, taus, rx_locs, rx_dirs, max_items=None):
    """complex64 [T, A, K]: the channel of antenna a for offset set t (taus: [T, C], already
    clipped), summed over the components."""
    dev = scene.grids.device
    taus = torch.as_tensor(taus, dtype=torch.float32, device=dev).reshape(-1, scene.num_comp)
    rx = torch.as_tensor(rx_locs, dtype=torch.float64, device=dev).reshape(-1, 3).contiguous()
    rd = torch.as_tensor(rx_dirs, dtype=torch.float32, device=dev).reshape(-1, 3).contiguous()
    T, A = taus.shape[0], rx.shape[0]
    out = torch.empty((T, A, scene.num_wl), dtype=torch.complex64, device=dev)
    lib = _lib.load()
    per_set = lib.mmn_iso_channels_workspace_bytes(ctypes.byref(scene.scene), 1, A)
    if per_set == 0:
        raise _lib.MmnError(_lib.MMN_ERR_INVALID_ARGUMENT, "mmn_iso_channels_workspace_bytes")
    sets = max(1, min(T, 65535 // max(A, 1), (1 << 30) // per_set))
    if max_items:
        sets = max(1, min(sets, max_items // A))
    nbytes = lib.mmn_iso_channels_workspace_bytes(ctypes.byref(scene.scene), sets, A)
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    for t0 in range(0, T, sets):
        t1 = min(T, t0 + sets)
        tt = taus[t0:t1].contiguous()
        o = out[t0:t1]
        _lib.check(lib.mmn_iso_channels(ctypes.byref(scene.scene), _vp(tt), t1 - t0, _vp(rx),
                                        _vp(rd), A, _vp(o), _vp(ws), nbytes, _stream(dev)),
                   "mmn_iso_channels")
    return out


def simulate_channels(bounding_box, bounding_box_lower, voxel_size, grid_res_x, grid_res_y,
                      grid_res_z, width, height, width_fov, height_fov, grid, rx_loc, rx_dir,
                      wavelengths, taus, tau_bounds, is_real_data, apply_tau_conversion=True,
                      sdf_indices=None):
    """_simulate_channels (isosurface_optimization.py:116): the channel complex64 [K] of
    one antenna, summed over the RSDF components ``sdf_indices`` (all by default), each at
    its offset clipped to its bounds."""
    del bounding_box_lower, grid_res_x, grid_res_y, grid_res_z   # implied by grid / box
    num = grid.shape[-1]
    idx = list(range(num)) if sdf_indices is None else [int(i) for i in sdf_indices]
    t = torch.as_tensor(taus).detach().to("cpu", torch.float32)
    tb = torch.as_tensor(tau_bounds).detach().to("cpu", torch.float32)
    sel = []
    for i in idx:
        ti = t[i]
        if apply_tau_conversion:
            ti = torch.clip(ti, tb[i, 0], tb[i, 1])
        sel.append(float(ti))
    scene = make_scene(torch.as_tensor(grid)[..., idx], bounding_box, voxel_size,
                       torch.as_tensor(wavelengths).cpu().numpy(), width, height, width_fov,
                       height_fov, is_real_data, device=torch.device("cuda", torch.cuda.current_device()))
    ch = simulate_channels_batch(scene, torch.tensor([sel]), torch.as_tensor(rx_loc).reshape(1, 3),
                                 torch.as_tensor(rx_dir).reshape(1, 3))
    return ch[0, 0]


def distance_indices(wavelengths, num_samples, fft_size=512, max_dist_real=0.55,
                     max_dist_all=0.55, min_dist=0.35, f_start=77.5e9):
    """The FFT window of the main loop (:448-458): (MIN_DIST_IDX, MAX_DIST_IDX,
    MAX_DIST_IDX_REAL)."""
    f_max = 3e8 / float(wavelengths[num_samples - 1])
    dist = torch.arange(0, fft_size) * 3e8 / (2 * (f_max - f_start)) * num_samples / fft_size
    return (int((dist < min_dist).sum()), int((dist < max_dist_all).sum()),
            int((dist < max_dist_real).sum()))


def channel_loss(output_ch, target_chs, is_real_data, fft_size, min_idx, max_idx, max_idx_real):
    """loss_fn (:211-246) over the last axis: zero-padded FFT of both channels (the
    reference forms it as a dense DFT), the target cut beyond max_idx_real for real data,
    the [min_idx, max_idx) window, unit-norm, L1 of the magnitudes' difference."""
    o = torch.fft.fft(output_ch.to(torch.complex64), n=fft_size, dim=-1)
    g = torch.fft.fft(target_chs.to(torch.complex64), n=fft_size, dim=-1)
    if is_real_data:
        g = g.clone()
        g[..., max_idx_real:] = 0
    o = o[..., min_idx:max_idx]
    g = g[..., min_idx:max_idx]
    o = o / torch.linalg.vector_norm(o, dim=-1, keepdim=True)
    g = g / torch.linalg.vector_norm(g, dim=-1, keepdim=True)
    return torch.sum(torch.abs(torch.abs(o) - torch.abs(g)), dim=-1)


def tau_grid(tau_bounds, step_size, skip=15):
    """The offset sets of the main loop (:476-486): per component an arange over its bounds,
    their meshgrid, the first ``skip`` entries of the first axis dropped."""
    tb = torch.as_tensor(tau_bounds, dtype=torch.float32)
    vecs = [torch.arange(tb[i, 0], tb[i, 1], step_size) for i in range(tb.shape[0])]
    grid = torch.stack(torch.meshgrid(*vecs, indexing="ij"), dim=-1)
    return grid[skip:, ...]


def search_taus(scene, tau_bounds, step_size, rx_locs, rx_dirs, channels, is_real_data,
                num_rx=50, fft_size=512, window=None, generator=None, skip=15):
    """The grid search of the main loop (:476-508): the loss of every offset set, summed
    over ``num_rx`` randomly chosen antennas.  Returns (tau_grid [..., C], all_losses [...]).
    All sets x antennas are simulated in batched launches."""
    dev = scene.grids.device
    grid = tau_grid(tau_bounds, step_size, skip)
    shape = grid.shape[:-1]
    taus = grid.reshape(-1, grid.shape[-1])
    tb = torch.as_tensor(tau_bounds, dtype=torch.float32)
    taus = torch.maximum(torch.minimum(taus, tb[:, 1]), tb[:, 0])      # clipped (:166-168)
    perm = torch.randperm(len(rx_locs), generator=generator)[:num_rx]
    rx = torch.as_tensor(rx_locs)[perm]
    rd = torch.as_tensor(rx_dirs)[perm]
    target = torch.as_tensor(channels)[perm].to(dev)
    K = scene.num_wl
    if window is None:
        raise ValueError("window = distance_indices(...) is required")
    min_idx, max_idx, max_idx_real = window
    ch = simulate_channels_batch(scene, taus, rx, rd)                    # [T, A, K]
    losses = channel_loss(ch, target[None, :, :K], is_real_data, fft_size, min_idx, max_idx,
                          max_idx_real).sum(dim=1)
    return grid, losses.reshape(shape).cpu()


def filter_channels(channels, rx_locs, rx_dirs, is_real_data, min_idx, max_idx, max_idx_real):
    """_filter_channels (:248-299): keep antennas whose windowed range profile has a strong,
    peaked maximum away from the window's edges; relax the thresholds if fewer than 20
    remain."""
    ch = np.abs(np.fft.fft(np.asarray(torch.as_tensor(channels).cpu()), axis=1))
    if is_real_data:
        ch[:, max_idx_real:] = 0
    ch = ch[:, min_idx:max_idx]
    ch_max = np.max(ch, axis=1)
    peaked = np.sum(ch, axis=1) / ch.shape[1] < ch_max * 0.7
    inner = np.logical_and(np.argmax(ch, axis=1) != 0, np.argmax(ch, axis=1) != ch.shape[1] - 1)
    keep = None
    for frac in (0.5, 0.1, 0.05):
        keep = np.logical_and(np.logical_and(ch_max > frac * np.max(ch_max), peaked), inner)
        if np.count_nonzero(keep) >= 20:
            break
    keep_t = torch.as_tensor(keep)
    return channels[keep_t], rx_locs[keep_t], rx_dirs[keep_t]


def select_tau(all_taus, all_losses):
    """_select_tau (:301-370): the offset of minimum loss, moved to the last (topmost)
    strong peak of the flipped loss when there is one."""
    from scipy.signal import find_peaks
    all_losses = np.asarray(all_losses)
    all_taus = np.asarray(all_taus)
    if all_losses.ndim == 1:
        min_idx = np.unravel_index(np.argmin(all_losses), all_losses.shape)
        threshold = 0.9
        if np.argmin(all_losses) == 0 or np.argmin(all_losses) == len(all_losses) - 1:
            threshold = 0.3
        flipped = np.nanmax(all_losses) - all_losses
        peaks, _ = find_peaks(flipped, height=flipped[min_idx] * threshold, prominence=1)
        if len(peaks) == 0:
            # (the reference puts the index tuple itself here, which the concatenation below
            # cannot take; the minimum's index is what it means)
            peaks = np.array([min_idx[0]])
        if min_idx[0] not in peaks and min_idx[0] != 0 and min_idx[0] != len(all_losses) - 1:
            peaks = np.concatenate((peaks, min_idx))
            peaks.sort()
        return all_taus[peaks[-1]]
    min_idx = np.unravel_index(np.argmin(all_losses), all_losses.shape)
    new_idx = list(min_idx)
    for i in range(len(min_idx)):
        sel = all_losses
        for j in range(len(min_idx)):
            if j < i:
                sel = sel[new_idx[j]]
            elif j > i:
                sel = sel[:, new_idx[j]]
        sel = np.nanmax(sel) - sel
        thr = max(max(sel) * 0.4, 2)
        peaks, _ = find_peaks(sel, height=thr, prominence=0.1)
        if len(peaks) == 0:
            peaks = [min_idx[i]]
        new_idx[i] = peaks[-1]
    taus = all_taus
    for i in new_idx:
        taus = taus[i]
    return taus


def final_point_cloud(sdf, taus, coords):
    """_get_final_point_cloud (:372-388): the voxels within 1 mm of each component's
    selected isosurface."""
    pts = []
    for c in range(sdf.shape[-1]):
        pts.append(coords[np.abs(sdf[..., c] - taus[c]) < 0.001, :])
    return np.concatenate(pts, axis=0)
