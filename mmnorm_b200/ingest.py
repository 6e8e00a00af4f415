"""Raw radar ingest on the GPU: 77 GHz ADC files (GenericLoader.load_radar_files,
src/utils/generic_loader.py:484-537) and the antenna position of every frame
(ImageProcessor.correlate_locs_and_meas, src/data_processing/image_processor.py:74-154).

    radar_data = load_radar_files(paths)                      # {timestamp: complex64 [N, 4]}
    data = correlate_locs_and_meas(robot_data, radar_data, robot_loc_data, params)
    data["radar_data"]  # list of complex64 [S, 4] device tensors, data["poses"] float64 [M, D]

Both steps are the reference's, with its skip rules; the samples are complex64 (the int16
values are exact) where the reference holds complex128.  The interpolation follows scipy's
linear interp1d, which evaluates float64 columns with numpy.interp (scipy 1.18, numpy 2.3
here; the reference pins numpy 1.24.3 and no scipy version).
"""
from __future__ import annotations

import os

import numpy as np
import torch

from . import _lib
from .ops import _stream, _vp

C = 2.99792458e8


def _device():
    if not torch.cuda.is_available():
        raise RuntimeError("mmnorm_b200 needs a CUDA device")
    return torch.device("cuda", torch.cuda.current_device())


def unpack_adc(raw_bytes, device=None):
    """complex64 [N, 4] device tensor from the bytes of one 77 GHz .bin file.  A file that
    is not whole rows of 8 int16 values is refused with ValueError, as the reference's
    reshape refuses it (generic_loader.py:533)."""
    dev = device or _device()
    raw = np.frombuffer(raw_bytes, dtype="<i2")
    if raw.size % 8:
        raise ValueError("77 GHz ADC data of %d int16 values is not whole rows of 8" % raw.size)
    n = raw.size // 8
    src = torch.as_tensor(raw[: n * 8].copy(), device=dev)
    out = torch.empty((n, 4), dtype=torch.complex64, device=dev)
    _lib.check(_lib.load().mmn_adc_unpack(_vp(src), n, _vp(out), _stream(dev)), "mmn_adc_unpack")
    return out


def file_timestamp(filename):
    """The timestamp of a .bin file name (generic_loader.py:526-529)."""
    try:
        return int(filename[8:18])
    except ValueError:
        return int(filename[9:21])


def load_radar_files(directory, device=None):
    """{timestamp: complex64 [N, 4]} for every .bin file in ``directory``, in name order."""
    out = {}
    for name in sorted(os.listdir(directory)):
        if name[-4:] != ".bin":
            continue
        with open(os.path.join(directory, name), "rb") as f:
            out[file_timestamp(name)] = unpack_adc(f.read(), device)
    return out


def correlate_locs_and_meas(robot_data, radar_data, robot_loc_data, params, radar_type="77_ghz",
                            is_optitrack=False):
    """{'radar_data': [complex64 [S, 4]], 'poses': float64 [M, D]} -- one entry per kept
    frame, in the reference's order (rows in file order, frames ascending).

    robot_data: 'all_radar_filenames', 'all_radar_created_ts'; robot_loc_data:
    'times_77', 'tx_77_locs'; params: num_frames, sweep_time, periodicity, num_samples,
    num_chirps, min_f (utilities.get_radar_parameters)."""
    dev = _device()
    num = radar_type[:2]
    times = np.asarray(robot_loc_data["times_%s" % num], np.float64)
    traj = np.asarray(robot_loc_data["tx_%s_locs" % num], np.float64)
    if traj.ndim == 1:
        traj = traj[:, None]
    order = np.argsort(times, kind="mergesort")   # interp1d sorts its abscissae
    times, traj = times[order], traj[order]
    frames = int(params["num_frames"])
    samples = int(params["num_samples"])
    stride = samples * int(params["num_chirps"])
    dt = float(params["sweep_time"]) + float(params["periodicity"])
    threshold = C / float(params["min_f"]) * (3 / 16)
    names = list(robot_data["all_radar_filenames"])
    created = np.asarray(robot_data["all_radar_created_ts"], np.float64)
    avail = np.full(len(names), -1, np.int64)
    for r, name in enumerate(names):
        if created[r] == -1 or int(name) not in radar_data:
            continue
        avail[r] = radar_data[int(name)].shape[0]
    dim = traj.shape[1]
    dim_out = 3 if is_optitrack else dim
    R = len(names)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    d_times, d_traj, d_created, d_avail = t(times), t(traj), t(created), t(avail)
    loc = torch.zeros((R, frames, dim_out), dtype=torch.float64, device=dev)
    keep = torch.zeros((R, frames), dtype=torch.uint8, device=dev)
    scratch = torch.empty((R, frames), dtype=torch.int32, device=dev)
    _lib.check(_lib.load().mmn_correlate_poses(
        _vp(d_times), _vp(d_traj), len(times), dim, _vp(d_created), _vp(d_avail), R, frames, dt,
        threshold, stride, samples, int(bool(is_optitrack)), _vp(loc), _vp(keep), _vp(scratch),
        _stream(dev)), "mmn_correlate_poses")
    kept = keep.bool().cpu().numpy()
    poses = loc[keep.bool()].cpu().numpy()
    radar = []
    for r, name in enumerate(names):
        js = np.flatnonzero(kept[r])
        if len(js) == 0:
            continue
        data = radar_data[int(name)]
        for j in js:
            radar.append(data[j * stride: j * stride + samples, :])
    return {"radar_data": radar, "poses": poses}
