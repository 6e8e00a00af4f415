"""Restatement of the reference's raw-radar ingest for checking mmnorm_b200.ingest.
TEST INFRASTRUCTURE ONLY.

* ``unpack``: GenericLoader.load_radar_files' 77 GHz branch (src/utils/generic_loader.py:
  521-535): little-endian int16, rows of 8 = I of lanes 0-3 then Q of lanes 0-3, as
  complex128;
* ``correlate``: ImageProcessor.correlate_locs_and_meas (src/data_processing/
  image_processor.py:74-154) with scipy interp1d per trajectory column and the same skip
  rules (outside the trajectory, within 3/16 wavelength of a frame already kept from the
  same file, file too short), written as a plain loop.
"""
from __future__ import annotations

import numpy as np
from scipy import interpolate

C = 2.99792458e8


def unpack(raw_bytes):
    a = np.frombuffer(raw_bytes, dtype="<i2")
    a = a[: a.size // 8 * 8].reshape(-1, 8)
    return a[:, [0, 1, 2, 3]] + 1j * a[:, [4, 5, 6, 7]]


def correlate(robot_data, radar_data, robot_loc_data, params, is_optitrack=False, num="77"):
    times = robot_loc_data["times_%s" % num]
    traj = np.asarray(robot_loc_data["tx_%s_locs" % num])
    columns = [interpolate.interp1d(times, traj[:, i]) for i in range(traj.shape[1])]
    frames, samples = params["num_frames"], params["num_samples"]
    stride = samples * params["num_chirps"]
    dt = params["sweep_time"] + params["periodicity"]
    thr = C / params["min_f"] * (3 / 16)
    poses, radar = [], []
    for r, name in enumerate(robot_data["all_radar_filenames"]):
        ts = robot_data["all_radar_created_ts"][r]
        if ts == -1 or int(name) not in radar_data:
            continue
        data = radar_data[int(name)]
        row = []
        for j in range(frames):
            start = ts + j * dt
            try:
                loc = np.zeros(len(columns))
                for k, f in enumerate(columns):
                    loc[k] = f([start])[0]
                if j != 0 and np.min(np.linalg.norm(np.array(row)[:, :3] - loc[:3], axis=1)) < thr:
                    continue
            except Exception:  # out of the trajectory, or no frame kept yet
                continue
            block = data[j * stride: j * stride + samples, :]
            if block.shape != (samples, 4):
                continue
            if is_optitrack:
                loc = np.array([-loc[0], loc[2], loc[1]])
            poses.append(loc)
            row.append(loc)
            radar.append(block)
    return radar, np.array(poses)
