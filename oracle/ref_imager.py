"""Runs the reference's own C++ OpenMP imager (src/data_processing/cpp/imaging.cpp),
compiled from source by oracle/build.py into oracle/_ref/.  TEST INFRASTRUCTURE ONLY:
the golden-fixture script, the tests and bench.py's reference/CPU-baseline leg use it.

The imager reads ``../utils/params.json`` relative to the working directory
(imaging.cpp:25, mmwave_common.h:20-56) and takes ``num_samples``, ``num_rx_antenna``,
``slope`` and ``max_f`` from it; it uses ``wavelength = c / max_f`` (imaging.cpp:31).
To make it compute the same image as the GPU path (``wavelength = c / min_f``) the
scratch params.json written here sets ``max_f`` to the sweep's start frequency.  It
prints a per-voxel progress line (imaging.cpp:121-128), so it runs in a child process
whose output is discarded.  Measurements are indexed ``[i][sample][rx]``
(imaging.cpp:108,111) and the result is divided by the TX count (imaging.cpp:119).
"""
from __future__ import annotations

import glob
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
C = 2.99792458e8


def available() -> bool:
    return bool(glob.glob(os.path.join(REF_DIR, "imaging*.so")))


def run(x_locs, y_locs, z_locs, antenna_locs, meas_asr, rx_offsets, slope, f_lo,
        fft_spacing=0.0, apply_ti_offset=False, use_interpolated=False, threads=None,
        timeout=3600):
    """Image with the reference imager.

    meas_asr: complex [A, S, R] measurements; rx_offsets [R, 3].
    Returns (complex64 image [NX,NY,NZ], seconds spent inside Imaging.image()).
    """
    if not available():
        raise RuntimeError("reference imager not built (python oracle/build.py)")
    meas_asr = np.asarray(meas_asr)
    A, S, R = meas_asr.shape
    with tempfile.TemporaryDirectory(prefix="mmn_ref_") as tmp:
        os.makedirs(os.path.join(tmp, "utils"))
        os.makedirs(os.path.join(tmp, "run"))
        params = {"robot_collected": {"77_ghz": {"synthetic": {
            "min_f": float(f_lo), "max_f": float(f_lo), "slope": float(slope),
            "num_samples": int(S), "num_rx_antenna": int(R)}}}}
        with open(os.path.join(tmp, "utils", "params.json"), "w") as f:
            json.dump(params, f)
        np.savez(os.path.join(tmp, "in.npz"), x=np.asarray(x_locs, np.float32),
                 y=np.asarray(y_locs, np.float32), z=np.asarray(z_locs, np.float32),
                 ant=np.asarray(antenna_locs, np.float32),
                 meas=meas_asr.astype(np.complex64),
                 rxo=np.asarray(rx_offsets, np.float32).reshape(-1, 3),
                 fsp=np.float32(fft_spacing), ti=bool(apply_ti_offset),
                 interp=bool(use_interpolated))
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(int(threads))
        cmd = [sys.executable, os.path.abspath(__file__), "--worker", tmp]
        proc = subprocess.run(cmd, cwd=os.path.join(tmp, "run"), env=env,
                              stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                              text=True, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError("reference imager failed:\n" + proc.stderr[-4000:])
        out = np.load(os.path.join(tmp, "out.npz"))
        return out["img"], float(out["seconds"])


def time_sample(x_locs, y_locs, z_locs, antenna_locs, meas_asr, rx_offsets, slope, f_lo,
                steps=1, warmup=0, threads=None, timeout=3600):
    """Times the reference imager's ``Imaging.image()`` on a voxel sample.

    Returns a dict: ``step_seconds`` (one per timed step, each a full image() call on the
    sample), ``conversion_seconds`` (an image() call on a single voxel: the pybind11
    conversion of the antenna and measurement lists, which every call pays once
    regardless of the voxel count), and ``threads``.
    """
    if not available():
        raise RuntimeError("reference imager not built (python oracle/build.py)")
    meas_asr = np.asarray(meas_asr)
    A, S, R = meas_asr.shape
    with tempfile.TemporaryDirectory(prefix="mmn_ref_") as tmp:
        os.makedirs(os.path.join(tmp, "utils"))
        os.makedirs(os.path.join(tmp, "run"))
        params = {"robot_collected": {"77_ghz": {"synthetic": {
            "min_f": float(f_lo), "max_f": float(f_lo), "slope": float(slope),
            "num_samples": int(S), "num_rx_antenna": int(R)}}}}
        with open(os.path.join(tmp, "utils", "params.json"), "w") as f:
            json.dump(params, f)
        np.savez(os.path.join(tmp, "in.npz"), x=np.asarray(x_locs, np.float32),
                 y=np.asarray(y_locs, np.float32), z=np.asarray(z_locs, np.float32),
                 ant=np.asarray(antenna_locs, np.float32), meas=meas_asr.astype(np.complex64),
                 rxo=np.asarray(rx_offsets, np.float32).reshape(-1, 3),
                 steps=int(steps), warmup=int(warmup))
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(int(threads))
        cmd = [sys.executable, os.path.abspath(__file__), "--time", tmp]
        proc = subprocess.run(cmd, cwd=os.path.join(tmp, "run"), env=env,
                              stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True,
                              timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError("reference imager failed:\n" + proc.stderr[-4000:])
        with open(os.path.join(tmp, "times.json")) as f:
            return json.load(f)


def _time_worker(tmp: str) -> None:
    sys.path.insert(0, REF_DIR)
    import imaging  # the reference's pybind11 module  # noqa: WPS433

    d = np.load(os.path.join(tmp, "in.npz"))
    locs = d["ant"].tolist()
    meas = d["meas"].tolist()
    rxo = d["rxo"].tolist()
    one = imaging.Imaging(d["x"][:1].tolist(), d["y"][:1].tolist(), d["z"][:1].tolist(),
                          "77_ghz", "synthetic", False)
    t0 = time.perf_counter()
    one.image(locs, meas, rxo, 0.0, False, False)
    conv = time.perf_counter() - t0
    im = imaging.Imaging(d["x"].tolist(), d["y"].tolist(), d["z"].tolist(), "77_ghz",
                         "synthetic", False)
    for _ in range(int(d["warmup"])):
        im.image(locs, meas, rxo, 0.0, False, False)
    times = []
    for _ in range(int(d["steps"])):
        t0 = time.perf_counter()
        im.image(locs, meas, rxo, 0.0, False, False)
        times.append(time.perf_counter() - t0)
    with open(os.path.join(tmp, "times.json"), "w") as f:
        json.dump({"step_seconds": times, "conversion_seconds": conv,
                   "threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))}, f)


def _worker(tmp: str) -> None:
    sys.path.insert(0, REF_DIR)
    import imaging  # the reference's pybind11 module  # noqa: WPS433

    d = np.load(os.path.join(tmp, "in.npz"))
    x, y, z = d["x"].tolist(), d["y"].tolist(), d["z"].tolist()
    locs = d["ant"].tolist()
    meas = d["meas"].tolist()
    rxo = d["rxo"].tolist()
    im = imaging.Imaging(x, y, z, "77_ghz", "synthetic", False)
    t0 = time.perf_counter()
    img = im.image(locs, meas, rxo, float(d["fsp"]), bool(d["ti"]), bool(d["interp"]))
    sec = time.perf_counter() - t0
    np.savez(os.path.join(tmp, "out.npz"), img=np.asarray(img, dtype=np.complex64),
             seconds=sec)


if __name__ == "__main__":
    if len(sys.argv) == 3 and sys.argv[1] == "--worker":
        _worker(sys.argv[2])
    elif len(sys.argv) == 3 and sys.argv[1] == "--time":
        _time_worker(sys.argv[2])
