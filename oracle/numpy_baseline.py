"""The fused backprojection + vote formula in NumPy on all host cores: a reported CPU
baseline (never the product).  TEST INFRASTRUCTURE: only bench.py's CPU-baseline leg runs
it.

Each worker process evaluates ``oracle.full_np`` (FP64 or FP32 throughout: range, phase,
complex exponential, multiply-accumulate over antennas and samples, vote) for one voxel at a time
over the whole aperture; voxels are spread over a ``spawn`` process pool (one process per
core), so no worker is forked from a process that already touched the GPU.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np

_G = {}


def _init(ant, rxo, meas, wavelength, slope, precision):
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    _G.update(ant=ant, rxo=rxo, meas=meas, wl=wavelength, sl=slope, prec=precision)


def _work(vox_chunk):
    from oracle import oracle as O
    out = []
    for v in vox_chunk:
        I, W = O.full_np(v[None, :], _G["ant"], _G["rxo"], _G["meas"], _G["wl"], _G["sl"],
                         precision=_G["prec"])
        out.append(I[0])
    return np.array(out)


def time_sample(vox, ant, rxo, meas, wavelength, slope, workers=None, target_seconds=10.0,
                precision="f64"):
    """Updates/s of the NumPy formula (``precision`` "f64" or "f32") over ``workers``
    processes on a voxel sample sized to about ``target_seconds`` (calibrated on one voxel
    per worker).  Returns a dict."""
    workers = workers or os.cpu_count() or 1
    vox = np.asarray(vox, np.float32)
    A, F = np.asarray(meas).shape
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers, initializer=_init, initargs=(ant, rxo, meas, wavelength, slope, precision)) as pool:
        # warm-up + calibration: one voxel per worker
        cal = [vox[i % len(vox)][None] for i in range(workers)]
        pool.map(_work, cal)
        t0 = time.perf_counter()
        pool.map(_work, cal)
        per_voxel = (time.perf_counter() - t0)  # one voxel per worker in parallel
        n = max(workers, int(target_seconds / max(per_voxel, 1e-6)) * workers)
        n = min(n, len(vox))
        chunks = [vox[i::workers][: (n + workers - 1) // workers] for i in range(workers)]
        t0 = time.perf_counter()
        pool.map(_work, chunks)
        dt = time.perf_counter() - t0
    done = sum(len(c) for c in chunks)
    return {"updates_per_s": done * A * F / dt, "seconds": dt, "voxels": done,
            "workers": workers}
