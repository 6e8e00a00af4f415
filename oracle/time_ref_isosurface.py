"""Times the isosurface channel simulation against the reference's own path on the same
B200: the reference ray-marching extension (built from source by oracle/build.py) plus the
torch steps of _simulate_channels (src/data_processing/isosurface_optimization.py:116-208),
as restated in oracle/iso_oracle.py, versus mmnorm_b200.isosurface.simulate_channels_batch.
TEST INFRASTRUCTURE: a measurement of the reference, not part of the product.

Workload: the reference's ray settings (2048 x 2048 rays, 80 degree half-angles, 512
wavelengths over 77.5-80.5 GHz, TI offset) on a 1 mm grid of 200 x 220 x 120 voxels holding
the RSDF of a 4 cm sphere on a +-8 mm shell, 8 antennas 0.28-0.40 m above it.  Wall-clock
after a warm-up, synchronised.  Prints one JSON line.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
C = 2.99792458e8


def main():
    import torch
    from mmnorm_b200 import isosurface
    from oracle import iso_oracle as IO
    dev = torch.device("cuda", 0)
    vs = 0.001
    x = -0.05 + vs * np.arange(200)
    y = -0.06 + vs * np.arange(220)
    z = -0.40 + vs * np.arange(120)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    r = np.sqrt((X - 0.05) ** 2 + (Y - 0.05) ** 2 + (Z + 0.33) ** 2) - 0.04
    sdf = np.where(np.abs(r) < 0.008, r, -50.0).astype(np.float32)[..., None]
    bbox = [x[0], y[0], z[0], x[-1], y[-1], z[-1]]
    wl = C / np.arange(77.5e9, 80.5e9, 3e9 / 512)
    rng = np.random.default_rng(0)
    A = 8
    loc = np.stack([rng.uniform(0.0, 0.1, A), rng.uniform(0.0, 0.1, A), np.zeros(A)], 1)
    dirs = np.tile(np.array([[0, 0, 1.0]], np.float32), (A, 1))
    W = H = 2048
    fov = 80.0
    scene = isosurface.make_scene(sdf, bbox, vs, wl, W, H, fov, fov, True)
    taus = torch.zeros((1, 1))
    isosurface.simulate_channels_batch(scene, taus, loc, dirs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ch = isosurface.simulate_channels_batch(scene, taus, loc, dirs)
    torch.cuda.synchronize()
    t_ours = time.perf_counter() - t0
    grid = torch.as_tensor(sdf, device=dev)
    wl_t = torch.as_tensor(wl, device=dev)
    IO.simulate_channels(bbox, vs, W, H, fov, fov, grid, torch.as_tensor(loc[0]), dirs[0], wl_t,
                         torch.zeros(1), True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    refs = [IO.simulate_channels(bbox, vs, W, H, fov, fov, grid, torch.as_tensor(loc[a]), dirs[a],
                                 wl_t, torch.zeros(1), True) for a in range(A)]
    torch.cuda.synchronize()
    t_ref = time.perf_counter() - t0
    rel = max(float((ch[0, a] - refs[a]).abs().norm() / refs[a].abs().norm()) for a in range(A))
    print(json.dumps({"grid": list(sdf.shape[:3]), "rays": W * H, "antennas": A,
                      "wavelengths": len(wl), "mmnorm_b200_s": t_ours,
                      "reference_path_s": t_ref, "speedup": t_ref / t_ours,
                      "max_rel_l2": rel}))


if __name__ == "__main__":
    main()
