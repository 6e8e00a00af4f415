"""Times the reference's own CUDA kernel (``cuda_image``, src/data_processing/cuda/
imaging_gpu.cu:12, compiled unmodified for sm_100a by oracle/build.py) on the B200 next
to this library's kernels, on the 128^3-voxel / 128x128-antenna / 256-frequency workload.
TEST INFRASTRUCTURE: a measurement of the reference, not part of the product.

Full matched filter: the reference evaluates an FP64 sin and cos per update, so it runs
on a leading slab of the grid (launch extent = grid_dim * 512 voxels, as its own multi-GPU
split does with start_ind, py_image_gpu.py:187,273); both kernels are timed on the same
slab.  Interpolated mode (range-FFT of 4096 bins): both kernels on the whole grid.
Kernel-only times with CUDA events, best of 3 after a warm-up.  Prints one JSON line.

Usage:  python oracle/time_ref_cuda.py [--slab-voxels N]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _time(fn, reps=3):
    import torch
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def main():
    import torch
    from mmnorm_b200 import _lib, ops, scenes
    from oracle import ref_cuda

    ap = argparse.ArgumentParser()
    ap.add_argument("--slab-voxels", type=int, default=65536)
    args = ap.parse_args()
    dev = torch.device("cuda", 0)
    sc = scenes.config1(sign=-1, device=dev)
    nx, ny, nz = sc.grid_shape
    V = sc.num_voxels
    A, F = sc.meas.shape
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    x, y, z = t(sc.x_locs), t(sc.y_locs), t(sc.z_locs)
    ant = t(sc.antenna_locs)
    rxo = t(np.zeros((1, 3), np.float32))
    mr, mi = t(sc.meas.real.reshape(-1)), t(sc.meas.imag.reshape(-1))
    wl, sl = np.float32(sc.wavelength), np.float32(sc.slope)
    out = {"workload": sc.name, "voxels": V, "antennas": A, "freqs": F}

    # ---- full matched filter on a leading slab
    grid = max(1, args.slab_voxels // 512)
    nslab = grid * 512
    pr = torch.zeros(V, device=dev)
    pi = torch.zeros(V, device=dev)
    ms_ref = _time(lambda: ref_cuda.cuda_image(pr, pi, x, y, z, ant.reshape(-1), mr, mi,
                                               rxo.reshape(-1), sl, wl, 0.0, nx, ny, nz, A, 1,
                                               F, 0, 0, start_ind=0, grid=grid))
    lib = _lib.load()
    ws_n = lib.mmn_cuda_image_workspace_bytes_for(nx, ny, nz, A, F, 0, nslab, 0)
    ws = torch.empty(ws_n, dtype=torch.uint8, device=dev)
    qr = torch.zeros(V, device=dev)
    qi = torch.zeros(V, device=dev)
    vp = ops._vp

    def ours_slab():
        rc = lib.mmn_cuda_image(vp(qr), vp(qi), vp(x), vp(y), vp(z), vp(ant), vp(mr), vp(mi),
                                vp(rxo), float(sl), float(wl), 0.0, nx, ny, nz, A, 1, F, 0, 0,
                                0, nslab, vp(ws), ws_n, ops._stream(dev))
        _lib.check(rc, "mmn_cuda_image")

    ms_ours = _time(ours_slab)
    upd = nslab * A * F
    a, b = pr[:nslab].cpu().numpy() + 1j * pi[:nslab].cpu().numpy(), \
        qr[:nslab].cpu().numpy() + 1j * qi[:nslab].cpu().numpy()
    out["full_matched_filter"] = {
        "slab_voxels": nslab, "updates": upd,
        "reference_kernel_ms": ms_ref, "reference_G_updates_per_s": upd / ms_ref / 1e6,
        "mmn_cuda_image_ms": ms_ours, "mmn_G_updates_per_s": upd / ms_ours / 1e6,
        "speedup": ms_ref / ms_ours,
        "rel_l2_between": float(np.linalg.norm(a - b) / np.linalg.norm(a))}

    # ---- interpolated mode (4096-bin range FFT), whole grid
    nb = 4096
    pad = torch.zeros((A, nb), dtype=torch.complex64, device=dev)
    pad[:, :F] = t(sc.meas)
    fft = torch.fft.fft(pad, dim=1)
    fr, fi = fft.real.contiguous().reshape(-1), fft.imag.contiguous().reshape(-1)
    fsp = float(np.float32(3e8 / (2 * (sc.f_hi - sc.f_lo)) * F / nb))
    ms_ref_i = _time(lambda: ref_cuda.cuda_image(pr, pi, x, y, z, ant.reshape(-1), fr, fi,
                                                 rxo.reshape(-1), sl, wl, fsp, nx, ny, nz, A,
                                                 1, nb, 0, 1))

    def ours_interp():
        rc = lib.mmn_cuda_image(vp(qr), vp(qi), vp(x), vp(y), vp(z), vp(ant), vp(fr), vp(fi),
                                vp(rxo), float(sl), float(wl), fsp, nx, ny, nz, A, 1, nb, 0, 0,
                                1, -1, vp(ws), ws_n, ops._stream(dev))
        _lib.check(rc, "mmn_cuda_image")

    ms_ours_i = _time(ours_interp)
    torch.cuda.synchronize()
    same = bool(torch.equal(pr, qr) and torch.equal(pi, qi))
    out["interpolated"] = {"pairs": V * A, "reference_kernel_ms": ms_ref_i,
                           "mmn_cuda_image_ms": ms_ours_i, "speedup": ms_ref_i / ms_ours_i,
                           "bit_identical": same}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
