"""Generates the golden fixtures in tests/golden/ by running the reference's OWN C++
imager (src/data_processing/cpp/imaging.cpp, compiled from source by
``python oracle/build.py``) on small seeded inputs.  The reference ships no tests or
golden vectors of its own, so these outputs pin the oracle to the reference.

Run from the repository root:  ``python tests/golden/make_golden.py``
Each fixture stores its inputs and the reference output, so the tests never need the
reference checkout or the compiled imager.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mmnorm_b200 import scenes  # noqa: E402
from oracle import ref_imager  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def _save(name, sc, x, y, z, meas_asr, rxo, ti, interp, fsp, bins=None):
    img, sec = ref_imager.run(x, y, z, sc.antenna_locs, meas_asr, rxo,
                              np.float32(sc.slope), sc.f_lo, fft_spacing=fsp,
                              apply_ti_offset=ti, use_interpolated=interp)
    np.savez_compressed(
        os.path.join(OUT, name + ".npz"), x=x, y=y, z=z, ant=sc.antenna_locs,
        meas=meas_asr.astype(np.complex64), rxo=np.asarray(rxo, np.float32),
        slope=np.float32(sc.slope), f_lo=np.float64(sc.f_lo),
        wavelength=np.float32(scenes.C / sc.f_lo), fsp=np.float32(fsp),
        ti=bool(ti), interp=bool(interp), ref_image=img,
        note="reference imager output (imaging.cpp), divided by TX count")
    print("%-14s image %s  %.2fs" % (name, img.shape, sec))


def main():
    # 1. tiny full matched filter, one RX, no TI offset
    sc = scenes.sphere_scene(seed=3, n_ap=8, nf=16, n_vox=6, n_pts=20)
    _save("full_r1", sc, sc.x_locs, sc.y_locs, sc.z_locs, sc.meas[:, :, None],
          np.zeros((1, 3), np.float32), False, False, 0.0)

    # 2. two RX antennas with offsets, TI 0.15 m offset
    sc = scenes.sphere_scene(seed=4, n_ap=8, nf=16, n_vox=5, n_pts=20)
    rng = np.random.default_rng(4)
    rxo = np.array([[0.0, -0.005, 0.0], [0.0, -0.005 - 0.0019, 0.0]], np.float32)
    m2 = np.stack([sc.meas, sc.meas * np.complex64(0.3 - 0.7j)
                   + (rng.standard_normal(sc.meas.shape) * 1e-3).astype(np.float32)],
                  axis=2)
    _save("full_r2_ti", sc, sc.x_locs, sc.y_locs, sc.z_locs, m2, rxo, True, False, 0.0)

    # 3. interpolated mode: zero-pad 64 samples to 512 bins and FFT
    #    (image_processor.py:22-35).  The range gate fft_spacing*bins = c/(2B)*64 = 2.4 m
    #    covers the 0.8 m round trip.
    sc = scenes.sphere_scene(seed=5, n_ap=8, nf=64, n_vox=6, n_pts=20, sign=+1)
    nb = 512
    pad = np.zeros((sc.meas.shape[0], nb, 1), np.complex64)
    pad[:, :64, 0] = sc.meas
    fft = np.fft.fft(pad, axis=1)
    bandwidth = sc.f_hi - sc.f_lo
    fsp = float(np.float32(3e8 / (2 * bandwidth) * 64 / nb))
    _save("interp_r1", sc, sc.x_locs, sc.y_locs, sc.z_locs, fft, np.zeros((1, 3)),
          False, True, fsp)

    # 4. config 0 (32x32 aperture, F=64, 48^3 grid) on a 12^3 sub-grid (every 4th voxel)
    sc = scenes.config0()
    _save("cfg0_sub12", sc, sc.x_locs[::4], sc.y_locs[::4], sc.z_locs[::4],
          sc.meas[:, :, None], np.zeros((1, 3), np.float32), False, False, 0.0)


if __name__ == "__main__":
    main()
