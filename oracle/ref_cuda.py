"""Launches the reference's own CUDA kernels -- ``cuda_image``
(src/data_processing/cuda/imaging_gpu.cu:12) and ``cuda_sn_est``
(src/data_processing/cuda/surface_normal_est.cu:14) -- compiled unmodified for sm_100a
by oracle/build.py into oracle/_ref/*.cubin.  TEST INFRASTRUCTURE ONLY (GPU parity
tests).  pycuda is not available, so the launch goes through cuda-python's driver API
with the argument order and launch shape of the reference's pycuda calls
(py_image_gpu.py:189-199: block=512, grid=V/512+1, start_ind=0, one GPU;
py_sn_est_gpu.py:229-246).
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_mods = {}


def available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, n + ".cubin"))
               for n in ("imaging_gpu", "surface_normal_est"))


def _check(res, what):
    err = res[0] if isinstance(res, tuple) else res
    if int(err) != 0:
        raise RuntimeError("%s failed with CUresult %d" % (what, int(err)))
    return res[1] if isinstance(res, tuple) and len(res) == 2 else res


def _function(module: str, name: str):
    import torch
    from cuda.bindings import driver as cu

    key = (module, name, torch.cuda.current_device())
    if key in _mods:
        return _mods[key]
    torch.cuda.init()
    torch.empty(1, device="cuda")  # make the primary context current
    _check(cu.cuInit(0), "cuInit")
    mod = _check(cu.cuModuleLoad(os.path.join(REF_DIR, module + ".cubin").encode()),
                 "cuModuleLoad")
    fn = _check(cu.cuModuleGetFunction(mod, name.encode()), "cuModuleGetFunction")
    _mods[key] = (mod, fn)
    return _mods[key]


def _launch(fn, grid, block, args, types):
    import torch
    from cuda.bindings import driver as cu

    stream = cu.CUstream(torch.cuda.current_stream().cuda_stream)
    _check(cu.cuLaunchKernel(fn, grid, 1, 1, block, 1, 1, 0, stream, (tuple(args), tuple(types)),
                             0), "cuLaunchKernel")


def cuda_image(p_r, p_i, x, y, z, ant, mr, mi, rxo, slope, wavelength, fft_spacing, nx, ny, nz,
               num_ant, num_rx, samples, is_ti, interp, start_ind=0, grid=None):
    """Reference cuda_image on torch float32 device tensors (SoA measurements)."""
    _, fn = _function("imaging_gpu", "cuda_image")
    block = 512
    if grid is None:
        grid = int(nx * ny * nz / block) + 1
    P, F, I = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
    args = [p_r.data_ptr(), p_i.data_ptr(), x.data_ptr(), y.data_ptr(), z.data_ptr(),
            ant.data_ptr(), mr.data_ptr(), mi.data_ptr(), rxo.data_ptr(), float(slope),
            float(wavelength), float(fft_spacing), int(nx), int(ny), int(nz), int(num_ant),
            int(num_rx), int(samples), int(start_ind), int(is_ti), int(interp)]
    types = [P] * 9 + [F] * 3 + [I] * 9
    _launch(fn, grid, block, args, types)


def cuda_sn_est(n_x, n_y, n_z, vx, vy, vz, p_r, p_i, x, y, z, ant, mr, mi, rxo, slope,
                wavelength, fft_spacing, nx, ny, nz, num_ant, num_rx, num_valid, samples, is_ti,
                start_ind=0):
    """Reference cuda_sn_est on torch device tensors."""
    _, fn = _function("surface_normal_est", "cuda_sn_est")
    block = 512
    grid = int(num_valid / block) + 1
    P, F, I = ctypes.c_void_p, ctypes.c_float, ctypes.c_int
    args = [n_x.data_ptr(), n_y.data_ptr(), n_z.data_ptr(), vx.data_ptr(), vy.data_ptr(),
            vz.data_ptr(), p_r.data_ptr(), p_i.data_ptr(), x.data_ptr(), y.data_ptr(),
            z.data_ptr(), ant.data_ptr(), mr.data_ptr(), mi.data_ptr(), rxo.data_ptr(),
            float(slope), float(wavelength), float(fft_spacing), int(nx), int(ny), int(nz),
            int(num_ant), int(num_rx), int(num_valid), int(samples), int(start_ind), int(is_ti)]
    types = [P] * 15 + [F] * 3 + [I] * 9
    _launch(fn, grid, block, args, types)
