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


class _DevPtr:
    """A raw device address with the data_ptr() accessor the launchers read."""

    def __init__(self, ptr):
        self.ptr = int(ptr)

    def data_ptr(self):
        return self.ptr


def cuda_image_in_out(x, y, z, ant, meas_r, meas_i, rxo, slope, wavelength, fft_spacing,
                      num_ant, num_rx, samples, is_ti, interp):
    """cuda_image with the reference's per-call transfers (py_image_gpu.py:189-199): each
    input through pycuda's drv.In -- a device allocation and a synchronous copy from the
    caller's (pageable) numpy array -- and the two outputs through drv.Out (allocation,
    launch, synchronous copy back), all freed before return.  Host numpy in, (p_r, p_i)
    float32 numpy out.  The per-call SourceModule build (py_image_gpu.py:56-179) is not
    included: pycuda serves it from its on-disk cache."""
    import numpy as np
    import torch
    from cuda.bindings import driver as cu

    torch.empty(1, device="cuda")  # make the primary context current
    nx, ny, nz = len(x), len(y), len(z)
    V = nx * ny * nz
    allocs = []

    def dev_in(arr):
        a = np.ascontiguousarray(arr, dtype=np.float32)
        d = _check(cu.cuMemAlloc(max(4, a.nbytes)), "cuMemAlloc")
        allocs.append(d)
        _check(cu.cuMemcpyHtoD(d, a.ctypes.data, a.nbytes), "cuMemcpyHtoD")
        return _DevPtr(d)

    def dev_out(n):
        d = _check(cu.cuMemAlloc(4 * n), "cuMemAlloc")
        allocs.append(d)
        return _DevPtr(d)

    try:
        p_r, p_i = dev_out(V), dev_out(V)
        args = [dev_in(a) for a in (x, y, z, ant, meas_r, meas_i, rxo)]
        cuda_image(p_r, p_i, *args, slope, wavelength, fft_spacing, nx, ny, nz, num_ant, num_rx,
                   samples, is_ti, interp)
        out_r = np.empty(V, np.float32)
        out_i = np.empty(V, np.float32)
        _check(cu.cuMemcpyDtoH(out_r.ctypes.data, p_r.ptr, 4 * V), "cuMemcpyDtoH")
        _check(cu.cuMemcpyDtoH(out_i.ctypes.data, p_i.ptr, 4 * V), "cuMemcpyDtoH")
    finally:
        for d in allocs:
            cu.cuMemFree(d)
    return out_r, out_i


def cuda_sn_est_in_out(valid_x, valid_y, valid_z, img_r, img_i, x, y, z, ant, meas_r, meas_i,
                       rxo, slope, wavelength, fft_spacing, num_ant, num_rx, samples, is_ti):
    """cuda_sn_est with the reference's per-call transfers (py_sn_est_gpu.py:229-246): the
    three outputs through drv.Out and every input through drv.In (int32 voxel index lists,
    float32 arrays), block 512, grid num_valid/512 + 1, start_ind 0, one GPU.  Host numpy
    in, (n_x, n_y, n_z) float32 numpy out."""
    import numpy as np
    import torch
    from cuda.bindings import driver as cu

    torch.empty(1, device="cuda")  # make the primary context current
    nx, ny, nz = len(x), len(y), len(z)
    nv = len(valid_x)
    allocs = []

    def dev_in(arr, dtype):
        a = np.ascontiguousarray(arr, dtype=dtype)
        d = _check(cu.cuMemAlloc(max(4, a.nbytes)), "cuMemAlloc")
        allocs.append(d)
        _check(cu.cuMemcpyHtoD(d, a.ctypes.data, a.nbytes), "cuMemcpyHtoD")
        return _DevPtr(d)

    def dev_out(n):
        d = _check(cu.cuMemAlloc(max(4, 4 * n)), "cuMemAlloc")
        allocs.append(d)
        return _DevPtr(d)

    try:
        outs = [dev_out(nv) for _ in range(3)]
        idx = [dev_in(a, np.int32) for a in (valid_x, valid_y, valid_z)]
        rest = [dev_in(a, np.float32) for a in (img_r, img_i, x, y, z, ant, meas_r, meas_i, rxo)]
        cuda_sn_est(*outs, *idx, *rest, slope, wavelength, fft_spacing, nx, ny, nz, num_ant,
                    num_rx, nv, samples, is_ti)
        res = []
        for o in outs:
            h = np.empty(nv, np.float32)
            _check(cu.cuMemcpyDtoH(h.ctypes.data, o.ptr, 4 * nv), "cuMemcpyDtoH")
            res.append(h)
    finally:
        for d in allocs:
            cu.cuMemFree(d)
    return tuple(res)
