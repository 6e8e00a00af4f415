"""Size-independent properties at the full workload sizes, where the oracle cannot run the
whole grid: the fused image and vote are linear in the measurements (128^3 voxels,
128x128 antennas, 256 frequencies), the plain and mixed forms agree within the plain
form's FP32 range error, and the adjoint satisfies <gI, I(m)> = <dL/dm, m> on the 64^3 /
64x64 / 128 differentiation workload.  (The oracle checks of the same sizes run on voxel
subsets in test_accuracy_gpu.py.)"""
import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float((a - b).abs().norm() / b.abs().norm())


def test_linearity_at_full_workload(cuda_dev):
    import torch
    from mmnorm_b200 import ops
    sc = scenes.config1(sign=-1, device=cuda_dev)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    x, y, z, ant = t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs)
    rxo = t(np.zeros((1, 3), np.float32))
    m1 = t(sc.meas)
    g = torch.Generator(device=cuda_dev).manual_seed(5)
    m2 = (torch.randn(m1.shape, generator=g, device=cuda_dev) +
          1j * torch.randn(m1.shape, generator=g, device=cuda_dev)).to(torch.complex64)
    a, b = 0.75 - 0.25j, -1.5 + 0.5j
    m3 = (a * m1 + b * m2).to(torch.complex64)
    i1, v1 = ops.backproject(x, y, z, ant, rxo, m1, sc.wavelength, sc.slope)
    i2, v2 = ops.backproject(x, y, z, ant, rxo, m2, sc.wavelength, sc.slope)
    i3, v3 = ops.backproject(x, y, z, ant, rxo, m3, sc.wavelength, sc.slope)
    torch.cuda.synchronize()
    assert _rel(i3, a * i1 + b * i2) < 2e-5
    assert _rel(v3, a * v1 + b * v2) < 2e-5
    # the plain FP32 form against the mixed form on the same inputs (FP32 range: ~1e-4)
    ip, vp = ops.backproject(x, y, z, ant, rxo, m1, sc.wavelength, sc.slope, mode="plain")
    torch.cuda.synchronize()
    assert _rel(ip, i1) < 1e-3


def test_adjoint_identity_at_differentiation_workload(cuda_dev):
    import torch
    from mmnorm_b200 import ops
    sc = scenes.config3(sign=+1, device=cuda_dev)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    args = [t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs),
            t(np.zeros((1, 3), np.float32)), t(sc.meas)]
    V = sc.num_voxels
    g = torch.Generator(device=cuda_dev).manual_seed(11)
    gI = (torch.randn(V, generator=g, device=cuda_dev) +
          1j * torch.randn(V, generator=g, device=cuda_dev)).to(torch.complex64)
    gW = (torch.randn((3, V), generator=g, device=cuda_dev) +
          1j * torch.randn((3, V), generator=g, device=cuda_dev)).to(torch.complex64)
    I, W = ops.backproject(*args, sc.wavelength, sc.slope)
    gm, _ = ops.backproject_backward(*args, sc.wavelength, sc.slope, gI, gW, want_pos=False)
    torch.cuda.synchronize()
    c128 = torch.complex128
    lhs = ((gI.conj().to(c128) * I.reshape(-1).to(c128)).sum() +
           (gW.conj().to(c128) * W.reshape(3, -1).to(c128)).sum()).real
    rhs = (gm.conj().to(c128) * args[5].to(c128)).sum().real
    assert abs(float(lhs - rhs)) <= 1e-4 * abs(float(lhs))
