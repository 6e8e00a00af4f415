"""torch.ops.mmnorm.* registration: schemas and fake (meta) shape propagation on CPU;
on the GPU the operators must return what mmnorm_b200.ops returns and the registered
autograd formula must give the adjoint kernels' gradients."""
import numpy as np
import pytest
import torch

import mmnorm_b200.torch_ops  # noqa: F401  (registers the operators)
from mmnorm_b200 import scenes


def test_operators_registered_with_fake_shapes():
    from torch._subclasses.fake_tensor import FakeTensorMode
    for name in ("backproject", "backproject_backward", "backproject_normals"):
        assert hasattr(torch.ops.mmnorm, name)
    with FakeTensorMode():
        x, y, z = torch.empty(4), torch.empty(5), torch.empty(6)
        ant, rxo = torch.empty(7, 3), torch.empty(1, 3)
        m = torch.empty(7, 32, dtype=torch.complex64)
        i, v = torch.ops.mmnorm.backproject(x, y, z, ant, rxo, m, 4e-3, 1e8, "mixed", 0.0,
                                            False, None)
        assert i.shape == (4, 5, 6) and v.shape == (3, 4, 5, 6) and i.dtype == torch.complex64
        out = torch.ops.mmnorm.backproject_normals(x, y, z, ant, rxo, m, 4e-3, 1e8, "mixed",
                                                   0.0, False, 0.05)
        assert [tuple(o.shape) for o in out] == [(4, 5, 6), (3, 4, 5, 6), (4, 5, 6, 3),
                                                 (4, 5, 6)]
        gm, gp = torch.ops.mmnorm.backproject_backward(x, y, z, ant, rxo, m, 4e-3, 1e8, False,
                                                       None, i, v)
        assert gm.shape == (7, 32) and gp.shape == (7, 3)
        imgs, votes = torch.ops.mmnorm.backproject_batched(
            [x, y], [y, z], [z, x], [ant, ant], [rxo, rxo], [m, m], [4e-3, 4e-3], [1e8, 1e8],
            [False, True], 8)
        assert [tuple(t.shape) for t in imgs] == [(4, 5, 6), (5, 6, 4)]
        assert tuple(votes[1].shape) == (3, 5, 6, 4)


@pytest.mark.gpu
def test_operators_match_ops_and_autograd(cuda_dev):
    from mmnorm_b200 import ops
    sc = scenes.sphere_scene(seed=9, n_ap=8, nf=40, n_vox=8, n_pts=20)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    x, y, z, ant = t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs)
    rxo = t(np.zeros((1, 3), np.float32))
    rng = np.random.default_rng(9)
    pos0 = t(rng.normal(0, 5e-4, sc.antenna_locs.shape).astype(np.float32))
    i0, v0 = ops.backproject(x, y, z, ant, rxo, t(sc.meas), sc.wavelength, sc.slope)
    i1, v1 = torch.ops.mmnorm.backproject(x, y, z, ant, rxo, t(sc.meas), sc.wavelength,
                                          sc.slope, "mixed", 0.0, False, None)
    assert torch.equal(i0, i1) and torch.equal(v0, v1)
    out = torch.ops.mmnorm.backproject_normals(x, y, z, ant, rxo, t(sc.meas), sc.wavelength,
                                               sc.slope, "mixed", 0.0, False, 0.05)
    n0, m0 = ops.surface_normals(i0, v0, 0.05)
    assert torch.equal(out[3], m0)
    assert torch.equal(torch.nan_to_num(out[2], 3.0), torch.nan_to_num(n0, 3.0))

    def loss(img, vote):
        return (img.abs() ** 2).sum() * 1e-6 + (vote.real ** 2).sum() * 1e-9

    grads = []
    for use_op in (True, False):
        meas = t(sc.meas).requires_grad_(True)
        pos = pos0.clone().requires_grad_(True)
        if use_op:
            img, vote = torch.ops.mmnorm.backproject(x, y, z, ant, rxo, meas, sc.wavelength,
                                                     sc.slope, "mixed", 0.0, False, pos)
        else:
            img, vote = ops.backproject_differentiable(x, y, z, ant, rxo, meas, sc.wavelength,
                                                       sc.slope, pos_offsets=pos)
        loss(img, vote).backward()
        grads.append((meas.grad.clone(), pos.grad.clone()))
    assert torch.equal(grads[0][0], grads[1][0]) and torch.equal(grads[0][1], grads[1][1])

    # the batched operator: the same results as a BatchPlan over the same objects
    objs = [dict(x_locs=x, y_locs=y, z_locs=z, antenna_locs=ant, rx_offsets=rxo,
                 meas=t(sc.meas), wavelength=sc.wavelength, slope=sc.slope),
            dict(x_locs=x[:5].contiguous(), y_locs=y, z_locs=z, antenna_locs=ant[:30].contiguous(),
                 rx_offsets=rxo, meas=t(sc.meas[:30]), wavelength=sc.wavelength, slope=sc.slope)]
    plan = ops.BatchPlan(objs, items_per_slot=8)
    plan.run()
    ref = plan.results()
    imgs, votes = torch.ops.mmnorm.backproject_batched(
        [o["x_locs"] for o in objs], [o["y_locs"] for o in objs], [o["z_locs"] for o in objs],
        [o["antenna_locs"] for o in objs], [o["rx_offsets"] for o in objs],
        [o["meas"] for o in objs], [sc.wavelength] * 2, [sc.slope] * 2, [False, False], 8)
    for (ri, rv), gi, gv in zip(ref, imgs, votes):
        assert torch.equal(ri, gi) and torch.equal(rv, gv)
