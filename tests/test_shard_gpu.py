"""The slab epilogue entry points on one GPU: two x-slabs imaged separately, their
maxima combined as the all-reduce would, and each slab's normals finished against the
global maximum must reproduce the whole-grid image, mask and normals."""
import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu


def test_two_slabs_match_whole_grid(cuda_dev):
    import torch
    from mmnorm_b200 import ops, shard
    sc = scenes.sphere_scene(seed=5, n_ap=16, nf=64, n_vox=20, spacing=3e-3, n_pts=60)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    x, y, z = t(sc.x_locs), t(sc.y_locs), t(sc.z_locs)
    ant, rxo, meas = t(sc.antenna_locs), t(np.zeros((1, 3), np.float32)), t(sc.meas)
    img, vote = ops.backproject(x, y, z, ant, rxo, meas, sc.wavelength, sc.slope)
    nrm, mask = ops.surface_normals(img, vote, 0.05)
    m_all = ops.image_max_abs(img)
    torch.cuda.synchronize()
    assert float(m_all) == float(img.abs().max())

    parts = []
    for r in range(2):
        x0, x1 = shard.split_bounds(x.numel(), 2, r)
        parts.append(ops.backproject(x[x0:x1].contiguous(), y, z, ant, rxo, meas,
                                     sc.wavelength, sc.slope))
    mx = torch.maximum(ops.image_max_abs(parts[0][0]), ops.image_max_abs(parts[1][0]))
    outs = [ops.surface_normals_from_max(i, v, mx, 0.05) for i, v in parts]
    torch.cuda.synchronize()
    img2 = torch.cat([p[0] for p in parts], 0)
    rel = float((img2 - img).abs().norm() / img.abs().norm())
    assert rel <= 2e-5
    # the maximum is taken over slightly different sums: allow for voxels at the threshold
    mask2 = torch.cat([o[1] for o in outs], 0)
    mag = img.abs()
    thr = 0.05 * float(m_all)
    border = (mag - thr).abs() <= 1e-4 * thr
    assert bool(((mask2 == mask) | border).all())
    both = mask & mask2
    n2 = torch.cat([o[0] for o in outs], 0)
    cos = (n2[both] * nrm[both]).sum(-1).clamp(-1, 1)
    assert float(torch.rad2deg(torch.arccos(cos)).max()) < 0.05


def test_sharded_single_rank_equals_ops(cuda_dev):
    import torch
    from mmnorm_b200 import ops, shard
    sc = scenes.sphere_scene(seed=6, n_ap=12, nf=40, n_vox=12, spacing=4e-3, n_pts=40)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    args = (t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs),
            t(np.zeros((1, 3), np.float32)), t(sc.meas), sc.wavelength, sc.slope)
    res = shard.surface_normals(*args)
    img, vote = ops.backproject(*args)
    nrm, mask = ops.surface_normals(img, vote, 0.05)
    torch.cuda.synchronize()
    assert torch.equal(res["image"], img) and torch.equal(res["mask"], mask)
    assert torch.equal(torch.nan_to_num(res["normals"], 7.0), torch.nan_to_num(nrm, 7.0))


def test_sharded_backward_single_rank_equals_ops(cuda_dev):
    """One rank: both decompositions of the sharded adjoint are the library's adjoint."""
    import torch
    from mmnorm_b200 import ops, shard
    sc = scenes.sphere_scene(seed=8, n_ap=10, nf=40, n_vox=10, spacing=4e-3, n_pts=30)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=cuda_dev)
    args = (t(sc.x_locs), t(sc.y_locs), t(sc.z_locs), t(sc.antenna_locs),
            t(np.zeros((1, 3), np.float32)), t(sc.meas), sc.wavelength, sc.slope)
    rng = np.random.default_rng(8)
    V = sc.num_voxels
    gI = t((rng.standard_normal(V) + 1j * rng.standard_normal(V)).astype(np.complex64))
    gW = t((rng.standard_normal((3, V)) + 1j * rng.standard_normal((3, V))).astype(np.complex64))
    shp = (len(sc.x_locs), len(sc.y_locs), len(sc.z_locs))
    gm, gp = ops.backproject_backward(*args, gI, gW)
    for dec in ("slabs", "antennas"):
        gm2, gp2 = shard.backproject_backward(*args, gI.view(shp), gW.view((3,) + shp),
                                              decomposition=dec)
        torch.cuda.synchronize()
        assert torch.equal(gm, gm2) and torch.equal(gp, gp2), dec
