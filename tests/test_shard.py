"""Multi-process logic of the sharded imaging path (mmnorm_b200.shard) on CPU ranks
(gloo), with the FP64 oracle standing in for the kernels: slab and antenna
decompositions must reproduce the single-process result, the normal mask must use the
maximum over the whole grid (not the slab's), and ranks with empty slabs must still
take part in every collective."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch

from mmnorm_b200 import scenes, shard


class OracleBackend:
    """CPU stand-in for shard.CudaBackend: the FP64 oracle, results rounded to the
    kernels' output types."""

    def __init__(self):
        from oracle import oracle as O
        self.O = O

    def backproject(self, x, y, z, ant, rxo, meas, wavelength, slope, **kw):
        xs, ys, zs = x.numpy(), y.numpy(), z.numpy()
        X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
        vox = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
        I, W = self.O.full(vox, ant.numpy(), rxo.numpy(), meas.numpy(), wavelength, slope)
        shp = (len(xs), len(ys), len(zs))
        return (torch.from_numpy(I.astype(np.complex64)).view(shp),
                torch.from_numpy(np.ascontiguousarray(W.T).astype(np.complex64)).view((3,) + shp))

    def max_abs(self, image):
        return image.abs().max().reshape(1).to(torch.float32)

    def backward(self, x, y, z, ant, rxo, meas, wavelength, slope, grad_image, grad_vote,
                 pos_offsets=None, is_ti_radar=False):
        X, Y, Z = np.meshgrid(x.numpy(), y.numpy(), z.numpy(), indexing="ij")
        vox = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
        a = ant.numpy().astype(np.float64)
        if pos_offsets is not None:
            a = a + pos_offsets.numpy()
        gI = grad_image.reshape(-1).numpy().astype(np.complex128)
        gW = (np.zeros((gI.size, 3), np.complex128) if grad_vote is None else
              grad_vote.reshape(3, -1).numpy().T.astype(np.complex128))
        gm, gp = self.O.full_backward(vox, a.astype(np.float32), rxo.numpy(), meas.numpy(),
                                      wavelength, slope, gI, gW, is_ti=is_ti_radar)
        return (torch.from_numpy(gm.astype(np.complex64)),
                torch.from_numpy(gp.astype(np.float32)))

    def normals_from_max(self, image, vote, max_abs, filter_percent):
        shp = tuple(image.shape)
        I = image.reshape(-1).numpy()
        W = vote.reshape(3, -1).numpy().T
        mag = np.abs(I)
        mask = mag > np.float32(max_abs.item()) * np.float32(filter_percent)
        raw = np.real(np.conj(I)[:, None] * W) / np.where(mag > 0, mag, 1)[:, None]
        unit = (raw / np.linalg.norm(raw, axis=1, keepdims=True)).astype(np.float32)
        unit[~mask] = np.nan
        return torch.from_numpy(unit).view(shp + (3,)), torch.from_numpy(mask).view(shp)


def _inputs(nx=6):
    sc = scenes.sphere_scene(seed=7, n_ap=6, nf=24, n_vox=5, spacing=6e-3, n_pts=30)
    # x-planes in two groups 0.3 m apart around the sphere's near cap (z = 0.35 m): the
    # two groups' maxima differ by an order of magnitude, so a slab-local mask would differ
    x = np.concatenate([sc.x_locs[:3], sc.x_locs[:3] + 0.3])[:nx].astype(np.float32)
    z = (0.35 + 6e-3 * np.arange(-2, 3)).astype(np.float32)
    t = torch.from_numpy
    return dict(x_locs=t(x), y_locs=t(sc.y_locs), z_locs=t(z),
                antenna_locs=t(sc.antenna_locs), rx_offsets=t(np.zeros((1, 3), np.float32)),
                meas=t(sc.meas), wavelength=sc.wavelength, slope=sc.slope)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, decomposition, nx):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        res = shard.surface_normals(**_inputs(nx), decomposition=decomposition, gather=True,
                                    backend=OracleBackend())
        np.savez(os.path.join(out_dir, "r%d.npz" % rank),
                 image=res["image"].numpy(), vote=res["vote"].numpy(),
                 normals=res["normals"].numpy(), mask=res["mask"].numpy(),
                 max_abs=res["max_abs"].numpy(), x_range=np.array(res["x_range"]))
    finally:
        dist.destroy_process_group()


def _run(world, decomposition, nx=6):
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(world, _free_port(), d, decomposition, nx), nprocs=world)
        return [dict(np.load(os.path.join(d, "r%d.npz" % r))) for r in range(world)]


def _single(nx=6):
    res = shard.surface_normals(**_inputs(nx), backend=OracleBackend())
    return {k: (v.numpy() if isinstance(v, torch.Tensor) else v) for k, v in res.items()}


def test_split_bounds_cover_and_balance():
    for n in range(0, 40):
        for world in range(1, 9):
            b = [shard.split_bounds(n, world, r) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
            sizes = [e - s for s, e in b]
            assert max(sizes) - min(sizes) <= 1
    b = [shard.split_bounds(12, 5, r, unit=4) for r in range(5)]
    assert all(s % 4 == 0 and e % 4 == 0 for s, e in b)
    with pytest.raises(ValueError):
        shard.split_bounds(10, 2, 0, unit=4)


def test_slabs_two_ranks_match_single_process(oracle):
    ref = _single()
    outs = _run(2, "slabs")
    # rank 0's slab maximum is well below the grid's: its slab-local mask would differ
    mags = np.abs(ref["image"])
    local_mask = mags[:3] > 0.05 * mags[:3].max()
    assert (local_mask != ref["mask"][:3]).any()
    for o in outs:
        assert tuple(o["x_range"]) == (0, 6)
        np.testing.assert_array_equal(o["image"], ref["image"])
        np.testing.assert_array_equal(o["vote"], ref["vote"])
        np.testing.assert_array_equal(o["mask"], ref["mask"])
        np.testing.assert_array_equal(o["normals"], ref["normals"])   # NaN == NaN here
        assert o["max_abs"][0] == ref["max_abs"][0]


def test_slabs_with_empty_ranks(oracle):
    ref = _single(nx=2)
    outs = _run(3, "slabs", nx=2)            # rank 2 owns no x-plane
    for o in outs:
        np.testing.assert_array_equal(o["image"], ref["image"])
        np.testing.assert_array_equal(o["mask"], ref["mask"])


def test_antennas_two_ranks_match_single_process(oracle):
    ref = _single()
    outs = _run(2, "antennas")
    for o in outs:
        rel = np.linalg.norm(o["image"] - ref["image"]) / np.linalg.norm(ref["image"])
        assert rel < 1e-6
        relw = np.linalg.norm(o["vote"] - ref["vote"]) / np.linalg.norm(ref["vote"])
        assert relw < 1e-6
        m = ref["mask"]
        np.testing.assert_array_equal(o["mask"], m)
        np.testing.assert_allclose(o["normals"][m], ref["normals"][m], atol=1e-5)


def _grads(nx):
    rng = np.random.default_rng(nx)
    shp = (nx, 5, 5)
    gI = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(np.complex64)
    gW = (rng.standard_normal((3,) + shp) + 1j * rng.standard_normal((3,) + shp)).astype(np.complex64)
    pos = rng.normal(0, 5e-4, (36, 3)).astype(np.float32)
    return torch.from_numpy(gI), torch.from_numpy(gW), torch.from_numpy(pos)


def _bwd_worker(rank, world, port, out_dir, decomposition, nx):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        gI, gW, pos = _grads(nx)
        gm, gp = shard.backproject_backward(**_inputs(nx), grad_image=gI, grad_vote=gW,
                                            decomposition=decomposition, pos_offsets=pos,
                                            backend=OracleBackend())
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), gm=gm.numpy(), gp=gp.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("decomposition,world,nx", [("slabs", 2, 6), ("slabs", 3, 2),
                                                    ("antennas", 2, 6)])
def test_sharded_backward_matches_single_process(decomposition, world, nx):
    """The adjoint split over ranks gives every rank the single-process gradients: slab
    partial sums all-reduced (an empty slab at world 3 with 2 planes still joins the
    collective), antenna rows all-gathered (each row computed whole: bitwise equal)."""
    import torch.multiprocessing as mp
    gI, gW, pos = _grads(nx)
    gm1, gp1 = shard.backproject_backward(**_inputs(nx), grad_image=gI, grad_vote=gW,
                                          pos_offsets=pos, backend=OracleBackend())
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_bwd_worker, args=(world, _free_port(), d, decomposition, nx), nprocs=world)
        res = [dict(np.load(os.path.join(d, "r%d.npz" % r))) for r in range(world)]
    for r in res:
        assert r["gm"].shape == tuple(gm1.shape) and r["gp"].shape == tuple(gp1.shape)
        if decomposition == "antennas":
            np.testing.assert_array_equal(r["gm"], gm1.numpy())
            np.testing.assert_array_equal(r["gp"], gp1.numpy())
        else:
            rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
            assert rel(r["gm"], gm1.numpy()) < 1e-6 and rel(r["gp"], gp1.numpy()) < 1e-5
        np.testing.assert_array_equal(r["gm"], res[0]["gm"])  # every rank holds the same
