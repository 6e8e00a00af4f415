"""Batched persistent launch (one kernel over a cost-sorted (object, voxel tile, antenna
split) work list): every object's image and vote must match its individually launched
result within the mixed form's tolerance, for several work granularities (which change
the antenna splits), under CUDA-graph capture and replay, and for every kernel variant
that has a persistent form."""
import numpy as np
import pytest

from mmnorm_b200 import scenes

pytestmark = pytest.mark.gpu
TOL = 2e-5


def _objects(dev):
    import torch
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    specs = [  # (seed, aperture side, F, grid side, spacing, R, ti)
        (1, 8, 64, 12, 4e-3, 1, False),
        (2, 12, 17, 9, 3e-3, 1, False),
        (3, 6, 100, 16, 2e-3, 2, True),
        (4, 7, 40, 10, 4e-3, 1, False),     # 49 antennas: odd count
        (5, 16, 96, 8, 3e-3, 1, False),
        (6, 10, 33, 20, 2e-3, 3, True),
    ]
    objs, scs = [], []
    for seed, n_ap, nf, n_vox, sp, R, ti in specs:
        sc = scenes.sphere_scene(seed=seed, n_ap=n_ap, nf=nf, n_vox=n_vox, spacing=sp, n_pts=20)
        ant = np.repeat(sc.antenna_locs, R, axis=0)
        rng = np.random.default_rng(seed)
        meas = np.repeat(sc.meas, R, axis=0) * np.exp(1j * rng.uniform(0, 6.28, (ant.shape[0], 1)))
        rxo = np.array([[0.0, -0.005 - 0.0019 * k, 0.0] for k in range(R)], np.float32) \
            if R > 1 else np.zeros((1, 3), np.float32)
        objs.append(dict(x_locs=t(sc.x_locs), y_locs=t(sc.y_locs), z_locs=t(sc.z_locs),
                         antenna_locs=t(ant.astype(np.float32)), rx_offsets=t(rxo),
                         meas=t(meas.astype(np.complex64)), wavelength=sc.wavelength,
                         slope=sc.slope, is_ti_radar=ti))
    # an object with an empty aperture
    o = dict(objs[0])
    o["antenna_locs"] = t(np.zeros((0, 3), np.float32))
    o["meas"] = t(np.zeros((0, 64), np.complex64))
    objs.append(o)
    return objs


def _individual(objs):
    from mmnorm_b200 import ops
    out = []
    for ob in objs:
        img, vote = ops.backproject(ob["x_locs"], ob["y_locs"], ob["z_locs"], ob["antenna_locs"],
                                    ob["rx_offsets"], ob["meas"], ob["wavelength"], ob["slope"],
                                    is_ti_radar=ob["is_ti_radar"])
        out.append((img.clone(), vote.clone()))
    return out


def _rel(a, b):
    import torch
    nb = float(b.abs().norm())
    return float((a - b).abs().norm()) / nb if nb > 0 else float(a.abs().norm())


@pytest.mark.parametrize("items_per_slot", [1, 8, 64])
def test_batched_matches_individual(cuda_dev, items_per_slot):
    import torch
    from mmnorm_b200 import ops
    objs = _objects(cuda_dev)
    ref = _individual(objs)
    plan = ops.BatchPlan(objs, items_per_slot=items_per_slot)
    plan.run()
    torch.cuda.synchronize()
    info = plan.info()
    assert info["items"] > 0
    for (img, vote), (ri, rv) in zip(plan.results(), ref):
        assert _rel(img, ri) <= TOL
        assert _rel(vote, rv) <= TOL


def test_batched_graph_replay(cuda_dev):
    import torch
    from mmnorm_b200 import ops
    objs = _objects(cuda_dev)
    plan = ops.BatchPlan(objs, items_per_slot=16)
    plan.run()
    torch.cuda.synchronize()
    first = [(i.clone(), v.clone()) for i, v in plan.results()]
    for im in plan.images:
        im.zero_()
    plan.capture()
    for _ in range(2):
        plan.replay()
        torch.cuda.synchronize()
        for (img, vote), (fi, fv) in zip(plan.results(), first):
            assert torch.equal(img, fi) and torch.equal(vote, fv)


def test_batched_every_persistent_variant(cuda_dev):
    import torch
    from mmnorm_b200 import ops
    objs = _objects(cuda_dev)[:4]
    ref = _individual(objs)
    try:
        for v in ops.variants("mixed"):
            ops.set_variant("mixed", v["index"])
            plan = ops.BatchPlan(objs, items_per_slot=8)
            plan.run()
            torch.cuda.synchronize()
            for (img, vote), (ri, rv) in zip(plan.results(), ref):
                assert _rel(img, ri) <= TOL, v["name"]
                assert _rel(vote, rv) <= TOL, v["name"]
    finally:
        ops.set_variant("mixed", 0)
