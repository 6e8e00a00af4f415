"""GPU connected components and RSDF (mmnorm_b200.rsdf) against the restatement of
sdf.py's steps in oracle/rsdf_oracle.py: the same component partition (root = smallest
flat index), the same labels and valid components, and RSDF values equal bit for bit."""
import numpy as np
import pytest
from scipy import ndimage

pytestmark = pytest.mark.gpu


def _field(shape, seed, level=0.2, smooth=1.5):
    """Blobby mask from smoothed noise, random float64 unit normals on it, NaN elsewhere."""
    rng = np.random.default_rng(seed)
    noise = ndimage.gaussian_filter(rng.standard_normal(shape), smooth)
    mask = noise > level * noise.std()
    n = rng.standard_normal(shape + (3,))
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    n[~mask] = np.nan
    return n, mask


@pytest.mark.parametrize("shape,seed", [((20, 17, 13), 1), ((9, 31, 7), 2), ((1, 5, 40), 3)])
def test_components_match_scipy(cuda_dev, shape, seed):
    import torch
    from mmnorm_b200 import rsdf
    _, mask = _field(shape, seed)
    root, count = rsdf.component_roots(torch.as_tensor(mask, device=cuda_dev))
    root, count = root.cpu().numpy(), count.cpu().numpy()
    lab, n = ndimage.label(mask, structure=ndimage.generate_binary_structure(3, 1))
    assert np.all((root >= 0) == mask)
    flat_idx = np.arange(mask.size).reshape(shape)
    for k in range(1, n + 1):
        sel = lab == k
        assert np.all(root[sel] == flat_idx[sel].min())
        assert count[flat_idx[sel].min()] == sel.sum()
    assert count.sum() == mask.sum()


@pytest.mark.parametrize("shape,seed,dx", [((16, 14, 12), 4, 0.01), ((24, 24, 24), 5, 0.01),
                                           ((30, 9, 20), 6, 0.006)])
def test_rsdf_matches_sequential_search(cuda_dev, shape, seed, dx):
    from oracle import rsdf_oracle as RO
    from mmnorm_b200 import rsdf
    normals, _ = _field(shape, seed, level=-0.1)
    x = np.arange(shape[0]) * dx
    y = np.arange(shape[1]) * dx - 0.05
    z = np.arange(shape[2]) * dx + 0.3
    out, labeled, valid, coords = rsdf.compute_rsdf(normals, x, y, z)
    lab_o, mask_o = RO.components(normals)
    valid_o = RO.valid_labels(lab_o, mask_o, x)
    np.testing.assert_array_equal(labeled, lab_o)
    np.testing.assert_array_equal(valid, valid_o)
    assert len(valid) > 0
    ref = RO.rsdf(normals, RO.coords(x, y, z), lab_o, valid_o, x)
    np.testing.assert_array_equal(np.isnan(out), np.isnan(ref))
    np.testing.assert_array_equal(out[~np.isnan(ref)], ref[~np.isnan(ref)])


def test_rsdf_one_large_component(cuda_dev):
    """A 48^3 slab-shaped component: deep search, frontiers over a thousand voxels (the
    multi-block scan), every voxel reached."""
    from oracle import rsdf_oracle as RO
    from mmnorm_b200 import rsdf
    shape = (48, 48, 48)
    rng = np.random.default_rng(7)
    n = rng.standard_normal(shape + (3,))
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    dx = 0.004
    x = np.arange(48) * dx
    out, labeled, valid, _ = rsdf.compute_rsdf(n, x, x, x)
    assert len(valid) == 1 and not np.isnan(out).any()
    ref = RO.rsdf(n, RO.coords(x, x, x), labeled, valid, x)
    np.testing.assert_array_equal(out, ref)


def test_rsdf_matches_reference_fixture(cuda_dev):
    """Against outputs of the reference's own sdf._find_connected_components and
    sdf._construct_rsdf_components (tests/golden/make_golden_next.py; cc3d's partition
    from scipy): the same labels, valid components and RSDF values, bit for bit."""
    from conftest import load_golden
    from mmnorm_b200 import rsdf
    g = load_golden("rsdf_ref")
    for c in range(int(g["cases"])):
        p = "c%d_" % c
        out, labeled, valid, _ = rsdf.compute_rsdf(g[p + "normals"], g[p + "x"], g[p + "y"],
                                                   g[p + "z"])
        np.testing.assert_array_equal(labeled, g[p + "labeled"])
        np.testing.assert_array_equal(valid, g[p + "valid"])
        ref = g[p + "rsdf"]
        np.testing.assert_array_equal(np.isnan(out), np.isnan(ref))
        np.testing.assert_array_equal(out[~np.isnan(ref)], ref[~np.isnan(ref)])
