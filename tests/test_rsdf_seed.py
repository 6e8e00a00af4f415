"""CPU checks of the RSDF host steps that pick each component's start voxel (no GPU).

compute_rsdf takes the start voxel of every component from that component's own voxel list
(flat indices in C order) instead of masking the whole coordinate grid; the rows, their
order and dtype are the same, so numpy's mean / norm / argmin -- and the chosen voxel --
must be identical to the reference's formulation (sdf.py:187-193), restated by rsdf._seed.
The coordinate grid itself is built by broadcasting instead of meshgrid + concatenate."""
import numpy as np
import pytest
from scipy import ndimage

from mmnorm_b200 import rsdf


def _axes(rng, n, dtype):
    return tuple(np.sort(rng.uniform(-0.1, 0.1, k)).astype(dtype) for k in n)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_coordinate_grid_matches_meshgrid(dtype):
    rng = np.random.default_rng(1)
    x, y, z = _axes(rng, (5, 7, 3), dtype)
    m1, m2, m3 = np.meshgrid(y, x, z)
    ref = np.concatenate((m2[..., None], m1[..., None], m3[..., None]), axis=-1)
    got = rsdf.coordinate_grid(x, y, z)
    assert got.dtype == ref.dtype and np.array_equal(got, ref)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_seed_from_voxel_list_matches_reference_formulation(dtype):
    rng = np.random.default_rng(2)
    shape = (24, 20, 16)
    x, y, z = _axes(rng, shape, dtype)
    coords = rsdf.coordinate_grid(x, y, z)
    for trial in range(6):
        mask = ndimage.binary_dilation(rng.random(shape) > 0.985, iterations=2)
        labels, count = ndimage.label(mask)
        normals = np.full(shape + (3,), np.nan)
        normals[mask] = 1.0
        labeled = np.where(mask, labels + 1, 1)
        for comp in range(2, count + 2):
            ref = tuple(rsdf._seed(normals, coords, labeled, comp))
            flat = np.flatnonzero(labeled == comp)  # ascending = C order
            got = np.unravel_index(rsdf._seed_from_voxels(flat, shape, (x, y, z)), shape)
            assert tuple(int(v) for v in got) == tuple(int(v) for v in ref), (trial, comp)


def test_seed_ties_resolve_to_the_first_voxel():
    # a symmetric component: several voxels at the same distance from the mean
    shape = (5, 5, 5)
    x = y = z = np.arange(5, dtype=np.float64) * 0.002
    coords = rsdf.coordinate_grid(x, y, z)
    mask = np.zeros(shape, bool)
    mask[1:4, 1:4, 2] = True
    mask[2, 2, 2] = False  # a ring: the mean falls in the hole
    normals = np.full(shape + (3,), np.nan)
    normals[mask] = 1.0
    labeled = np.where(mask, 2, 1)
    ref = tuple(int(v) for v in rsdf._seed(normals, coords, labeled, 2))
    got = np.unravel_index(rsdf._seed_from_voxels(np.flatnonzero(mask), shape, (x, y, z)), shape)
    assert tuple(int(v) for v in got) == ref
