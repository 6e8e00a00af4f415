"""The RSDF restatement itself (CPU): on a constant normal field the breadth-first
integral is path independent and equals the signed distance to the seed's plane; the
components are a partition into 6-connected sets."""
import numpy as np

from oracle import rsdf_oracle as RO


def test_constant_normals_give_plane_distance():
    shape = (11, 9, 7)
    nrm = np.array([0.3, -0.5, 0.8])
    nrm /= np.linalg.norm(nrm)
    normals = np.broadcast_to(nrm, shape + (3,)).copy()
    dx = 0.01
    x = np.arange(shape[0]) * dx
    y = np.arange(shape[1]) * dx
    z = np.arange(shape[2]) * dx
    lab, mask = RO.components(normals)
    valid = RO.valid_labels(lab, mask, x)
    assert list(valid) == [2]
    coords = RO.coords(x, y, z)
    out = RO.rsdf(normals, coords, lab, valid, x)
    seed = np.argwhere(out == 0)[0]
    expect = (coords - coords[tuple(seed)]) @ nrm
    np.testing.assert_allclose(out, expect, atol=1e-12)


def test_components_partition():
    rng = np.random.default_rng(0)
    mask = rng.random((8, 9, 10)) > 0.55
    normals = np.where(mask[..., None], 1.0, np.nan) * np.ones(3)
    lab, m = RO.components(normals)
    assert np.all((lab >= 2) == mask) and np.all(lab[~mask] == 1)
    # 6-neighbours inside the mask share a label
    for ax in range(3):
        a = np.moveaxis(lab, ax, 0)
        b = np.moveaxis(mask, ax, 0)
        both = b[1:] & b[:-1]
        assert np.all(a[1:][both] == a[:-1][both])
    # labels numbered by first voxel in C order
    firsts = [np.flatnonzero(lab.ravel() == k)[0] for k in range(2, lab.max() + 1)]
    assert firsts == sorted(firsts)


def test_restatement_matches_reference_fixture():
    """The restatement against outputs of the reference's own functions
    (tests/golden/make_golden_next.py): labels, valid components, RSDF bit for bit."""
    from conftest import load_golden
    g = load_golden("rsdf_ref")
    for c in range(int(g["cases"])):
        p = "c%d_" % c
        normals, x, y, z = g[p + "normals"], g[p + "x"], g[p + "y"], g[p + "z"]
        lab, mask = RO.components(normals)
        np.testing.assert_array_equal(lab, g[p + "labeled"])
        valid = RO.valid_labels(lab, mask, x)
        np.testing.assert_array_equal(valid, g[p + "valid"])
        out = RO.rsdf(normals, RO.coords(x, y, z), lab, valid, x)
        ref = g[p + "rsdf"]
        np.testing.assert_array_equal(np.isnan(out), np.isnan(ref))
        np.testing.assert_array_equal(out[~np.isnan(ref)], ref[~np.isnan(ref)])
