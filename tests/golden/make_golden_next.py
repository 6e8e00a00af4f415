"""Golden fixtures for the steps after the normals, produced by running the reference's
OWN Python functions (not a restatement) on seeded inputs:

* sdf._find_connected_components and sdf._construct_rsdf_components
  (src/data_processing/sdf.py:94-224)                                  -> rsdf_ref.npz
* GenericLoader.load_radar_files, 77 GHz branch
  (src/utils/generic_loader.py:484-537)                                 -> ingest_ref.npz
* ImageProcessor.correlate_locs_and_meas
  (src/data_processing/image_processor.py:74-154)                       -> ingest_ref.npz

The reference modules import packages this image does not have; they are replaced in
sys.modules by stand-ins before the import, none of which takes part in the arithmetic
that is pinned:
  trimesh, PIL, skimage, open3d, matplotlib   (unused by these functions)
  cc3d.connected_components(mask, connectivity=6)
      -> scipy.ndimage.label with the 6-neighbour cross: the same partition; the label
         NUMBERS are scipy's (components numbered by first voxel in C order), so the
         numbering is the one thing here not pinned to cc3d
  data_processing.cuda.py_image_gpu / py_sn_est_gpu (pycuda; imported at module top)
utilities.get_radar_parameters is replaced by one returning each session's parameters
(the reference reads them from src/utils/params.json).

Usage:  python tests/golden/make_golden_next.py --ref-root <mmNorm checkout>
(or MMNORM_REF_ROOT in the environment).  Writes next to this file.
"""
from __future__ import annotations

import argparse
import importlib.util
import os
import sys
import tempfile
import types

import numpy as np
from scipy import ndimage

HERE = os.path.dirname(os.path.abspath(__file__))


def _stub(name, **attrs):
    mod = types.ModuleType(name)
    for k, v in attrs.items():
        setattr(mod, k, v)
    sys.modules[name] = mod
    return mod


def _cc3d_connected_components(mask, connectivity=6):
    assert connectivity == 6
    lab, _ = ndimage.label(mask, structure=ndimage.generate_binary_structure(3, 1))
    return lab


def _import_reference(ref_root, params):
    src = os.path.join(ref_root, "src")
    sys.path.insert(0, src)
    for name in ("trimesh", "open3d", "matplotlib", "matplotlib.pyplot"):
        _stub(name)
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    pil = _stub("PIL")
    pil.Image = _stub("PIL.Image")
    sk = _stub("skimage")
    sk.filters = _stub("skimage.filters")
    _stub("cc3d", connected_components=_cc3d_connected_components)
    _stub("data_processing.cuda.py_image_gpu")
    _stub("data_processing.cuda.py_sn_est_gpu")
    from utils import utilities
    utilities.load_param_json = lambda: {"processing": {"use_cuda": True}}
    utilities.get_radar_parameters = lambda radar_type="77_ghz", is_sim=False, \
        aperture_type="normal": dict(params)
    from utils import generic_loader
    from data_processing import image_processor
    spec = importlib.util.spec_from_file_location(
        "ref_sdf", os.path.join(src, "data_processing", "sdf.py"))
    sdf = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(sdf)
    return sdf, generic_loader, image_processor


def _normal_field(shape, seed, level, smooth=1.5):
    """Blobby mask from smoothed noise, float64 unit normals on it, NaN elsewhere."""
    rng = np.random.default_rng(seed)
    noise = ndimage.gaussian_filter(rng.standard_normal(shape), smooth)
    mask = noise > level * noise.std()
    n = rng.standard_normal(shape + (3,))
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    n[~mask] = np.nan
    return n


RSDF_CASES = [  # (shape, seed, level, dx): several components, boundary-touching ones
    ((16, 14, 12), 4, 0.2, 0.01),
    ((20, 9, 15), 5, -0.1, 0.006),
    ((12, 12, 24), 6, 0.0, 0.004),
    ((10, 10, 10), 7, -9.0, 0.01),   # one component filling the grid
    ((24, 20, 16), 8, 0.4, 0.01),    # several valid components searched one after another
]


def make_rsdf(sdf):
    out = {}
    for c, (shape, seed, level, dx) in enumerate(RSDF_CASES):
        normals = _normal_field(shape, seed, level)
        x = np.arange(shape[0]) * dx
        y = np.arange(shape[1]) * dx - 0.05
        z = np.arange(shape[2]) * dx + 0.3
        m1, m2, m3 = np.meshgrid(y, x, z)                       # sdf.py:283-284
        coords = np.concatenate((m2[..., None], m1[..., None], m3[..., None]), axis=-1)
        labeled, valid = sdf._find_connected_components(normals, x)
        rsdf = sdf._construct_rsdf_components(normals, coords, labeled, valid, x)
        p = "c%d_" % c
        out.update({p + "normals": normals, p + "x": x, p + "y": y, p + "z": z,
                    p + "labeled": labeled.astype(np.int32), p + "valid": np.asarray(valid),
                    p + "rsdf": rsdf})
        print("rsdf case %d: shape %s, %d components, %d valid, %d voxels with a value"
              % (c, shape, labeled.max() - 1, len(valid), int((~np.isnan(rsdf)).sum())))
    out["cases"] = np.array(len(RSDF_CASES))
    np.savez_compressed(os.path.join(HERE, "rsdf_ref.npz"), **out)


INGEST_PARAMS = dict(num_frames=40, num_samples=4, num_chirps=2, sweep_time=0.0004,
                     periodicity=0.003, min_f=77.5e9)


def _session(seed, dim):
    """Trajectory with pauses (repeated positions are dropped), rows of radar files with a
    missing timestamp, a missing file and a short file."""
    rng = np.random.default_rng(seed)
    p = INGEST_PARAMS
    n = 300
    times = 1.7e9 + np.cumsum(rng.uniform(0.001, 0.02, n))
    steps = rng.uniform(0, 1.2e-3, (n, 3)) * (rng.random((n, 1)) > 0.3)
    traj = np.concatenate([np.cumsum(steps, axis=0), rng.standard_normal((n, dim - 3))], axis=1)
    rows = 8
    names = [str(1000 + r) for r in range(rows)]
    created = list(times[0] + np.linspace(-0.3, times[-1] - times[0] - 0.05, rows))
    created[3] = -1
    radar = {}
    per_file = p["num_frames"] * p["num_samples"] * p["num_chirps"]
    for r, name in enumerate(names):
        if r == 5:
            continue
        length = per_file if r != 6 else 12 * p["num_samples"] * p["num_chirps"] + 3
        radar[int(name)] = (rng.integers(-2000, 2000, (length, 4)) +
                            1j * rng.integers(-2000, 2000, (length, 4))).astype(np.complex64)
    return names, created, radar, times, traj


SESSIONS = [(11, 3, False), (12, 7, False), (13, 3, True)]  # (seed, trajectory columns, optitrack)


def make_ingest(generic_loader, image_processor):
    out = {}
    # --- load_radar_files on a directory of .bin files (both name layouts, a non-.bin file)
    rng = np.random.default_rng(20)
    with tempfile.TemporaryDirectory() as tmp:
        d = os.path.join(tmp, "radar_data")
        os.makedirs(d)
        files = {"adc_data1700000001.bin": 8 * 37, "adc_data1700000042.bin": 8 * 5,
                 "adc_data_170000000123.bin": 8 * 64, "notes.txt": 10,
                 "adc_data1700000100.bin": 0}
        names = sorted(files)
        for k, name in enumerate(names):
            raw = rng.integers(-32768, 32768, files[name], dtype=np.int64).astype("<i2")
            with open(os.path.join(d, name), "wb") as f:
                f.write(raw.tobytes())
            out["file%d_name" % k] = np.array(name)
            out["file%d_raw" % k] = raw
        self_ = types.SimpleNamespace(_find_obj_angles=lambda: (0, 0, 0),
                                      _get_path=lambda *a, **kw: tmp)
        loaded = generic_loader.GenericLoader.load_radar_files(self_, "77_ghz")
        out["files"] = np.array(len(names))
        for i, (ts, arr) in enumerate(sorted(loaded.items())):
            out["loaded%d_ts" % i] = np.array(ts)
            out["loaded%d_data" % i] = arr
        out["loaded"] = np.array(len(loaded))
        print("load_radar_files: %d files -> %d arrays" % (len(names), len(loaded)))
    # --- correlate_locs_and_meas on seeded sessions
    proc = image_processor.ImageProcessor.__new__(image_processor.ImageProcessor)
    for s, (seed, dim, opti) in enumerate(SESSIONS):
        names, created, radar, times, traj = _session(seed, dim)
        proc.is_optitrack = opti
        proc.radar_type = "77_ghz"
        robot = {"all_radar_filenames": names, "all_radar_created_ts": created}
        locs = {"times_77": times, "tx_77_locs": traj}
        res = proc.correlate_locs_and_meas("77_ghz", robot, radar,
                                           {"aperture size": "normal"}, robot_loc_data=locs)
        p = "s%d_" % s
        out[p + "names"] = np.array(names)
        out[p + "created"] = np.array(created, np.float64)
        out[p + "times"] = times
        out[p + "traj"] = traj
        out[p + "optitrack"] = np.array(opti)
        out[p + "file_keys"] = np.array(sorted(radar), np.int64)
        for key in sorted(radar):
            out[p + "file_%d" % key] = radar[key]
        out[p + "poses"] = np.asarray(res["poses"], np.float64)
        out[p + "radar"] = np.asarray(res["radar_data"]).astype(np.complex64)
        print("session %d: %d frames kept" % (s, len(res["radar_data"])))
    out["sessions"] = np.array(len(SESSIONS))
    for k, v in INGEST_PARAMS.items():
        out["param_" + k] = np.array(v)
    np.savez_compressed(os.path.join(HERE, "ingest_ref.npz"), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get("MMNORM_REF_ROOT"))
    args = ap.parse_args()
    if not args.ref_root or not os.path.isdir(args.ref_root):
        raise SystemExit("pass --ref-root (or MMNORM_REF_ROOT): the mmNorm checkout")
    sdf, generic_loader, image_processor = _import_reference(args.ref_root, INGEST_PARAMS)
    make_rsdf(sdf)
    make_ingest(generic_loader, image_processor)


if __name__ == "__main__":
    main()
