"""Raw radar ingest (mmnorm_b200.ingest) against the restatement of the reference's
loader and frame correlation (oracle/ingest_oracle.py): ADC samples exactly, the same kept
frames in the same order, positions bit for bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_adc_unpack_exact(cuda_dev):
    from oracle import ingest_oracle as IO
    from mmnorm_b200 import ingest
    rng = np.random.default_rng(0)
    raw = rng.integers(-32768, 32767, 8 * 1000, dtype=np.int16).astype("<i2").tobytes()
    got = ingest.unpack_adc(raw).cpu().numpy()
    ref = IO.unpack(raw)
    assert got.shape == ref.shape == (1000, 4)
    np.testing.assert_array_equal(got.astype(np.complex128), ref)
    with pytest.raises(ValueError):  # not whole rows: the reference's reshape refuses it
        ingest.unpack_adc(raw + b"\x01\x00")
    assert ingest.unpack_adc(b"").shape == (0, 4)


def _session(seed, dim, frames=60, samples=16, chirps=2):
    rng = np.random.default_rng(seed)
    n = 400
    times = 1.7e9 + np.cumsum(rng.uniform(0.001, 0.02, n))
    # a trajectory that pauses now and then (repeated positions get dropped)
    steps = rng.uniform(0, 1.2e-3, (n, 3)) * (rng.random((n, 1)) > 0.3)
    xyz = np.cumsum(steps, axis=0)
    traj = np.concatenate([xyz, rng.standard_normal((n, dim - 3))], axis=1)
    params = dict(num_frames=frames, num_samples=samples, num_chirps=chirps, sweep_time=0.0004,
                  periodicity=0.003, min_f=77.5e9)
    rows = 9
    names = [str(1000 + r) for r in range(rows)]
    created = list(times[0] + np.linspace(-0.3, times[-1] - times[0] - 0.05, rows))
    created[3] = -1                                   # a row without a timestamp
    radar = {}
    for r, name in enumerate(names):
        if r == 5:
            continue                                  # a missing file
        length = frames * samples * chirps if r != 7 else 20 * samples * chirps + 3   # short
        radar[int(name)] = (rng.standard_normal((length, 4)) +
                            1j * rng.standard_normal((length, 4))).astype(np.complex64)
    robot = {"all_radar_filenames": names, "all_radar_created_ts": created}
    locs = {"times_77": times, "tx_77_locs": traj}
    return robot, radar, locs, params


@pytest.mark.parametrize("dim,opti", [(3, False), (7, False), (3, True)])
def test_correlate_matches_reference_loop(cuda_dev, dim, opti):
    import torch
    from oracle import ingest_oracle as IO
    from mmnorm_b200 import ingest
    robot, radar, locs, params = _session(dim, dim)
    radar_dev = {k: torch.as_tensor(v, device=cuda_dev) for k, v in radar.items()}
    out = ingest.correlate_locs_and_meas(robot, radar_dev, locs, params, is_optitrack=opti)
    ref_radar, ref_poses = IO.correlate(robot, radar, locs, params, is_optitrack=opti)
    assert len(ref_radar) > 20
    # some frames of the session are dropped as repeats, some for being outside the track
    assert len(ref_radar) < 8 * params["num_frames"]
    np.testing.assert_array_equal(out["poses"], ref_poses)
    assert len(out["radar_data"]) == len(ref_radar)
    for a, b in zip(out["radar_data"], ref_radar):
        np.testing.assert_array_equal(a.cpu().numpy(), b)


def _fixture_session(g, s):
    p = "s%d_" % s
    robot = {"all_radar_filenames": [str(n) for n in g[p + "names"]],
             "all_radar_created_ts": list(g[p + "created"])}
    radar = {int(k): g[p + "file_%d" % k] for k in g[p + "file_keys"]}
    locs = {"times_77": g[p + "times"], "tx_77_locs": g[p + "traj"]}
    params = {k: g["param_" + k].item() for k in ("num_frames", "num_samples", "num_chirps",
                                                  "sweep_time", "periodicity", "min_f")}
    return robot, radar, locs, params, bool(g[p + "optitrack"])


def test_load_radar_files_matches_reference_fixture(cuda_dev, tmp_path):
    """The reference's own GenericLoader.load_radar_files (77 GHz branch) on a directory of
    .bin files with both file-name layouts, an empty file and a non-.bin file
    (tests/golden/make_golden_next.py): same timestamps, samples exactly."""
    from conftest import load_golden
    from mmnorm_b200 import ingest
    g = load_golden("ingest_ref")
    for k in range(int(g["files"])):
        (tmp_path / str(g["file%d_name" % k])).write_bytes(g["file%d_raw" % k].tobytes())
    got = ingest.load_radar_files(str(tmp_path))
    ref = {int(g["loaded%d_ts" % i]): g["loaded%d_data" % i] for i in range(int(g["loaded"]))}
    assert sorted(got) == sorted(ref)
    for ts, arr in ref.items():
        np.testing.assert_array_equal(got[ts].cpu().numpy().astype(np.complex128), arr)


def test_correlate_matches_reference_fixture(cuda_dev):
    """The reference's own ImageProcessor.correlate_locs_and_meas on seeded sessions
    (tests/golden/make_golden_next.py): the same kept frames in the same order, positions
    bit for bit, the same sample rows."""
    import torch
    from conftest import load_golden
    from mmnorm_b200 import ingest
    g = load_golden("ingest_ref")
    for s in range(int(g["sessions"])):
        robot, radar, locs, params, opti = _fixture_session(g, s)
        radar_dev = {k: torch.as_tensor(v, device=cuda_dev) for k, v in radar.items()}
        out = ingest.correlate_locs_and_meas(robot, radar_dev, locs, params, is_optitrack=opti)
        ref_poses = g["s%d_poses" % s]
        ref_radar = g["s%d_radar" % s]
        assert len(ref_radar) > 20
        np.testing.assert_array_equal(out["poses"], ref_poses)
        got = np.stack([a.cpu().numpy() for a in out["radar_data"]])
        np.testing.assert_array_equal(got, ref_radar)
