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
    raw = rng.integers(-32768, 32767, 8 * 1000 + 5, dtype=np.int16).astype("<i2").tobytes()
    got = ingest.unpack_adc(raw).cpu().numpy()
    ref = IO.unpack(raw)
    assert got.shape == ref.shape == (1000, 4)
    np.testing.assert_array_equal(got.astype(np.complex128), ref)


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
