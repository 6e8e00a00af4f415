"""The raw-ingest restatement (oracle/ingest_oracle.py) against outputs of the reference's
own GenericLoader.load_radar_files and ImageProcessor.correlate_locs_and_meas
(tests/golden/make_golden_next.py).  CPU only."""
import numpy as np

from conftest import load_golden
from oracle import ingest_oracle as IO


def test_unpack_matches_reference_loader():
    g = load_golden("ingest_ref")
    by_name = {str(g["file%d_name" % k]): g["file%d_raw" % k] for k in range(int(g["files"]))}
    ref = {int(g["loaded%d_ts" % i]): g["loaded%d_data" % i] for i in range(int(g["loaded"]))}
    for name, raw in by_name.items():
        if not name.endswith(".bin"):
            continue
        ts = int(name[8:18]) if name[8:18].isdigit() else int(name[9:21])
        np.testing.assert_array_equal(IO.unpack(raw.tobytes()), ref[ts])


def test_correlate_matches_reference_loop():
    g = load_golden("ingest_ref")
    for s in range(int(g["sessions"])):
        p = "s%d_" % s
        robot = {"all_radar_filenames": [str(n) for n in g[p + "names"]],
                 "all_radar_created_ts": list(g[p + "created"])}
        radar = {int(k): g[p + "file_%d" % k] for k in g[p + "file_keys"]}
        locs = {"times_77": g[p + "times"], "tx_77_locs": g[p + "traj"]}
        params = {k: g["param_" + k].item() for k in ("num_frames", "num_samples", "num_chirps",
                                                      "sweep_time", "periodicity", "min_f")}
        radar_out, poses = IO.correlate(robot, radar, locs, params,
                                        is_optitrack=bool(g[p + "optitrack"]))
        np.testing.assert_array_equal(poses, g[p + "poses"])
        np.testing.assert_array_equal(np.stack(radar_out), g[p + "radar"])
