"""Times the GPU RSDF (mmnorm_b200.rsdf.compute_rsdf) against the reference's sequential
breadth-first search (restated in oracle/rsdf_oracle.py after src/data_processing/sdf.py:
122-224) on open spherical caps of unit normals, 3 voxels thick, on 64^3 and 128^3 grids at
2 mm, and checks the two agree bit for bit (the 64^3 case).  TEST INFRASTRUCTURE: a
measurement of the reference, not part of the product.  Prints one JSON line.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    import torch
    from mmnorm_b200 import rsdf
    from oracle import rsdf_oracle as RO
    out = {}
    for n, thick in ((64, 3), (128, 3)):
        c = (n - 1) / 2
        g = np.indices((n, n, n)).astype(np.float64)
        r = np.sqrt(((g - c) ** 2).sum(0))
        shell = (r > n * 0.35) & (r < n * 0.35 + thick) & (g[2] < c + n * 0.1)
        nrm = np.stack([(g[k] - c) / np.maximum(r, 1e-9) for k in range(3)], -1)
        nrm[~shell] = np.nan
        x = np.arange(n) * 0.002
        rsdf.compute_rsdf(nrm, x, x, x)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res, lab, valid, _ = rsdf.compute_rsdf(nrm, x, x, x)
        torch.cuda.synchronize()
        rec = {"voxels_in_mask": int(shell.sum()), "components": int(len(valid)),
               "gpu_s": time.perf_counter() - t0}
        if n == 64:
            t0 = time.perf_counter()
            ref = RO.rsdf(nrm, RO.coords(x, x, x), lab, valid, x)
            rec["python_bfs_s"] = time.perf_counter() - t0
            rec["bit_identical"] = bool(np.array_equal(np.nan_to_num(ref, nan=7.0),
                                                       np.nan_to_num(res, nan=7.0)))
        out["cap%d" % n] = rec
    print(json.dumps(out))


if __name__ == "__main__":
    main()
