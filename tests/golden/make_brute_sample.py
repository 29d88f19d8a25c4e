"""Regenerate tests/golden/golden_brute_sample.npz from the reference's own
sample grids.

The reference ships four text grids of `x y z delta w` rows for its
brute-force estimator (sample-data/delta-nanoer.dat, delta-nano.dat,
delta-micro.dat, delta-tinier.dat: 2^3, 4^3, 16^3 and 32^3 points at 5 Mpc/h
spacing, w = 1) and no expected output for them.  This script stores each
grid's points (float32, as bruteGPU reads them into its columns) with the
strict FP64 oracle's histogram for the configured binning, 100 bins over
[0, 200) Mpc/h (bin 0 below, bin 101 above): per-bin pair counts, sum of
w_i delta_i w_j delta_j and sum of w_i w_j.  Run from the repository root
where the reference tree is present:
    python tests/golden/make_brute_sample.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT]

from oracle import oracle  # noqa: E402

REF = "/root/reference/sample-data"
NAMES = ("delta-nanoer", "delta-nano", "delta-micro", "delta-tinier")
RMIN, RMAX, NBINS = 0.0, 200.0, 100


def main():
    out = {"rmin": RMIN, "rmax": RMAX, "nbins": NBINS}
    for name in NAMES:
        pts = np.loadtxt(os.path.join(REF, name + ".dat"), dtype=np.float64).astype(np.float32)
        assert pts.ndim == 2 and pts.shape[1] == 5
        ds, ws, ct = oracle.brute(pts, RMIN, RMAX, NBINS, nthreads=8)
        key = name.replace("-", "_")
        out[key + "_points"] = pts
        out[key + "_dsum"] = ds
        out[key + "_wsum"] = ws
        out[key + "_counts"] = ct
        print(name, len(pts), "points,", int(ct.sum()), "pairs")
    np.savez_compressed(os.path.join(os.path.dirname(__file__), "golden_brute_sample.npz"), **out)


if __name__ == "__main__":
    main()
