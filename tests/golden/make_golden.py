"""Regenerate the golden fixtures of tests/golden from the strict CPU oracle.

The reference ships no expected outputs for its pair-counting path, so these
fixtures pin the oracle (and through it the engine) against regressions:
seeded small catalogues (inputs) and the oracle's FP64 per-bin and per-cell
sums (outputs).  Run from the repository root:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "turbo-octo-spice_b200"), os.path.join(ROOT, "tests")]

from helpers import FIELDS, GRIDS, small_catalog  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    los, px, meta = small_catalog(n=60, seed=21, size_deg=2.0, max_pixels=96)
    for name, g in GRIDS.items():
        bins, cells, ids, st = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=1,
                                         nthreads=4, subsamples=True)
        absb = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=2, nthreads=4)[0]
        out = dict(sightlines=los, pixels=px, order=6, coord=g.type, axes=g.axes_array(),
                   scale=meta["scale"], num_pairs=bins["num_pairs"], cell_ids=ids,
                   cell_num_pairs=cells["num_pairs"])
        for f in FIELDS:
            out[f] = bins[f]
            out["abs_" + f] = absb[f]
        path = os.path.join(os.path.dirname(__file__), f"golden_{name}.npz")
        np.savez_compressed(path, **out)
        print(path, int(bins["num_pairs"].sum()), "pairs,", len(ids), "cells")


if __name__ == "__main__":
    main()
