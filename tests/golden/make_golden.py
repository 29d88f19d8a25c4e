"""Regenerate the golden fixtures of tests/golden.

Each fixture holds a seeded catalogue (inputs) and two sets of outputs:
- the reference's own XiEstimator, built from its unchanged sources against
  the stand-in headers of oracle/refshim (oracle/_ref/libtosref.so, built by
  `make -C oracle ref` where the reference tree is present): raw per-bin
  XiBin totals (`ref_*`), the finalized xi (`ref_final_*`), the occupied
  cells and their pair counts, and the five reference counters;
- the strict CPU oracle's FP64 sums (mode 1) and sums of absolute values
  (mode 2), the tolerance scale of the weighted-sum checks.
golden_edges.npz adds a catalogue built to hit the reference's quirks: pixel
distances on a 1 Mpc/h lattice (separations exactly on bin edges), a
sightline without pixels, two sightlines at one position (cos theta = 1, the
Polar r == 0 skip) and reversed pixel order.
golden_plates_cartesian.npz bins the sightlines by plate (PlateBins) with a
platelist of every case PlateBins meets (helpers.plate_catalog) and a scale
at which the maximum angle is below 1.5 degrees, where PlateBins' ring test
skips nearby plates.
Run from the repository root (needs the reference tree for the `ref_*` part);
name fixtures to regenerate only those:
    python tests/golden/make_golden.py [name ...]
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "turbo-octo-spice_b200"), os.path.join(ROOT, "tests")]

from helpers import FIELDS, GRIDS, plate_catalog, small_catalog  # noqa: E402
from oracle import oracle  # noqa: E402
import tos_b200 as T  # noqa: E402


def edge_catalog():
    """Catalogue whose pixel pairs sit on bin edges, plus degenerate sightlines."""
    n, npx = 12, 200
    rng = np.random.default_rng(2)
    los = np.zeros(n, dtype=T.SIGHTLINE_DTYPE)
    px = np.zeros(n * npx, dtype=T.PIXEL_DTYPE)
    for s in range(n):
        los[s]["ra"] = 3.0 + s * 2e-3
        los[s]["dec"] = 0.3 + (s % 3) * 1.5e-3
        los[s]["pixel_offset"] = s * npx
        los[s]["num_pixels"] = npx
        d = 3800.0 + s * 3.0 + np.arange(npx, dtype=np.float64)
        sl = slice(s * npx, (s + 1) * npx)
        px[sl]["distance"] = d.astype(np.float32)
        px[sl]["loglam"] = (3.6 + 1e-4 * np.arange(npx)).astype(np.float32)
        px[sl]["value"] = rng.normal(0, 0.2, npx).astype(np.float32)
        px[sl]["weight"] = rng.uniform(0.5, 2, npx).astype(np.float32)
    los[4]["num_pixels"] = 0                                # no pixels
    los[7]["ra"], los[7]["dec"] = los[6]["ra"], los[6]["dec"]  # same direction
    o = int(los[9]["pixel_offset"])
    px[o:o + npx] = px[o:o + npx][::-1].copy()              # reversed order
    return los, px, {"scale": 3586.0}


def write(name, los, px, order, g, scale):
    bins, cells, ids, st = oracle.xi(los, px, order, g.type, g.axes_array(), scale, mode=1, nthreads=4,
                                     subsamples=True)
    absb = oracle.xi(los, px, order, g.type, g.axes_array(), scale, mode=2, nthreads=4)[0]
    out = dict(sightlines=los, pixels=px, order=order, coord=g.type, axes=g.axes_array(), scale=scale,
               num_pairs=bins["num_pairs"], cell_ids=ids, cell_num_pairs=cells["num_pairs"])
    for f in FIELDS:
        out[f] = bins[f]
        out["abs_" + f] = absb[f]
    if oracle.ref_available():
        rb, rf, rc, rids, rst = oracle.ref_xi(los, px, order, g.type, g.axes_array(), scale, nthreads=4,
                                              subsamples=True)
        out["ref_num_pairs"] = rb["num_pairs"]
        for f in FIELDS:
            out["ref_" + f] = rb[f]
            out["ref_final_" + f] = rf[f]
        out["ref_cell_ids"] = rids
        out["ref_cell_num_pairs"] = rc["num_pairs"]
        out["ref_counters"] = np.array([rst[k] for k in oracle.REF_COUNTERS], dtype=np.uint64)
        out["ref_max_ang"] = np.array([rst["max_ang"], rst["cos_max_ang"]])
    else:
        print("reference build absent: fixture without ref_* outputs")
    path = os.path.join(os.path.dirname(__file__), f"golden_{name}.npz")
    np.savez_compressed(path, **out)
    print(path, int(bins["num_pairs"].sum()), "pairs,", len(ids), "cells")


def write_plates(name, los, px, plates, g, scale):
    bins, cells, ids, st = oracle.xi_plates(los, px, plates, g.type, g.axes_array(), scale, mode=1, nthreads=4,
                                            subsamples=True)
    absb = oracle.xi_plates(los, px, plates, g.type, g.axes_array(), scale, mode=2, nthreads=4)[0]
    out = dict(sightlines=los, pixels=px, platelist=plates, coord=g.type, axes=g.axes_array(), scale=scale,
               num_pairs=bins["num_pairs"], cell_ids=ids, cell_num_pairs=cells["num_pairs"],
               num_sightline_pairs=st["num_sightline_pairs"])
    for f in FIELDS:
        out[f] = bins[f]
        out["abs_" + f] = absb[f]
    if oracle.ref_available():
        rb, rf, rc, rids, rst = oracle.ref_xi_plates(los, px, plates, g.type, g.axes_array(), scale, nthreads=4,
                                                     subsamples=True)
        out["ref_num_pairs"] = rb["num_pairs"]
        for f in FIELDS:
            out["ref_" + f] = rb[f]
            out["ref_final_" + f] = rf[f]
        out["ref_cell_ids"] = rids
        out["ref_cell_num_pairs"] = rc["num_pairs"]
        out["ref_counters"] = np.array([rst[k] for k in oracle.REF_COUNTERS], dtype=np.uint64)
        out["ref_max_ang"] = np.array([rst["max_ang"], rst["cos_max_ang"]])
    else:
        print("reference build absent: fixture without ref_* outputs")
    path = os.path.join(os.path.dirname(__file__), f"golden_{name}.npz")
    np.savez_compressed(path, **out)
    print(path, int(bins["num_pairs"].sum()), "pairs,", len(ids), "cells")


def main(names):
    def want(name):
        return not names or name in names

    los, px, meta = small_catalog(n=60, seed=21, size_deg=2.0, max_pixels=96)
    for name, g in GRIDS.items():
        if want(name):
            write(name, los, px, 6, g, meta["scale"])
    # a wider patch (the angular cut rejects sightline pairs) on an offset grid
    los, px, meta = small_catalog(n=160, seed=8, size_deg=7.0, max_pixels=48)
    if want("wide_offset"):
        write("wide_offset", los, px, 6, T.Grid.cartesian("[3:183]*45", "[2.5:182.5]*36"), meta["scale"])
    los, px, meta = edge_catalog()
    if want("edges_cartesian"):
        write("edges_cartesian", los, px, 6, GRIDS["cartesian"], meta["scale"])
    if want("edges_polar"):
        write("edges_polar", los, px, 6, GRIDS["polar"], meta["scale"])
    los, px, plates, meta = plate_catalog()
    if want("plates_cartesian"):
        write_plates("plates_cartesian", los, px, plates, GRIDS["cartesian"], 4.0 * meta["scale"])


if __name__ == "__main__":
    main(sys.argv[1:])
