"""bench.py on the host: its default command line (one GPU, at least three
warm-up steps) and the reduced-catalogue helper of the jackknife section."""
import sys

import numpy as np

import bench
from helpers import small_catalog


def test_defaults(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert a.gpus == 1 and a.impl == "engine" and a.workload == "full"
    assert a.warmup >= 3 and a.steps >= 1
    assert a.sightlines == 160000 and a.grid == "cartesian"


def test_reduced_keeps_selected_sightlines():
    los, px, _ = small_catalog(n=9, seed=3, size_deg=2.0, max_pixels=15)
    keep = np.array([True, False, True, True, False, False, True, False, True])
    r_los, r_px = bench.reduced(los, px, keep)
    assert len(r_los) == keep.sum()
    assert len(r_px) == int(los["num_pixels"][keep].sum())
    for k, s in enumerate(np.nonzero(keep)[0]):
        o, n = int(r_los[k]["pixel_offset"]), int(r_los[k]["num_pixels"])
        so = int(los[s]["pixel_offset"])
        assert np.array_equal(r_px[o:o + n], px[so:so + n])
        assert r_los[k]["ra"] == los[s]["ra"]
