"""Host-side logic: synthetic workloads have the configured shapes."""
import math

import numpy as np

from tos_b200 import synth


def test_small_patch_shapes():
    los, px, meta = synth.small_patch(300, seed=2)
    n = los["num_pixels"].astype(int)
    assert n.min() >= 143 and n.max() <= 622
    assert np.all(np.diff(los["pixel_offset"].astype(np.int64)) == n[:-1])
    assert int(n.sum()) == len(px)
    # pixels ascending in loglam and distance within every sightline (HDF5Delta order)
    for s in range(0, 300, 37):
        o, k = int(los[s]["pixel_offset"]), int(los[s]["num_pixels"])
        assert np.all(np.diff(px["loglam"][o:o + k]) > 0)
        assert np.all(np.diff(px["distance"][o:o + k]) > 0)
    assert px["loglam"].min() >= math.log10(3600) - 1e-6
    assert 0.15 < px["value"].std() < 0.25
    assert 0.5 <= px["weight"].min() and px["weight"].max() <= 2.0
    assert abs(meta["scale"] - 3586.0) < 3.0
    ra, dec = np.rad2deg(los["ra"]), np.rad2deg(los["dec"])
    assert ra.min() >= 180 and ra.max() <= 190 and dec.min() >= 20 and dec.max() <= 30


def test_survey_mask_area():
    cells, v, cap = synth.survey_mask(7)
    area = len(cells) * 4 * math.pi / 768 * (180 / math.pi) ** 2
    assert 8500 < area < 11500


def test_grf_unit_variance():
    pts = synth.grf_grid(16, box=64.0, seed=1)
    assert pts.shape == (4096, 5)
    assert abs(pts[:, 3].std() - 1.0) < 1e-5
    assert np.all(pts[:, 4] == 1)
    assert pts[:, 0].min() == 2.0 and pts[:, 0].max() == 62.0
