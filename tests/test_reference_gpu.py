"""GPU parity against the reference's own XiEstimator, through the C ABI.

The golden fixtures hold the outputs of the reference built from its
unchanged sources (oracle/ref_harness.cc).  For every fixture the engine must
give the reference's pair counts per bin and per cell bit for bit, its sums
within a relative 1e-6 per bin of the FP64 oracle (judged against
max(|sum|, 1e-6 * A), A the sum of absolute values of the terms), and, against
the reference's own float-product sums, within 1e-6 relative for the positive
sums and 1e-6 of A for the signed ones (the reference rounds w*delta and the
products to float).

At survey density (a 20,000-sightline catalogue at the full survey's 16
sightlines per square degree, on a sky mask with edges), six primary cells
are checked against the live reference where oracle/_ref is built, else the
oracle in reference arithmetic: the two costliest cells, two at the mask
edge and two near the median, in (r_par, r_perp) and in (r, mu).  These are
the geometries where the grid sweep's monotonicity guard and the Polar
column window are tested at the density they are timed at.
"""
import os

import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth  # noqa: F401  (T.synth)
from helpers import FIELDS
from oracle import oracle, parity

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = ["golden_cartesian", "golden_polar", "golden_observing", "golden_wide_offset",
            "golden_edges_cartesian", "golden_edges_polar"]


@pytest.mark.parametrize("fixture", FIXTURES)
def test_engine_matches_reference_fixture(engine, fixture):
    z = np.load(os.path.join(GOLDEN, fixture + ".npz"))
    g = T.Grid.from_axes(int(z["coord"]), z["axes"])
    cat = T.Catalog(engine, z["sightlines"], z["pixels"], int(z["order"]))
    bins, cells, st = T.xi_run(engine, cat, g, float(z["scale"]), subsamples=True)
    assert np.array_equal(cat.cells(), z["ref_cell_ids"])
    cat.close()
    assert np.array_equal(bins["num_pairs"], z["ref_num_pairs"])
    assert np.array_equal(cells["num_pairs"], z["ref_cell_num_pairs"])
    cnt = z["ref_counters"]
    assert st["num_sightline_pairs_used"] == cnt[1] and st["num_pixel_pairs"] == cnt[3]
    assert st["num_pixel_pairs_used"] == cnt[4]
    ref = {f: z["ref_" + f] for f in FIELDS}
    ref["num_pairs"] = z["ref_num_pairs"]
    fp64 = {f: z[f] for f in FIELDS}
    fp64["num_pairs"] = z["num_pairs"]
    absb = {f: z["abs_" + f] for f in FIELDS}
    out = parity.compare(bins, ref, fp64, absb)
    assert out["counts_equal"]
    assert out["max_rel_err_vs_fp64"] <= parity.REL_TOL, out
    assert out["max_rel_err_vs_reference"] <= 1e-6, out


@pytest.fixture(scope="module")
def survey_20k():
    los, px, meta = T.synth.full_survey(20000, seed=7, area_deg2=1250.0)
    return los, px, meta


@pytest.mark.parametrize("binning", ["cartesian", "polar"])
def test_survey_density_cells_match_reference(engine, survey_20k, binning):
    los, px, meta = survey_20k
    g = T.Grid.cartesian() if binning == "cartesian" else T.Grid.polar("[0:200]*50", "[0:1]*20")
    cat = T.Catalog(engine, los, px, 6)
    bins, rows, st = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    ids = cat.cells()
    pos_of = np.searchsorted(ids, cat.sightline_cells())
    cat.close()
    pix = np.bincount(pos_of, weights=los["num_pixels"].astype(np.float64), minlength=len(ids))
    sel = parity.pick_cells(rows["num_pairs"].sum(axis=1), pix, n_median=2, n_costly=2, n_edge=2)
    assert len(sel) == 6
    out = parity.check_cells(rows[sel], sel, ids[sel], los, px, 6, g.type, g.axes_array(), meta["scale"])
    assert out["counts_equal"], out
    assert out["reference_counts_equal_fp64_oracle"], out
    assert out["max_rel_err_vs_fp64"] <= parity.REL_TOL, out
    assert out["max_rel_err_vs_reference"] <= 1e-6, out
    assert out["pairs_compared"] > 10**9  # cells at the density of the timed survey
    # both sweeps of the timed configuration ran on this catalogue
    if binning == "cartesian":
        assert st["num_grid_items"] > 0.99 * st["num_sightline_pairs_used"]
