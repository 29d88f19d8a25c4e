"""CPU tests that pin the oracle to the reference's own code.

The golden fixtures hold the outputs of the reference's XiEstimator built from
its unchanged sources (turbooctospice/XiEstimator.cc and the grid classes,
with ThreadPool.cc, against the stand-in headers of oracle/refshim; see
oracle/ref_harness.cc).  The oracle in reference-arithmetic mode (mode 0)
must reproduce them: pair counts per bin and per cell bit for bit, and the
seven XiBin sums exactly (the same float products, the same double sums in
the same order).  The FP64 mode (mode 1) must give the same pair counts.

Where oracle/_ref has been built (here; the built library also travels with
the repository to GPU hosts) the live reference is compared on more
catalogues: a wide patch where the angular cut rejects pairs, every grid of
the GPU tests, the quirk catalogue, and seeded primary cells of the
2,000-sightline configuration.  No GPU needed.
"""
import math
import os

import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth  # noqa: F401  (T.synth)
from helpers import FIELDS, GRIDS, small_catalog
from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = ["golden_cartesian", "golden_polar", "golden_observing", "golden_wide_offset",
            "golden_edges_cartesian", "golden_edges_polar"]
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built (no reference tree)")

EXTRA_GRIDS = {
    "cartesian_offset": T.Grid.cartesian("[3:183]*45", "[2.5:182.5]*36"),
    "cartesian_z3": T.Grid.cartesian(z="[3.55:3.75]*3"),
    "polar_offset": T.Grid.polar("[5:150]*29", "[0.1:0.95]*17"),
    "observing_fine": T.Grid.observing("[0:0.02]*40", "[0:175]*7"),
    "cartesian_gap": T.Grid.cartesian("[12:196]*46", "[0:200]*50"),
    "observing_gap": T.Grid.observing("[0.004:0.05]*23", "[5:175]*1"),
}


def _load(fixture):
    z = np.load(os.path.join(GOLDEN, fixture + ".npz"))
    assert "ref_num_pairs" in z.files, "fixture lacks the reference outputs (regenerate with the reference tree)"
    return z


def assert_same_as_reference(orc_bins, ref_bins, exact=True):
    assert np.array_equal(orc_bins["num_pairs"], ref_bins["num_pairs"])
    for f in FIELDS:
        if exact:
            assert np.array_equal(orc_bins[f], ref_bins[f]), f
        else:  # summation order may differ: rounding of the double sums only
            np.testing.assert_allclose(orc_bins[f], ref_bins[f], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("fixture", FIXTURES)
def test_oracle_reproduces_reference_fixture(fixture):
    z = _load(fixture)
    los, px, axes = z["sightlines"], z["pixels"], z["axes"]
    order, coord, scale = int(z["order"]), int(z["coord"]), float(z["scale"])
    b0, c0, ids, st = oracle.xi(los, px, order, coord, axes, scale, mode=0, nthreads=4, subsamples=True)
    assert np.array_equal(b0["num_pairs"], z["ref_num_pairs"])
    assert np.array_equal(ids, z["ref_cell_ids"])
    assert np.array_equal(c0["num_pairs"], z["ref_cell_num_pairs"])
    for f in FIELDS:
        assert np.array_equal(b0[f], z["ref_" + f]), f
    cnt = z["ref_counters"]
    assert st["num_sightline_pairs_used"] == cnt[1]
    assert st["num_pixels"] == cnt[2] and st["num_pixel_pairs"] == cnt[3] and st["num_pixel_pairs_used"] == cnt[4]
    np.testing.assert_array_equal([st["max_ang"], st["cos_max_ang"]], z["ref_max_ang"])
    # the FP64 mode bins the same pairs
    b1 = oracle.xi(los, px, order, coord, axes, scale, mode=1, nthreads=4)[0]
    assert np.array_equal(b1["num_pairs"], z["ref_num_pairs"])
    # XiBin::finalize of the raw totals is the reference's finalized xi_
    fin = T.finalize(b0)
    for f in FIELDS:
        assert np.array_equal(fin[f], z["ref_final_" + f]), f


@needs_ref
@pytest.mark.parametrize("name", sorted(dict(GRIDS, **EXTRA_GRIDS)))
def test_oracle_matches_live_reference(name):
    g = dict(GRIDS, **EXTRA_GRIDS)[name]
    los, px, meta = small_catalog(n=150, seed=31, size_deg=7.0, max_pixels=40)
    rb, rf, rc, rids, rst = oracle.ref_xi(los, px, 6, g.type, g.axes_array(), meta["scale"], nthreads=4,
                                          subsamples=True)
    ob, oc, oids, ost = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=0, nthreads=4,
                                  subsamples=True)
    if g.type != T.OBSERVING:  # QuasarGrid's max angle is 175 "radians" (arcmin misread): no cut
        assert rst["num_sightline_pairs_used"] < rst["num_sightline_pairs"]  # the cut is active
    assert ost["num_pixel_pairs_used"] == rst["num_pixel_pairs_used"] > 0
    assert np.array_equal(oids, rids)
    assert np.array_equal(oc["num_pairs"], rc["num_pairs"])
    assert_same_as_reference(ob, rb, exact=False)


@needs_ref
def test_small_configuration_cells_match_live_reference():
    """Four seeded primary cells of the 2,000-sightline configuration."""
    los, px, meta = T.synth.small_patch(2000, seed=1)
    g = GRIDS["cartesian"]
    cells = np.unique(T.synth.ang2pix_ring(64, 0.5 * math.pi - los["dec"], los["ra"]))
    pick = np.sort(np.random.default_rng(0).choice(len(cells), size=4, replace=False))
    rb, _, rc, rids, rst = oracle.ref_xi(los, px, 6, g.type, g.axes_array(), meta["scale"], cell_subset=cells[pick],
                                         subsamples=True)
    _, oc, oids, ost = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=0, cell_subset=pick,
                                 subsamples=True)
    assert np.array_equal(rids, cells[pick]) and np.array_equal(oids, cells)
    for k, c in enumerate(pick):
        assert_same_as_reference(oc[c], rc[k], exact=False)
    assert ost["num_pixel_pairs_used"] == rst["num_pixel_pairs_used"]


@needs_ref
def test_fast_math_reference_build_counts():
    """The reference is built with -O3 -ffast-math (SConstruct:32); on the
    golden catalogues that build bins the same pairs as the strict one."""
    for fixture in FIXTURES:
        z = _load(fixture)
        rb = oracle.ref_xi(z["sightlines"], z["pixels"], int(z["order"]), int(z["coord"]), z["axes"],
                           float(z["scale"]), nthreads=4, kind="fast")[0]
        assert np.array_equal(rb["num_pairs"], z["ref_num_pairs"]), fixture


@needs_ref
def test_healpix_cells_match_reference():
    """Cell of each direction: the oracle's RING ang2pix and the vectorised
    one of tos_b200.synth against HealpixBins::ang2pix of the reference build,
    on random directions and on directions within 0.01 rad of the poles."""
    rng = np.random.default_rng(5)
    ra = np.concatenate([rng.uniform(0, 2 * math.pi, 3000), rng.uniform(0, 2 * math.pi, 500)])
    dec = np.concatenate([np.arcsin(rng.uniform(-1, 1, 3000)),
                          np.sign(rng.uniform(-1, 1, 500)) * (0.5 * math.pi - rng.uniform(0, 0.01, 500))])
    for order in (3, 6):
        ref = np.array([oracle.ref_radec2pix(order, r, d) for r, d in zip(ra, dec)])
        orc = np.array([oracle.radec2pix(order, r, d) for r, d in zip(ra, dec)])
        assert np.array_equal(ref, orc)
        vec = T.synth.ang2pix_ring(1 << order, 0.5 * math.pi - dec, ra)
        far = np.abs(np.sin(dec)) < 0.99
        assert np.array_equal(vec[far], ref[far])


@needs_ref
def test_disc_superset_bound():
    """The stand-in query_disc_inclusive adds a pixel-radius bound to the
    query radius; it must exceed every direction's distance to its own
    pixel centre, or a neighbour cell could be missed."""
    rng = np.random.default_rng(6)
    v = rng.normal(size=(200000, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    for order in (3, 6):
        worst, bound = oracle.ref_max_centre_distance(order, v)
        assert worst < 0.8 * bound, (order, worst, bound)


# ---- PlateBins (sky cells = BOSS plates)

def test_oracle_reproduces_reference_plate_fixture():
    """The plate fixture: a platelist with a repeated plate id, a plate
    without sightlines and sightlines on an unlisted plate, at a maximum
    angle below 1.5 degrees (PlateBins' ring test skips nearby plates)."""
    z = _load("golden_plates_cartesian")
    los, px, plates, axes = z["sightlines"], z["pixels"], z["platelist"], z["axes"]
    coord, scale = int(z["coord"]), float(z["scale"])
    b0, c0, ids, st = oracle.xi_plates(los, px, plates, coord, axes, scale, mode=0, nthreads=4, subsamples=True)
    assert np.array_equal(b0["num_pairs"], z["ref_num_pairs"])
    assert np.array_equal(ids, z["ref_cell_ids"])
    assert np.array_equal(c0["num_pairs"], z["ref_cell_num_pairs"])
    for f in FIELDS:
        assert np.array_equal(b0[f], z["ref_" + f]), f
    cnt = z["ref_counters"]
    assert st["num_sightline_pairs"] == cnt[0] and st["num_sightline_pairs_used"] == cnt[1]
    assert st["num_pixels"] == cnt[2] and st["num_pixel_pairs"] == cnt[3] and st["num_pixel_pairs_used"] == cnt[4]
    assert z["ref_max_ang"][0] < math.radians(1.5)
    b1 = oracle.xi_plates(los, px, plates, coord, axes, scale, mode=1, nthreads=4)[0]
    assert np.array_equal(b1["num_pairs"], z["ref_num_pairs"])


@needs_ref
@pytest.mark.parametrize("name", ["cartesian", "polar", "observing"])
@pytest.mark.parametrize("scale_factor", [1.0, 4.0])
def test_plate_bins_match_live_reference(name, scale_factor):
    """The oracle's plate cells against the reference's own PlateBins (its
    constructor reading the platelist through the CCfits stand-in): the
    cells, every counter and the sums bit for bit."""
    from helpers import plate_catalog
    los, px, plates, meta = plate_catalog(n=80, seed=5, size_deg=7.0, max_pixels=32)
    g = GRIDS[name]
    scale = scale_factor * meta["scale"]
    rb, _, rc, rids, rst = oracle.ref_xi_plates(los, px, plates, g.type, g.axes_array(), scale, nthreads=4,
                                                subsamples=True)
    ob, oc, oids, ost = oracle.xi_plates(los, px, plates, g.type, g.axes_array(), scale, mode=0, nthreads=4,
                                         subsamples=True)
    assert rst["num_pixel_pairs_used"] > 0
    for k in ("num_sightline_pairs", "num_sightline_pairs_used", "num_pixels", "num_pixel_pairs",
              "num_pixel_pairs_used"):
        assert ost[k] == rst[k], k
    assert np.array_equal(oids, rids)
    assert np.array_equal(oc["num_pairs"], rc["num_pairs"])
    assert_same_as_reference(ob, rb, exact=True)
