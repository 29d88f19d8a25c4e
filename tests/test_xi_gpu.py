"""GPU parity of the XiEstimator pair count (through the C ABI) against the
CPU oracle and the committed golden fixtures.

Pass criteria (per bin): pair counts bit-exact; every weighted sum within a
relative error of REL_TOL = 1e-6 of the FP64 oracle (zero where the oracle is
zero).  Against the engine's all-FP64 path (TOS_XI_EXACT) the fast paths give
identical pair counts; the sums of the run sweeps (FP64 sums over whole
rows) and of the Polar diagonal sweep (FP64 sums along diagonals), each
converted on a 62-bit scale, agree to FAST_TOL = 1e-10 of the bin's sum of
absolute values of the terms, the quantisation of the FP64 path's positive
sums (42-bit per run) included."""
import os

import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth  # noqa: F401  (T.synth)
from helpers import FIELDS, GRIDS, REL_TOL, assert_counts_equal, assert_sums_close, small_catalog, truncate
from oracle import oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

EXTRA_GRIDS = {
    # non power-of-two widths and positive minima: edge re-binning on both axes,
    # truncation of (-1, 0) to bin 0
    "cartesian_offset": T.Grid.cartesian("[3:183]*45", "[2.5:182.5]*36"),
    # several z bins: the z index varies inside an item (per-pair FP64 path)
    "cartesian_z3": T.Grid.cartesian(z="[3.55:3.75]*3"),
    "polar_offset": T.Grid.polar("[5:150]*29", "[0.1:0.95]*17"),
    "observing_fine": T.Grid.observing("[0:0.02]*40", "[0:175]*7"),
    # first-axis minimum several bins above 0: separations below it wrap in
    # ref_u32 and are rejected, the accepted range starts at a threshold > 0
    "cartesian_gap": T.Grid.cartesian("[12:196]*46", "[0:200]*50"),
    "observing_gap": T.Grid.observing("[0.004:0.05]*23", "[5:175]*1"),
}
FAST_TOL = 1e-10
ALL_GRIDS = dict(GRIDS, **EXTRA_GRIDS)


def run_both(engine, los, px, grid, scale, order=6, subsamples=True):
    cat = T.Catalog(engine, los, px, order)
    bins, cells, st = T.xi_run(engine, cat, grid, scale, subsamples=subsamples)
    ids = cat.cells()
    cat.close()
    obins, ocells, oids, ost = oracle.xi(los, px, order, grid.type, grid.axes_array(), scale, mode=1,
                                         subsamples=subsamples)
    ost["abs"] = oracle.xi(los, px, order, grid.type, grid.axes_array(), scale, mode=2)[0]
    return bins, cells, ids, st, obins, ocells, oids, ost


@pytest.mark.parametrize("name", ["cartesian", "polar", "observing"])
def test_golden_fixture(engine, name):
    z = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    g = GRIDS[name]
    cat = T.Catalog(engine, z["sightlines"], z["pixels"], int(z["order"]))
    bins, cells, st = T.xi_run(engine, cat, g, float(z["scale"]), subsamples=True)
    assert np.array_equal(cat.cells(), z["cell_ids"])
    assert_counts_equal(bins, {"num_pairs": z["num_pairs"]})
    assert np.array_equal(cells["num_pairs"], z["cell_num_pairs"])
    ref = {f: z[f] for f in FIELDS}
    assert_sums_close(bins, ref, {f: z["abs_" + f] for f in FIELDS})
    assert st["num_pixel_pairs_used"] == int(z["num_pairs"].sum())


@pytest.mark.parametrize("name", sorted(ALL_GRIDS))
def test_parity_vs_oracle(engine, name):
    los, px, meta = small_catalog(n=150, seed=3, size_deg=3.0)
    g = ALL_GRIDS[name]
    bins, cells, ids, st, obins, ocells, oids, ost = run_both(engine, los, px, g, meta["scale"])
    assert np.array_equal(ids, oids)
    assert_counts_equal(bins, obins)
    assert bins["num_pairs"].sum() > 1000
    errs = assert_sums_close(bins, obins, ost["abs"])
    for c in range(len(ids)):
        assert np.array_equal(cells[c]["num_pairs"], ocells[c]["num_pairs"]), f"cell {ids[c]}"
    assert st["num_sightline_pairs_used"] == ost["num_sightline_pairs_used"]
    assert st["num_pixel_pairs"] == ost["num_pixel_pairs"]
    assert st["num_pixel_pairs_used"] == ost["num_pixel_pairs_used"]
    assert st["num_index_overflow"] == ost["num_index_overflow"]
    print(name, errs, "rechecks", st["num_edge_rechecks"], "evaluated", st["num_pixel_pairs_evaluated"])


@pytest.mark.parametrize("name", ["cartesian", "polar", "observing", "cartesian_offset", "polar_offset",
                                  "cartesian_gap", "observing_gap"])
def test_fast_paths_match_fp64_path(engine, name):
    los, px, meta = small_catalog(n=120, seed=8, size_deg=2.5)
    g = ALL_GRIDS[name]
    cat = T.Catalog(engine, los, px, 6)
    fast, fc, st = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    exact, ec, est = T.xi_run(engine, cat, g, meta["scale"], subsamples=True, exact=True)
    assert est["num_run_items"] == 0
    assert_counts_equal(fast, exact)
    assert np.array_equal(fc["num_pairs"], ec["num_pairs"])
    if g.type == T.POLAR:
        # the diagonal sweep takes every item (z index constant here)
        assert st["num_run_items"] == 0
        assert st["num_diag_items"] == st["num_sightline_pairs_used"] > 0
    else:
        assert st["num_run_items"] > 0.9 * st["num_sightline_pairs_used"]
    ref_abs = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=2)[0]
    for f in FIELDS:
        err = np.abs(fast[f] - exact[f])
        bound = FAST_TOL * np.abs(ref_abs[f])
        assert np.all(err <= bound), (f, float(np.max(err - bound)))


def test_deterministic_and_subsamples_sum(engine):
    los, px, meta = small_catalog(n=150, seed=13, size_deg=3.0)
    g = GRIDS["cartesian"]
    cat = T.Catalog(engine, los, px, 6)
    a, ca, _ = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    b, cb, _ = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    c, _, _ = T.xi_run(engine, cat, g, meta["scale"], subsamples=False)
    assert np.array_equal(a, b) and np.array_equal(ca, cb) and np.array_equal(a, c)
    assert np.array_equal(ca["num_pairs"].sum(axis=0), a["num_pairs"])
    for f in FIELDS:  # combined = per-cell values added in ascending cell order
        s = np.zeros(len(a))
        for k in range(ca.shape[0]):
            s = s + ca[k][f]
        assert np.array_equal(s, a[f])


def test_reference_arithmetic_mode(engine):
    # against the reference's own float-product arithmetic (mode 0) the
    # difference is the float rounding of w*delta products: ~1e-7 relative
    los, px, meta = small_catalog(n=100, seed=17, size_deg=2.5)
    g = GRIDS["cartesian"]
    cat = T.Catalog(engine, los, px, 6)
    bins, _, _ = T.xi_run(engine, cat, g, meta["scale"])
    ref, _, _, _ = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=0)
    assert_counts_equal(bins, ref)
    for f in ("wgt", "wi", "wj", "z"):  # positive sums: no cancellation
        nz = ref[f] != 0
        rel = np.abs(bins[f][nz] - ref[f][nz]) / np.abs(ref[f][nz])
        assert rel.max() < 1e-5, (f, rel.max())


def test_edge_cases(engine):
    los, px, meta = small_catalog(n=40, seed=23, size_deg=1.0, max_pixels=80)
    g = GRIDS["cartesian"]
    # one sightline: no pairs
    cat = T.Catalog(engine, los[:1], px[: int(los[0]["num_pixels"])], 6)
    bins, _, st = T.xi_run(engine, cat, g, meta["scale"])
    assert bins["num_pairs"].sum() == 0 and st["num_sightline_pairs_used"] == 0
    cat.close()
    # sightlines without pixels, duplicated positions, and reversed pixel order
    los2 = los.copy()
    los2[5]["num_pixels"] = 0
    los2[6]["ra"], los2[6]["dec"] = los2[7]["ra"], los2[7]["dec"]  # cos(theta) = 1
    bins, _, _, st, obins, _, _, ost = run_both(engine, los2, px, g, meta["scale"], subsamples=False)
    assert_counts_equal(bins, obins)
    assert_sums_close(bins, obins, ost["abs"])
    px_rev = px.copy()
    for s in range(len(los2)):
        o, n = int(los2[s]["pixel_offset"]), int(los2[s]["num_pixels"])
        px_rev[o:o + n] = px[o:o + n][::-1]
    cat = T.Catalog(engine, los2, px_rev, 6)  # unsorted: no column pruning
    rb, _, rst = T.xi_run(engine, cat, g, meta["scale"])
    assert_counts_equal(rb, obins)
    assert_sums_close(rb, obins, ost["abs"])
    assert rst["num_pixel_pairs_evaluated"] == rst["num_pixel_pairs"]


def test_pixels_on_bin_edges(engine):
    # distances on a 1 Mpc/h lattice: |d1 - d2| falls exactly on r_par edges,
    # transverse separations from a fixed angle
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
        px[s * npx:(s + 1) * npx]["distance"] = d.astype(np.float32)
        px[s * npx:(s + 1) * npx]["loglam"] = (3.6 + 1e-4 * np.arange(npx)).astype(np.float32)
        px[s * npx:(s + 1) * npx]["value"] = rng.normal(0, 0.2, npx).astype(np.float32)
        px[s * npx:(s + 1) * npx]["weight"] = rng.uniform(0.5, 2, npx).astype(np.float32)
    for name in ("cartesian", "polar", "cartesian_offset"):
        g = ALL_GRIDS[name]
        bins, _, _, st, obins, _, _, ost = run_both(engine, los, px, g, 3586.0, subsamples=False)
        assert_counts_equal(bins, obins)
        assert_sums_close(bins, obins, ost["abs"])


def test_invalid_inputs(engine):
    los, px, meta = small_catalog(n=10, seed=1, size_deg=1.0, max_pixels=20)
    bad = px.copy()
    bad[3]["distance"] = np.nan
    with pytest.raises(T.TosError) as e:
        T.Catalog(engine, los, bad, 6)
    assert e.value.status == 1
    los_bad = los.copy()
    los_bad[2]["pixel_offset"] = len(px)  # range past the pixel array
    with pytest.raises(T.TosError):
        T.Catalog(engine, los_bad, px, 6)
    cat = T.Catalog(engine, los, px, 6)
    with pytest.raises(T.TosError):
        T.xi_run(engine, cat, T.Grid.cartesian(), -1.0)
    # bins so fine that a separation's index would wrap 32 bits
    with pytest.raises(T.TosError) as e:
        T.xi_run(engine, cat, T.Grid.cartesian("[0:1e-6]*50"), meta["scale"])
    assert e.value.status == 5  # TOS_ERR_UNSUPPORTED


def test_full_size_small_config_cell_subset(engine):
    """The small configuration at full size (2,000 sightlines): the GPU's
    per-cell sums for a seeded subset of cells equal the oracle's for the same
    primary cells, and whole-run invariants hold."""
    los, px, meta = T.synth.small_patch(2000, seed=1)
    g = GRIDS["cartesian"]
    cat = T.Catalog(engine, los, px, 6)
    bins, cells, st = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    ids = cat.cells()
    assert st["num_pixel_pairs_used"] == int(bins["num_pairs"].sum())
    assert np.array_equal(cells["num_pairs"].sum(axis=0), bins["num_pairs"])
    rng = np.random.default_rng(0)
    subset = np.sort(rng.choice(len(ids), size=4, replace=False))
    _, ocells, oids, _ = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=1,
                                   cell_subset=subset, subsamples=True)
    _, acells, _, _ = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=2,
                                cell_subset=subset, subsamples=True)
    assert np.array_equal(ids, oids)
    for c in subset:
        assert_counts_equal(cells[c], ocells[c])
        assert_sums_close(cells[c], ocells[c], acells[c])


def drop_pixels(los, px, frac, seed):
    """Remove a random fraction of the pixels of every other sightline (as
    masking does): those sightlines are no longer contiguous on the grid."""
    rng = np.random.default_rng(seed)
    los2 = los.copy()
    out, off = [], 0
    for s in range(len(los)):
        o, n = int(los[s]["pixel_offset"]), int(los[s]["num_pixels"])
        p = px[o:o + n]
        if s % 2 == 1 and n > 4:
            p = p[np.sort(rng.choice(n, size=max(2, int(n * (1 - frac))), replace=False))]
        out.append(p)
        los2[s]["pixel_offset"] = off
        los2[s]["num_pixels"] = len(p)
        off += len(p)
    return los2, np.concatenate(out)


@pytest.mark.parametrize("name", ["cartesian", "observing", "cartesian_gap"])
def test_pointer_sweep_on_gapped_sightlines(engine, name):
    los, px, meta = small_catalog(n=120, seed=21, size_deg=2.5)
    los, px = drop_pixels(los, px, 0.1, seed=4)
    g = ALL_GRIDS[name]
    bins, cells, ids, st, obins, ocells, oids, ost = run_both(engine, los, px, g, meta["scale"])
    assert_counts_equal(bins, obins)
    assert_sums_close(bins, obins, ost["abs"])
    # both sweeps ran: grid pairs and pairs with a gapped sightline
    assert 0 < st["num_grid_items"] < st["num_run_items"]
    assert st["num_run_items"] == st["num_sightline_pairs_used"]


@pytest.mark.parametrize("name", ["cartesian", "polar", "observing"])
def test_tuned_launch_shape_gives_identical_results(engine, name):
    """TOS_XI_TUNE times the dominant kernel with every CTA count per SM on
    a sample of the sightline pairs and keeps the fastest on the engine.  A
    warp sweeps an item on its own and every add is an integer add, so the
    tuning run and the runs after it give the untuned results bit for bit."""
    los, px, meta = small_catalog(n=300, seed=21, size_deg=4.0)
    g = GRIDS[name]
    cat = T.Catalog(engine, los, px, 6)
    a, ac, _ = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    b, bc, st = T.xi_run(engine, cat, g, meta["scale"], subsamples=True, tune=True)
    c, cc, _ = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    cat.close()
    assert st["num_grid_items"] + st["num_diag_items"] > 0.9 * st["num_sightline_pairs_used"]
    for x, y in ((a, b), (ac, bc), (a, c), (ac, cc)):
        assert np.array_equal(x, y)
