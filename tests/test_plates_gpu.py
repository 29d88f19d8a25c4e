"""GPU parity of plate-binned catalogues (tos_catalog_create_plates, the
reference's PlateBins) against the CPU oracle's plate cells, which the CPU
tests pin to the reference's own PlateBins (tests/test_reference_pin.py).

Pass criteria as for HEALPix cells: the occupied cells, every counter
(candidates num_sightline_pairs included: they count the plates PlateBins'
ring test |theta - 1.5 deg| < max_ang admits) and the per-bin and per-cell
pair counts bit-exact; every weighted sum within REL_TOL = 1e-6 of the FP64
oracle."""
import math
import os

import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth
from helpers import FIELDS, GRIDS, assert_counts_equal, assert_sums_close, plate_catalog
from oracle import oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
COUNTERS = ("num_sightline_pairs", "num_sightline_pairs_used", "num_pixels", "num_pixel_pairs",
            "num_pixel_pairs_used")


def run_plates(engine, los, px, plates, grid, scale):
    cat = T.Catalog(engine, los, px, platelist=plates)
    bins, cells, st = T.xi_run(engine, cat, grid, scale, subsamples=True)
    ids = cat.cells()
    cat.close()
    obins, ocells, oids, ost = oracle.xi_plates(los, px, plates, grid.type, grid.axes_array(), scale, mode=1,
                                                subsamples=True)
    oabs = oracle.xi_plates(los, px, plates, grid.type, grid.axes_array(), scale, mode=2)[0]
    return bins, cells, ids, st, obins, ocells, oids, ost, oabs


def check(bins, cells, ids, st, obins, ocells, oids, ost, oabs):
    assert np.array_equal(ids, oids)
    assert_counts_equal(bins, obins)
    assert np.array_equal(cells["num_pairs"], ocells["num_pairs"])
    for k in COUNTERS:
        assert st[k] == ost[k], (k, st[k], ost[k])
    assert_sums_close(bins, obins, oabs)


def test_plate_golden_fixture(engine):
    """The committed fixture, whose reference outputs came from the
    reference's own PlateBins: a repeated plate id, an empty plate, an
    unlisted plate, and a maximum angle below 1.5 degrees."""
    z = np.load(os.path.join(GOLDEN, "golden_plates_cartesian.npz"))
    cat = T.Catalog(engine, z["sightlines"], z["pixels"], platelist=z["platelist"])
    bins, cells, st = T.xi_run(engine, cat, GRIDS["cartesian"], float(z["scale"]), subsamples=True)
    assert np.array_equal(cat.cells(), z["ref_cell_ids"])
    assert_counts_equal(bins, {"num_pairs": z["ref_num_pairs"]})
    assert np.array_equal(cells["num_pairs"], z["ref_cell_num_pairs"])
    assert_sums_close(bins, {f: z[f] for f in FIELDS}, {f: z["abs_" + f] for f in FIELDS})
    for k, v in zip(COUNTERS, z["ref_counters"]):
        assert st[k] == int(v), k


@pytest.mark.parametrize("name", ["cartesian", "polar", "observing"])
@pytest.mark.parametrize("scale_factor", [1.0, 4.0])
def test_plates_vs_oracle(engine, name, scale_factor):
    """Full forests (the grid and diagonal sweeps run), maximum angle above
    and below 1.5 degrees."""
    los, px, plates, meta = plate_catalog(n=140, seed=23, size_deg=7.0, max_pixels=None)
    check(*run_plates(engine, los, px, plates, GRIDS[name], scale_factor * meta["scale"]))


def test_plate_groups_pair_within_their_group(engine):
    """Two catalogues on the same plates in one resident catalogue: a plate
    cell is (group, plate), and each group's row equals its own run."""
    los_a, px_a, plates, meta = plate_catalog(n=90, seed=3, size_deg=6.0, max_pixels=40)
    los_b, px_b = synth.small_patch(90, seed=4, size_deg=6.0)[:2]
    from helpers import truncate
    los_b, px_b = truncate(los_b, px_b, 40)
    los_b, _ = synth.plate_tiling(los_b, 2.0)  # the same lattice: same plate ids and centres
    los, px = synth.merge_groups([(los_a, px_a), (los_b, px_b)])
    g = GRIDS["cartesian"]
    scale = 2.0 * meta["scale"]
    cat = T.Catalog(engine, los, px, platelist=plates)
    _, rows, st = T.xi_run(engine, cat, g, scale, per_group=True)
    cat.close()
    total = 0
    for k, (lk, pk) in enumerate(((los_a, px_a), (los_b, px_b))):
        ob, _, _, ost = oracle.xi_plates(lk, pk, plates, g.type, g.axes_array(), scale, mode=1)
        oabs = oracle.xi_plates(lk, pk, plates, g.type, g.axes_array(), scale, mode=2)[0]
        assert_counts_equal(rows[k], ob)
        assert_sums_close(rows[k], ob, oabs)
        total += ost["num_sightline_pairs"]
    assert st["num_sightline_pairs"] == total


def test_plate_ring_edge_is_settled_on_the_host(engine):
    """Sightlines at an angle from a plate centre within 1e-12 rad of
    1.5 deg + max_ang (where the device and host acos may round apart): the
    engine takes the host libm's decision, so its candidate count equals the
    oracle's."""
    los, px, plates, meta = plate_catalog(n=60, seed=8, size_deg=5.0, max_pixels=16)
    g = GRIDS["cartesian"]
    scale = 4.0 * meta["scale"]
    max_ang = g.max_angular_scale(scale)
    deg2rad = (math.atan(1.0) * 4) / 180.0
    ring = 1.5 * deg2rad
    # plate of sightline 30 (on the platelist): put sightlines 0..5 due north
    # of its centre at ring + max_ang (+ a few ulps either way)
    p = int(los["plate"][30])
    row = plates[plates["plate"] == p][-1]
    pra, pdec = float(row["ra_center"]) * deg2rad, float(row["dec_center"]) * deg2rad
    los = los.copy()
    for s, eps in enumerate((-2e-15, -1e-15, 0.0, 1e-15, 2e-15, 4e-15)):
        los["ra"][s] = pra
        los["dec"][s] = pdec + ring + max_ang + eps
        los["plate"][s] = p + 100000  # an unlisted plate: the primaries are theirs alone
    check(*run_plates(engine, los, px, plates, g, scale))


def test_plate_catalogue_edge_cases(engine):
    los, px, plates, meta = plate_catalog(n=40, seed=2, size_deg=4.0, max_pixels=16)
    g = GRIDS["cartesian"]
    # an empty platelist: every sightline a primary, nobody a neighbour
    cat = T.Catalog(engine, los, px, platelist=np.zeros(0, dtype=T.PLATE_DTYPE))
    bins, _, st = T.xi_run(engine, cat, g, meta["scale"])
    assert int(bins["num_pairs"].sum()) == 0 and st["num_sightline_pairs"] == 0
    assert st["num_pixels"] == int(los["num_pixels"].astype(np.int64).sum())
    # HEALPix-region jackknife has no meaning on plate cells
    with pytest.raises(T.TosError) as ex:
        T.xi_run_jackknife(engine, cat, g, meta["scale"], 1)
    assert ex.value.status == 5  # TOS_ERR_UNSUPPORTED
    cat.close()
    # plate ids are >= 0 (cell id = group * 2^32 + plate)
    bad = los.copy()
    bad["plate"][3] = -7
    with pytest.raises(T.TosError) as ex:
        T.Catalog(engine, bad, px, platelist=plates)
    assert ex.value.status == 1  # TOS_ERR_INVALID_ARG
    with pytest.raises(ValueError):
        T.Catalog(engine, los, px, 6, platelist=plates)
