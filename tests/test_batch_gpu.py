"""Batched catalogues: several mock catalogues resident as the sightline
groups of one catalogue and counted by one tos_xi_run with TOS_XI_PER_GROUP
(the batched form of running XiEstimator once per catalogue).

Pass criteria, per group and bin: pair counts bit-exact against the group's
catalogue run alone and against the FP64 oracle on it; sums within
REL_TOL = 1e-6 of the oracle and within SAME_TOL = 1e-10 of the bin's sum
of absolute values of the terms from the lone run (the two runs convert to
different fixed-point scales).  No pair crosses groups, also when two groups
hold sightlines at identical sky positions."""
import ctypes as C

import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth  # noqa: F401  (T.synth)
from helpers import FIELDS, GRIDS, assert_counts_equal, assert_same_count, assert_sums_close, small_catalog
from oracle import oracle

pytestmark = pytest.mark.gpu
SAME_TOL = 1e-10


def parts_three():
    a_los, a_px, meta = small_catalog(n=120, seed=3, size_deg=3.0, max_pixels=160)
    b_los, b_px, _ = small_catalog(n=90, seed=5, size_deg=2.5, max_pixels=160)
    # C: A's sky positions and pixel grid, new values and weights
    rng = np.random.default_rng(99)
    c_px = a_px.copy()
    c_px["value"] = rng.normal(0, 0.2, len(c_px)).astype(np.float32)
    c_px["weight"] = rng.uniform(0.5, 2.0, len(c_px)).astype(np.float32)
    return [(a_los, a_px), (b_los, b_px), (a_los.copy(), c_px)], meta["scale"]


def interleave(parts, group_ids):
    """Merge parts with the given group ids, sightlines interleaved round-robin
    (each group keeps its own order, which fixes its pairs' (i, j) order)."""
    los, px = T.synth.merge_groups(parts)
    los["group"] = np.concatenate([np.full(len(p[0]), g, np.uint32) for p, g in zip(parts, group_ids)])
    owner = np.concatenate([np.full(len(p[0]), k) for k, p in enumerate(parts)])
    rank = np.concatenate([np.arange(len(p[0])) for p in parts])
    order = np.lexsort((owner, rank))
    return los[order], px


def abs_sums(los, px, grid, scale, order=6):
    return oracle.xi(los, px, order, grid.type, grid.axes_array(), scale, mode=2)[0]


@pytest.mark.parametrize("name", ["cartesian", "polar", "observing"])
def test_groups_equal_lone_runs(engine, name):
    g = GRIDS[name]
    parts, scale = parts_three()
    gids = [7, 3, 12]
    los, px = interleave(parts, gids)
    cat = T.Catalog(engine, los, px, 6)
    assert list(cat.groups()) == sorted(gids)
    bins, rows, st = T.xi_run(engine, cat, g, scale, per_group=True)
    cat.close()
    assert rows.shape == (3, g.nbins)
    used = 0
    for r, gid in enumerate(sorted(gids)):
        k = gids.index(gid)
        p_los, p_px = parts[k]
        lone = T.Catalog(engine, p_los, p_px, 6)
        lb, _, lst = T.xi_run(engine, lone, g, scale)
        lone.close()
        used += lst["num_sightline_pairs_used"]
        a = abs_sums(p_los, p_px, g, scale)
        assert_same_count(rows[r], lb, a, SAME_TOL)
        ob = oracle.xi(p_los, p_px, 6, g.type, g.axes_array(), scale, mode=1)[0]
        assert_counts_equal(rows[r], ob)
        assert_sums_close(rows[r], ob, a)
    assert st["num_sightline_pairs_used"] == used
    # out_bins: the groups' rows added in ascending group order
    for f in FIELDS:
        assert np.array_equal(bins[f], rows[0][f] + rows[1][f] + rows[2][f])
    assert np.array_equal(bins["num_pairs"], rows["num_pairs"].sum(axis=0))


def test_one_group_per_group_equals_plain(engine):
    los, px, meta = small_catalog(n=100, seed=8, size_deg=3.0, max_pixels=200)
    g = GRIDS["cartesian"]
    cat = T.Catalog(engine, los, px, 6)
    b0, _, _ = T.xi_run(engine, cat, g, meta["scale"])
    b1, rows, _ = T.xi_run(engine, cat, g, meta["scale"], per_group=True)
    cat.close()
    assert rows.shape == (1, g.nbins)
    for f in FIELDS + ("num_pairs",):
        assert np.array_equal(b0[f], b1[f]), f
        assert np.array_equal(b0[f], rows[0][f]), f


def test_identical_positions_do_not_pair(engine):
    los, px, meta = small_catalog(n=60, seed=4, size_deg=2.0, max_pixels=100)
    g = GRIDS["cartesian"]
    both_los, both_px = T.synth.merge_groups([(los, px), (los.copy(), px.copy())])
    cat = T.Catalog(engine, both_los, both_px, 6)
    bins, rows, st = T.xi_run(engine, cat, g, meta["scale"], per_group=True)
    # the cells of the two groups hold the same HEALPix pixels
    cells = cat.cells()
    assert np.array_equal(cells[cells >> 32 == 0], cells[cells >> 32 == 1] & 0xFFFFFFFF)
    cat.close()
    lone = T.Catalog(engine, los, px, 6)
    lb, _, lst = T.xi_run(engine, lone, g, meta["scale"])
    lone.close()
    for r in range(2):
        for f in FIELDS + ("num_pairs",):
            assert np.array_equal(rows[r][f], lb[f]), (r, f)
    assert st["num_sightline_pairs_used"] == 2 * lst["num_sightline_pairs_used"]


def test_per_group_argument_errors(engine):
    los, px, meta = small_catalog(n=20, seed=2, size_deg=2.0, max_pixels=50)
    cat = T.Catalog(engine, los, px, 6)
    g = GRIDS["cartesian"]
    out = np.zeros(g.nbins, dtype=T.XIBIN_DTYPE)
    rows = np.zeros((4, g.nbins), dtype=T.XIBIN_DTYPE)
    L = T.lib()
    st = T.XiStats()
    s = L.tos_xi_run(engine.handle, cat.handle, C.byref(g.c_struct()), meta["scale"], T.XI_PER_GROUP,
                     T._ptr(out), None, C.byref(st))
    assert s == 1
    s = L.tos_xi_run(engine.handle, cat.handle, C.byref(g.c_struct()), meta["scale"],
                     T.XI_PER_GROUP | T.XI_SUBSAMPLES, T._ptr(out), T._ptr(rows), C.byref(st))
    assert s == 1
    cat.close()
