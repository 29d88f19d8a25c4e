"""Exact delete-one-region jackknife in one pass (tos_xi_run_jackknife).

Pass criteria: for every (group, region) subsample, the one-pass result has
the pair counts of a separate tos_xi_run on the catalogue without that
region's sightlines, bit-exact, and its sums within SAME_TOL = 1e-10 of the
bin's sum of absolute values of the terms (FP64 oracle, mode 2); the run's
totals and per-group rows match tos_xi_run the same way."""
import math

import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth  # noqa: F401  (T.synth)
from helpers import FIELDS, GRIDS, assert_counts_equal, assert_same_count, assert_sums_close, small_catalog
from oracle import oracle

pytestmark = pytest.mark.gpu
SAME_TOL = 1e-10
ORDER, REGION_ORDER = 6, 4


def regions_of(los, region_order):
    theta = 0.5 * math.pi - los["dec"]
    return T.synth.ang2pix_ring(1 << region_order, theta, los["ra"])


def subset(los, px, keep):
    """Sightlines where keep is true, compact pixel layout."""
    idx = np.nonzero(keep)[0]
    out_los = los[idx].copy()
    parts, off = [], 0
    for k, s in enumerate(idx):
        o, n = int(los[s]["pixel_offset"]), int(los[s]["num_pixels"])
        parts.append(px[o:o + n])
        out_los[k]["pixel_offset"] = off
        off += n
    return out_los, (np.concatenate(parts) if parts else px[:0].copy())


def lone_run(engine, los, px, g, scale):
    cat = T.Catalog(engine, los, px, ORDER)
    b, _, st = T.xi_run(engine, cat, g, scale)
    cat.close()
    return b, st


def abs_sums(los, px, g, scale):
    return oracle.xi(los, px, ORDER, g.type, g.axes_array(), scale, mode=2)[0]


@pytest.mark.parametrize("name", ["cartesian", "polar", "observing"])
def test_drop_region_equals_reduced_run(engine, name):
    g = GRIDS[name]
    los, px, meta = small_catalog(n=200, seed=6, size_deg=8.0, max_pixels=120)
    scale = meta["scale"]
    cat = T.Catalog(engine, los, px, ORDER)
    ids, bins, groups, drop, st = T.xi_run_jackknife(engine, cat, g, scale, REGION_ORDER)
    full, _, fst = T.xi_run(engine, cat, g, scale)
    cat.close()
    reg = regions_of(los, REGION_ORDER)
    assert np.array_equal(ids, np.unique(reg))
    assert len(ids) >= 4
    assert_same_count(bins, full, abs_sums(los, px, g, scale), SAME_TOL)
    assert_same_count(groups[0], full, abs_sums(los, px, g, scale), SAME_TOL)
    assert st["num_sightline_pairs_used"] == fst["num_sightline_pairs_used"]
    assert st["num_pixel_pairs_used"] == fst["num_pixel_pairs_used"]
    for k, rid in enumerate(ids):
        r_los, r_px = subset(los, px, reg != rid)
        rb, _ = lone_run(engine, r_los, r_px, g, scale)
        assert_same_count(drop[k], rb, abs_sums(r_los, r_px, g, scale), SAME_TOL)
        assert drop[k]["num_pairs"].sum() < full["num_pairs"].sum()


def test_drop_region_with_groups(engine):
    g = GRIDS["cartesian"]
    los, px, meta = small_catalog(n=160, seed=9, size_deg=8.0, max_pixels=100)
    rng = np.random.default_rng(5)
    px2 = px.copy()
    px2["value"] = rng.normal(0, 0.2, len(px2)).astype(np.float32)
    parts = {4: (los, px2), 1: (los, px)}  # same sky positions in both groups
    m_los, m_px = T.synth.merge_groups([parts[4], parts[1]])
    m_los["group"] = np.r_[np.full(len(los), 4, np.uint32), np.full(len(los), 1, np.uint32)]
    cat = T.Catalog(engine, m_los, m_px, ORDER)
    ids, bins, groups, drop, st = T.xi_run_jackknife(engine, cat, g, meta["scale"], REGION_ORDER)
    cat.close()
    reg = regions_of(los, REGION_ORDER)
    ur = np.unique(reg)
    assert np.array_equal(ids, np.r_[(1 << 32) + ur, (4 << 32) + ur])
    for r, gid in enumerate((1, 4)):
        p_los, p_px = parts[gid]
        lb, _ = lone_run(engine, p_los, p_px, g, meta["scale"])
        assert_same_count(groups[r], lb, abs_sums(p_los, p_px, g, meta["scale"]), SAME_TOL)
    for f in FIELDS:
        assert np.array_equal(bins[f], groups[0][f] + groups[1][f])
    for k, key in enumerate(ids):
        gid, rid = int(key) >> 32, int(key) & 0xFFFFFFFF
        p_los, p_px = parts[gid]
        r_los, r_px = subset(p_los, p_px, reg != rid)
        rb, _ = lone_run(engine, r_los, r_px, g, meta["scale"])
        assert_same_count(drop[k], rb, abs_sums(r_los, r_px, g, meta["scale"]), SAME_TOL)


def test_jackknife_run_arguments(engine):
    los, px, meta = small_catalog(n=30, seed=2, size_deg=3.0, max_pixels=40)
    cat = T.Catalog(engine, los, px, ORDER)
    g = GRIDS["cartesian"]
    with pytest.raises(T.TosError):
        T.xi_run_jackknife(engine, cat, g, meta["scale"], ORDER + 1)  # coarser than the cells only
    with pytest.raises(T.TosError):
        T.xi_run_jackknife(engine, cat, g, meta["scale"], -1)
    # a jackknife run leaves no per-cell sums behind for the covariance calls
    T.xi_run_jackknife(engine, cat, g, meta["scale"], 3)
    with pytest.raises(T.TosError):
        T.cell_covariance(engine, cat, g.nbins)
    cat.close()


def test_subsample_covariance(engine):
    """The jackknife covariance of the one-pass subsamples against numpy:
    xi_k = didj/wgt (0 where wgt <= 0), cov = (N-1)/N sum (xi_k - mean)^T (xi_k - mean),
    to 1e-10 of the largest |cov| entry (FP64, different summation order)."""
    g = GRIDS["cartesian"]
    los, px, meta = small_catalog(n=200, seed=6, size_deg=8.0, max_pixels=120)
    cat = T.Catalog(engine, los, px, ORDER)
    ids, bins, groups, drop, st = T.xi_run_jackknife(engine, cat, g, meta["scale"], REGION_ORDER)
    cat.close()
    xi, mean, cov = T.subsample_covariance(engine, drop)
    wgt = drop["wgt"].astype(np.float64)
    X = np.where(wgt > 0, drop["didj"] / np.where(wgt > 0, wgt, 1.0), 0.0)
    assert np.array_equal(xi, X)
    n = len(ids)
    m = X.mean(axis=0)
    C = (n - 1) / n * (X - m).T @ (X - m)
    assert np.allclose(mean, m, rtol=0, atol=1e-12 * np.abs(m).max())
    assert np.abs(cov - C).max() <= 1e-10 * np.abs(C).max()
    assert np.allclose(cov, cov.T, rtol=0, atol=1e-12 * np.abs(C).max())


def test_jackknife_run_exact_path(engine):
    """TOS_XI_EXACT (every pixel pair in FP64, the pixel-pair kernel's direct
    adds on the 42-bit scale of positive fields) routes pairs to the same
    region slots: identical pair counts per subsample, and sums within
    REL_TOL of the FP64 oracle."""
    g = GRIDS["cartesian"]
    los, px, meta = small_catalog(n=120, seed=12, size_deg=6.0, max_pixels=80)
    cat = T.Catalog(engine, los, px, ORDER)
    ids, bins, _, drop, _ = T.xi_run_jackknife(engine, cat, g, meta["scale"], REGION_ORDER)
    ids2, bins2, _, drop2, st2 = T.xi_run_jackknife(engine, cat, g, meta["scale"], REGION_ORDER, exact=True)
    cat.close()
    assert st2["num_run_items"] == 0
    assert np.array_equal(ids, ids2)
    assert_counts_equal(bins2, bins)
    ob = oracle.xi(los, px, ORDER, g.type, g.axes_array(), meta["scale"], mode=1)[0]
    assert_counts_equal(bins2, ob)
    assert_sums_close(bins2, ob, abs_sums(los, px, g, meta["scale"]))
    for k in range(len(ids)):
        assert np.array_equal(drop2[k]["num_pairs"], drop[k]["num_pairs"])
