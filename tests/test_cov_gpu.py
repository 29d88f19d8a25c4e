"""GPU covariances of the pair count against numpy on the oracle's per-cell
sums: the reference's per-cell covariance (XiEstimator.cc:60-97) and the
leave-one-region-out jackknife over coarser HEALPix regions."""
import numpy as np
import pytest

import tos_b200 as T
from helpers import GRIDS, small_catalog
from oracle import oracle

pytestmark = pytest.mark.gpu


def cell_samples(cells):
    """x_c[b] = didj/wgt (0 where wgt = 0), W_c = sum of wgt over bins with wgt > 0."""
    wgt = cells["wgt"]
    ok = wgt > 0
    x = np.where(ok, cells["didj"] / np.where(ok, wgt, 1.0), 0.0)
    return x, np.where(ok, wgt, 0.0).sum(axis=1)


def weighted_cov(x, w):
    W = w.sum()
    mean = (w[:, None] * x).sum(axis=0) / W
    d = x - mean
    return mean, (w[:, None] * d).T @ d / W


def assert_close(got, ref, rtol):
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) <= rtol * scale, (np.max(np.abs(got - ref)), scale)


@pytest.mark.parametrize("name", ["cartesian", "polar"])
def test_cell_covariance_matches_oracle(engine, name):
    los, px, meta = small_catalog(n=150, seed=31, size_deg=3.0)
    g = GRIDS[name]
    cat = T.Catalog(engine, los, px, 6)
    bins, cells, _ = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    mean, cov, W = T.cell_covariance(engine, cat, g.nbins)
    _, ocells, _, _ = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=1, subsamples=True)
    ox, ow = cell_samples(ocells)
    omean, ocov = weighted_cov(ox, ow)
    assert len(ocells) > 4
    np.testing.assert_allclose(W, ow.sum(), rtol=1e-12)
    assert_close(mean, omean, 1e-9)
    assert_close(cov, ocov, 1e-8)
    # and exactly the covariance of the engine's own per-cell output
    gx, gw = cell_samples(cells)
    gmean, gcov = weighted_cov(gx, gw)
    assert_close(cov, gcov, 1e-12)


def test_jackknife_matches_oracle(engine):
    los, px, meta = small_catalog(n=200, seed=32, size_deg=4.0)
    g = GRIDS["cartesian"]
    order, region_order = 6, 5
    cat = T.Catalog(engine, los, px, order)
    T.xi_run(engine, cat, g, meta["scale"])
    ids, xi, cov = T.jackknife(engine, cat, region_order, g.nbins)
    _, ocells, oids, _ = oracle.xi(los, px, order, g.type, g.axes_array(), meta["scale"], mode=1,
                                   subsamples=True)
    # region of a cell: that of any of its sightlines (cells nest in regions)
    cell_of = np.array([oracle.radec2pix(order, r, d) for r, d in zip(los["ra"], los["dec"])])
    reg_of = np.array([oracle.radec2pix(region_order, r, d) for r, d in zip(los["ra"], los["dec"])])
    cell_region = {c: reg for c, reg in zip(cell_of, reg_of)}
    regions = np.array(sorted(set(cell_region[c] for c in oids)))
    assert np.array_equal(ids, regions) and len(regions) >= 3
    D, G = ocells["didj"].sum(axis=0), ocells["wgt"].sum(axis=0)
    oxi = []
    for k in regions:
        m = np.array([cell_region[c] == k for c in oids])
        Gk = G - ocells["wgt"][m].sum(axis=0)
        Dk = D - ocells["didj"][m].sum(axis=0)
        oxi.append(np.where(Gk > 0, Dk / np.where(Gk > 0, Gk, 1.0), 0.0))
    oxi = np.array(oxi)
    n = len(regions)
    d = oxi - oxi.mean(axis=0)
    ocov = (n - 1) / n * d.T @ d
    assert_close(xi, oxi, 1e-9)
    assert_close(cov, ocov, 1e-7)


def test_covariance_needs_a_run(engine):
    los, px, meta = small_catalog(n=20, seed=2, size_deg=1.0, max_pixels=50)
    cat = T.Catalog(engine, los, px, 6)
    with pytest.raises(T.TosError):
        T.cell_covariance(engine, cat, 2500)
