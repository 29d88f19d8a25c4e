"""GPU parity of the brute-force cubic-grid estimator against the FP64 oracle."""
import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth  # noqa: F401  (T.synth)
from oracle import oracle

pytestmark = pytest.mark.gpu


def grid_points(n, spacing, seed, weights=False):
    rng = np.random.default_rng(seed)
    c = (np.arange(n) + 0.5) * spacing
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    w = rng.uniform(0.5, 2.0, n ** 3) if weights else np.ones(n ** 3)
    return np.stack([X.ravel(), Y.ravel(), Z.ravel(), rng.normal(size=n ** 3), w], 1).astype(np.float32)


@pytest.mark.parametrize("n,spacing,rmax,nbins,weights", [
    (16, 5.0, 200.0, 50, False),   # the reference's delta-micro geometry: 16^3 at 5 Mpc/h
    (20, 4.0, 60.0, 30, True),     # many pairs exactly on bin edges (r = 4*sqrt(k))
    (32, 4.0, 200.0, 100, False),  # the benchmark binning on a 32^3 grid
])
def test_brute_grid_vs_oracle(engine, n, spacing, rmax, nbins, weights):
    pts = grid_points(n, spacing, seed=n, weights=weights)
    ds, ws, ct, ms = T.brute_run(engine, pts, 0.0, rmax, nbins)
    ods, ows, oct_ = oracle.brute(pts, 0.0, rmax, nbins)
    assert np.array_equal(ct, oct_), np.nonzero(ct != oct_)[0][:10]
    assert int(ct.sum()) == len(pts) * (len(pts) - 1) // 2
    nz = ows != 0
    assert np.max(np.abs(ws[nz] - ows[nz]) / np.abs(ows[nz])) < 1e-9
    nzd = ods != 0
    assert np.max(np.abs(ds[nzd] - ods[nzd]) / np.abs(ods[nzd])) < 1e-6


@pytest.mark.parametrize("key", ["delta_nanoer", "delta_nano", "delta_micro", "delta_tinier"])
def test_brute_on_reference_sample_grids(engine, key):
    """The reference's own sample grids (sample-data/delta-*.dat, 2^3 to 32^3
    points at 5 Mpc/h), stored with the FP64 oracle's histogram for 100 bins
    over [0, 200) Mpc/h in tests/golden/golden_brute_sample.npz: separations
    10, 20, 30 ... Mpc/h fall exactly on bin edges."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_brute_sample.npz"))
    pts = z[key + "_points"]
    ds, ws, ct, _ = T.brute_run(engine, pts, float(z["rmin"]), float(z["rmax"]), int(z["nbins"]))
    assert np.array_equal(ct, z[key + "_counts"]), np.nonzero(ct != z[key + "_counts"])[0][:10]
    ows, ods = z[key + "_wsum"], z[key + "_dsum"]
    nz = ows != 0
    assert np.max(np.abs(ws[nz] - ows[nz]) / np.abs(ows[nz])) < 1e-9
    nzd = ods != 0
    assert np.max(np.abs(ds[nzd] - ods[nzd]) / np.abs(ods[nzd])) < 1e-6


def test_brute_random_points(engine):
    rng = np.random.default_rng(5)
    pts = np.concatenate([rng.uniform(0, 120, (3000, 3)), rng.normal(size=(3000, 1)),
                          rng.uniform(0.5, 2, (3000, 1))], 1).astype(np.float32)
    ds, ws, ct, _ = T.brute_run(engine, pts, 5.0, 100.0, 19)
    ods, ows, oct_ = oracle.brute(pts, 5.0, 100.0, 19)
    assert np.array_equal(ct, oct_)
    np.testing.assert_allclose(ws, ows, rtol=1e-9)
    nzd = ods != 0
    assert np.max(np.abs(ds[nzd] - ods[nzd]) / np.abs(ods[nzd])) < 1e-6


@pytest.mark.parametrize("nbins", [322, 323, 686, 687, 1000, 4096])
def test_brute_many_bins(engine, nbins):
    """Bin counts whose shared-memory windows do not fit the default 8 warps
    per block (above 686 bins the block holds fewer warps; above 322, fewer
    than 16), up to the 4096 limit, where a block holds one warp."""
    pts = grid_points(12, 5.0, seed=nbins, weights=True)
    ds, ws, ct, _ = T.brute_run(engine, pts, 0.0, 90.0, nbins)
    ods, ows, oct_ = oracle.brute(pts, 0.0, 90.0, nbins)
    assert np.array_equal(ct, oct_), np.nonzero(ct != oct_)[0][:10]
    nz = ows != 0
    assert np.max(np.abs(ws[nz] - ows[nz]) / np.abs(ows[nz])) < 1e-9
    nzd = ods != 0
    assert np.max(np.abs(ds[nzd] - ods[nzd]) / np.abs(ods[nzd])) < 1e-6


def test_brute_rejects_too_many_bins(engine):
    pts = grid_points(4, 5.0, seed=1)
    with pytest.raises(T.TosError) as e:
        T.brute_run(engine, pts, 0.0, 90.0, 4097)
    assert e.value.status == 1


def test_brute_full_config_rows_vs_oracle(engine):
    """The 64^3 benchmark grid: pairs (i, j) with i < 256 and j > i, the
    difference of the engine's all-pairs counts over the grid and over its
    rows [256, n), against the FP64 oracle bin by bin."""
    pts = T.synth.grf_grid(64, 256.0, seed=3)
    m = 256
    full = T.brute_run(engine, pts, 0.0, 200.0, 100)
    tail = T.brute_run(engine, pts[m:], 0.0, 200.0, 100)
    ods, ows, oct_ = oracle.brute_rows(pts, m, 0.0, 200.0, 100)
    ct = full[2].astype(np.int64) - tail[2].astype(np.int64)
    assert np.array_equal(ct, oct_.astype(np.int64))
    assert int(oct_.sum()) == sum(len(pts) - 1 - i for i in range(m))
    ws = full[1] - tail[1]
    np.testing.assert_array_equal(ws, ows)  # w = 1: weight sums are counts
    ds = full[0] - tail[0]
    nzd = ods != 0
    assert np.max(np.abs(ds[nzd] - ods[nzd]) / np.abs(ods[nzd])) < 1e-6


def test_brute_full_config_invariants(engine):
    pts = T.synth.grf_grid(64, 256.0, seed=3)
    ds, ws, ct, ms = T.brute_run(engine, pts, 0.0, 200.0, 100)
    n = len(pts)
    assert int(ct.sum()) == n * (n - 1) // 2
    np.testing.assert_allclose(ws, ct.astype(np.float64), rtol=0, atol=0)  # w = 1: sum of weights = count
    assert ct[0] == 0  # no pair below r = 0


def test_brute_tune_pick_gives_identical_results(engine):
    """The autotuner times every launch shape on the points and keeps the
    fastest for this bin count; counts and sums are exact integer sums, so the
    tuned shape gives the same results bit for bit."""
    pts = T.synth.grf_grid(24, 96.0, seed=9)
    before = T.brute_run(engine, pts, 0.0, 80.0, 40)
    k, w = T.brute_tune(engine, pts, 0.0, 80.0, 40)
    assert k in (1, 2, 4) and w in (4, 8, 16)
    after = T.brute_run(engine, pts, 0.0, 80.0, 40)
    for a, b in zip(before[:3], after[:3]):
        assert np.array_equal(a, b)
    ods, ows, oct_ = oracle.brute(pts, 0.0, 80.0, 40)
    assert np.array_equal(after[2], oct_)
