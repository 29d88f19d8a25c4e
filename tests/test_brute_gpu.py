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


def test_brute_full_config_invariants(engine):
    pts = T.synth.grf_grid(64, 256.0, seed=3)
    ds, ws, ct, ms = T.brute_run(engine, pts, 0.0, 200.0, 100)
    n = len(pts)
    assert int(ct.sum()) == n * (n - 1) // 2
    np.testing.assert_allclose(ws, ct.astype(np.float64), rtol=0, atol=0)  # w = 1: sum of weights = count
    assert ct[0] == 0  # no pair below r = 0
