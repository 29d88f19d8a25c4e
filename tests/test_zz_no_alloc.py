"""tos_brute_run_noalloc: the brute-force pair count for callers that cannot
allocate GPU memory (their own pool owns every byte, or a cudaMalloc would
synchronise the device where they cannot afford it).  Through the C ABI, two
calls in a row with different inputs must give the results of tos_brute_run
(the allocating entry point) on the same points: counts bit-exact, weight
sums to 1e-9 and signal sums to 1e-6 relative, the tolerances of the brute
parity tests.  The second call also shows that the shared static scratch is
cleared between calls.

This file sorts last so that a run stopping at the first failure has run
every other test before it; it also passes alone in a fresh process."""
import numpy as np
import pytest

import tos_b200 as T

pytestmark = pytest.mark.gpu


def make_points(n, seed):
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.uniform(0, 90, (n, 3)), rng.normal(size=(n, 1)),
                           rng.uniform(0.5, 2, (n, 1))], 1).astype(np.float32)


def run_noalloc(engine, pts, rmin, rmax, nbins):
    import torch
    dev = torch.device("cuda", 0)
    d_pts = torch.from_numpy(pts).to(dev)
    d_ds = torch.zeros(nbins + 2, dtype=torch.float64, device=dev)
    d_ws = torch.zeros(nbins + 2, dtype=torch.float64, device=dev)
    d_ct = torch.zeros(nbins + 2, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    T.brute_run_noalloc(engine, d_pts.data_ptr(), len(pts), rmin, rmax, nbins, d_ds.data_ptr(),
                        d_ws.data_ptr(), d_ct.data_ptr())
    return d_ds.cpu().numpy(), d_ws.cpu().numpy(), d_ct.cpu().numpy().astype(np.uint64)


def check_same(got, ref):
    ds, ws, ct = got
    rds, rws, rct = ref[:3]
    assert np.array_equal(ct, rct), np.nonzero(ct != rct)[0][:10]
    nz = rws != 0
    assert np.max(np.abs(ws[nz] - rws[nz]) / np.abs(rws[nz])) < 1e-9
    assert np.all(ws[~nz] == 0)
    nzd = rds != 0
    assert np.max(np.abs(ds[nzd] - rds[nzd]) / np.abs(rds[nzd])) < 1e-6


def test_noalloc_matches_allocating_entry_point_twice(engine):
    pytest.importorskip("torch")
    a = make_points(4000, seed=1)
    b = make_points(2500, seed=2)
    # first call: the larger case; second call: fewer points and bins, so any
    # sums left in the shared scratch by the first call would show
    check_same(run_noalloc(engine, a, 0.0, 120.0, 40), T.brute_run(engine, a, 0.0, 120.0, 40))
    check_same(run_noalloc(engine, b, 5.0, 80.0, 17), T.brute_run(engine, b, 5.0, 80.0, 17))


def test_noalloc_at_the_bin_limit(engine):
    pytest.importorskip("torch")
    a = make_points(3000, seed=3)
    check_same(run_noalloc(engine, a, 0.0, 100.0, 4096), T.brute_run(engine, a, 0.0, 100.0, 4096))


def test_noalloc_rejects_sizes_beyond_its_scratch(engine):
    with pytest.raises(T.TosError) as e:
        T.brute_run_noalloc(engine, 1, (1 << 18) + 1, 0.0, 100.0, 10, 1, 1, 1)
    assert e.value.status == 1 and "at most 262144 points" in str(e.value)
    with pytest.raises(T.TosError):
        T.brute_run_noalloc(engine, 1, 100, 0.0, 100.0, 4097, 1, 1, 1)
