"""CPU tests of the oracle: against a second, literal restatement of the
reference loop, against hand-computed bin edges, and against the committed
golden fixtures.  No GPU needed."""
import math
import os

import numpy as np
import pytest

from helpers import FIELDS, GRIDS, as_matrix, small_catalog
from oracle import oracle
import ref_loop

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["cartesian", "polar", "observing"])
@pytest.mark.parametrize("mode", [0, 1])
def test_oracle_matches_literal_loop(name, mode):
    los, px, meta = small_catalog(n=14, seed=5, size_deg=1.0, max_pixels=40)
    g = GRIDS[name]
    bins, _, _, st = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], mode=mode, nthreads=2)
    ref, rst = ref_loop.xi(los, px, g.type, g.axes_array(), meta["scale"], mode=mode)
    m = as_matrix(bins)
    assert np.array_equal(m[:, 7], ref[:, 7])
    assert m[:, 7].sum() > 0
    # identical expression order and accumulation order -> identical sums
    np.testing.assert_allclose(m[:, :7], ref[:, :7], rtol=1e-13, atol=1e-13)
    for k in ("num_sightline_pairs_used", "num_pixel_pairs", "num_pixel_pairs_used"):
        assert st[k] == rst[k]


def test_oracle_thread_count_invariant():
    los, px, meta = small_catalog(n=60, seed=9, size_deg=2.0, max_pixels=64)
    g = GRIDS["cartesian"]
    a = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], nthreads=1)[0]
    b = oracle.xi(los, px, 6, g.type, g.axes_array(), meta["scale"], nthreads=7)[0]
    assert np.array_equal(a["num_pairs"], b["num_pairs"])
    for f in FIELDS:  # per-cell sums are merged in cell order: identical
        assert np.array_equal(a[f], b[f])


def _axes(spec):
    return np.array(spec, dtype=np.float64)


def test_cartesian_bin_edges_known_answers():
    # [0:200]*50 x [0:200]*50 x [3.556:3.735]*1; both pixels on one line of
    # sight direction (c = 1): r_perp comes only from the float rounding of d1*d1.
    ax = _axes([0, 200, 50, 0, 200, 50, 3.556, 3.735, 1])
    d1 = np.float32(4000.0)  # d1*d1 = 1.6e7 exactly representable -> r_perp = 0
    for dpar, expect in [(0.0, 0), (3.999, 0), (4.0, 1), (7.5, 1), (8.0, 2), (199.5, 49), (200.0, None)]:
        d2 = np.float32(4000.0 + dpar)
        idx = oracle.bin_pair(1, ax, 3586.0, d1, np.float32(3.6), d2, np.float32(3.6), 1.0)
        if expect is None:
            assert idx is None
        else:
            assert idx == expect * 50, (dpar, idx)
    # transverse: same distance, angle chosen so r_perp^2 = 2 d^2 (1-c) hits 4 Mpc/h
    d = np.float32(4096.0)
    for rp, expect in [(3.9, 0), (4.1, 1), (7.99, 1), (8.01, 2), (199.9, 49), (200.1, None)]:
        c = 1.0 - rp * rp / (2.0 * float(d) * float(d))
        idx = oracle.bin_pair(1, ax, 3586.0, d, np.float32(3.6), d, np.float32(3.6), c)
        if expect is None:
            assert idx is None
        else:
            assert idx == expect, (rp, idx)


def test_polar_quirks():
    ax = _axes([0, 200, 50, 0, 1, 20, 3.556, 3.735, 1])
    d = np.float32(4096.0)
    # identical pixel positions: r == 0 is skipped (XiEstimator.cc:192)
    assert oracle.bin_pair(0, ax, 3586.0, d, np.float32(3.6), d, np.float32(3.6), 1.0) is None
    # purely radial separation: mu = 1 -> bin 20 is outside [0:1]*20 -> skipped
    assert oracle.bin_pair(0, ax, 3586.0, d, np.float32(3.6), np.float32(4106.0), np.float32(3.6), 1.0) is None
    # transverse separation: mu = 0, r = 10 -> r bin 2, mu bin 0
    c = 1.0 - 100.0 / (2.0 * 4096.0 * 4096.0)
    assert oracle.bin_pair(0, ax, 3586.0, d, np.float32(3.6), d, np.float32(3.6), c) == 2 * 20


def test_unchecked_z_index_overflow():
    # z axis [3.5:3.6]*2: zbin = trunc((0.5*(l1+l2) - 3.5) * 1/2) -> 0 for z < 5.5;
    # a loglam pair far above the axis gives zbin = 1 -> idx = 1 + 2*b (aliasing)
    ax = _axes([0, 200, 50, 0, 200, 50, 3.5, 3.6, 2])
    d = np.float32(4000.0)
    idx = oracle.bin_pair(1, ax, 3586.0, d, np.float32(5.6), d, np.float32(5.6), 1.0)
    assert idx == 1
    # zbin = 6000 runs past the 5000-bin grid: the reference writes out of
    # bounds (undefined behaviour); the oracle and the engine count it instead
    l = np.float32(12003.5)
    idx = oracle.bin_pair(1, ax, 3586.0, d, l, d, l, 1.0)
    assert idx == 0xFFFFFFFF


def test_healpix_known_pixels_and_cross_check():
    from tos_b200 import synth
    # nside = 1: north pole -> 0, equator at phi = 0 -> 4, south pole -> 8
    assert oracle.radec2pix(0, 0.0, math.pi / 2) == 0
    assert oracle.radec2pix(0, 0.0, 0.0) == 4
    assert oracle.radec2pix(0, 0.0, -math.pi / 2) == 8
    # nside = 8: independent vectorised restatement (tos_b200.synth) on random points
    rng = np.random.default_rng(1)
    ra = rng.uniform(0, 2 * math.pi, 20000)
    dec = np.arcsin(rng.uniform(-1, 1, 20000))
    mine = synth.ang2pix_ring(8, 0.5 * math.pi - dec, ra)
    orc = np.array([oracle.radec2pix(3, r, d) for r, d in zip(ra, dec)])
    # the vectorised version has no sin(theta) refinement near the poles
    far = np.abs(np.cos(0.5 * math.pi - dec)) < 0.99
    assert np.array_equal(mine[far], orc[far])
    assert orc.min() >= 0 and orc.max() < 768
    counts = np.bincount(orc, minlength=768)
    assert counts.min() > 0  # equal-area pixels all receive points


def test_brute_oracle_literal():
    rng = np.random.default_rng(4)
    c = np.arange(4) * 5.0 + 2.5
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel(), rng.normal(size=64), rng.uniform(0.5, 2, 64)], 1).astype(np.float32)
    ds, ws, ct = oracle.brute(pts, 0.0, 10.0, 5, nthreads=3)
    eds, ews, ect = np.zeros(7), np.zeros(7), np.zeros(7, dtype=np.int64)
    p = pts.astype(np.float64)
    for i in range(64):
        for j in range(i + 1, 64):
            r = math.sqrt(((p[i, :3] - p[j, :3]) ** 2).sum())
            k = 0 if r < 0 else (6 if r >= 10.0 else min(int(math.floor(r / 2.0)), 4) + 1)
            eds[k] += p[i, 4] * p[i, 3] * p[j, 4] * p[j, 3]
            ews[k] += p[i, 4] * p[j, 4]
            ect[k] += 1
    assert np.array_equal(ct.astype(np.int64), ect)
    np.testing.assert_allclose(ds, eds, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(ws, ews, rtol=1e-12)


@pytest.mark.parametrize("fixture", ["golden_cartesian", "golden_polar", "golden_observing"])
def test_oracle_reproduces_golden(fixture):
    path = os.path.join(GOLDEN, fixture + ".npz")
    if not os.path.exists(path):
        pytest.skip("golden fixture not generated")
    z = np.load(path)
    los, px = z["sightlines"], z["pixels"]
    axes = z["axes"]
    bins, cells, ids, st = oracle.xi(los, px, int(z["order"]), int(z["coord"]), axes, float(z["scale"]),
                                     mode=1, nthreads=4, subsamples=True)
    assert np.array_equal(bins["num_pairs"], z["num_pairs"])
    assert np.array_equal(ids, z["cell_ids"])
    assert np.array_equal(cells["num_pairs"], z["cell_num_pairs"])
    for f in FIELDS:
        np.testing.assert_allclose(bins[f], z[f], rtol=1e-12, atol=0)


def test_plate_ring_covers_the_disc_above_1p5_degrees():
    """PlateBins' neighbour test |theta - 1.5 deg| < max_ang holds for every
    plate with a sightline within max_ang when max_ang > 1.5 deg and every
    sightline lies within 1.5 deg of its plate's centre: then plate cells
    bin the same pairs as HEALPix cells.  Below 1.5 deg the ring skips plates
    whose centre is nearer than 1.5 deg - max_ang, and pairs are lost."""
    from helpers import GRIDS, small_catalog
    from tos_b200 import synth
    los, px, meta = small_catalog(n=120, seed=9, size_deg=6.0, max_pixels=24)
    los, plates = synth.plate_tiling(los, 2.0)
    g = GRIDS["cartesian"]
    for factor, same in ((1.0, True), (4.0, False)):
        scale = factor * meta["scale"]
        hb, _, _, hst = oracle.xi(los, px, 6, g.type, g.axes_array(), scale, mode=1, nthreads=4)
        pb, _, _, pst = oracle.xi_plates(los, px, plates, g.type, g.axes_array(), scale, mode=1, nthreads=4)
        assert (hst["max_ang"] > math.radians(1.5)) == same
        if same:
            assert np.array_equal(pb["num_pairs"], hb["num_pairs"])
            assert pst["num_sightline_pairs_used"] == hst["num_sightline_pairs_used"]
        else:
            assert 0 < pb["num_pairs"].sum() < hb["num_pairs"].sum()


def _numpy_brute(pts, rmin, rmax, nbins):
    """All pairs i < j of the brute-force histogram in FP64 from the float
    coordinates (gpu/brute.cu:40-48 with bucketxi's double separation):
    bin 0 below rmin, nbins + 1 at or above rmax."""
    p = pts.astype(np.float64)
    spacing = (rmax - rmin) / nbins
    cnt = np.zeros(nbins + 2, dtype=np.int64)
    wsum = np.zeros(nbins + 2)
    for i in range(len(p) - 1):
        d = p[i + 1:, :3] - p[i, :3]
        r = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        k = np.floor((r - rmin) / spacing)
        idx = np.where(r < rmin, 0, np.where(r >= rmax, nbins + 1, np.minimum(k, nbins - 1) + 1)).astype(np.int64)
        cnt += np.bincount(idx, minlength=nbins + 2)
        wsum += np.bincount(idx, weights=p[i, 4] * p[i + 1:, 4], minlength=nbins + 2)
    return cnt, wsum


def test_brute_oracle_on_reference_sample_grids():
    """The reference's own sample grids (sample-data/delta-*.dat: 2^3 to 32^3
    points at 5 Mpc/h, kept in tests/golden/golden_brute_sample.npz by
    make_brute_sample.py): the oracle reproduces the stored histogram, and an
    independent FP64 pair loop bins the same pairs (many separations, 5 sqrt(k)
    Mpc/h, fall exactly on the 2 Mpc/h bin edges)."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_brute_sample.npz"))
    rmin, rmax, nbins = float(z["rmin"]), float(z["rmax"]), int(z["nbins"])
    for key in ("delta_nanoer", "delta_nano", "delta_micro", "delta_tinier"):
        pts = z[key + "_points"]
        ds, ws, ct = oracle.brute(pts, rmin, rmax, nbins, nthreads=4)
        assert np.array_equal(ct, z[key + "_counts"]), key
        assert int(ct.sum()) == len(pts) * (len(pts) - 1) // 2
        np.testing.assert_allclose(ws, z[key + "_wsum"], rtol=1e-12)
        np.testing.assert_allclose(ds, z[key + "_dsum"], rtol=1e-9, atol=1e-9 * np.abs(z[key + "_dsum"]).max())
        if len(pts) <= 4096:
            cnt, wsum = _numpy_brute(pts, rmin, rmax, nbins)
            assert np.array_equal(cnt, ct.astype(np.int64)), key
            np.testing.assert_allclose(wsum, ws, rtol=1e-12)
