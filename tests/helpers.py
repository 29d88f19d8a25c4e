"""Shared helpers for the tests: small catalogues and result comparison."""
import numpy as np

from tos_b200 import PIXEL_DTYPE, SIGHTLINE_DTYPE, Grid, synth

FIELDS = ("didj", "di", "dj", "wgt", "wi", "wj", "z")


def truncate(los, px, max_pixels):
    """Keep at most max_pixels leading pixels of each sightline (compact layout)."""
    los2 = los.copy()
    out = []
    off = 0
    for s in range(len(los)):
        n = min(int(los[s]["num_pixels"]), max_pixels)
        o = int(los[s]["pixel_offset"])
        out.append(px[o:o + n])
        los2[s]["pixel_offset"] = off
        los2[s]["num_pixels"] = n
        off += n
    return los2, (np.concatenate(out) if out else np.zeros(0, dtype=PIXEL_DTYPE))


def small_catalog(n=120, seed=11, size_deg=3.0, max_pixels=None):
    los, px, meta = synth.small_patch(n, seed=seed, size_deg=size_deg)
    if max_pixels:
        los, px = truncate(los, px, max_pixels)
    return los, px, meta


def plate_catalog(n=90, seed=17, size_deg=6.0, max_pixels=48, spacing_deg=2.0):
    """A small catalogue on BOSS-like plates (synth.plate_tiling) with the
    platelist cases PlateBins meets: a plate listed twice (its second row,
    with a moved centre, is the one kept), a listed plate without sightlines
    and three sightlines on a plate missing from the platelist.  Returns
    (sightlines, pixels, platelist, meta)."""
    los, px, meta = small_catalog(n=n, seed=seed, size_deg=size_deg, max_pixels=max_pixels)
    los, plates = synth.plate_tiling(los, spacing_deg)
    used = np.unique(los["plate"])
    dup = plates[plates["plate"] == used[1]].copy()  # moved far enough to change the count
    dup["ra_center"] += np.float32(1.0)
    dup["dec_center"] -= np.float32(0.8)
    empty = np.zeros(1, dtype=plates.dtype)
    empty["plate"] = 9000
    empty["ra_center"] = plates["ra_center"][0]
    empty["dec_center"] = plates["dec_center"][0]
    plates = np.concatenate([plates, dup, empty])
    los = los.copy()
    los["plate"][[1, 5, 9]] = 8999  # not in the platelist
    return los, px, plates, meta


def as_matrix(bins):
    """XiBin structured array -> (n, 8) float64 with the count in column 7."""
    m = np.zeros((len(bins), 8))
    for k, f in enumerate(FIELDS):
        m[:, k] = bins[f]
    m[:, 7] = bins["num_pairs"]
    return m


def assert_counts_equal(gpu, ref):
    g = np.asarray(gpu["num_pairs"], dtype=np.int64)
    r = np.asarray(ref["num_pairs"], dtype=np.int64)
    bad = np.nonzero(g != r)[0]
    assert len(bad) == 0, f"{len(bad)} bins differ in pair count, first {bad[:10]}: gpu {g[bad[:10]]} ref {r[bad[:10]]}"


def rel_errors(gpu, ref, ref_abs=None):
    """Per-field worst relative error.  For each bin the error |gpu - ref| is
    divided by max(|ref|, 1e-6 * A) where A is the bin's sum of absolute
    values of the terms (FP64 oracle, mode 2): a signed sum that cancels to
    below 1e-6 of its own magnitude is judged against that magnitude, since no
    summation order (the FP64 oracle's included) determines it to 1e-6 of
    itself.  Also returns the plain |gpu - ref| / |ref| worst case."""
    out = {}
    for f in FIELDS:
        g, r = np.asarray(gpu[f], dtype=np.float64), np.asarray(ref[f], dtype=np.float64)
        a = np.abs(np.asarray(ref_abs[f], dtype=np.float64)) if ref_abs is not None else np.abs(r)
        denom = np.maximum(np.abs(r), 1e-6 * a)
        err = np.abs(g - r)
        nz = denom > 0
        out[f] = float(np.max(err[nz] / denom[nz])) if nz.any() else 0.0
        out[f + "_plain"] = float(np.max(err[r != 0] / np.abs(r[r != 0]))) if (r != 0).any() else 0.0
        out[f + "_at_zero"] = float(np.max(np.abs(g[~nz]))) if (~nz).any() else 0.0
    return out


# Relative tolerance of the weighted sums against the FP64 oracle, per bin.
REL_TOL = 1e-6


def assert_sums_close(gpu, ref, ref_abs=None, rel=REL_TOL):
    errs = rel_errors(gpu, ref, ref_abs)
    for f in FIELDS:
        assert errs[f] <= rel, f"field {f}: relative error {errs[f]:.3e} > {rel:.1e} ({errs})"
        assert errs[f + "_at_zero"] == 0.0, f"field {f} nonzero where the oracle is exactly 0"
    return errs


def assert_same_count(gpu, ref, ref_abs, tol):
    """Two engine counts of the same pairs (e.g. batched and alone): pair
    counts equal, and per bin and field |gpu - ref| <= tol * A with A the
    bin's sum of absolute values of the terms (FP64 oracle, mode 2); the
    two runs may convert to different fixed-point scales."""
    assert_counts_equal(gpu, ref)
    for f in FIELDS:
        g, r = np.asarray(gpu[f], dtype=np.float64), np.asarray(ref[f], dtype=np.float64)
        a = np.abs(np.asarray(ref_abs[f], dtype=np.float64))
        bad = np.nonzero(np.abs(g - r) > tol * a)[0]
        assert len(bad) == 0, f"field {f}: {len(bad)} bins differ, first {bad[:5]}: {g[bad[:5]]} vs {r[bad[:5]]}"


GRIDS = {
    "cartesian": Grid.cartesian(),
    "polar": Grid.polar(),
    "observing": Grid.observing(),
}
