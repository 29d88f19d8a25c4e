"""Parity of the engine's per-cell results against the reference, on a chosen
set of primary cells.

TEST INFRASTRUCTURE: the checker that tests/ and bench.py (after its timed
steps) run on the engine's output; the engine never loads it.

For the chosen cells (HEALPix ids and their positions in the ascending list
of occupied cells):
- the reference's own XiEstimator (oracle/_ref/libtosref.so, strict build;
  where it has not been built, the oracle in reference-arithmetic mode,
  which the golden fixtures pin to it bit for bit) gives the pair counts the
  engine must equal bin by bin, and its float-product sums;
- the FP64 oracle (mode 1) gives the sums the engine must match to a
  relative 1e-6 per bin, judged against max(|sum|, 1e-6 * A) with A the sum
  of absolute values of the terms (mode 2), so that a bin whose signed sum
  cancels is judged against its own magnitude.
"""
from __future__ import annotations

import os

import numpy as np

from . import oracle

FIELDS = ("didj", "di", "dj", "wgt", "wi", "wj", "z")
POSITIVE = ("wgt", "wi", "wj", "z")
SIGNED = ("didj", "di", "dj")
REL_TOL = 1e-6


def pick_cells(pairs_per_cell, pixels_per_cell, n_median=16, n_costly=4, n_edge=4, seed=0):
    """Positions of the cells to check: the n_costly cells with the most
    binned pairs, n_edge occupied cells with the fewest pairs per own pixel
    (cells at the edge of the sky mask, where the neighbour discs are cut),
    and n_median cells nearest the median pair count (seeded tie-break)."""
    cost = np.asarray(pairs_per_cell, dtype=np.float64)
    pix = np.asarray(pixels_per_cell, dtype=np.float64)
    rng = np.random.default_rng(seed)
    chosen = list(np.argsort(cost)[::-1][:n_costly])
    live = np.nonzero((cost > 0) & (pix > 0))[0]
    ratio = cost[live] / pix[live]
    for k in live[np.argsort(ratio)]:
        if len(chosen) >= n_costly + n_edge:
            break
        if k not in chosen:
            chosen.append(int(k))
    order = np.argsort(np.abs(cost - np.median(cost[cost > 0])) + rng.uniform(0, 1e-3, len(cost)))
    for k in order:
        if len(chosen) >= n_costly + n_edge + n_median:
            break
        if k not in chosen and cost[k] > 0:
            chosen.append(int(k))
    return np.sort(np.array(chosen, dtype=np.int64))


def compare(rows, ref_rows, fp64_rows, abs_rows):
    """Per-bin comparison of engine rows with the reference's rows (counts,
    float-product sums) and the FP64 oracle's (sums).  Returns a summary."""
    out = {"bins_compared": int(np.asarray(rows["num_pairs"]).size)}
    out["counts_equal"] = bool(np.array_equal(rows["num_pairs"], ref_rows["num_pairs"]))
    out["reference_counts_equal_fp64_oracle"] = bool(np.array_equal(ref_rows["num_pairs"], fp64_rows["num_pairs"]))
    out["pairs_compared"] = int(np.asarray(ref_rows["num_pairs"]).sum())
    worst, worst_ref = {}, {}
    for f in FIELDS:
        g = np.asarray(rows[f], dtype=np.float64)
        r = np.asarray(fp64_rows[f], dtype=np.float64)
        a = np.abs(np.asarray(abs_rows[f], dtype=np.float64))
        denom = np.maximum(np.abs(r), 1e-6 * a)
        err = np.abs(g - r)
        nz = denom > 0
        worst[f] = float(np.max(err[nz] / denom[nz])) if nz.any() else 0.0
        if (~nz).any() and np.any(g[~nz] != 0):
            worst[f] = float("inf")
        # against the reference's float products: relative for positive sums,
        # relative to the absolute-value sum for the signed ones
        rr = np.asarray(ref_rows[f], dtype=np.float64)
        scale = np.abs(rr) if f in POSITIVE else a
        ok = scale > 0
        worst_ref[f] = float(np.max(np.abs(g - rr)[ok] / scale[ok])) if ok.any() else 0.0
    out["max_rel_err_vs_fp64"] = max(worst.values())
    out["max_rel_err_vs_fp64_by_field"] = worst
    out["max_rel_err_vs_reference"] = max(worst_ref.values())
    out["rel_tol"] = REL_TOL
    out["pass"] = bool(out["counts_equal"] and out["max_rel_err_vs_fp64"] <= REL_TOL)
    return out


def check_cells(rows, cell_pos, cell_ids, los, px, order, grid_type, axes, scale, nthreads=0):
    """Compare engine rows (one per chosen cell, in cell_pos order) with the
    reference and the FP64 oracle run on the same primary cells."""
    nthreads = nthreads or (os.cpu_count() or 1)
    cell_pos = np.asarray(cell_pos, dtype=np.int64)
    cell_ids = np.asarray(cell_ids, dtype=np.int64)
    if oracle.ref_available("strict"):
        _, _, ref_rows, rids, rst = oracle.ref_xi(los, px, order, grid_type, axes, scale, nthreads=nthreads,
                                                  cell_subset=cell_ids, subsamples=True)
        assert np.array_equal(rids, cell_ids), "reference ran other cells"
        checker = "reference XiEstimator built from its sources (oracle/_ref/libtosref.so)"
    else:
        _, ref_all, oids, _ = oracle.xi(los, px, order, grid_type, axes, scale, mode=0, nthreads=nthreads,
                                        cell_subset=cell_pos.astype(np.uint32), subsamples=True)
        assert np.array_equal(oids[cell_pos], cell_ids), "oracle cells differ"
        ref_rows = ref_all[cell_pos]
        checker = "oracle in reference arithmetic (pinned to the reference by tests/golden)"
    _, fp_all, oids, _ = oracle.xi(los, px, order, grid_type, axes, scale, mode=1, nthreads=nthreads,
                                   cell_subset=cell_pos.astype(np.uint32), subsamples=True)
    assert np.array_equal(oids[cell_pos], cell_ids), "oracle cells differ"
    fp_rows = fp_all[cell_pos]
    del fp_all
    _, ab_all, _, _ = oracle.xi(los, px, order, grid_type, axes, scale, mode=2, nthreads=nthreads,
                                cell_subset=cell_pos.astype(np.uint32), subsamples=True)
    ab_rows = ab_all[cell_pos]
    del ab_all
    out = compare(rows, ref_rows, fp_rows, ab_rows)
    out["checker"] = checker
    out["cells"] = int(len(cell_ids))
    return out
