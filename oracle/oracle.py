"""ctypes wrappers of the CPU oracle (oracle/xi_oracle.c) and of the
reference's own XiEstimator built from its unchanged sources
(oracle/ref_harness.cc -> oracle/_ref/libtosref*.so).

TEST INFRASTRUCTURE: used by tests/, __graft_entry__.smoke() and the CPU
legs of bench.py only, as the checker or the timed reference CPU path.
The engine never loads either library.  The oracle is pinned to the
reference build: tests/golden holds the reference build's outputs for the
golden catalogues, and tests compare the oracle with them (and with the
live reference build wherever oracle/_ref has been built).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
XIBIN_DTYPE = np.dtype([("didj", "<f8"), ("di", "<f8"), ("dj", "<f8"), ("wgt", "<f8"), ("wi", "<f8"),
                        ("wj", "<f8"), ("z", "<f8"), ("num_pairs", "<i8")])


class OrcStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("num_sightline_pairs_used", "num_pixels", "num_pixel_pairs",
                                          "num_pixel_pairs_used", "num_index_overflow")] + [
        ("max_ang", C.c_double), ("cos_max_ang", C.c_double), ("num_sightline_pairs", C.c_uint64)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


_libs = {}


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(kind: str = "strict") -> C.CDLL:
    """kind: 'strict' (parity reference) or 'fast' (reference build flags, timing)."""
    if kind not in _libs:
        path = os.path.join(_HERE, f"liboracle_{kind}.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, sz, i32, dbl = C.c_void_p, C.c_size_t, C.c_int, C.c_double
        L.orc_xi.argtypes = [vp, vp, vp, vp, sz, vp, i32, i32, vp, dbl, i32, i32, vp, sz, vp, vp, vp,
                             C.POINTER(OrcStats)]
        L.orc_xi.restype = C.c_long
        L.orc_xi_plates.argtypes = [vp, vp, vp, vp, vp, sz, vp, vp, vp, vp, sz, i32, vp, dbl, i32, i32, vp, sz,
                                    vp, vp, vp, C.POINTER(OrcStats)]
        L.orc_xi_plates.restype = C.c_long
        L.orc_cell_costs.argtypes = [vp, vp, vp, sz, i32, i32, vp, dbl, vp]
        L.orc_cell_costs.restype = C.c_long
        L.orc_brute.argtypes = [vp, sz, dbl, dbl, i32, i32, vp, vp, vp]
        L.orc_brute.restype = C.c_int
        L.orc_brute_rows.argtypes = [vp, sz, sz, dbl, dbl, i32, i32, vp, vp, vp]
        L.orc_brute_rows.restype = C.c_int
        L.orc_radec2pix.argtypes = [i32, dbl, dbl]
        L.orc_radec2pix.restype = C.c_int64
        L.orc_bin_pair.argtypes = [i32, vp, dbl, C.c_float, C.c_float, C.c_float, C.c_float, dbl,
                                   C.POINTER(C.c_uint32)]
        L.orc_bin_pair.restype = C.c_int
        _libs[kind] = L
    return _libs[kind]


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def xi(sightlines, pixels, order: int, coord: int, axes, scale: float, mode: int = 1, nthreads: int = 0,
       cell_subset=None, subsamples: bool = False, kind: str = "strict"):
    """Oracle pair count.  Returns (bins, cells or None, cell_ids, stats).
    mode 0: reference arithmetic (float products); mode 1: FP64 sums;
    mode 2: FP64 sums of absolute values of the signed terms."""
    L = lib(kind)
    ra = np.ascontiguousarray(sightlines["ra"], dtype=np.float64)
    dec = np.ascontiguousarray(sightlines["dec"], dtype=np.float64)
    off = np.ascontiguousarray(sightlines["pixel_offset"], dtype=np.uint64)
    npx = np.ascontiguousarray(sightlines["num_pixels"], dtype=np.uint32)
    px = np.ascontiguousarray(pixels)
    axes = np.ascontiguousarray(axes, dtype=np.float64)
    nb = int(axes[2] * axes[5] * axes[8])
    ncells = L.orc_cell_costs(_p(ra), _p(dec), _p(npx), len(ra), order, coord, _p(axes), scale, None)
    bins = np.zeros(nb, dtype=XIBIN_DTYPE)
    cells = np.zeros((ncells, nb), dtype=XIBIN_DTYPE) if subsamples else None
    ids = np.zeros(ncells, dtype=np.int64)
    sub = None if cell_subset is None else np.ascontiguousarray(cell_subset, dtype=np.uint32)
    st = OrcStats()
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    r = L.orc_xi(_p(ra), _p(dec), _p(off), _p(npx), len(ra), _p(px), order, coord, _p(axes), scale, mode,
                 nthreads, _p(sub), 0 if sub is None else len(sub), _p(bins), _p(cells), _p(ids), C.byref(st))
    if r < 0:
        raise ValueError("oracle rejected the input")
    return bins, cells, ids, st.as_dict()


def _platelist(platelist):
    """(plate ids int32, RACEN float32, DECCEN float32) of a platelist given as
    a structured array with fields plate, ra_center, dec_center (degrees)."""
    return (np.ascontiguousarray(platelist["plate"], dtype=np.int32),
            np.ascontiguousarray(platelist["ra_center"], dtype=np.float32),
            np.ascontiguousarray(platelist["dec_center"], dtype=np.float32))


def xi_plates(sightlines, pixels, platelist, coord: int, axes, scale: float, mode: int = 1, nthreads: int = 0,
              cell_subset=None, subsamples: bool = False, kind: str = "strict"):
    """Oracle pair count with sightlines binned by their plate (PlateBins):
    cells are the sightlines' plate ids, neighbours the platelist plates
    whose centres pass PlateBins' ring test.  Returns (bins, cells or None,
    cell_ids, stats); stats also has num_sightline_pairs (candidates)."""
    L = lib(kind)
    ra = np.ascontiguousarray(sightlines["ra"], dtype=np.float64)
    dec = np.ascontiguousarray(sightlines["dec"], dtype=np.float64)
    plate = np.ascontiguousarray(sightlines["plate"], dtype=np.int32)
    off = np.ascontiguousarray(sightlines["pixel_offset"], dtype=np.uint64)
    npx = np.ascontiguousarray(sightlines["num_pixels"], dtype=np.uint32)
    px = np.ascontiguousarray(pixels)
    axes = np.ascontiguousarray(axes, dtype=np.float64)
    lp, lra, ldec = _platelist(platelist)
    nb = int(axes[2] * axes[5] * axes[8])
    ncells = len(np.unique(plate))
    bins = np.zeros(nb, dtype=XIBIN_DTYPE)
    cells = np.zeros((ncells, nb), dtype=XIBIN_DTYPE) if subsamples else None
    ids = np.zeros(ncells, dtype=np.int64)
    sub = None if cell_subset is None else np.ascontiguousarray(cell_subset, dtype=np.uint32)
    st = OrcStats()
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    r = L.orc_xi_plates(_p(ra), _p(dec), _p(plate), _p(off), _p(npx), len(ra), _p(px), _p(lp), _p(lra), _p(ldec),
                        len(lp), coord, _p(axes), scale, mode, nthreads, _p(sub), 0 if sub is None else len(sub),
                        _p(bins), _p(cells), _p(ids), C.byref(st))
    if r < 0:
        raise ValueError("oracle rejected the input")
    return bins, cells, ids, st.as_dict()


def cell_costs(sightlines, order: int, coord: int, axes, scale: float, kind: str = "strict"):
    L = lib(kind)
    ra = np.ascontiguousarray(sightlines["ra"], dtype=np.float64)
    dec = np.ascontiguousarray(sightlines["dec"], dtype=np.float64)
    npx = np.ascontiguousarray(sightlines["num_pixels"], dtype=np.uint32)
    axes = np.ascontiguousarray(axes, dtype=np.float64)
    n = L.orc_cell_costs(_p(ra), _p(dec), _p(npx), len(ra), order, coord, _p(axes), scale, None)
    cost = np.zeros(n, dtype=np.uint64)
    L.orc_cell_costs(_p(ra), _p(dec), _p(npx), len(ra), order, coord, _p(axes), scale, _p(cost))
    return cost


def brute(points, rmin: float, rmax: float, nbins: int, nthreads: int = 0, kind: str = "strict"):
    L = lib(kind)
    pts = np.ascontiguousarray(points, dtype=np.float32)
    dsum = np.zeros(nbins + 2)
    wsum = np.zeros(nbins + 2)
    cnt = np.zeros(nbins + 2, dtype=np.uint64)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    L.orc_brute(_p(pts), len(pts), rmin, rmax, nbins, nthreads, _p(dsum), _p(wsum), _p(cnt))
    return dsum, wsum, cnt


def brute_rows(points, rows: int, rmin: float, rmax: float, nbins: int, nthreads: int = 0, kind: str = "strict"):
    """Pairs (i, j) with i < rows and i < j: the first rows of the grid against every later row."""
    L = lib(kind)
    pts = np.ascontiguousarray(points, dtype=np.float32)
    dsum = np.zeros(nbins + 2)
    wsum = np.zeros(nbins + 2)
    cnt = np.zeros(nbins + 2, dtype=np.uint64)
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    L.orc_brute_rows(_p(pts), len(pts), rows, rmin, rmax, nbins, nthreads, _p(dsum), _p(wsum), _p(cnt))
    return dsum, wsum, cnt


def radec2pix(order: int, ra: float, dec: float) -> int:
    return int(lib().orc_radec2pix(order, ra, dec))


def bin_pair(coord: int, axes, scale: float, d1, l1, d2, l2, c):
    """Flat index of one pixel pair (None when skipped, 0xFFFFFFFF when it overflows the grid)."""
    axes = np.ascontiguousarray(axes, dtype=np.float64)
    out = C.c_uint32()
    ok = lib().orc_bin_pair(coord, _p(axes), scale, d1, l1, d2, l2, c, C.byref(out))
    return int(out.value) if ok else None


# ---- the reference's own XiEstimator (oracle/_ref, built by `make -C oracle ref`)

REF_DIR = os.path.join(_HERE, "_ref")
_ref_libs = {}


def ref_available(kind: str = "strict") -> bool:
    name = {"strict": "libtosref.so", "fast": "libtosref_fast.so", "brute": "libtosref_brute.so"}[kind]
    return os.path.exists(os.path.join(REF_DIR, name))


def ref_lib(kind: str = "strict") -> C.CDLL:
    """kind: 'strict' (parity pin), 'fast' (the reference's -O3 -ffast-math) or 'brute' (gpu/brute.cu)."""
    if kind not in _ref_libs:
        name = {"strict": "libtosref.so", "fast": "libtosref_fast.so", "brute": "libtosref_brute.so"}[kind]
        path = os.path.join(REF_DIR, name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (make -C oracle ref needs the reference tree)")
        L = C.CDLL(path)
        vp, sz, i32, dbl = C.c_void_p, C.c_size_t, C.c_int, C.c_double
        if kind == "brute":
            L.tosref_brute.argtypes = [vp, sz, dbl, dbl, i32, C.c_long, vp]
            L.tosref_brute.restype = C.c_int
        else:
            L.tosref_xi.argtypes = [vp, vp, vp, vp, sz, vp, i32, i32, vp, dbl, i32, vp, sz, vp, vp, vp, vp, sz,
                                    vp, vp, vp, C.c_char_p, sz]
            L.tosref_xi.restype = C.c_long
            L.tosref_xi_plates.argtypes = [vp, vp, vp, vp, vp, sz, vp, vp, vp, vp, sz, i32, vp, dbl, i32, vp, sz,
                                           vp, vp, vp, vp, sz, vp, vp, vp, C.c_char_p, sz]
            L.tosref_xi_plates.restype = C.c_long
            L.tosref_radec2pix.argtypes = [i32, dbl, dbl]
            L.tosref_radec2pix.restype = C.c_int64
            L.tosref_max_centre_distance.argtypes = [i32, vp, sz, C.POINTER(C.c_double)]
            L.tosref_max_centre_distance.restype = C.c_double
        _ref_libs[kind] = L
    return _ref_libs[kind]


REF_COUNTERS = ("num_sightline_pairs", "num_sightline_pairs_used", "num_pixels", "num_pixel_pairs",
                "num_pixel_pairs_used")


def ref_xi(sightlines, pixels, order: int, coord: int, axes, scale: float, nthreads: int = 0, cell_subset=None,
           subsamples: bool = False, kind: str = "strict"):
    """The reference XiEstimator::run over the catalogue (cell_subset: HEALPix
    ids of the primary cells to run, default all).  Returns (bins, final,
    cells or None, cell_ids, stats): raw per-bin totals (the per-cell rows
    summed in ascending cell order), the finalized xi_, the per-cell rows of
    the cells run, their ids, and the reference counters plus run_seconds,
    the wall time of XiEstimator::run alone."""
    L = ref_lib(kind)
    ra = np.ascontiguousarray(sightlines["ra"], dtype=np.float64)
    dec = np.ascontiguousarray(sightlines["dec"], dtype=np.float64)
    off = np.ascontiguousarray(sightlines["pixel_offset"], dtype=np.uint64)
    npx = np.ascontiguousarray(sightlines["num_pixels"], dtype=np.uint32)
    px = np.ascontiguousarray(pixels)
    axes = np.ascontiguousarray(axes, dtype=np.float64)
    nb = int(axes[2] * axes[5] * axes[8])
    sub = None if cell_subset is None else np.ascontiguousarray(cell_subset, dtype=np.int64)
    cap = len(sub) if sub is not None else len(ra)
    bins = np.zeros(nb, dtype=XIBIN_DTYPE)
    final = np.zeros(nb, dtype=XIBIN_DTYPE)
    cells = np.zeros((cap, nb), dtype=XIBIN_DTYPE) if subsamples else None
    ids = np.zeros(cap, dtype=np.int64)
    cnt = np.zeros(5, dtype=np.uint64)
    ang = np.zeros(2)
    err = C.create_string_buffer(512)
    secs = C.c_double()
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    n = L.tosref_xi(_p(ra), _p(dec), _p(off), _p(npx), len(ra), _p(px), order, coord, _p(axes), scale, nthreads,
                    _p(sub), 0 if sub is None else len(sub), _p(bins), _p(final), _p(cells), _p(ids), cap,
                    _p(cnt), _p(ang), C.byref(secs), err, 512)
    if n < 0:
        raise ValueError("reference XiEstimator failed: " + err.value.decode())
    st = {k: int(v) for k, v in zip(REF_COUNTERS, cnt)}
    st["max_ang"], st["cos_max_ang"] = float(ang[0]), float(ang[1])
    st["run_seconds"] = secs.value
    return bins, final, (cells[:n] if cells is not None else None), ids[:n], st


def ref_xi_plates(sightlines, pixels, platelist, coord: int, axes, scale: float, nthreads: int = 0,
                  cell_subset=None, subsamples: bool = False, kind: str = "strict"):
    """ref_xi with the reference's PlateBins (cell ids = plate ids; the
    platelist is handed to PlateBins' own constructor)."""
    L = ref_lib(kind)
    ra = np.ascontiguousarray(sightlines["ra"], dtype=np.float64)
    dec = np.ascontiguousarray(sightlines["dec"], dtype=np.float64)
    plate = np.ascontiguousarray(sightlines["plate"], dtype=np.int32)
    off = np.ascontiguousarray(sightlines["pixel_offset"], dtype=np.uint64)
    npx = np.ascontiguousarray(sightlines["num_pixels"], dtype=np.uint32)
    px = np.ascontiguousarray(pixels)
    axes = np.ascontiguousarray(axes, dtype=np.float64)
    lp, lra, ldec = _platelist(platelist)
    nb = int(axes[2] * axes[5] * axes[8])
    sub = None if cell_subset is None else np.ascontiguousarray(cell_subset, dtype=np.int64)
    cap = len(sub) if sub is not None else len(ra)
    bins = np.zeros(nb, dtype=XIBIN_DTYPE)
    final = np.zeros(nb, dtype=XIBIN_DTYPE)
    cells = np.zeros((cap, nb), dtype=XIBIN_DTYPE) if subsamples else None
    ids = np.zeros(cap, dtype=np.int64)
    cnt = np.zeros(5, dtype=np.uint64)
    ang = np.zeros(2)
    err = C.create_string_buffer(512)
    secs = C.c_double()
    if nthreads <= 0:
        nthreads = os.cpu_count() or 1
    n = L.tosref_xi_plates(_p(ra), _p(dec), _p(plate), _p(off), _p(npx), len(ra), _p(px), _p(lp), _p(lra), _p(ldec),
                           len(lp), coord, _p(axes), scale, nthreads, _p(sub), 0 if sub is None else len(sub),
                           _p(bins), _p(final), _p(cells), _p(ids), cap, _p(cnt), _p(ang), C.byref(secs), err, 512)
    if n < 0:
        raise ValueError("reference XiEstimator failed: " + err.value.decode())
    st = {k: int(v) for k, v in zip(REF_COUNTERS, cnt)}
    st["max_ang"], st["cos_max_ang"] = float(ang[0]), float(ang[1])
    st["run_seconds"] = secs.value
    return bins, final, (cells[:n] if cells is not None else None), ids[:n], st


def ref_radec2pix(order: int, ra: float, dec: float) -> int:
    return int(ref_lib().tosref_radec2pix(order, ra, dec))


def ref_max_centre_distance(order: int, dirs):
    """(largest direction-to-own-pixel-centre distance over dirs, the bound
    the stand-in query_disc_inclusive adds to the radius)."""
    d = np.ascontiguousarray(dirs, dtype=np.float64)
    bound = C.c_double()
    worst = ref_lib().tosref_max_centre_distance(order, _p(d), len(d), C.byref(bound))
    return float(worst), float(bound.value)


def ref_brute_gpu(points, rmin: float, rmax: float, nbins: int, chunksize: int = 4096):
    """The reference's bruteGPU (gpu/brute.cu:63-225) on the GPU: xi per bin
    (FP32 histograms).  Needs a CUDA device."""
    L = ref_lib("brute")
    pts = np.ascontiguousarray(points, dtype=np.float32)
    xi = np.zeros(nbins)
    r = L.tosref_brute(_p(pts), len(pts), rmin, rmax, nbins, chunksize, _p(xi))
    if r < 0:
        raise ValueError("reference bruteGPU rejected the input")
    return xi
