"""ctypes wrapper of the CPU oracle (oracle/xi_oracle.c).

TEST INFRASTRUCTURE: used by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py only, as the checker or the timed reference CPU path.
The engine never loads it.  Parity unpinned: the reference ships no expected
outputs for this path and cannot be built here; see the header of
xi_oracle.c for what the oracle is checked against.
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
        ("max_ang", C.c_double), ("cos_max_ang", C.c_double)]

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
        L.orc_cell_costs.argtypes = [vp, vp, vp, sz, i32, i32, vp, dbl, vp]
        L.orc_cell_costs.restype = C.c_long
        L.orc_brute.argtypes = [vp, sz, dbl, dbl, i32, i32, vp, vp, vp]
        L.orc_brute.restype = C.c_int
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


def radec2pix(order: int, ra: float, dec: float) -> int:
    return int(lib().orc_radec2pix(order, ra, dec))


def bin_pair(coord: int, axes, scale: float, d1, l1, d2, l2, c):
    """Flat index of one pixel pair (None when skipped, 0xFFFFFFFF when it overflows the grid)."""
    axes = np.ascontiguousarray(axes, dtype=np.float64)
    out = C.c_uint32()
    ok = lib().orc_bin_pair(coord, _p(axes), scale, d1, l1, d2, l2, c, C.byref(out))
    return int(out.value) if ok else None
