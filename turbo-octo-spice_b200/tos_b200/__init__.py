"""Python bindings of the B200 pair-counting engine (ctypes over include/tos_b200.h).

The engine is the in-tree shared library ``lib/libtos_b200.so`` built by the
package Makefile.  There is no Python or CPU implementation of the hot path
here: every compute call goes through the library, and loading fails loudly
when it has not been built.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libtos_b200.so")

TOS_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "OOM", 3: "CUDA", 4: "TIMEOUT", 5: "UNSUPPORTED",
                6: "NO_DEVICE", 7: "INTERNAL"}
POLAR, CARTESIAN, OBSERVING = 0, 1, 2
XI_SUBSAMPLES = 0x1
XI_EXACT = 0x2
XI_PER_GROUP = 0x4
XI_TUNE = 0x8

# numpy views of the C structs
PIXEL_DTYPE = np.dtype([("value", "<f4"), ("loglam", "<f4"), ("weight", "<f4"), ("distance", "<f4")])
SIGHTLINE_DTYPE = np.dtype([("ra", "<f8"), ("dec", "<f8"), ("forest_id", "<i4"), ("plate", "<i4"),
                            ("pixel_offset", "<u8"), ("num_pixels", "<u4"), ("group", "<u4")])
XIBIN_DTYPE = np.dtype([("didj", "<f8"), ("di", "<f8"), ("dj", "<f8"), ("wgt", "<f8"), ("wi", "<f8"),
                        ("wj", "<f8"), ("z", "<f8"), ("num_pairs", "<i8")])
# one platelist row: PLATE, RACEN, DECCEN (degrees), the columns PlateBins reads
PLATE_DTYPE = np.dtype([("plate", "<i4"), ("ra_center", "<f4"), ("dec_center", "<f4")])


class TosError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class _Axis(C.Structure):
    _fields_ = [("min", C.c_double), ("max", C.c_double), ("nbins", C.c_int32), ("reserved", C.c_int32)]


class _Grid(C.Structure):
    _fields_ = [("type", C.c_int32), ("reserved", C.c_int32), ("axis", _Axis * 3)]


class XiStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "num_sightlines", "num_sightline_pairs", "num_sightline_pairs_used", "num_pixels",
        "num_pixel_pairs", "num_pixel_pairs_used", "num_pixel_pairs_evaluated", "num_edge_rechecks",
        "num_index_overflow", "num_cells", "num_direct_runs", "num_window_flushes")] + [(n, C.c_double) for n in (
            "max_ang", "cos_max_ang", "ms_expand", "ms_pairs", "ms_total", "ms_device")] + [
        ("num_run_items", C.c_uint64), ("ms_runs", C.c_double), ("num_grid_items", C.c_uint64), ("ms_grid", C.c_double),
        ("num_diag_items", C.c_uint64), ("ms_diag", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class RequestInfo(C.Structure):
    _fields_ = [("submit_s", C.c_double), ("start_s", C.c_double), ("end_s", C.c_double),
                ("slot", C.c_int32), ("reserved", C.c_int32), ("workspace_bytes", C.c_uint64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class ServerStatus(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("budget_bytes", "resident_bytes", "in_use_bytes", "peak_bytes",
                                           "queued", "running", "completed")] + [
        ("slots", C.c_uint32), ("reserved", C.c_uint32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


_lib = None


def lib() -> C.CDLL:
    """The engine library (loaded once). Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"engine library not built: {LIB_PATH} (run make in {PKG_ROOT})")
        L = C.CDLL(LIB_PATH)
        vp, sz, i32, u32, dbl = C.c_void_p, C.c_size_t, C.c_int, C.c_uint32, C.c_double
        u64 = C.c_uint64
        L.tos_last_error.restype = C.c_char_p
        L.tos_abi_version.restype = C.c_int
        L.tos_engine_create.argtypes = [i32, C.POINTER(vp)]
        L.tos_engine_destroy.argtypes = [vp]
        L.tos_engine_destroy.restype = None
        L.tos_catalog_create.argtypes = [vp, vp, sz, vp, sz, i32, C.POINTER(vp)]
        L.tos_catalog_destroy.argtypes = [vp]
        L.tos_catalog_destroy.restype = None
        L.tos_catalog_num_cells.argtypes = [vp, C.POINTER(sz)]
        L.tos_catalog_cells.argtypes = [vp, vp, sz]
        L.tos_catalog_sightline_cells.argtypes = [vp, vp, sz]
        L.tos_catalog_num_groups.argtypes = [vp, C.POINTER(sz)]
        L.tos_catalog_groups.argtypes = [vp, vp, sz]
        L.tos_grid_max_angular_scale.argtypes = [C.POINTER(_Grid), dbl, C.POINTER(dbl)]
        L.tos_grid_num_bins.argtypes = [C.POINTER(_Grid)]
        L.tos_grid_num_bins.restype = sz
        L.tos_xi_run.argtypes = [vp, vp, C.POINTER(_Grid), dbl, u32, vp, vp, C.POINTER(XiStats)]
        L.tos_xibin_finalize.argtypes = [vp, sz]
        L.tos_xibin_finalize.restype = None
        L.tos_brute_run.argtypes = [vp, vp, sz, dbl, dbl, i32, vp, vp, vp, C.POINTER(dbl)]
        L.tos_brute_run_noalloc.argtypes = [vp, vp, sz, dbl, dbl, i32, vp, vp, vp, C.POINTER(dbl)]
        L.tos_brute_tune.argtypes = [vp, vp, sz, dbl, dbl, i32, C.POINTER(i32), C.POINTER(i32)]
        L.tos_xi_cell_covariance.argtypes = [vp, vp, vp, vp, vp]
        L.tos_xi_jackknife.argtypes = [vp, vp, i32, sz, C.POINTER(sz), vp, vp, vp]
        L.tos_xi_subsample_covariance.argtypes = [vp, vp, sz, sz, vp, vp, vp]
        L.tos_xi_run_jackknife.argtypes = [vp, vp, C.POINTER(_Grid), dbl, u32, i32, sz, C.POINTER(sz),
                                           vp, vp, vp, vp, C.POINTER(XiStats)]
        L.tos_server_create.argtypes = [i32, i32, u64, C.POINTER(vp)]
        L.tos_server_destroy.argtypes = [vp]
        L.tos_server_destroy.restype = None
        L.tos_server_attach.argtypes = [vp, vp]
        L.tos_server_detach.argtypes = [vp, vp]
        L.tos_server_submit.argtypes = [vp, vp, C.POINTER(_Grid), dbl, u32, C.POINTER(u64)]
        L.tos_server_wait.argtypes = [vp, u64, vp, vp, C.POINTER(XiStats), C.POINTER(RequestInfo)]
        L.tos_server_status_get.argtypes = [vp, C.POINTER(ServerStatus)]
        L.tos_server_poll.argtypes = [vp, u64, C.POINTER(C.c_int)]
        L.tos_server_set_policy.argtypes = [vp, i32, dbl]
        L.tos_catalog_device_bytes.argtypes = [vp, C.POINTER(u64)]
        L.tos_comoving_distance.argtypes = [dbl, vp, sz, vp]
        L.tos_fill_distances.argtypes = [dbl, vp, sz]
        L.tos_catalog_create_dc.argtypes = [vp, vp, sz, vp, sz, i32, dbl, C.POINTER(vp)]
        L.tos_catalog_distances.argtypes = [vp, vp, sz]
        L.tos_catalog_create_plates.argtypes = [vp, vp, sz, vp, sz, vp, sz, dbl, C.POINTER(vp)]
        L.tos_forests_assemble.argtypes = [vp, sz, vp, sz, C.POINTER(sz), vp, sz, C.POINTER(sz)]
        for name in ("tos_engine_create", "tos_catalog_create", "tos_catalog_num_cells", "tos_catalog_cells",
                     "tos_catalog_sightline_cells", "tos_grid_max_angular_scale", "tos_xi_run",
                     "tos_brute_run", "tos_brute_tune", "tos_comoving_distance", "tos_fill_distances"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _check(status: int):
    if status != TOS_OK:
        raise TosError(status, lib().tos_last_error().decode(errors="replace"))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


@dataclass(frozen=True)
class Axis:
    """Linear axis "[min:max]*nbins" (likely's uniform binning)."""
    min: float
    max: float
    nbins: int

    @staticmethod
    def parse(spec: str) -> "Axis":
        s = spec.strip()
        if not (s.startswith("[") and "]*" in s and ":" in s):
            raise ValueError(f"bad binning specification: {spec}")
        rng, n = s[1:].split("]*")
        lo, hi = rng.split(":")
        return Axis(float(lo), float(hi), int(n))

    @property
    def width(self) -> float:
        return (self.max - self.min) / self.nbins


@dataclass(frozen=True)
class Grid:
    """A three-axis binning grid with its coordinate type (AbsTwoPointGrid + subclass)."""
    type: int
    axes: tuple

    @staticmethod
    def cartesian(rpar="[0:200]*50", rperp="[0:200]*50", z="[3.556:3.735]*1") -> "Grid":
        return Grid(CARTESIAN, tuple(Axis.parse(a) for a in (rpar, rperp, z)))

    @staticmethod
    def polar(r="[0:200]*50", mu="[0:1]*20", z="[3.556:3.735]*1") -> "Grid":
        return Grid(POLAR, tuple(Axis.parse(a) for a in (r, mu, z)))

    @staticmethod
    def observing(dloglam="[0:0.05]*25", theta="[5:175]*1", z="[3.556:3.735]*1") -> "Grid":
        return Grid(OBSERVING, tuple(Axis.parse(a) for a in (dloglam, theta, z)))

    @staticmethod
    def from_axes(coord_type: int, axes) -> "Grid":
        """Grid of a coordinate type from nine values (min, max, nbins) x 3."""
        a = np.asarray(axes, dtype=np.float64).reshape(3, 3)
        return Grid(int(coord_type), tuple(Axis(float(x[0]), float(x[1]), int(x[2])) for x in a))

    def c_struct(self) -> _Grid:
        g = _Grid()
        g.type = self.type
        for k, a in enumerate(self.axes):
            g.axis[k].min, g.axis[k].max, g.axis[k].nbins = a.min, a.max, a.nbins
        return g

    @property
    def nbins(self) -> int:
        return int(self.axes[0].nbins * self.axes[1].nbins * self.axes[2].nbins)

    def axes_array(self) -> np.ndarray:
        return np.array([[a.min, a.max, a.nbins] for a in self.axes], dtype=np.float64).ravel()

    def max_angular_scale(self, scale: float) -> float:
        out = C.c_double()
        _check(lib().tos_grid_max_angular_scale(C.byref(self.c_struct()), scale, C.byref(out)))
        return out.value


class Engine:
    """A CUDA device owned by the engine (tos_engine)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().tos_engine_create(device, C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            lib().tos_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Catalog:
    """Sightlines and pixels resident on the device, binned into HEALPix cells
    (HealpixBins) or, with a platelist, into their plates (PlateBins)."""

    def __init__(self, engine: Engine, sightlines: np.ndarray, pixels: np.ndarray, healpix_order: int = None,
                 omega_matter: float = None, platelist: np.ndarray = None):
        """With omega_matter, each pixel's comoving distance is computed on the
        device from its loglam (tos_catalog_create_dc; the pixels' own
        distances are ignored), with the same bits as fill_distances.  With
        platelist (PLATE_DTYPE rows: PLATE, RACEN, DECCEN in degrees) the
        cells are the sightlines' `plate` ids (tos_catalog_create_plates) and
        healpix_order must be None."""
        sightlines = np.ascontiguousarray(sightlines, dtype=SIGHTLINE_DTYPE)
        pixels = np.ascontiguousarray(pixels, dtype=PIXEL_DTYPE)
        h = C.c_void_p()
        if platelist is not None:
            if healpix_order is not None:
                raise ValueError("a plate catalogue takes no HEALPix order")
            plates = np.ascontiguousarray(platelist, dtype=PLATE_DTYPE)
            _check(lib().tos_catalog_create_plates(engine.handle, _ptr(sightlines), len(sightlines), _ptr(pixels),
                                                   len(pixels), _ptr(plates) if len(plates) else None, len(plates),
                                                   0.0 if omega_matter is None else float(omega_matter),
                                                   C.byref(h)))
        elif healpix_order is None:
            raise ValueError("healpix_order is needed without a platelist")
        elif omega_matter is None:
            _check(lib().tos_catalog_create(engine.handle, _ptr(sightlines), len(sightlines), _ptr(pixels),
                                            len(pixels), healpix_order, C.byref(h)))
        else:
            _check(lib().tos_catalog_create_dc(engine.handle, _ptr(sightlines), len(sightlines), _ptr(pixels),
                                               len(pixels), healpix_order, float(omega_matter), C.byref(h)))
        self._h = h
        self.engine = engine
        self.n_sightlines = len(sightlines)
        self.n_pixels = int(sightlines["num_pixels"].astype(np.int64).sum())

    def distances(self) -> np.ndarray:
        """The resident per-pixel comoving distances (compact sightline order)."""
        out = np.zeros(self.n_pixels, dtype=np.float32)
        _check(lib().tos_catalog_distances(self._h, _ptr(out), len(out)))
        return out

    @property
    def handle(self):
        return self._h

    def num_cells(self) -> int:
        n = C.c_size_t()
        _check(lib().tos_catalog_num_cells(self._h, C.byref(n)))
        return n.value

    def cells(self) -> np.ndarray:
        n = self.num_cells()
        out = np.zeros(n, dtype=np.int64)
        _check(lib().tos_catalog_cells(self._h, _ptr(out), n))
        return out

    def sightline_cells(self) -> np.ndarray:
        out = np.zeros(self.n_sightlines, dtype=np.int64)
        _check(lib().tos_catalog_sightline_cells(self._h, _ptr(out), self.n_sightlines))
        return out

    def device_bytes(self) -> int:
        n = C.c_uint64()
        _check(lib().tos_catalog_device_bytes(self._h, C.byref(n)))
        return n.value

    def num_groups(self) -> int:
        n = C.c_size_t()
        _check(lib().tos_catalog_num_groups(self._h, C.byref(n)))
        return n.value

    def groups(self) -> np.ndarray:
        n = self.num_groups()
        out = np.zeros(n, dtype=np.uint32)
        _check(lib().tos_catalog_groups(self._h, _ptr(out), n))
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().tos_catalog_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def xi_run(engine: Engine, catalog: Catalog, grid: Grid, scale: float, subsamples: bool = False,
           exact: bool = False, per_group: bool = False, tune: bool = False):
    """Pair count of XiEstimator::run. Returns (bins, rows or None, stats dict);
    bins/rows are raw (unfinalized) XiBin sums as XIBIN_DTYPE arrays.  rows
    are per cell with subsamples=True, per sightline group (ascending group
    id, one xi per batched catalogue) with per_group=True.  tune=True first
    times the dominant kernel's launch shapes on a sample of the sightline
    pairs and keeps the fastest on the engine (TOS_XI_TUNE)."""
    nb = grid.nbins
    bins = np.zeros(nb, dtype=XIBIN_DTYPE)
    cells = None
    if subsamples:
        cells = np.zeros((catalog.num_cells(), nb), dtype=XIBIN_DTYPE)
    elif per_group:
        cells = np.zeros((catalog.num_groups(), nb), dtype=XIBIN_DTYPE)
    flags = ((XI_SUBSAMPLES if subsamples else 0) | (XI_EXACT if exact else 0) |
             (XI_PER_GROUP if per_group else 0) | (XI_TUNE if tune else 0))
    st = XiStats()
    _check(lib().tos_xi_run(engine.handle, catalog.handle, C.byref(grid.c_struct()), scale, flags, _ptr(bins),
                            _ptr(cells) if cells is not None else None, C.byref(st)))
    return bins, cells, st.as_dict()


def xi_run_jackknife(engine: Engine, catalog: Catalog, grid: Grid, scale: float, region_order: int,
                     exact: bool = False):
    """Exact delete-one-region jackknife in one pass (tos_xi_run_jackknife).
    Returns (region_ids, bins, group_rows, drop_rows, stats): region ids
    (group << 32 | HEALPix RING pixel of region_order), the whole catalogue's
    sums, per-group sums (ascending group id) and for every region the sums of
    the catalogue without that region's sightlines, all raw XiBin arrays."""
    L = lib()
    g = grid.c_struct()
    flags = XI_EXACT if exact else 0
    n = C.c_size_t()
    _check(L.tos_xi_run_jackknife(engine.handle, catalog.handle, C.byref(g), scale, flags, region_order, 0,
                                  C.byref(n), None, None, None, None, None))
    nk, nb = n.value, grid.nbins
    ids = np.zeros(nk, dtype=np.int64)
    bins = np.zeros(nb, dtype=XIBIN_DTYPE)
    groups = np.zeros((catalog.num_groups(), nb), dtype=XIBIN_DTYPE)
    drop = np.zeros((nk, nb), dtype=XIBIN_DTYPE)
    st = XiStats()
    _check(L.tos_xi_run_jackknife(engine.handle, catalog.handle, C.byref(g), scale, flags, region_order, nk,
                                  C.byref(n), _ptr(ids), _ptr(bins), _ptr(groups), _ptr(drop), C.byref(st)))
    return ids, bins, groups, drop, st.as_dict()


class Server:
    """Request server over resident catalogues (tos_server): worker slots with
    their own streams, admission in arrival order under a device-memory budget."""

    def __init__(self, device: int = 0, slots: int = 4, memory_budget_bytes: int = 150 * 10**9):
        h = C.c_void_p()
        _check(lib().tos_server_create(device, slots, memory_budget_bytes, C.byref(h)))
        self._h = h

    def attach(self, catalog: Catalog):
        _check(lib().tos_server_attach(self._h, catalog.handle))

    def set_policy(self, policy: str = "fifo", max_wait_s: float = 5.0):
        """Admission order: "fifo" (arrival order) or "shortest" (least
        estimated work first, with requests older than max_wait_s first)."""
        _check(lib().tos_server_set_policy(self._h, {"fifo": 0, "shortest": 1}[policy], max_wait_s))

    def detach(self, catalog: Catalog):
        _check(lib().tos_server_detach(self._h, catalog.handle))

    def submit(self, catalog: Catalog, grid: Grid, scale: float, subsamples: bool = False,
               per_group: bool = False, exact: bool = False) -> "ServerRequest":
        flags = ((XI_SUBSAMPLES if subsamples else 0) | (XI_EXACT if exact else 0) |
                 (XI_PER_GROUP if per_group else 0))
        rid = C.c_uint64()
        _check(lib().tos_server_submit(self._h, catalog.handle, C.byref(grid.c_struct()), scale, flags,
                                       C.byref(rid)))
        rows = catalog.num_cells() if subsamples else catalog.num_groups() if per_group else 0
        return ServerRequest(self, rid.value, grid.nbins, rows)

    def status(self) -> dict:
        st = ServerStatus()
        _check(lib().tos_server_status_get(self._h, C.byref(st)))
        return st.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            lib().tos_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class ServerRequest:
    """A submitted request; wait() blocks and returns (bins, rows or None, stats, info)."""

    def __init__(self, server: Server, rid: int, nbins: int, n_rows: int):
        self.server, self.id, self.nbins, self.n_rows = server, rid, nbins, n_rows

    def done(self) -> bool:
        """Non-blocking: has the request finished?"""
        d = C.c_int()
        _check(lib().tos_server_poll(self.server._h, self.id, C.byref(d)))
        return bool(d.value)

    def wait(self):
        bins = np.zeros(self.nbins, dtype=XIBIN_DTYPE)
        rows = np.zeros((self.n_rows, self.nbins), dtype=XIBIN_DTYPE) if self.n_rows else None
        st, info = XiStats(), RequestInfo()
        _check(lib().tos_server_wait(self.server._h, self.id, _ptr(bins),
                                     _ptr(rows) if rows is not None else None, C.byref(st), C.byref(info)))
        return bins, rows, st.as_dict(), info.as_dict()


def subsample_covariance(engine: Engine, rows: np.ndarray):
    """Jackknife covariance of delete-one subsample rows (n, nbins) XiBin
    arrays, e.g. one group's rows of xi_run_jackknife.  Returns (xi, mean, cov)."""
    rows = np.ascontiguousarray(rows, dtype=XIBIN_DTYPE)
    n, nb = rows.shape
    xi = np.zeros((n, nb))
    mean = np.zeros(nb)
    cov = np.zeros((nb, nb))
    _check(lib().tos_xi_subsample_covariance(engine.handle, _ptr(rows), n, nb, _ptr(xi), _ptr(mean), _ptr(cov)))
    return xi, mean, cov


def finalize(bins: np.ndarray) -> np.ndarray:
    """XiBin::finalize on a copy."""
    out = np.ascontiguousarray(bins.copy(), dtype=XIBIN_DTYPE)
    lib().tos_xibin_finalize(_ptr(out), len(out))
    return out


def brute_run(engine: Engine, points: np.ndarray, rmin: float, rmax: float, nbins: int):
    """All-pairs isotropic xi(r) (bruteGPU). points: (n, 5) float32 rows x, y, z, delta, w.
    Returns dsum, wsum, counts (nbins+2 each, bin 0 underflow, nbins+1 overflow) and kernel ms."""
    pts = np.ascontiguousarray(points, dtype=np.float32)
    if pts.ndim != 2 or pts.shape[1] != 5:
        raise ValueError("points must be (n, 5)")
    dsum = np.zeros(nbins + 2)
    wsum = np.zeros(nbins + 2)
    counts = np.zeros(nbins + 2, dtype=np.uint64)
    ms = C.c_double()
    _check(lib().tos_brute_run(engine.handle, _ptr(pts), len(pts), rmin, rmax, nbins, _ptr(dsum), _ptr(wsum),
                               _ptr(counts), C.byref(ms)))
    return dsum, wsum, counts, ms.value


def brute_tune(engine: Engine, points: np.ndarray, rmin: float, rmax: float, nbins: int):
    """tos_brute_tune: time the brute-force kernel's launch shapes on a sample
    of the points and keep the fastest on the engine for this bin count.
    Returns (diagonals per lane, warps per CTA) of the pick."""
    pts = np.ascontiguousarray(points, dtype=np.float32)
    if pts.ndim != 2 or pts.shape[1] != 5:
        raise ValueError("points must be (n, 5)")
    k, w = C.c_int(), C.c_int()
    _check(lib().tos_brute_tune(engine.handle, _ptr(pts), len(pts), rmin, rmax, nbins, C.byref(k), C.byref(w)))
    return k.value, w.value


def brute_run_noalloc(engine: Engine, points_ptr: int, n_points: int, rmin: float, rmax: float,
                      nbins: int, dsum_ptr: int, wsum_ptr: int, counts_ptr: int) -> float:
    """tos_brute_run_noalloc: the brute-force count on device buffers with no
    device allocation (for callers that cannot allocate GPU memory).  The
    arguments are device addresses: points (n, 5) float32, dsum and wsum
    float64 (nbins+2), counts uint64 (nbins+2).  Returns the kernel ms."""
    ms = C.c_double()
    _check(lib().tos_brute_run_noalloc(engine.handle, C.c_void_p(points_ptr), n_points, rmin, rmax, nbins,
                                       C.c_void_p(dsum_ptr), C.c_void_p(wsum_ptr), C.c_void_p(counts_ptr),
                                       C.byref(ms)))
    return ms.value


def cell_covariance(engine: Engine, cat: "Catalog", nbins: int):
    """Covariance of the per-cell xi of the last xi_run on `cat` (the
    reference's do_cov).  Returns (mean[nbins], cov[nbins, nbins], total weight)."""
    mean = np.zeros(nbins)
    cov = np.zeros((nbins, nbins))
    W = C.c_double()
    _check(lib().tos_xi_cell_covariance(engine.handle, cat.handle, _ptr(mean), _ptr(cov), C.byref(W)))
    return mean, cov, W.value


def jackknife(engine: Engine, cat: "Catalog", region_order: int, nbins: int):
    """Leave-one-region-out jackknife of the last xi_run on `cat` over HEALPix
    regions of region_order.  Returns (region ids, xi_jk[N, nbins], cov)."""
    n = C.c_size_t()
    _check(lib().tos_xi_jackknife(engine.handle, cat.handle, region_order, 0, C.byref(n), None, None, None))
    ids = np.zeros(n.value, dtype=np.int64)
    xi = np.zeros((n.value, nbins))
    cov = np.zeros((nbins, nbins))
    _check(lib().tos_xi_jackknife(engine.handle, cat.handle, region_order, n.value, C.byref(n), _ptr(ids),
                                  _ptr(xi), _ptr(cov)))
    return ids, xi, cov


def fill_distances(omega_matter: float, pixels: np.ndarray) -> np.ndarray:
    """tos_fill_distances on the host: a copy of the pixels with each distance
    computed from its loglam (h5healxi.cc:38-40, 196-203)."""
    out = np.ascontiguousarray(pixels, dtype=PIXEL_DTYPE).copy()
    _check(lib().tos_fill_distances(omega_matter, _ptr(out), len(out)))
    return out


class _Forest(C.Structure):
    _fields_ = [("name", C.c_char_p), ("ra", C.c_double), ("dec", C.c_double), ("z", C.c_double),
                ("plate", C.c_int32), ("reserved", C.c_int32), ("n", C.c_uint64),
                ("delta", C.c_void_p), ("weight", C.c_void_p), ("r_comov", C.c_void_p), ("loglam", C.c_void_p)]


def assemble_forests(forests):
    """Sightlines and pixels (SIGHTLINE_DTYPE, PIXEL_DTYPE arrays) from forests
    as HDF5Delta::loadForests reads them (tos_forests_assemble): forests is a
    sequence of dicts with the group's name, its ra, dec, z and plate
    attributes and its delta, weight, r_comov and loglam datasets."""
    keep = []
    arr = (_Forest * max(1, len(forests)))()
    for k, f in enumerate(forests):
        cols = [np.ascontiguousarray(f[c], dtype=np.float32) for c in ("delta", "weight", "r_comov", "loglam")]
        n = len(cols[0])
        if any(len(c) < n for c in cols[1:]):
            raise ValueError(f"forest {f['name']!r}: datasets shorter than delta")
        name = f["name"].encode() if isinstance(f["name"], str) else bytes(f["name"])
        keep.append((name, cols))
        arr[k] = _Forest(name, float(f["ra"]), float(f["dec"]), float(f.get("z", 0.0)), int(f.get("plate", 0)), 0,
                         n, *[c.ctypes.data for c in cols])
    n_los, n_px = C.c_size_t(), C.c_size_t()
    L = lib()
    arr = C.cast(arr, C.c_void_p)
    _check(L.tos_forests_assemble(arr, len(forests), None, 0, C.byref(n_los), None, 0, C.byref(n_px)))
    los = np.zeros(max(1, n_los.value), dtype=SIGHTLINE_DTYPE)
    px = np.zeros(max(1, n_px.value), dtype=PIXEL_DTYPE)
    _check(L.tos_forests_assemble(arr, len(forests), _ptr(los), len(los), C.byref(n_los), _ptr(px), len(px),
                                  C.byref(n_px)))
    del keep
    return los[:n_los.value], px[:n_px.value]


def comoving_distance(omega_matter: float, z) -> np.ndarray:
    z = np.ascontiguousarray(z, dtype=np.float64)
    out = np.zeros_like(z)
    _check(lib().tos_comoving_distance(omega_matter, _ptr(z), z.size, _ptr(out)))
    return out


def header_symbols() -> list:
    """Function names declared in include/tos_b200.h."""
    import re
    path = os.path.join(os.path.dirname(PKG_ROOT), "include", "tos_b200.h")
    text = open(path).read()
    return sorted(set(re.findall(r"^\s*(?:[a-z_0-9]+\s*\**\s+)+\**\s*(tos_[a-z_0-9]+)\s*\(", text, re.M)))
