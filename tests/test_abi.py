"""C-ABI library checks that need no GPU: it loads, exports every entry point
declared in include/tos_b200.h, reports a missing device cleanly, and its
host-only helpers (grid geometry, cosmology) are correct."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import Grid, synth


def test_library_exports_every_declared_symbol():
    lib = T.lib()
    declared = T.header_symbols()
    assert len(declared) >= 15
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", T.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(declared) <= exported
    assert lib.tos_abi_version() == 1


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="host has a GPU")
def test_engine_create_reports_missing_device():
    with pytest.raises(T.TosError) as e:
        T.Engine(0)
    assert e.value.status == 6  # TOS_ERR_NO_DEVICE, never a crash or exit()


def test_grid_geometry():
    g = Grid.cartesian()
    assert g.nbins == 2500
    assert T.lib().tos_grid_num_bins(C.byref(g.c_struct())) == 2500
    # CartesianGrid::maxAngularScale = r_perp,max / scale
    assert g.max_angular_scale(3586.0) == 200.0 / 3586.0
    p = Grid.polar(mu="[0.5:1]*10")
    assert p.max_angular_scale(1000.0) == 200.0 * math.sqrt(1 - 0.25) / 1000.0
    q = Grid.observing()
    assert q.max_angular_scale(1.0) == 175.0  # QuasarGrid: no scaling (arcmin used as radians)
    bad = Grid(T.CARTESIAN, (T.Axis(0, 200, 50), T.Axis(0, 200, 0), T.Axis(0, 1, 1)))
    with pytest.raises(T.TosError):
        bad.max_angular_scale(1.0)


def test_axis_parse():
    a = T.Axis.parse("[3.556:3.735]*1")
    assert (a.min, a.max, a.nbins) == (3.556, 3.735, 1)
    with pytest.raises(ValueError):
        T.Axis.parse("3.556:3.735")


def test_comoving_distance_matches_fp64_quadrature():
    z = np.linspace(0.0, 4.0, 401)
    a = T.comoving_distance(0.3, z)
    b = synth.comoving_distance_fp64(z, 0.3)
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-9)
    # D_C(1.9605) ~ 3586 Mpc/h (the angular scale of the configurations)
    assert abs(T.comoving_distance(0.3, [1.9605])[0] - 3586.0) < 2.0


def test_fill_distances_matches_fp64_integral():
    """tos_fill_distances (host): z from loglam (h5healxi.cc:38-40) and D_C from
    the table, against an FP64 quadrature of the same integral, to within one
    float rounding."""
    los, px, meta = synth.small_patch(200, seed=3)
    got = T.fill_distances(0.3, px)["distance"].astype(np.float64)
    z = 10.0 ** (px["loglam"].astype(np.float64) - np.log10(1216.0)) - 1.0
    ref = synth.comoving_distance_fp64(z, 0.3)
    assert np.max(np.abs(got - ref) / ref) < 1.2e-7


def _loader_restated(forests):
    """HDF5Delta::loadForests (HDF5Delta.cc:40-93) restated in Python: groups
    in byte-wise name order, pixels with finite delta and weight and weight
    > 0, empty forests dropped, forests numbered in that order."""
    los, px = [], []
    for f in sorted(forests, key=lambda f: f["name"].encode()):
        kept = [(d, l, w, r) for d, w, r, l in zip(f["delta"], f["weight"], f["r_comov"], f["loglam"])
                if np.isfinite(np.float32(d)) and np.isfinite(np.float32(w)) and np.float32(w) > 0]
        if kept:
            los.append((f["ra"], f["dec"], len(los), f["plate"], len(px), len(kept), 0))
            px.extend(kept)
    return (np.array(los, dtype=T.SIGHTLINE_DTYPE), np.array(px, dtype=T.PIXEL_DTYPE).reshape(-1))


def test_forests_assemble_follows_the_loader():
    rng = np.random.default_rng(12)
    names = ["10", "9", "B", "a", "a0", "Z", "los-003", "los-001", "los-002", "empty", "allbad"]
    forests = []
    for k, name in enumerate(names):
        n = 0 if name == "empty" else int(rng.integers(1, 40))
        delta = rng.normal(size=n).astype(np.float32)
        weight = rng.uniform(0.1, 2, n).astype(np.float32)
        bad = rng.uniform(size=n) < 0.2
        delta[bad & (rng.uniform(size=n) < 0.5)] = np.nan
        weight[bad & (rng.uniform(size=n) < 0.5)] = rng.choice([0.0, -1.0, np.inf, np.nan])
        if name == "allbad":
            weight[:] = 0.0
        forests.append(dict(name=name, ra=0.1 * k, dec=-0.05 * k, z=2.0 + 0.1 * k, plate=3000 + k, delta=delta,
                            weight=weight, r_comov=rng.uniform(3000, 4000, n).astype(np.float32),
                            loglam=np.sort(rng.uniform(3.56, 3.74, n)).astype(np.float32)))
    los, px = T.assemble_forests(forests)
    rlos, rpx = _loader_restated(forests)
    assert np.array_equal(los, rlos)
    assert np.array_equal(px.view(np.uint32), rpx.view(np.uint32))  # bit for bit
    assert [int(x) for x in los["forest_id"]] == list(range(len(los)))
    assert len(los) == len(names) - 2  # "empty" and "allbad" are dropped


def test_forests_assemble_round_trip_and_capacity():
    """A catalogue split into named forests comes back unchanged; a buffer
    that is too small is refused."""
    import ctypes as C
    from helpers import small_catalog
    los0, px0, _ = small_catalog(n=25, seed=4, size_deg=2.0, max_pixels=30)
    forests = []
    for s in range(len(los0)):
        o, n = int(los0[s]["pixel_offset"]), int(los0[s]["num_pixels"])
        p = px0[o:o + n]
        forests.append(dict(name=f"{s:06d}", ra=los0[s]["ra"], dec=los0[s]["dec"], plate=int(los0[s]["plate"]),
                            delta=p["value"], weight=p["weight"], r_comov=p["distance"], loglam=p["loglam"]))
    los, px = T.assemble_forests(forests[::-1])  # the order given does not matter
    assert np.array_equal(los, los0) and np.array_equal(px, px0)
    L = T.lib()
    arr = (T._Forest * 1)(T._Forest(b"x", 0.0, 0.0, 0.0, 0, 0, 3, *[np.ones(3, np.float32).ctypes.data] * 4))
    nl, npx = C.c_size_t(), C.c_size_t()
    small_l = np.zeros(1, dtype=T.SIGHTLINE_DTYPE)
    small_p = np.zeros(2, dtype=T.PIXEL_DTYPE)
    st = L.tos_forests_assemble(C.cast(arr, C.c_void_p), 1, small_l.ctypes.data, 1, C.byref(nl),
                                small_p.ctypes.data, 2, C.byref(npx))
    assert st == 1 and nl.value == 1 and npx.value == 3  # TOS_ERR_INVALID_ARG, sizes reported
