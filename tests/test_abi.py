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
