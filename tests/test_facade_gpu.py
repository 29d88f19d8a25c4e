"""The C++ XiEstimator facade end to end, driven like h5healxi drives the
reference's class (h5healxi.cc:279-290): run with do_cov, save_results,
save_subsamples.  Its files must carry exactly what the C ABI returns through
the Python binding on the same catalogue: .data / .details from the finalized
bins, .cov from tos_xi_cell_covariance, and one -<cell>.data per cell."""
import os
import subprocess

import numpy as np
import pytest

import tos_b200 as T
from helpers import GRIDS, small_catalog

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIBDIR = os.path.join(ROOT, "turbo-octo-spice_b200", "lib")


@pytest.fixture(scope="module")
def facade(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("facade") / "facade_main")
    subprocess.run(["g++", "-std=c++17", "-O1", os.path.join(HERE, "facade", "facade_main.cc"), "-o", exe,
                    f"-L{LIBDIR}", "-ltos_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def write_catalogue(path, los, px):
    with open(path, "wb") as f:
        f.write(np.uint64(len(los)).tobytes())
        for s in range(len(los)):
            o, n = int(los[s]["pixel_offset"]), int(los[s]["num_pixels"])
            f.write(np.float64(los[s]["ra"]).tobytes() + np.float64(los[s]["dec"]).tobytes())
            f.write(np.uint32(n).tobytes())
            f.write(np.ascontiguousarray(px[o:o + n]).tobytes())


def test_facade_files_match_c_abi(engine, facade, tmp_path):
    los, px, meta = small_catalog(n=100, seed=41, size_deg=2.5)
    g = GRIDS["cartesian"]
    cat_path = str(tmp_path / "cat.bin")
    write_catalogue(cat_path, los, px)
    base = str(tmp_path / "xi")
    r = subprocess.run([facade, cat_path, "1", "[0:200]*50", "[0:200]*50", "[3.556:3.735]*1",
                        repr(meta["scale"]), "6", base], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # the same through the C ABI
    cat = T.Catalog(engine, los, px, 6)
    bins, cells, _ = T.xi_run(engine, cat, g, meta["scale"], subsamples=True)
    _, cov, _ = T.cell_covariance(engine, cat, g.nbins)
    fin = T.finalize(bins.copy())
    data = np.loadtxt(base + ".data")
    assert np.array_equal(data[:, 0], np.arange(g.nbins))
    np.testing.assert_array_equal(data[:, 1], fin["didj"])
    det = np.loadtxt(base + ".details")
    for col, f in ((4, "didj"), (5, "di"), (6, "dj"), (7, "wgt"), (9, "z")):
        np.testing.assert_array_equal(det[:, col], fin[f])
    np.testing.assert_array_equal(det[:, 8], bins["num_pairs"])
    c = np.loadtxt(base + ".cov")
    assert len(c) == g.nbins * (g.nbins + 1) // 2
    np.testing.assert_array_equal(c[:, 2], cov[c[:, 0].astype(int), c[:, 1].astype(int)])
    ids = cat.cells()
    for k, cid in enumerate(ids):
        sub = np.loadtxt(f"{base}-{cid}.data")
        w = cells[k]["wgt"]
        np.testing.assert_array_equal(sub[:, 2], w)
        np.testing.assert_array_equal(sub[:, 1], np.where(w > 0, cells[k]["didj"] / np.where(w > 0, w, 1), 0))
        np.testing.assert_array_equal(sub[:, 3], cells[k]["num_pairs"])
