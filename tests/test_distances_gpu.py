"""Pixel distances computed on the device from loglam (tos_catalog_create_dc)
against the host fill (tos_fill_distances): the same float for every pixel,
bit for bit, on a small patch and on a 20,000-sightline survey (11 M
pixels); the pair counts of the two catalogues are then identical; loglam
below log10(1216) (z < 0) is refused as on the host."""
import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth  # noqa: F401  (T.synth)
from helpers import GRIDS, small_catalog

pytestmark = pytest.mark.gpu


def compact(los, px):
    return np.concatenate([px[int(o):int(o) + int(n)] for o, n in zip(los["pixel_offset"], los["num_pixels"])])


def test_device_distances_equal_host_fill(engine):
    los, px, meta = small_catalog(n=300, seed=41, size_deg=4.0)
    host = T.fill_distances(0.3, px)
    zeroed = px.copy()
    zeroed["distance"] = 0.0
    a = T.Catalog(engine, los, host, 6)
    b = T.Catalog(engine, los, zeroed, 6, omega_matter=0.3)
    da, db = a.distances(), b.distances()
    assert np.array_equal(da, compact(los, host)["distance"])
    assert np.array_equal(da, db)
    g = GRIDS["cartesian"]
    ra = T.xi_run(engine, a, g, meta["scale"])[0]
    rb = T.xi_run(engine, b, g, meta["scale"])[0]
    a.close()
    b.close()
    assert np.array_equal(ra, rb)


def test_device_distances_full_survey_geometry(engine):
    los, px, meta = T.synth.full_survey(20000, seed=7, area_deg2=1250.0)
    host = T.fill_distances(0.3, px)
    b = T.Catalog(engine, los, px, 6, omega_matter=0.3)
    db = b.distances()
    b.close()
    assert len(db) > 10**6
    assert np.array_equal(db, compact(los, host)["distance"])


def test_device_distances_refuse_negative_redshift(engine):
    los, px, meta = small_catalog(n=40, seed=42, size_deg=2.0)
    bad = px.copy()
    bad["loglam"][3] = 3.0  # below log10(1216): z < 0
    with pytest.raises(T.TosError) as e:
        T.Catalog(engine, los, bad, 6, omega_matter=0.3)
    assert e.value.status == 1
