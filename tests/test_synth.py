"""Host-side helpers of the synthetic catalogues (no GPU): merging mock
catalogues into one catalogue of sightline groups, the seeded mock draw, and
the plate layout of the plate-cell tests."""
import numpy as np

from tos_b200 import synth
from helpers import small_catalog


def test_merge_groups_offsets_and_groups():
    a_los, a_px, _ = small_catalog(n=7, seed=1, size_deg=2.0, max_pixels=20)
    b_los, b_px, _ = small_catalog(n=5, seed=2, size_deg=2.0, max_pixels=30)
    los, px = synth.merge_groups([(a_los, a_px), (b_los, b_px)])
    assert len(los) == 12 and len(px) == len(a_px) + len(b_px)
    assert list(los["group"]) == [0] * 7 + [1] * 5
    for s in range(12):
        src_los, src_px = (a_los, a_px) if s < 7 else (b_los, b_px)
        t = s if s < 7 else s - 7
        o, n = int(los[s]["pixel_offset"]), int(los[s]["num_pixels"])
        so = int(src_los[t]["pixel_offset"])
        assert n == int(src_los[t]["num_pixels"])
        assert np.array_equal(px[o:o + n], src_px[so:so + n])
    # the inputs are untouched
    assert a_los["group"].max() == 0 and int(b_los[0]["pixel_offset"]) == 0


def test_mock_draw_is_seeded_and_log_uniform():
    c1 = synth.mock_counts(256, seed=11)
    c2 = synth.mock_counts(256, seed=11)
    assert np.array_equal(c1, c2)
    assert c1.min() >= 2000 and c1.max() <= 40000
    # log-uniform: about half the mocks below the geometric mean
    gm = np.sqrt(2000 * 40000)
    assert 0.35 < np.mean(c1 < gm) < 0.65
    # the first mocks of a longer draw are the same mocks
    assert np.array_equal(synth.mock_counts(300, seed=11)[:256], c1)


def test_cap_patch_density():
    los, px, meta = synth.cap_patch(400, seed=3, area_deg2=25.0)
    v = np.stack([np.cos(los["dec"]) * np.cos(los["ra"]), np.cos(los["dec"]) * np.sin(los["ra"]),
                  np.sin(los["dec"])], 1)
    centre = v.mean(0)
    centre /= np.linalg.norm(centre)
    cap = np.degrees(np.arccos(np.clip(v @ centre, -1, 1))).max()
    # a 25 deg^2 cap has a radius of about 2.82 deg
    assert 2.3 < cap < 3.1


def test_plate_tiling_puts_every_sightline_near_its_plate():
    """BOSS-like plates: ids unique, every sightline on a listed plate whose
    centre is within 1.5 degrees (a plate's field radius is 1.49 degrees), the
    nearest one, so the plate-cell tests start from a realistic layout."""
    import math
    los, _, _ = small_catalog(n=300, seed=4, size_deg=8.0, max_pixels=4)
    out, plates = synth.plate_tiling(los, 2.0)
    assert len(np.unique(plates["plate"])) == len(plates)
    assert np.isin(out["plate"], plates["plate"]).all()
    by_id = {int(p["plate"]): p for p in plates}

    def unit(ra, dec):
        return np.array([math.cos(dec) * math.cos(ra), math.cos(dec) * math.sin(ra), math.sin(dec)])

    for s in range(len(out)):
        p = by_id[int(out["plate"][s])]
        u = unit(float(out["ra"][s]), float(out["dec"][s]))
        d = math.degrees(math.acos(min(1.0, float(u @ unit(math.radians(float(p["ra_center"])),
                                                            math.radians(float(p["dec_center"])))))))
        assert d < 1.5, (s, d)
    # only the plate id changes
    assert np.array_equal(out["ra"], los["ra"]) and np.array_equal(out["num_pixels"], los["num_pixels"])
