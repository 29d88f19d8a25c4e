"""Host-side helpers of the batched configuration (no GPU): merging mock
catalogues into one catalogue of sightline groups, and the seeded mock draw."""
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
