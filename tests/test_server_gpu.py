"""The request server (tos_server): continuous admission of xi requests to
worker slots under a device-memory budget, and chunk-level scheduling of
their sweeps.

Pass criteria: every request's result is bit-identical to tos_xi_run on the
same catalogue alone (bins, per-group rows, pair counts), whatever else runs
beside it; requests on different slots overlap in time; under a budget that
holds one workspace at a time they run one after another and still give the
same results; FIFO starts requests in arrival order, shortest-first may
reorder them but gives the same results, and a short request that arrives
while a long one sweeps finishes first; requests and catalogues that cannot
fit are refused."""
import numpy as np
import pytest

import tos_b200 as T
from tos_b200 import synth  # noqa: F401  (T.synth)
from helpers import FIELDS, GRIDS, small_catalog

pytestmark = pytest.mark.gpu
ALL = FIELDS + ("num_pairs",)


@pytest.fixture(scope="module")
def catalogs(engine):
    a = small_catalog(n=150, seed=21, size_deg=3.0, max_pixels=200)
    b = small_catalog(n=300, seed=22, size_deg=4.0, max_pixels=300)
    c1 = small_catalog(n=80, seed=23, size_deg=2.0, max_pixels=150)
    c2 = small_catalog(n=120, seed=24, size_deg=2.5, max_pixels=150)
    c_los, c_px = T.synth.merge_groups([(c1[0], c1[1]), (c2[0], c2[1])])
    cats = {
        "a": (T.Catalog(engine, a[0], a[1], 6), a[2]["scale"]),
        "b": (T.Catalog(engine, b[0], b[1], 6), b[2]["scale"]),
        "c": (T.Catalog(engine, c_los, c_px, 6), c1[2]["scale"]),
    }
    yield cats
    for cat, _ in cats.values():
        cat.close()


def mix():
    """(catalogue, grid, per_group) of a mixed stream: both binnings of the
    serving mix and a batched (per-group) request."""
    out = []
    for rep in range(2):
        for key in ("b", "a", "c"):
            out.append((key, "cartesian", key == "c"))
            out.append((key, "polar", False))
    out.append(("a", "observing", False))
    return out


def alone(engine, cats, key, gname, per_group):
    cat, scale = cats[key]
    bins, rows, _ = T.xi_run(engine, cat, GRIDS[gname], scale, per_group=per_group)
    return bins, rows


def assert_identical(x, y, what):
    for f in ALL:
        assert np.array_equal(x[f], y[f]), f"{what}: field {f} differs"


@pytest.mark.parametrize("policy", ["fifo", "shortest"])
def test_results_same_alone_and_in_mix(engine, catalogs, policy):
    ref = {}
    for key, gname, pg in mix():
        ref[(key, gname, pg)] = alone(engine, catalogs, key, gname, pg)
    with T.Server(0, slots=3, memory_budget_bytes=40 * 10**9) as srv:
        srv.set_policy(policy, max_wait_s=5.0)
        for cat, _ in catalogs.values():
            srv.attach(cat)
        reqs = []
        for key, gname, pg in mix():
            cat, scale = catalogs[key]
            reqs.append(((key, gname, pg), srv.submit(cat, GRIDS[gname], scale, per_group=pg)))
        infos = []
        for k, r in reqs:
            bins, rows, st, info = r.wait()
            rb, rr = ref[k]
            assert_identical(bins, rb, str(k))
            if k[2]:
                assert rows.shape == rr.shape
                for g in range(rows.shape[0]):
                    assert_identical(rows[g], rr[g], f"{k} group {g}")
            infos.append(info)
        status = srv.status()
    assert status["completed"] == len(reqs)
    assert status["queued"] == 0 and status["running"] == 0
    assert {i["slot"] for i in infos} == {0, 1, 2}
    # requests on different slots ran at the same time
    ev = sorted([(i["start_s"], 1) for i in infos] + [(i["end_s"], -1) for i in infos])
    live, most = 0, 0
    for _, d in ev:
        live += d
        most = max(most, live)
    assert most >= 2
    for i in infos:
        assert i["submit_s"] <= i["start_s"] <= i["end_s"]
    if policy == "fifo":  # requests start in arrival order
        starts = [i["start_s"] for i in infos]
        assert starts == sorted(starts)


def test_budget_for_one_workspace_serialises(engine, catalogs):
    cat, scale = catalogs["b"]
    g = GRIDS["cartesian"]
    ref, _ = alone(engine, catalogs, "b", "cartesian", False)
    with T.Server(0, slots=2, memory_budget_bytes=40 * 10**9) as probe:
        probe.attach(cat)
        _, _, _, info = probe.submit(cat, g, scale).wait()
        held = probe.status()["in_use_bytes"] - probe.status()["resident_bytes"]
    need = max(info["workspace_bytes"], held)
    budget = cat.device_bytes() + int(need * 1.5)
    with T.Server(0, slots=2, memory_budget_bytes=budget) as srv:
        srv.attach(cat)
        reqs = [srv.submit(cat, g, scale) for _ in range(4)]
        infos = []
        for r in reqs:
            bins, _, _, info = r.wait()
            assert_identical(bins, ref, "serialised")
            infos.append(info)
        st = srv.status()
    assert st["peak_bytes"] <= budget
    infos.sort(key=lambda i: i["start_s"])
    for p, q in zip(infos, infos[1:]):
        assert q["start_s"] >= p["end_s"]  # one workspace at a time


def test_refusals(engine, catalogs):
    cat, scale = catalogs["a"]
    with T.Server(0, slots=1, memory_budget_bytes=1000) as srv:
        with pytest.raises(T.TosError) as e:
            srv.attach(cat)
        assert e.value.status == 2  # TOS_ERR_OOM
    with T.Server(0, slots=1, memory_budget_bytes=cat.device_bytes() + 10**6) as srv:
        srv.attach(cat)
        with pytest.raises(T.TosError) as e:
            srv.submit(cat, GRIDS["cartesian"], scale)  # its workspace cannot fit
        assert e.value.status == 2
    with T.Server(0, slots=1, memory_budget_bytes=10**10) as srv:
        other, oscale = catalogs["b"]
        with pytest.raises(T.TosError):
            srv.submit(other, GRIDS["cartesian"], oscale)  # not attached
        srv.attach(cat)
        r = srv.submit(cat, GRIDS["polar"], scale)
        with pytest.raises(T.TosError):
            srv.detach(cat)  # a request is unfinished
        while not r.done():  # poll without blocking
            pass
        r.wait()
        with pytest.raises(T.TosError):
            r.done()  # the id is released by wait
        srv.detach(cat)


def test_destroy_with_requests_in_flight(engine, catalogs):
    """Destroying a server finishes the running request and ends the queued
    ones; nothing hangs and the ids are gone afterwards."""
    cat, scale = catalogs["b"]
    srv = T.Server(0, slots=1, memory_budget_bytes=40 * 10**9)
    srv.attach(cat)
    reqs = [srv.submit(cat, GRIDS["polar"], scale) for _ in range(4)]
    srv.close()  # joins the running request, drops the three queued ones
    for r in reqs:
        with pytest.raises(T.TosError):
            r.wait()  # the server handle is gone: a clean error, not a crash


def test_subsample_rows_through_the_server(engine, catalogs):
    """A request for per-cell rows returns tos_xi_run's per-cell sums."""
    cat, scale = catalogs["a"]
    g = GRIDS["cartesian"]
    rb, rc, _ = T.xi_run(engine, cat, g, scale, subsamples=True)
    with T.Server(0, slots=2, memory_budget_bytes=10**10) as srv:
        srv.attach(cat)
        bins, rows, _, _ = srv.submit(cat, g, scale, subsamples=True).wait()
    assert rows.shape == rc.shape
    assert_identical(bins, rb, "bins")
    for c in range(rows.shape[0]):
        assert_identical(rows[c], rc[c], f"cell {c}")


def test_short_request_overtakes_long_sweep(engine, catalogs):
    """A long request's sweep runs as a chain of chunks; with the
    shortest-first order a short request submitted while it sweeps takes the
    GPU at the long one's next chunk and finishes first.  Both results equal
    their lone runs."""
    import time
    los, px, meta = T.synth.full_survey(20000, seed=7, area_deg2=1250.0)
    big = T.Catalog(engine, los, px, 6)
    small, s_scale = catalogs["a"]
    g = GRIDS["cartesian"]
    ref_big = T.xi_run(engine, big, g, meta["scale"])[0]
    ref_small = T.xi_run(engine, small, g, s_scale)[0]
    try:
        with T.Server(0, slots=2, memory_budget_bytes=40 * 10**9) as srv:
            srv.set_policy("shortest", max_wait_s=30.0)
            srv.attach(big)
            srv.attach(small)
            rb = srv.submit(big, g, meta["scale"])
            time.sleep(0.05)
            rs = srv.submit(small, g, s_scale)
            bb, _, st_b, ib = rb.wait()
            bs, _, _, i_s = rs.wait()
    finally:
        big.close()
    assert st_b["num_sightline_pairs_used"] > 2 * 131072  # several chunks
    assert_identical(bb, ref_big, "long request")
    assert_identical(bs, ref_small, "short request")
    assert i_s["start_s"] < ib["end_s"] and i_s["end_s"] < ib["end_s"]
