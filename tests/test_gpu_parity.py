"""Parity of the B200 engine (through the C ABI) with the CPU oracle and the
reference's golden journeys.  Integer work: results must be identical."""
import ctypes as C

import numpy as np
import pytest

import fixture as F
import oracle_lib
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

pytestmark = pytest.mark.gpu
CASES = F.load_cases()


def run_batch(engine, qarr, n, plain=False):
    out = (A.Result * max(1, n))()
    lib = A.lib()
    recs = []
    if plain:
        for i in range(n):
            rc = lib.b2r_search_plain(engine.handle, C.byref(qarr[i]), C.byref(out[i]))
            assert rc == 0, lib.b2r_last_error()
            recs.append(records(out[i]) if out[i].round_times is None or not bool(out[i].round_times)
                        else ("rows", out[i].n_rows, out[i].base_day))
        return recs, out
    rc = lib.b2r_search_batch(engine.handle, qarr, n, out)
    assert rc == 0, lib.b2r_last_error()
    return [records(out[i]) for i in range(n)], out


@pytest.fixture(scope="module")
def golden_engines():
    lib = A.lib()
    res = {}
    for name, spec in CASES["timetables"].items():
        ftt = F.FixtureTimetable(spec, lib)
        dtt = R.Timetable(ftt.desc, owner=ftt)
        eng = R.Engine(dtt, max_slots=64)
        res[name] = (ftt, dtt, eng)
    return res


@pytest.mark.parametrize("plain", [False, True], ids=["batched", "plain"])
def test_golden_cases_on_gpu(golden_engines, plain):
    by_tt = {}
    for c in CASES["cases"]:
        by_tt.setdefault(c["timetable"], []).append(c)
    for name, cases in by_tt.items():
        ftt, dtt, eng = golden_engines[name]
        qs = [F.FixtureQuery(A.lib(), ftt, c["query"]) for c in cases]
        arr = (A.Query * len(qs))()
        for i, q in enumerate(qs):
            arr[i] = q.q
        out = (A.Result * len(qs))()
        if plain:
            for i in range(len(qs)):
                assert A.lib().b2r_search_plain(eng.handle, C.byref(arr[i]), C.byref(out[i])) == 0
                got = F.journeys_to_records(ftt, out[i])
                assert got == F.strip_expected(cases[i]["expected"]), cases[i]["name"]
        else:
            assert A.lib().b2r_search_batch(eng.handle, arr, len(qs), out) == 0
            for i, c in enumerate(cases):
                got = F.journeys_to_records(ftt, out[i])
                assert got == F.strip_expected(c["expected"]), c["name"]


def oracle_records(desc, q):
    r = oracle_lib.OracleResult(desc, q)
    return records(r.view), r


@pytest.fixture(scope="module")
def c1():
    h = HostTimetable.generate(1)
    dtt = R.Timetable(h.desc, owner=h)
    return h, dtt, R.Engine(dtt, max_slots=256)


@pytest.fixture(scope="module")
def c2():
    h = HostTimetable.generate(2)
    dtt = R.Timetable(h.desc, owner=h)
    return h, dtt, R.Engine(dtt, max_slots=256)


def test_workload1_batched_matches_oracle(c1):
    h, dtt, eng = c1
    qs = QuerySet(h, 1, 300)
    got, _ = run_batch(eng, qs.arr, qs.n)
    n_j = 0
    for i in range(qs.n):
        exp, _ = oracle_records(h.desc, qs.arr[i])
        assert got[i] == exp, i
        n_j += len(exp)
    assert n_j > 100


def test_workload1_plain_matches_batched(c1):
    h, dtt, eng = c1
    qs = QuerySet(h, 1, 40, seed=77)
    got_b, _ = run_batch(eng, qs.arr, qs.n)
    got_p, _ = run_batch(eng, qs.arr, qs.n, plain=True)
    assert got_b == got_p


def test_workload2_intermodal_matches_oracle(c2):
    h, dtt, eng = c2
    qs = QuerySet(h, 2, 96)
    got, _ = run_batch(eng, qs.arr, qs.n)
    for i in range(qs.n):
        exp, _ = oracle_records(h.desc, qs.arr[i])
        assert got[i] == exp, i


def test_workload3_range_fwd_bwd_matches_oracle(c2):
    h, dtt, eng = c2
    qs = QuerySet(h, 3, 48)
    got, _ = run_batch(eng, qs.arr, qs.n)
    dirs = set()
    for i in range(qs.n):
        exp, _ = oracle_records(h.desc, qs.arr[i])
        assert got[i] == exp, i
        dirs.add(qs.arr[i].direction)
    assert dirs == {0, 1}


@pytest.mark.parametrize("workload", [1, 2])
def test_one_to_all_rows_match_oracle(workload, c1, c2):
    h, dtt, eng = c1 if workload == 1 else c2
    qs = QuerySet(h, 1, 12, seed=5 + workload)
    arr = (A.Query * qs.n)()
    for i in range(qs.n):
        arr[i] = qs.arr[i]
        arr[i].kind = A.B2R_ONE_TO_ALL
        arr[i].n_destination = 0
        arr[i].direction = i % 2
    out = (A.Result * qs.n)()
    assert A.lib().b2r_search_batch(eng.handle, arr, qs.n, out) == 0
    n = h.desc.n_locations
    for i in range(qs.n):
        r = out[i]
        rows = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n,)).reshape(r.n_rows, n)
        o = oracle_lib.OracleResult(h.desc, arr[i])
        orows, _, base_day = o.state()
        assert r.base_day == base_day
        assert np.array_equal(rows, orows[: r.n_rows]), i


@pytest.mark.parametrize("lb_mode", ["host", "device", False])
def test_lower_bound_modes_give_identical_journeys(c2, lb_mode):
    """Lower bounds only prune: journeys are the same with bounds computed
    on the device, on the host, or without bounds (nigiri's GPU raptor runs
    without them, gpu/raptor.h:60)."""
    h, dtt, eng = c2
    other = R.Engine(dtt, max_slots=128, use_lower_bounds=lb_mode)
    qs = QuerySet(h, 2, 64, seed=31)
    a, _ = run_batch(eng, qs.arr, qs.n)
    b, _ = run_batch(other, qs.arr, qs.n)
    assert a == b


FIXTURE_QUERIES = [
    # parents and children (dijkstra_test.cc's feed): exact, equivalent,
    # range, both directions
    ("gtfs_dijkstra", dict(start=[["D1", 0, 0]], dest=[["C2", 0, 0]], start_time=28630500)),
    ("gtfs_dijkstra", dict(start=[["D", 0, 0]], dest=[["C", 0, 0]], start_time=28630500,
                           start_mode="equivalent", dest_mode="equivalent")),
    ("gtfs_dijkstra", dict(start=[["A", 0, 0], ["D1", 5, 0]], dest=[["C", 0, 0]],
                           interval=[28630440, 28630680], dest_mode="equivalent")),
    ("gtfs_dijkstra", dict(start=[["C2", 0, 0]], dest=[["D", 0, 0]], interval=[28630620, 28630740],
                           direction="bwd", dest_mode="equivalent", start_mode="equivalent")),
    # start_times_test.cc's feed: a walk to the start over a whole day
    ("hrd_simple", dict(start=[["0000001", 15, 0]], dest=[["0000002", 0, 0]],
                        interval=[26425440, 26426880])),
    ("hrd_simple", dict(start=[["0000002", 0, 0]], dest=[["0000001", 10, 0]],
                        interval=[26425440, 26426880], direction="bwd")),
]


@pytest.mark.parametrize("tt_name,q", FIXTURE_QUERIES)
def test_fixture_queries_match_oracle(golden_engines, tt_name, q):
    """Engine against the oracle on the fixtures of nigiri's start-time and
    Dijkstra tests (the oracle is pinned on their known answers)."""
    ftt, _, eng = golden_engines[tt_name]
    fq = F.FixtureQuery(A.lib(), ftt, q)
    res = A.Result()
    assert A.lib().b2r_search_batch(eng.handle, C.byref(fq.q), 1, C.byref(res)) == 0
    exp = oracle_lib.OracleResult(ftt.desc, fq.q).records()
    assert records(res) == exp
