"""The CPU oracle against the golden journey printouts of nigiri's own
routing tests (tests/golden/cases.json, made by make_fixtures.py)."""
import ctypes as C

import pytest

import fixture as F
import oracle_lib
from nigiri_b200 import _abi as A

CASES = F.load_cases()


@pytest.fixture(scope="module")
def timetables():
    lib = A.lib()
    return {k: F.FixtureTimetable(v, lib) for k, v in CASES["timetables"].items()}


@pytest.mark.parametrize("case", CASES["cases"], ids=[c["name"] for c in CASES["cases"]])
def test_oracle_matches_golden(case, timetables):
    tt = timetables[case["timetable"]]
    q = F.FixtureQuery(A.lib(), tt, case["query"])
    r = oracle_lib.OracleResult(tt.desc, q.q)
    assert F.journeys_to_records(tt, r.view) == F.strip_expected(case["expected"])


INTERVAL_CASES = [c for c in CASES["cases"] if "interval" in c["query"]]


@pytest.mark.parametrize("case", INTERVAL_CASES, ids=[c["name"] for c in INTERVAL_CASES])
def test_oracle_pong_matches_golden_in_window(case, timetables):
    """pong_search against the same golden printouts: inside the query's
    interval its journeys print exactly as range RAPTOR's, and outside it
    they respect the interval-extension flags (test/raptor_search.cc:198-237
    runs every interval query of nigiri's tests this way)."""
    tt = timetables[case["timetable"]]
    qd = dict(case["query"], algorithm="pong")
    q = F.FixtureQuery(A.lib(), tt, qd)
    r = oracle_lib.OracleResult(tt.desc, q.q)
    got = F.journeys_to_records(tt, r.view)
    lo, hi = qd["interval"]
    key = "dep" if qd.get("direction", "fwd") == "fwd" else "arr"
    if not qd.get("extend_earlier"):
        assert all(j[key] >= lo for j in got)
    if not qd.get("extend_later"):
        assert all(j[key] < hi for j in got)
    assert F.in_window(qd, got) == F.in_window(qd, F.strip_expected(case["expected"]))


def test_golden_cases_cover_both_directions_and_intermodal():
    names = [c["name"] for c in CASES["cases"]]
    assert any("backward" in n or n.endswith("_bwd") for n in names)
    assert any("intermodal" in n for n in names)
    assert sum(len(c["expected"]) for c in CASES["cases"]) >= 40


def _names(tt):
    by_id = {x["id"]: x["name"] for x in tt.spec["locations"]}
    return {idx: by_id.get(i, i) for i, idx in tt.loc_idx.items()}


@pytest.mark.parametrize("ka", CASES["known_answers"], ids=[k["name"] for k in CASES["known_answers"]])
def test_oracle_known_answers(ka, timetables):
    """Intermediate results pinned by nigiri's own tests: the start labels of
    an interval search (start_times_test.cc) and Dijkstra lower bounds over
    a timetable with parent stations (dijkstra_test.cc)."""
    tt = timetables[ka["timetable"]]
    q = F.FixtureQuery(A.lib(), tt, ka["query"])
    L = oracle_lib.lib()
    name = _names(tt)
    if ka["kind"] == "starts":
        cap = 1 << 14
        tas, tst = (C.c_int32 * cap)(), (C.c_int32 * cap)()
        stop = (C.c_uint32 * cap)()
        n = C.c_uint32()
        assert L.or_get_starts(C.byref(tt.desc), C.byref(q.q), tas, tst, stop, cap, C.byref(n)) == 0
        # the test's own order: descending by (time_at_start, time_at_stop,
        # stop), duplicates removed
        got = sorted({(tas[i], tst[i], stop[i]) for i in range(n.value)}, reverse=True)
        assert [[a, b, name[s]] for a, b, s in got] == ka["expected"]
    elif ka["kind"] == "departures":
        r = oracle_lib.OracleResult(tt.desc, q.q)
        deps = sorted(j["dep"] for j in F.journeys_to_records(tt, r.view))
        if "expected" in ka:
            assert deps == ka["expected"]
        if "not_before" in ka:
            assert all(d >= ka["not_before"] for d in deps)
    elif ka["kind"] == "departure_range":  # the first and last departure of the results
        r = oracle_lib.OracleResult(tt.desc, q.q)
        deps = sorted(j["dep"] for j in F.journeys_to_records(tt, r.view))
        assert deps and [deps[0], deps[-1]] == ka["expected"]
    elif ka["kind"] == "earliest_alternative":
        legs = (A.Leg * 3)()
        qq = q.q
        rc = L.or_earliest_alternative(C.byref(tt.desc), C.byref(qq), tt.loc_idx["A"],
                                       tt.loc_idx["C"], qq.start_time, ka["to_dep"], legs)
        assert rc == (1 if ka["expected"] else 0)
        if rc == 1:
            assert [legs[i].kind for i in range(3)] == [A.B2R_LEG_FOOTPATH, A.B2R_LEG_TRANSPORT,
                                                       A.B2R_LEG_FOOTPATH]
    else:
        dists = (C.c_uint16 * tt.desc.n_locations)()
        assert L.or_lower_bounds(C.byref(tt.desc), C.byref(q.q), dists) == 0
        for loc, value in ka["expected"]:
            assert dists[tt.loc_idx[loc]] == value, loc
