"""pong_search (src/routing/raptor/pong.cc) on the engine and in the oracle.

CPU: on generated timetables the oracle's pong prints, inside each query's
interval, exactly the journeys of its range RAPTOR -- the agreement nigiri's
own test harness (test/raptor_search.cc:198-237) and benchmark cross-check
require of every interval query.  GPU: the engine's pong against the
oracle's, complete result lists, on the golden interval cases and on range
queries of the generated workloads (both directions, station and
intermodal, with and without filters)."""
import ctypes as C

import pytest

import fixture as F
import oracle_lib
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200.timetable import HostTimetable, QuerySet

CASES = F.load_cases()
INTERVAL_CASES = [c for c in CASES["cases"] if "interval" in c["query"]]


def with_start_footpaths(arr, n):
    """Station queries walking from the start as from the destination.  A
    pong that may end on a walk from the origin while its ping may not start
    with one finds journeys the ping cannot see, and fails as the reference
    does ("no pong", pong.cc:328-333)."""
    out = (A.Query * n)()
    for i in range(n):
        out[i] = arr[i]
        if out[i].start_match_mode != A.B2R_MATCH_INTERMODAL:
            out[i].use_start_footpaths = 1
    return out


def as_pong(arr, n, filters=False):
    out = (A.Query * n)()
    for i in range(n):
        out[i] = arr[i]
        out[i].algorithm = A.B2R_ALGO_PONG
        if filters and i % 3 != 0:
            out[i].allowed_claszes = 0xFFFF & ~(1 << (10 if i % 3 == 1 else 9))
            out[i].require_bike_transport = 1 if i % 3 == 2 else 0
    return out


def intermodal_ranges(h, n, seed):
    """Workload-2 queries (intermodal offset sets) as 90-minute ranges."""
    qs = QuerySet(h, 2, n, seed=seed)
    arr = (A.Query * qs.n)()
    for i in range(qs.n):
        arr[i] = qs.arr[i]
        arr[i].is_interval = 1
        arr[i].interval_from = qs.arr[i].start_time
        arr[i].interval_to = qs.arr[i].start_time + 90
        arr[i].direction = i % 2
    return qs, arr


def window(q, recs):
    """The journeys anchored in q's interval (departure forward, arrival
    backward), as printed: without journey::dest_, which pong leaves at the
    location its backward search ended (the query's start)."""
    lo, hi = q.interval_from, q.interval_to
    out = []
    for r in recs:
        dep = min(r["start"], r["dest_time"])
        arr = max(r["start"], r["dest_time"])
        anchor = dep if q.direction == A.B2R_FORWARD else arr
        if lo <= anchor < hi:
            out.append({k: v for k, v in r.items() if k != "dest"})
    return out


@pytest.fixture(scope="module")
def tt1():
    return HostTimetable.generate(1)


def pareto(recs):
    return [(r["start"], r["dest_time"], r["transfers"]) for r in recs]


def test_oracle_pong_agrees_with_range_raptor_in_window(tt1):
    """The agreement nigiri's benchmark checks between pong and range RAPTOR
    (exe/benchmark.cc: the Pareto sets on the common interval), here on 40
    generated range queries in both directions.  The legs may differ: pong
    reconstructs backward, and its forward pass only replaces inner rides."""
    qs = QuerySet(tt1, 3, 40, seed=515)
    rq = with_start_footpaths(qs.arr, qs.n)
    pq = as_pong(rq, qs.n)
    n_in = 0
    for i in range(qs.n):
        rr = oracle_lib.OracleResult(tt1.desc, rq[i]).records()
        pr = oracle_lib.OracleResult(tt1.desc, pq[i]).records()
        assert pareto(window(rq[i], pr)) == pareto(window(rq[i], rr)), i
        n_in += len(window(rq[i], rr))
    assert n_in > 40


# ------------------------------------------------------------------ GPU

@pytest.fixture(scope="module")
def engines():
    from nigiri_b200 import routing as R
    out = {}
    for w in (1, 2):
        h = HostTimetable.generate(w)
        dtt = R.Timetable(h.desc, owner=h)
        out[w] = (h, dtt, R.Engine(dtt, max_slots=128))
    return out


@pytest.fixture(scope="module")
def golden():
    from nigiri_b200 import routing as R
    lib = A.lib()
    res = {}
    for name, spec in CASES["timetables"].items():
        ftt = F.FixtureTimetable(spec, lib)
        dtt = R.Timetable(ftt.desc, owner=ftt)
        res[name] = (ftt, dtt, R.Engine(dtt, max_slots=32))
    return res


def batch(eng, qarr, n):
    out = (A.Result * n)()
    assert A.lib().b2r_search_batch(eng.handle, qarr, n, out) == 0, A.lib().b2r_last_error()
    return out


@pytest.mark.gpu
def test_pong_golden_cases_match_oracle(golden):
    for c in INTERVAL_CASES:
        ftt, _, eng = golden[c["timetable"]]
        fq = F.FixtureQuery(A.lib(), ftt, dict(c["query"], algorithm="pong"))
        out = batch(eng, C.pointer(fq.q), 1)
        exp = oracle_lib.OracleResult(ftt.desc, fq.q)
        assert out[0].status == A.B2R_OK, c["name"]
        assert records(out[0]) == exp.records(), c["name"]
        assert (out[0].interval_from, out[0].interval_to) == \
            (exp.view.interval_from, exp.view.interval_to), c["name"]


@pytest.mark.gpu
@pytest.mark.parametrize("workload,filters", [(1, False), (2, False), (2, True)],
                         ids=["w1", "w2", "w2_filters"])
def test_pong_range_queries_match_oracle(engines, workload, filters):
    h, _, eng = engines[workload]
    qs = QuerySet(h, 3, 48, seed=600 + workload)
    pq = as_pong(with_start_footpaths(qs.arr, qs.n), qs.n, filters)
    out = batch(eng, pq, qs.n)
    n_j = 0
    for i in range(qs.n):
        exp = oracle_lib.OracleResult(h.desc, pq[i])
        assert out[i].status == A.B2R_OK, i
        assert records(out[i]) == exp.records(), i
        assert (out[i].interval_from, out[i].interval_to) == \
            (exp.view.interval_from, exp.view.interval_to), i
        n_j += out[i].n_journeys
    assert n_j > 40


@pytest.mark.gpu
def test_pong_intermodal_ranges_match_oracle(engines):
    h, _, eng = engines[2]
    qs, arr = intermodal_ranges(h, 24, seed=77)
    pq = as_pong(arr, qs.n)
    out = batch(eng, pq, qs.n)
    for i in range(qs.n):
        exp = oracle_lib.OracleResult(h.desc, pq[i])
        assert records(out[i]) == exp.records(), i


@pytest.mark.gpu
def test_pong_mixed_with_range_raptor_in_one_batch(engines):
    """Pong and range-RAPTOR queries share the resident slots of one batch;
    each gets the result of its own algorithm."""
    h, _, eng = engines[1]
    qs = QuerySet(h, 3, 32, seed=901)
    mixed = with_start_footpaths(qs.arr, qs.n)
    for i in range(qs.n):
        mixed[i].algorithm = A.B2R_ALGO_PONG if i % 2 else A.B2R_ALGO_RAPTOR
    out = batch(eng, mixed, qs.n)
    for i in range(qs.n):
        assert records(out[i]) == oracle_lib.OracleResult(h.desc, mixed[i]).records(), i
