"""Edge cases of the batched engine against the oracle: an empty batch,
starts that overlap the destinations (search.h:354-378), searches that
reach nothing within their travel-time bound, and queries whose start labels
exceed a slot's capacity inside a batch of ordinary queries (reported per
query, the others unaffected)."""
import ctypes as C

import pytest

import oracle_lib
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    h = HostTimetable.generate(1)
    dtt = R.Timetable(h.desc, owner=h)
    return h, dtt


def oracle(desc, q):
    r = oracle_lib.OracleResult(desc, q)  # owns the records its view points to
    return r.view.status, records(r.view)


def run(eng, arr, n):
    out = (A.Result * max(1, n))()
    assert A.lib().b2r_search_batch(eng.handle, arr, n, out) == 0, A.lib().b2r_last_error()
    return [(out[i].status, records(out[i])) for i in range(n)]


def test_empty_batch(c1):
    h, dtt = c1
    eng = R.Engine(dtt, max_slots=32)
    assert A.lib().b2r_search_batch(eng.handle, None, 0, None) == 0
    assert eng.stats().super_steps == 0


def test_starts_overlapping_destinations_match_oracle(c1):
    h, dtt = c1
    eng = R.Engine(dtt, max_slots=32)
    qs = QuerySet(h, 1, 16, seed=31)
    arr = (A.Query * qs.n)()
    for i in range(qs.n):
        arr[i] = qs.arr[i]
        arr[i].destination = qs.arr[i].start  # the start offsets are the destinations too
        arr[i].n_destination = qs.arr[i].n_start
        if i % 2:  # half as 1 h range queries
            arr[i].is_interval = 1
            arr[i].interval_from = qs.arr[i].start_time
            arr[i].interval_to = qs.arr[i].start_time + 60
    got = run(eng, arr, qs.n)
    for i in range(qs.n):
        assert got[i] == oracle(h.desc, arr[i]), i
    assert all(not recs for _, recs in got)


def test_searches_reaching_nothing_match_oracle(c1):
    h, dtt = c1
    eng = R.Engine(dtt, max_slots=32)
    qs = QuerySet(h, 1, 24, seed=32)
    arr = (A.Query * qs.n)()
    for i in range(qs.n):
        arr[i] = qs.arr[i]
        day = qs.arr[i].start_time - qs.arr[i].start_time % 1440
        arr[i].start_time = day + 3 * 60  # 03:00 UTC, before the first departures
        arr[i].max_travel_time = 10
    got = run(eng, arr, qs.n)
    for i in range(qs.n):
        assert got[i] == oracle(h.desc, arr[i]), i


def test_queries_beyond_slot_capacity_fail_alone(c1):
    h, dtt = c1
    eng = R.Engine(dtt, max_slots=32, max_starts=16)
    qs = QuerySet(h, 1, 24, seed=33)
    arr = (A.Query * qs.n)()
    for i in range(qs.n):
        arr[i] = qs.arr[i]
        if i % 4 == 0:  # a 6 h range: more start labels than a slot holds
            arr[i].is_interval = 1
            arr[i].interval_from = qs.arr[i].start_time
            arr[i].interval_to = qs.arr[i].start_time + 360
    got = run(eng, arr, qs.n)
    n_cap = 0
    for i in range(qs.n):
        status, recs = got[i]
        if status == A.B2R_ERR_CAPACITY:
            n_cap += 1
            assert not recs
        else:
            assert got[i] == oracle(h.desc, arr[i]), i
    assert n_cap >= 3
    assert sum(1 for s, _ in got if s == A.B2R_OK) >= qs.n - n_cap
