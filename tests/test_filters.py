"""Query filters: allowed transport classes, required bike / car transport
and no compulsory reservation (routing/query.h:91-94, raptor.h:491-575 and
1177-1217, reconstruct.cc:239-250 and 455-515).

CPU: the timetable data behind the filters and properties of the oracle's
filtered journeys.  GPU: the engine against the oracle with filters on, for
one-to-one (both directions, ranges) and one-to-all searches."""
import ctypes as C

import numpy as np
import pytest

import fixture as F
import oracle_lib
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200.timetable import HostTimetable, QuerySet

CASES = F.load_cases()
BUS, TRAM, SUBWAY, SUBURBAN, REGIONAL = 10, 9, 8, 7, 6


def arr(ptr, n, dtype):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype).copy()


# (allowed classes, bikes, cars, no reservation) cycled over the queries
FILTERS = [
    (0xFFFF, 0, 0, 0),
    (0xFFFF & ~(1 << BUS), 0, 0, 0),
    (0xFFFF, 1, 0, 0),
    (0xFFFF, 1, 0, 1),
    ((1 << BUS) | (1 << TRAM), 0, 0, 1),
    (0xFFFF, 0, 1, 0),
    ((1 << SUBWAY) | (1 << SUBURBAN) | (1 << REGIONAL), 1, 0, 0),
]


def filtered(qs: QuerySet, n=None, kind=None):
    n = qs.n if n is None else n
    out = (A.Query * n)()
    for i in range(n):
        out[i] = qs.arr[i]
        mask, bikes, cars, resv = FILTERS[i % len(FILTERS)]
        out[i].allowed_claszes = mask
        out[i].require_bike_transport = bikes
        out[i].require_car_transport = cars
        out[i].no_compulsory_reservation = resv
        if kind is not None:
            out[i].kind = kind
    return out


@pytest.fixture(scope="module")
def tt1():
    return HostTimetable.generate(1)


def route_data(d):
    nr = d.n_routes
    rsi = arr(d.route_stop_index, nr + 1, np.int64)
    return (rsi, arr(d.route_clasz, nr, np.int64), arr(d.route_flags, nr, np.int64),
            arr(d.route_section_flags, int(rsi[-1]), np.int64))


def test_generated_routes_carry_classes_and_flags(tt1):
    """Every class of the mix occurs; each flag is on all, some and no
    sections of some routes; route flags follow register_route's rule
    (timetable.cc:136-156) from the per-section flags."""
    rsi, clasz, flags, sec = route_data(tt1.desc)
    assert set(clasz.tolist()) == {BUS, TRAM, SUBWAY, SUBURBAN, REGIONAL}
    kinds = {f: set() for f in range(4)}
    for r in range(tt1.desc.n_routes):
        n_sec = rsi[r + 1] - rsi[r] - 1
        s = sec[rsi[r]: rsi[r] + n_sec]
        for f in range(4):
            cnt = int(((s >> f) & 1).sum())
            all_ = cnt == n_sec and n_sec != 0
            some = cnt != 0
            assert ((flags[r] >> (2 * f)) & 1) == all_, (r, f)
            assert ((flags[r] >> (2 * f + 1)) & 1) == some, (r, f)
            kinds[f].add("all" if all_ else "some" if some else "none")
    for f in range(4):
        assert kinds[f] == {"all", "some", "none"}, f


def test_fixture_route_flags_from_sections():
    """b2r_tt_build derives the all / some bits from per-section flags: in
    the bike test's timetable 1 the chained transport T3>T5 has bikes on
    some sections, T4>T6 on all, T0 / T2 on none."""
    ftt = F.FixtureTimetable(CASES["timetables"]["gtfs_bikes_1"], A.lib())
    rsi, clasz, flags, sec = route_data(ftt.desc)
    by_stops = {}
    for r in range(ftt.desc.n_routes):
        stops = tuple(ftt.loc_name[int(w) & 0x0FFFFFFF]
                      for w in arr(ftt.desc.route_stops, int(rsi[-1]), np.int64)[rsi[r]:rsi[r + 1]])
        by_stops.setdefault(stops, []).append(int(flags[r]) & 3)
    assert sorted(by_stops[("A", "B", "C")]) == [0, 3]   # none (T0, T2), all (T1)
    assert sorted(by_stops[("C", "D", "E", "F")]) == [2, 3]  # some (T3>T5), all (T4>T6)
    assert set(clasz.tolist()) == {BUS}


def test_tt_build_rejects_unknown_class():
    spec = CASES["timetables"]["gtfs_clasz"]
    bad = dict(spec, routes=[dict(r, clasz=16) for r in spec["routes"]])
    with pytest.raises(AssertionError):
        F.FixtureTimetable(bad, A.lib())
    assert "route_clasz" in A.lib().b2r_last_error().decode()


def check_journeys_respect_filters(d, q, res):
    """Every transport leg of a filtered journey rides a route of an allowed
    class.  In journeys with a single ride, every section ridden carries the
    required flags; with more rides, opt_transfers (optimize_footpaths.cc,
    which looks at no flags) may move a transfer stop along a transport past
    a section without them, as the reference does."""
    rsi, clasz, flags, sec = route_data(d)
    troute = arr(d.transport_route, d.n_transports, np.int64)
    req = ((1 if q.require_bike_transport else 0) | (2 if q.require_car_transport else 0) |
           (8 if q.no_compulsory_reservation else 0))
    n_legs = 0
    for ji in range(res.n_journeys):
        j = res.journeys[ji]
        rides = [res.legs[li] for li in range(j.first_leg, j.first_leg + j.n_legs)
                 if res.legs[li].kind == A.B2R_LEG_TRANSPORT]
        for L in rides:
            n_legs += 1
            r = troute[L.transport]
            assert (q.allowed_claszes >> int(clasz[r])) & 1
            if len(rides) == 1:
                for s in range(L.stop_from, L.stop_to - 1):
                    assert (int(sec[rsi[r] + s]) & req) == req
    return n_legs


def test_oracle_filtered_journeys_respect_filters(tt1):
    qs = QuerySet(tt1, 1, 70, seed=4242)
    fq = filtered(qs)
    changed = 0
    legs = 0
    for i in range(qs.n):
        r = oracle_lib.OracleResult(tt1.desc, fq[i])
        legs += check_journeys_respect_filters(tt1.desc, fq[i], r.view)
        if i % len(FILTERS) != 0:
            plain = oracle_lib.OracleResult(tt1.desc, qs.arr[i])
            changed += records(plain.view) != r.records()
    assert legs > 50
    assert changed > 5  # the filters bite on this timetable


# ------------------------------------------------------------------ GPU

@pytest.fixture(scope="module")
def engines():
    from nigiri_b200 import routing as R
    out = {}
    for w in (1, 2):
        h = HostTimetable.generate(w)
        dtt = R.Timetable(h.desc, owner=h)
        out[w] = (h, dtt, R.Engine(dtt, max_slots=256))
    return out


def batch(eng, qarr, n):
    out = (A.Result * n)()
    assert A.lib().b2r_search_batch(eng.handle, qarr, n, out) == 0, A.lib().b2r_last_error()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("workload,qkind,n", [(1, 1, 140), (2, 2, 70), (2, 3, 42)],
                         ids=["w1_fwd_bwd", "w2_intermodal", "w2_range"])
def test_filtered_searches_match_oracle(engines, workload, qkind, n):
    h, _, eng = engines[workload]
    qs = QuerySet(h, qkind, n, seed=900 + qkind)
    fq = filtered(qs)
    out = batch(eng, fq, qs.n)
    for i in range(qs.n):
        exp = oracle_lib.OracleResult(h.desc, fq[i])
        assert records(out[i]) == exp.records(), i


@pytest.mark.gpu
def test_filtered_one_to_all_rows_match_oracle(engines):
    h, _, eng = engines[2]
    qs = QuerySet(h, 1, 14, seed=77)
    fq = filtered(qs, kind=A.B2R_ONE_TO_ALL)
    for i in range(qs.n):
        fq[i].n_destination = 0
        fq[i].direction = i % 2
    out = batch(eng, fq, qs.n)
    n = h.desc.n_locations
    for i in range(qs.n):
        r = out[i]
        rows = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n,)).reshape(r.n_rows, n)
        orows, _, base_day = oracle_lib.OracleResult(h.desc, fq[i]).state()
        assert r.base_day == base_day
        assert np.array_equal(rows, orows[: r.n_rows]), i
