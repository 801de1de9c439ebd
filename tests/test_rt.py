"""The real-time overlay (rt_timetable): routing with delayed, cancelled and
added runs as raptor<Dir, Rt = true> does (raptor.h:228-241, 577-678,
1068-1175; start_times.cc:177-215; reconstruct.cc:381-452).

CPU: the oracle's Rt restatement gives the golden journeys of nigiri's
test/routing/rt_routing_test.cc on the feed the GTFS reader builds, with the
update each test applies restated as the overlay it leaves.  GPU: the engine
bound to the overlay gives the same golden journeys, and on generated
timetables with generated overlays (delays from a stop on, cancellations,
added runs) the same answers as the oracle for one-to-one, range and
one-to-all queries in both directions."""
import ctypes as C
import random

import numpy as np
import pytest

import fixture as F
import oracle_lib
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

CASES = F.load_cases()
RT_CASES = CASES["rt_cases"]


@pytest.fixture(scope="module")
def feed():
    return F.GtfsFixture("gtfs_rt_routing", A.lib())


@pytest.mark.parametrize("case", RT_CASES, ids=lambda c: c["name"])
def test_oracle_rt_golden_journeys(case, feed):
    ov = F.rt_overlay_of_case(feed, case["rt"])
    q = F.FixtureQuery(A.lib(), feed, case["query"])
    r = oracle_lib.OracleResult(feed.desc, q.q, ov.desc)
    assert F.journeys_to_records(feed, r.view) == F.strip_expected(case["expected"])


def test_oracle_without_the_overlay_misses_the_delayed_connection(feed):
    """Without the update, RE 2 has left B before RE 1 arrives: the golden
    connection exists only in real time."""
    case = RT_CASES[0]
    q = F.FixtureQuery(A.lib(), feed, case["query"])
    r = oracle_lib.OracleResult(feed.desc, q.q)
    assert F.journeys_to_records(feed, r.view) != F.strip_expected(case["expected"])


def query_days(h, qs):
    """The traffic day indices around the queries' start times."""
    first = h.desc.date_range_from - 5
    out = set()
    for i in range(qs.n):
        q = qs.arr[i]
        t = q.interval_from if q.is_interval else q.start_time
        d = t // 1440 - first
        out.update((d - 1, d))
    return sorted(x for x in out if 0 <= x < 512)


def ridden_trips(answers):
    """(transport, traffic day) of the static rides in oracle answers."""
    out = []
    for kind, recs in answers.values():
        if kind != "journeys":
            continue
        for j in recs:
            for leg in j["legs"]:
                if leg[0] == A.B2R_LEG_TRANSPORT and leg[-1] == 0xFFFFFFFF:
                    out.append((leg[5], leg[6]))
    return sorted(set(out))


def generated_overlay(h, seed, days_near, focus=(), n_delayed=600, n_cancelled=200, n_added=600):
    """A real-time state on a generated timetable: runs delayed from some
    stop on (later, never faster), runs cancelled, and added runs that copy
    a trip's times shifted later, all on traffic days in `days_near`.  The
    delayed and cancelled trips leave the static schedule on their day.
    The trips in `focus` ((transport, day) pairs, e.g. the ones the static
    answers ride) are changed first."""
    rnd = random.Random(seed)
    near = set(days_near)
    focus = list(focus)
    d = h.desc
    first = d.date_range_from - 5
    nr = d.n_routes
    rsi = np.ctypeslib.as_array(d.route_stop_index, shape=(nr + 1,))
    rstops = np.ctypeslib.as_array(d.route_stops, shape=(int(rsi[-1]),))
    tfrom = np.ctypeslib.as_array(d.route_transport_from, shape=(nr,))
    tto = np.ctypeslib.as_array(d.route_transport_to, shape=(nr,))
    sfrom = np.ctypeslib.as_array(d.route_stop_time_from, shape=(nr,))
    st = np.ctypeslib.as_array(d.route_stop_times, shape=(d.n_route_stop_times,))
    changed, runs, used = {}, [], set()

    def active_day(t):
        words = F.transport_days(d, t)
        days = [x for x in range(512) if (words[x // 64] >> (x % 64)) & 1]
        return words, days

    def trip_times(r, t, day):  # rt_transport_stop_times_ order, minutes since the epoch
        n_s = int(rsi[r + 1] - rsi[r])
        n_t = int(tto[r] - tfrom[r])
        out = []
        for s in range(n_s):
            for arr in ((True,) if s == n_s - 1 else ((False,) if s == 0 else (True, False))):
                slot = 2 * s - (1 if arr else 0)
                ev = int(st[int(sfrom[r]) + n_t * slot + (t - int(tfrom[r]))])
                out.append((first + day) * 1440 + (ev & 31) * 1440 + (ev >> 5))
        return out

    wanted = n_delayed + n_cancelled + n_added
    for _ in range(200 * wanted):  # bounded: a timetable may have few such trips
        if len(runs) + len(changed) >= wanted:
            break
        if focus:
            t, day = focus.pop(0)
            r = int(d.transport_route[t])
            words, days = active_day(t)
            if t in used or day not in days:
                continue
        else:
            r = rnd.randrange(nr)
            if tto[r] == tfrom[r]:
                continue
            t = rnd.randrange(int(tfrom[r]), int(tto[r]))
            words, days = active_day(t)
            days = [x for x in days if x in near]
            if not days or t in used:
                continue
            day = rnd.choice(days)
        stops = [int(x) for x in rstops[int(rsi[r]):int(rsi[r + 1])]]
        times = trip_times(r, t, day)
        kind = rnd.randrange(3)
        if kind < 2:  # delayed or cancelled: the trip leaves the schedule on that day
            used.add(t)
            words = list(words)
            words[day // 64] &= ~(1 << (day % 64))
            changed[t] = words
            if kind == 0:
                k = rnd.randrange(1, len(times) + 1)
                delay = rnd.randint(1, 40)
                times = times[:len(times) - k] + [x + delay for x in times[len(times) - k:]]
                runs.append(dict(stops=stops, times=times, static_transport=t, static_day=day,
                                 clasz=int(d.route_clasz[r]) if d.route_clasz else 10))
        else:  # an added run: the trip's times a few minutes later
            shift = rnd.randint(1, 30)
            runs.append(dict(stops=[F.stop_word(x & 0x0FFFFFFF) for x in stops],
                             times=[x + shift for x in times],
                             clasz=int(d.route_clasz[r]) if d.route_clasz else 10))
    return F.RtOverlay(sorted(changed.items()), runs)


def test_oracle_rides_generated_real_time_runs():
    """The generated overlay is ridden: on the city timetable some of the
    oracle's journeys use real-time runs, and some answers change."""
    h = HostTimetable.generate(1)
    qs = QuerySet(h, 1, 60, seed=7001)
    static = oracle_lib.answers(h.desc, qs.arr, range(qs.n))
    ov = generated_overlay(h, 71, query_days(h, qs), focus=ridden_trips(static))
    assert ov.desc.n_rt_transports >= 30 and ov.desc.n_changed >= 30
    with_rt = oracle_lib.answers(h.desc, qs.arr, range(qs.n), rt=ov.desc)
    rt_legs = sum(1 for i in range(qs.n) for j in with_rt[i][1] for leg in j["legs"]
                  if leg[0] == A.B2R_LEG_TRANSPORT and leg[-1] != 0xFFFFFFFF)
    assert rt_legs > 0
    assert any(with_rt[i] != static[i] for i in range(qs.n))


def bound_engine(desc, ov, max_slots=256):
    lib = A.lib()
    tt = R.Timetable(desc, owner=None)
    eng = R.Engine(tt, max_slots=max_slots)
    rt = C.c_void_p()
    assert lib.b2r_rt_upload(tt.handle, C.byref(ov.desc), C.byref(rt)) == 0, lib.b2r_last_error()
    assert lib.b2r_engine_set_rt(eng.handle, rt) == 0, lib.b2r_last_error()
    return tt, eng, rt


@pytest.mark.gpu
@pytest.mark.parametrize("case", RT_CASES, ids=lambda c: c["name"])
def test_engine_rt_golden_journeys(case, feed):
    lib = A.lib()
    ov = F.rt_overlay_of_case(feed, case["rt"])
    tt, eng, rt = bound_engine(feed.desc, ov, max_slots=32)
    q = F.FixtureQuery(lib, feed, case["query"])
    res = A.Result()
    assert lib.b2r_search_batch(eng.handle, C.byref(q.q), 1, C.byref(res)) == 0, lib.b2r_last_error()
    assert F.journeys_to_records(feed, res) == F.strip_expected(case["expected"])
    # the same engine without the overlay: the static answer again
    assert lib.b2r_engine_set_rt(eng.handle, None) == 0
    res2 = A.Result()
    assert lib.b2r_search_batch(eng.handle, C.byref(q.q), 1, C.byref(res2)) == 0
    want = oracle_lib.OracleResult(feed.desc, q.q).records()
    assert records(res2) == want
    del eng
    lib.b2r_rt_destroy(rt)


@pytest.mark.gpu
@pytest.mark.parametrize("workload,n", [(1, 120), (2, 48), (3, 24)])
def test_engine_rt_generated_matches_oracle(workload, n):
    """Generated overlay on the city / regional timetable: one-to-one
    (intermodal on the regional one), range queries of both directions, and
    one-to-all rows."""
    lib = A.lib()
    h = HostTimetable.generate(1 if workload == 1 else 2)
    qs = QuerySet(h, workload, n, seed=7000 + workload)
    static = oracle_lib.answers(h.desc, qs.arr, range(qs.n))
    ov = generated_overlay(h, 70 + workload, query_days(h, qs), focus=ridden_trips(static))
    tt, eng, rt = bound_engine(h.desc, ov)
    arr = (A.Query * (qs.n + 8))()
    for i in range(qs.n):
        arr[i] = qs.arr[i]
    for i in range(8):  # one-to-all, both directions
        arr[qs.n + i] = qs.arr[i]
        arr[qs.n + i].kind = A.B2R_ONE_TO_ALL
        arr[qs.n + i].n_destination = 0
        arr[qs.n + i].is_interval = 0
        arr[qs.n + i].direction = i % 2
    n_all = qs.n + 8
    out = (A.Result * n_all)()
    assert lib.b2r_search_batch(eng.handle, arr, n_all, out) == 0, lib.b2r_last_error()
    want = oracle_lib.answers(h.desc, arr, range(n_all), rt=ov.desc)
    n_loc = h.desc.n_locations
    n_rt_legs, bad = 0, []
    for i in range(n_all):
        r = out[i]
        w = want[i]
        if w[0] == "rows":
            got = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n_loc,)).reshape(r.n_rows, n_loc)
            ok = r.base_day == w[1] and np.array_equal(got, w[2][: r.n_rows])
        else:
            got = records(r)
            ok = r.status == 0 and got == w[1]
            n_rt_legs += sum(1 for j in got for leg in j["legs"] if leg[0] == A.B2R_LEG_TRANSPORT
                             and leg[-1] != 0xFFFFFFFF)
        if not ok:
            bad.append(i)
    assert bad == [], f"{len(bad)} queries differ, first {bad[:5]}"
    assert n_rt_legs > 0  # real-time runs are ridden
    del eng
    lib.b2r_rt_destroy(rt)
