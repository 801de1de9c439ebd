"""The GTFS reader (b2r_tt_load_gtfs) on the feeds of nigiri's routing tests:
the timetables it builds give the golden journeys and known answers of
those tests (through the oracle on the CPU, through the engine on the
GPU), and match the timetables restated by hand for them."""
import ctypes as C

import numpy as np
import pytest

import fixture as F
import oracle_lib
from nigiri_b200 import _abi as A

CASES = F.load_cases()
FEEDS = sorted(CASES["gtfs_feeds"])
RESTATED = [f for f in FEEDS if f in CASES["timetables"]]
ALL_CASES = [c for c in CASES["cases"] if c["timetable"] in CASES["gtfs_feeds"]] + CASES["gtfs_cases"]


@pytest.fixture(scope="module")
def loaded():
    return {name: F.GtfsFixture(name, A.lib()) for name in FEEDS}


def routes_of(tt):
    """(stop ids, class, section flags, [(transport name, UTC days, times)])
    per route, independent of route and bitfield numbering."""
    d = tt.desc
    nr, nt = d.n_routes, d.n_transports
    arr = lambda p, n, dt: np.ctypeslib.as_array(p, shape=(n,)).astype(dt).copy() if n else np.zeros(0, dt)
    rsi = arr(d.route_stop_index, nr + 1, np.int64)
    stops = arr(d.route_stops, int(rsi[-1]), np.int64)
    tf = arr(d.route_transport_from, nr, np.int64)
    tto = arr(d.route_transport_to, nr, np.int64)
    sf = arr(d.route_stop_time_from, nr, np.int64)
    st = arr(d.route_stop_times, d.n_route_stop_times, np.int64)
    tbf = arr(d.transport_traffic_days, nt, np.int64)
    bfs = arr(d.bitfields, 8 * d.n_bitfields, np.uint64).reshape(-1, 8) if d.n_bitfields else None
    clasz = arr(d.route_clasz, nr, np.int64)
    sec = arr(d.route_section_flags, int(rsi[-1]), np.int64) if d.route_section_flags else np.zeros(int(rsi[-1]), np.int64)
    out = []
    for r in range(nr):
        n = rsi[r + 1] - rsi[r]
        n_t = tto[r] - tf[r]
        names = tuple(tt.loc_name[int(w) & 0x0FFFFFFF] for w in stops[rsi[r]:rsi[r + 1]])
        flags = tuple(int(w) >> 28 for w in stops[rsi[r]:rsi[r + 1]])
        trs = []
        for x in range(n_t):
            t = tf[r] + x
            days = tuple(int(i) for i in range(512)
                         if (int(bfs[tbf[t]][i // 64]) >> (i % 64)) & 1)
            times = tuple(int(st[sf[r] + slot * n_t + x]) for slot in range(2 * (n - 1)))
            trs.append((tt.transport_names[t], days, times))
        out.append((names, flags, int(clasz[r]), tuple(int(x) for x in sec[rsi[r]:rsi[r + 1] - 1]), tuple(trs)))
    return sorted(out)


@pytest.mark.parametrize("name", RESTATED)
def test_reader_rebuilds_the_restated_timetable(name, loaded):
    """Same routes (stops, pickup / drop-off flags, class, section flags),
    same transports (names, UTC traffic days, UTC times) and the same
    footpaths, transfer times and parents as the hand-restated fixture."""
    got = loaded[name]
    want = F.FixtureTimetable(CASES["timetables"][name], A.lib())
    # traffic days are bits of the same internal interval in both
    assert routes_of(got) == routes_of(want)

    def locs(tt):
        d = tt.desc
        n = d.n_locations
        tr = np.ctypeslib.as_array(d.transfer_time, shape=(n,))
        par = np.ctypeslib.as_array(d.parent, shape=(n,)) if d.parent else np.full(n, 0xFFFFFFFF)
        fi = np.ctypeslib.as_array(d.footpaths_out_index, shape=(n + 1,))
        fo = np.ctypeslib.as_array(d.footpaths_out, shape=(int(fi[-1]),)) if fi[-1] else []
        out = {}
        for l in range(9, n):
            fps = sorted((tt.loc_name[int(w) & 0x7FFFFF], int(w) >> 23) for w in fo[fi[l]:fi[l + 1]])
            p = int(par[l])
            out[tt.loc_name[l]] = (int(tr[l]), None if p == 0xFFFFFFFF else tt.loc_name[p], tuple(fps))
        return out
    assert locs(got) == locs(want)


@pytest.mark.parametrize("case", ALL_CASES, ids=lambda c: c["name"])
def test_golden_cases_on_read_feeds(case, loaded):
    tt = loaded[case["timetable"]]
    q = F.FixtureQuery(A.lib(), tt, case["query"])
    r = oracle_lib.OracleResult(tt.desc, q.q)
    assert F.journeys_to_records(tt, r.view) == F.strip_expected(case["expected"])


@pytest.mark.parametrize("algo", ["raptor", "pong"])
@pytest.mark.parametrize("ka", CASES["gtfs_known_answers"], ids=lambda k: k["name"])
def test_known_answers_on_read_feeds(ka, algo, loaded):
    tt = loaded[ka["timetable"]]
    q = F.FixtureQuery(A.lib(), tt, dict(ka["query"], algorithm=algo))
    r = oracle_lib.OracleResult(tt.desc, q.q)
    got = [[j["dep"], j["arr"], j["transfers"]] for j in F.journeys_to_records(tt, r.view)]
    assert ka["contains"] in got, got


@pytest.mark.parametrize("case", CASES["gtfs_cases"], ids=lambda c: c["name"])
def test_pong_on_read_feeds_in_window(case, loaded):
    """The harness check of test/raptor_search.cc for the feed-only cases."""
    tt = loaded[case["timetable"]]
    qd = dict(case["query"], algorithm="pong")
    r = oracle_lib.OracleResult(tt.desc, F.FixtureQuery(A.lib(), tt, qd).q)
    got = F.journeys_to_records(tt, r.view)
    assert F.in_window(qd, got) == F.in_window(qd, F.strip_expected(case["expected"]))


@pytest.mark.parametrize("case", CASES["gtfs_seated_cases"], ids=lambda c: c["name"])
def test_stay_seated_known_answers(case, loaded):
    """join_split.complex (test/routing/join_split_test.cc): between stops
    reached only over stay-seated transfers there are journeys, and none
    has a transfer, in both trip orders of the feed."""
    tt = loaded[case["timetable"]]
    r = oracle_lib.OracleResult(tt.desc, F.FixtureQuery(A.lib(), tt, case["query"]).q)
    got = F.journeys_to_records(tt, r.view)
    assert (len(got) > 0) == case["nonempty"]
    assert all(j["transfers"] <= case["max_transfers_seen"] for j in got)


def transports_by_days(tt):
    """(stop names, first trip's route, UTC traffic dates) per transport."""
    import datetime
    d = tt.desc
    rsi = np.ctypeslib.as_array(d.route_stop_index, shape=(d.n_routes + 1,))
    rs = np.ctypeslib.as_array(d.route_stops, shape=(int(rsi[-1]),))
    tf = np.ctypeslib.as_array(d.route_transport_from, shape=(d.n_routes,))
    tto = np.ctypeslib.as_array(d.route_transport_to, shape=(d.n_routes,))
    tbf = np.ctypeslib.as_array(d.transport_traffic_days, shape=(d.n_transports,))
    bfs = np.ctypeslib.as_array(d.bitfields, shape=(8 * d.n_bitfields,)).reshape(-1, 8)
    base = datetime.date(1970, 1, 1) + datetime.timedelta(days=d.date_range_from - 5)
    out = []
    for r in range(d.n_routes):
        names = "-".join(tt.loc_name[int(w) & 0x0FFFFFFF] for w in rs[rsi[r]:rsi[r + 1]])
        for t in range(int(tf[r]), int(tto[r])):
            days = tuple((base + datetime.timedelta(days=i)).day for i in range(512)
                         if (int(bfs[tbf[t]][i // 64]) >> (i % 64)) & 1)
            out.append((names, tt.transport_names[t], days))
    return sorted(out)


@pytest.mark.parametrize("name", ["gtfs_join_split", "gtfs_join_split_rev"])
def test_stay_seated_transports(name, loaded):
    """The transports of join_split.complex's day table (UTC first-departure
    days in June 2025): i and k (01:00 local, days 11, 12, 16-19) continue
    seated into x (12-14, 19, 21; x1 replaces it on 20) and on into j and l
    (13-15, 17, 20, 21) where those run; the rest runs alone.  Per trip the
    days of the transports holding it add up to the test's transportsXDays
    (i 6, k 6, x 5, x1 1, j 6, l 6 = 30)."""
    want = []
    for first, a, c in (("i", "A", "C1"), ("k", "B", "C2")):
        want += [(f"{a}-{c}", first, (16, 17)), (f"{a}-{c}-D", first, (11, 18)),
                 (f"{a}-{c}-D-E", first, (12,)), (f"{a}-{c}-D-E", first, (19,)),
                 (f"{a}-{c}-D-F", first, (12,)), (f"{a}-{c}-D-F", first, (19,))]
    want += [("C-D-E", "x", (14, 21)), ("C-D-F", "x", (14, 21)), ("D1-E", "j", (15, 17)), ("D2-F", "l", (15, 17))]
    assert transports_by_days(loaded[name]) == sorted(want)


def test_python_reader_reads_a_feed_directory(tmp_path):
    """HostTimetable.load_gtfs on a directory of files (the clasz test's
    feed written out), with the stop ids and names it keeps."""
    from nigiri_b200.timetable import HostTimetable
    text = CASES["gtfs_feeds"]["gtfs_clasz"]["text"]
    name = None
    for line in text.splitlines():
        if line.startswith("# "):
            name = line[2:].strip()
            (tmp_path / name).write_text("")
        elif name:
            with open(tmp_path / name, "a") as f:
                f.write(line + "\n")
    spec = CASES["timetables"]["gtfs_clasz"]
    h = HostTimetable.load_gtfs(str(tmp_path), tuple(F._day(x) for x in spec["date_range"]))
    ids = [h.location_id(l) for l in range(h.desc.n_locations)]
    assert ids[9:] == ["A", "B", "C"]
    assert sorted(h.transport_name(t) for t in range(h.desc.n_transports)) == ["1", "2", "X"]


def test_reader_rejects_missing_time_zone():
    cfg = A.GtfsConfig()
    A.lib().b2r_gtfs_config_init(C.byref(cfg))
    cfg.date_range_from, cfg.date_range_to = 19000, 19002
    h = C.c_void_p()
    text = b"# stops.txt\nstop_id,stop_name\nA,A\n"
    assert A.lib().b2r_tt_load_gtfs(text, 1, C.byref(cfg), C.byref(h)) == A.B2R_ERR_INVALID_ARGUMENT
    assert b"time zone" in A.lib().b2r_last_error()


@pytest.mark.gpu
def test_golden_cases_on_read_feeds_gpu(loaded):
    """Feed text -> reader -> device image -> engine: the golden journeys."""
    from nigiri_b200 import routing as R
    for name in FEEDS:
        tt = loaded[name]
        dtt = R.Timetable(tt.desc, owner=tt)
        eng = R.Engine(dtt, max_slots=32)
        for c in ALL_CASES:
            if c["timetable"] != name:
                continue
            q = F.FixtureQuery(A.lib(), tt, c["query"])
            res = A.Result()
            assert A.lib().b2r_search_batch(eng.handle, C.byref(q.q), 1, C.byref(res)) == 0
            assert F.journeys_to_records(tt, res) == F.strip_expected(c["expected"]), c["name"]
        for c in CASES["gtfs_seated_cases"]:
            if c["timetable"] != name:
                continue
            q = F.FixtureQuery(A.lib(), tt, c["query"])
            res = A.Result()
            assert A.lib().b2r_search_batch(eng.handle, C.byref(q.q), 1, C.byref(res)) == 0
            exp = oracle_lib.OracleResult(tt.desc, q.q)
            assert F.journeys_to_records(tt, res) == F.journeys_to_records(tt, exp.view), c["name"]
            assert (res.n_journeys > 0) == c["nonempty"], c["name"]
        for ka in CASES["gtfs_known_answers"]:
            if ka["timetable"] != name:
                continue
            for algo in ("raptor", "pong"):
                q = F.FixtureQuery(A.lib(), tt, dict(ka["query"], algorithm=algo))
                res = A.Result()
                assert A.lib().b2r_search_batch(eng.handle, C.byref(q.q), 1, C.byref(res)) == 0
                assert res.status == 0, (ka["name"], algo)
                got = [[j["dep"], j["arr"], j["transfers"]] for j in F.journeys_to_records(tt, res)]
                assert ka["contains"] in got, (ka["name"], algo, got)
