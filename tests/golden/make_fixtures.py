"""Builds tests/golden/cases.json from nigiri's own routing tests.

Run in a checkout that has the nigiri sources (pass their root as argv[1]);
the output is committed so the test suite never reads the reference at run
time.

Two kinds of content end up in cases.json:
  * timetables: the reference tests' tiny GTFS / HRD fixtures, restated by
    hand as UTC event times (the conversion is written next to each one);
  * expected results: the golden journey printouts (`R"(...)"` strings) of
    the reference tests, parsed mechanically from the test sources into
    (departure, arrival, transfers, legs) records.
"""
from __future__ import annotations

import datetime as dt
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def day(s: str) -> int:
    return (dt.date.fromisoformat(s) - dt.date(1970, 1, 1)).days


def hm(s: str) -> int:
    h, m = s.split(":")[:2]
    return int(h) * 60 + int(m)


# ----------------------------------------------------------------------------
# Timetables (stop ids / names as printed by the reference tests).
# Route entries: {"stops": [id,...], "transports": [{"name", "day", "times"}]}
# where times = [dep(0), arr(1), dep(1), ..., arr(n-1)] in UTC minutes after
# midnight of `day` (may exceed 1440), i.e. nigiri's per-transport delta times
# relative to the UTC traffic day.
# ----------------------------------------------------------------------------

def get_index(route, svc):
    """Position at which `svc` may join `route` (a list of services sorted
    by minutes after midnight), or None -- nigiri's FIFO rule on times
    modulo 1440 at every stop (include/nigiri/loader/get_index.h:8-29)."""
    key = svc["times"][0] % 1440
    index = 0
    while index < len(route) and route[index]["times"][0] % 1440 < key:
        index += 1
    for i, x in enumerate(svc["times"]):
        earlier = index > 0 and x % 1440 < route[index - 1]["times"][i] % 1440
        later = index < len(route) and x % 1440 > route[index]["times"][i] % 1440
        if earlier or later:
            return None
    return index


def group_routes(services):
    """Services (in load order) -> routes: one route key per (stop sequence,
    transport class, per-section flags), split into sub-routes by get_index
    (gtfs/load_timetable.cc:277-309)."""
    keys = {}
    order = []
    for svc in services:
        k = (tuple(svc["stops"]), svc.get("clasz", 10),
             tuple(svc.get("sections", [0] * (len(svc["stops"]) - 1))),
             tuple(tuple(x) for x in svc.get("wc", ())))
        if k not in keys:
            keys[k] = [[svc]]
            order.append(k)
            continue
        for sub in keys[k]:
            idx = get_index(sub, svc)
            if idx is not None:
                sub.insert(idx, svc)
                break
        else:
            keys[k].append([svc])
    routes = []
    for k in order:
        for sub in keys[k]:
            route = {"stops": list(k[0]), "clasz": k[1], "sections": list(k[2]),
                     "transports": [
                         {kk: v for kk, v in x.items()
                          if kk not in ("stops", "clasz", "sections", "wc")} for x in sub]}
            if k[3]:
                route["stop_wc"] = [list(x) for x in k[3]]
            routes.append(route)
    return routes


def utc_service(name, stops, first_day, times):
    """Normalise a service whose UTC times are given relative to
    `first_day`: the first departure is moved below 24:00 and the traffic
    day shifted accordingly (README.md: first departures < 24:00)."""
    shift = times[0] // 1440
    d = dt.date.fromisoformat(first_day) + dt.timedelta(days=shift)
    return {"name": name, "stops": stops, "day": d.isoformat(),
            "times": [x - 1440 * shift for x in times]}


def hrd_abc():
    """test/loader/hrd/hrd_timetable.h files_abc(): two HRD services on
    30.03.2020 (bitfield 000005), local time UTC+2 (DST since 29.03 02:00):
      RE 1337 A 02:30 -> B 03:30, repeated 48 times every 30 min
      RE 7331 B 02:30 -> C 03:30, repeated 92 times every 15 min
    -> UTC: departures 00:30 + j*30 min (j = 0..48) and 00:30 + j*15 min
    (j = 0..92) after 2020-03-30 00:00, each run 60 min."""
    locs = [("0000001", "A"), ("0000002", "B"), ("0000003", "C"),
            ("0000004", "D"), ("0000005", "E"), ("0000006", "F"),
            ("0000007", "G"), ("0000008", "H"), ("0000009", "I"),
            ("0000010", "F_META")]
    services = []
    for j in range(49):
        dep = 30 + 30 * j
        services.append(utc_service("RE 1337", ["0000001", "0000002"], "2020-03-30",
                                    [dep, dep + 60]))
    for j in range(93):
        dep = 30 + 15 * j
        services.append(utc_service("RE 7331", ["0000002", "0000003"], "2020-03-30",
                                    [dep, dep + 60]))
    return {
        "date_range": ["2020-03-28", "2020-03-31"],
        "locations": [{"id": i, "name": n, "transfer_time": 2} for i, n in locs],
        "footpaths": [],
        "routes": group_routes(services),
    }


def gtfs_transfer_time():
    """test/routing/transfer_time_settings_test.cc test_files: agency
    Europe/Berlin (UTC+2 on 2019-05-01), service S1 on 2019-05-01 only.
      T1 (route 1) A 10:00 -> B 10:10      UTC 08:00 -> 08:10
      T2 (route 2) B 10:13 -> C 10:22      UTC 08:13 -> 08:22
      T3 (route 2) B 10:20 -> C 10:30      UTC 08:20 -> 08:30
      T4 (route 3) A 09:55 -> C 10:35      UTC 07:55 -> 08:35
    Stops are ~300 km apart: no footpaths; transfer time 2 min (GTFS
    loader default).  Printed trip names are the route short names."""
    d = "2019-05-01"
    services = [
        dict(utc_service("1", ["A", "B"], d, [hm("08:00"), hm("08:10")]), id="T1"),
        dict(utc_service("2", ["B", "C"], d, [hm("08:13"), hm("08:22")]), id="T2"),
        dict(utc_service("2", ["B", "C"], d, [hm("08:20"), hm("08:30")]), id="T3"),
        dict(utc_service("3", ["A", "C"], d, [hm("07:55"), hm("08:35")]), id="T4"),
    ]
    return {
        "date_range": ["2019-05-01", "2019-05-02"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in "ABC"],
        "footpaths": [],
        "routes": group_routes(services),
    }


def hrd_simple():
    """test/loader/hrd/hrd_timetable.h files_simple(): like files_abc() but
    the second service runs back from B to A:
      RE 1337 A 02:30 -> B 03:30, repeated 48 times every 30 min
      RE 7331 B 02:30 -> A 03:30, repeated 92 times every 15 min
    on 30.03.2020, local time UTC+2 -> UTC departures 00:30 + j*30 / j*15."""
    locs = [("0000001", "A"), ("0000002", "B"), ("0000003", "C"),
            ("0000004", "D"), ("0000005", "E"), ("0000006", "F"),
            ("0000007", "G"), ("0000008", "H"), ("0000009", "I"),
            ("0000010", "F_META")]
    services = []
    for j in range(49):
        dep = 30 + 30 * j
        services.append(utc_service("RE 1337", ["0000001", "0000002"], "2020-03-30",
                                    [dep, dep + 60]))
    for j in range(93):
        dep = 30 + 15 * j
        services.append(utc_service("RE 7331", ["0000002", "0000001"], "2020-03-30",
                                    [dep, dep + 60]))
    return {
        "date_range": ["2020-03-28", "2020-03-31"],
        "locations": [{"id": i, "name": n, "transfer_time": 2} for i, n in locs],
        "footpaths": [],
        "routes": group_routes(services),
    }


def gtfs_dijkstra():
    """test/routing/dijkstra_test.cc dijkstra_files(): agency Europe/Berlin
    (UTC+2 on 2024-06-08), service S on 2024-06-08 only.  C1, C2 are children
    of C and D1, D2 children of station D; transfers.txt (type 2) gives
    footpaths D1 <-> D2 of 600 s and C1 <-> C2 of 900 s.  The stop reader
    links each stop with its parent and the parent's children (stop.cc
    get_metas; no coordinates, so distance 0 and 2-minute walks, the existing
    10 and 15 minutes kept), and finalize()'s footpath closure
    (build_footpaths.cc:229-345) shortens the sibling walks to 4 minutes over
    the parent.
      AB_TRP A 09:00 -> B 09:30     UTC 07:00 -> 07:30
      BC_TRP B 10:00 -> C2 11:00    UTC 08:00 -> 09:00
      DB_TRP D1 09:30 -> B 09:45    UTC 07:30 -> 07:45
      DC_TRP D2 10:30 -> C1 11:30   UTC 08:30 -> 09:30
    Route type 0: kTram (9)."""
    d = "2024-06-08"
    services = [
        dict(utc_service("AB", ["A", "B"], d, [hm("07:00"), hm("07:30")]), id="AB_TRP", clasz=9),
        dict(utc_service("BC", ["B", "C2"], d, [hm("08:00"), hm("09:00")]), id="BC_TRP", clasz=9),
        dict(utc_service("DB", ["D1", "B"], d, [hm("07:30"), hm("07:45")]), id="DB_TRP", clasz=9),
        dict(utc_service("DC", ["D2", "C1"], d, [hm("08:30"), hm("09:30")]), id="DC_TRP", clasz=9),
    ]
    parents = {"C1": "C", "C2": "C", "D1": "D", "D2": "D"}
    return {
        "date_range": ["2024-06-07", "2024-06-09"],
        "locations": [{"id": x, "name": x, "transfer_time": 2, "parent": parents.get(x)}
                      for x in ["A", "B", "C", "C1", "C2", "D", "D1", "D2"]],
        "footpaths": [[a, b, w] for p, (x, y) in (("C", ("C1", "C2")), ("D", ("D1", "D2")))
                      for a, b, w in ((p, x, 2), (p, y, 2), (x, p, 2), (y, p, 2), (x, y, 4), (y, x, 4))],
        "routes": group_routes(services),
    }


def gtfs_clasz():
    """test/routing/clasz_filter_test.cc test_files: agency Europe/Berlin
    (UTC+1 on 2024-03-01), service S1 on 2024-03-01 only.  GTFS route types
    give the classes (src/loader/gtfs/route.cc:22-45, 105): 1100 -> kAir (0),
    3 -> kBus (10), 2 -> kRegional (6).
      AIR (route X, air)  A 10:00 -> C 11:00   UTC 09:00 -> 10:00
      T1  (route 1, bus)  A 10:00 -> B 10:55   UTC 09:00 -> 09:55
      T2  (route 2, rail) B 11:05 -> C 12:00   UTC 10:05 -> 11:00
    Stops are far apart: no footpaths, transfer time 2 min."""
    d = "2024-03-01"
    services = [
        dict(utc_service("X", ["A", "C"], d, [hm("09:00"), hm("10:00")]), id="AIR", clasz=0),
        dict(utc_service("1", ["A", "B"], d, [hm("09:00"), hm("09:55")]), id="T1", clasz=10),
        dict(utc_service("2", ["B", "C"], d, [hm("10:05"), hm("11:00")]), id="T2", clasz=6),
    ]
    return {
        "date_range": ["2024-03-01", "2024-03-02"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in "ABC"],
        "footpaths": [],
        "routes": group_routes(services),
    }


# Route flag bits (include/nigiri/types.h:417-423).
FLAG_BIKES, FLAG_RESERVATION_NOT_REQUIRED = 0, 3


def flag_service(name, stops, times, sections, flag):
    """A service of 2019-05-01 (UTC times) whose section s carries `flag`
    when sections[s] is true."""
    return dict(utc_service(name, stops, "2019-05-01", [hm(x) for x in times]), clasz=10,
                sections=[(1 << flag) if x else 0 for x in sections])


def gtfs_flags_1(flag):
    """Timetable 1 of test/routing/bike_transport_test.cc and of
    test/routing/no_compulsory_reservation_test.cc (same stops and times;
    the flag is bikes_allowed = 1, resp. pickup_type != 2, per trip --
    src/loader/gtfs/trip.cc:296-316).  Europe/Berlin, UTC+2 on 2019-05-01:
      T0 (route 0) A 08:00 - B 08:10 - C 08:20            no flag
      T1 (route 1) A 08:00 - B 08:15 - C 08:30            flag
      T2 (route 1) A 09:00 - B 09:15 - C 09:30            no flag
    Block 1 holds T3 (route 2, C 08:35 - D 08:40, flag), T5 (route 3,
    D 08:42 - E 08:50 - F 08:55, no flag), T4 (route 2, C 08:45 - D 08:50,
    flag) and T6 (route 3, D 08:52 - E 09:00 - F 09:05, flag).  The block's
    rule services (block::rule_services, src/loader/gtfs/trip.cc:31-106)
    chain trips whose first stop is the last stop of the one before: T3>T5
    and T4>T6, each one transport over C-D-E-F with per-section flags
    [1, 0, 0] and [1, 1, 1].  The route key includes the flags, so T0 / T2
    share a route, T1 has its own, and so has each chained transport.
    Printed names are the route short names of the first trip."""
    services = [
        flag_service("0", list("ABC"), ["08:00", "08:10", "08:10", "08:20"], [0, 0], flag),
        flag_service("1", list("ABC"), ["08:00", "08:15", "08:15", "08:30"], [1, 1], flag),
        flag_service("1", list("ABC"), ["09:00", "09:15", "09:15", "09:30"], [0, 0], flag),
        flag_service("2", list("CDEF"), ["08:35", "08:40", "08:42", "08:50", "08:50", "08:55"],
                     [1, 0, 0], flag),
        flag_service("2", list("CDEF"), ["08:45", "08:50", "08:52", "09:00", "09:00", "09:05"],
                     [1, 1, 1], flag),
    ]
    return {
        "date_range": ["2019-05-01", "2019-05-02"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in "ABCDEF"],
        "footpaths": [],
        "routes": group_routes(services),
    }


def gtfs_flags_2(flag):
    """Timetable 2 of the same two tests: blocks T1>T2 and T3>T4, the flag on
    every trip but T1 (UTC):
      T1>T2 (route 1) A 08:00 - B 08:10/08:15 - C 08:20 - D 08:25  [0, 1, 1]
      T3>T4 (route 1) A 08:00 - B 08:20/08:25 - C 08:30 - D 08:35  [1, 1, 1]"""
    services = [
        flag_service("1", list("ABCD"), ["08:00", "08:10", "08:15", "08:20", "08:20", "08:25"],
                     [0, 1, 1], flag),
        flag_service("1", list("ABCD"), ["08:00", "08:20", "08:25", "08:30", "08:30", "08:35"],
                     [1, 1, 1], flag),
    ]
    return {
        "date_range": ["2019-05-01", "2019-05-02"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in "ABCD"],
        "footpaths": [],
        "routes": group_routes(services),
    }


def gtfs_flags_3(flag):
    """Timetable 3 of the same two tests: blocks T1>T2>T3 and T4>T5>T6, the
    flag on every trip but T2 (UTC):
      T1>T2>T3 (route 1) A 08:00 - B 08:10/08:15 - C 08:20/08:25 - D 08:30  [1, 0, 1]
      T4>T5>T6 (route 1) A 08:00 - B 08:20/08:25 - C 08:30/08:35 - D 08:40  [1, 1, 1]"""
    services = [
        flag_service("1", list("ABCD"), ["08:00", "08:10", "08:15", "08:20", "08:25", "08:30"],
                     [1, 0, 1], flag),
        flag_service("1", list("ABCD"), ["08:00", "08:20", "08:25", "08:30", "08:35", "08:40"],
                     [1, 1, 1], flag),
    ]
    return {
        "date_range": ["2019-05-01", "2019-05-02"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in "ABCD"],
        "footpaths": [],
        "routes": group_routes(services),
    }


def gtfs_pong_lookahead():
    """test/routing/pong_minlookahead_test.cc kTimetable: agency
    Europe/London (UTC+1 on 2026-06-01), service MON on Mondays of
    2026-06-01..07 (only 2026-06-01 is a Monday), stops without coordinates
    (no footpaths), route type 2 -> kRegional (6); each trip is alone in its
    block:
      R0_MON (route R0) S0 05:00 -> S1 06:00   UTC 04:00 -> 05:00
      R1_MON (route R1) S1 08:00 -> S2 10:00   UTC 07:00 -> 09:00"""
    d = "2026-06-01"
    services = [
        dict(utc_service("R0", ["S0", "S1"], d, [hm("04:00"), hm("05:00")]), id="R0_MON", clasz=6),
        dict(utc_service("R1", ["S1", "S2"], d, [hm("07:00"), hm("09:00")]), id="R1_MON", clasz=6),
    ]
    return {
        "date_range": ["2026-06-01", "2026-06-07"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in ["S0", "S1", "S2"]],
        "footpaths": [],
        "routes": group_routes(services),
    }


def gtfs_pong_gap():
    """test/routing/pong_gap_truncation_test.cc test_files(): agency Etc/UTC,
    service S on 2024-06-19, stops ~150 km apart (no footpaths), route type 2
    -> kRegional (6):
      PH (route PH) A 09:59 -> B 11:00
      EA (route EA) A 10:05 -> C 10:20
      EB (route EB) C 10:30 -> B 11:00
      L  (route L)  A 15:00 -> B 15:30"""
    d = "2024-06-19"
    services = [
        dict(utc_service("PH", ["A", "B"], d, [hm("09:59"), hm("11:00")]), id="PH", clasz=6),
        dict(utc_service("EA", ["A", "C"], d, [hm("10:05"), hm("10:20")]), id="EA", clasz=6),
        dict(utc_service("EB", ["C", "B"], d, [hm("10:30"), hm("11:00")]), id="EB", clasz=6),
        dict(utc_service("L", ["A", "B"], d, [hm("15:00"), hm("15:30")]), id="L", clasz=6),
    ]
    return {
        "date_range": ["2024-06-18", "2024-06-20"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in "ACB"],
        "footpaths": [],
        "routes": group_routes(services),
    }


FLAG_CARS = 1
FLAG_WHEELCHAIR = 2


def gtfs_alternative_block(flag, first_has):
    """test/routing/pong_get_earliest_alternative_test.cc: agency
    Europe/Berlin (UTC+2 on 2024-06-19), service S on 2024-06-19, one block
    of two trips chained into one transport A 08:00 - B 08:15 - C 08:30
    (UTC) whose sections carry `flag` as [first_has, not first_has]:
    bikes [0, 1] (T_NO_BIKE > T_BIKE), cars [1, 0] (T_CAR > T_NO_CAR)."""
    s = dict(utc_service("R1", list("ABC"), "2024-06-19",
                         [hm("08:00"), hm("08:15"), hm("08:15"), hm("08:30")]), clasz=10,
             sections=[(1 << flag) if first_has else 0, 0 if first_has else (1 << flag)])
    return {
        "date_range": ["2024-06-18", "2024-06-20"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in "ABC"],
        "footpaths": [],
        "routes": group_routes([s]),
    }


TIMETABLES = {"hrd_abc": hrd_abc(), "gtfs_transfer_time": gtfs_transfer_time(),
              "gtfs_pong_lookahead": gtfs_pong_lookahead(), "gtfs_pong_gap": gtfs_pong_gap(),
              "gtfs_alternative_bikes": gtfs_alternative_block(FLAG_BIKES, False),
              "gtfs_alternative_cars": gtfs_alternative_block(FLAG_CARS, True),
              "hrd_simple": hrd_simple(), "gtfs_dijkstra": gtfs_dijkstra(),
              "gtfs_clasz": gtfs_clasz(),
              "gtfs_bikes_1": gtfs_flags_1(FLAG_BIKES), "gtfs_bikes_2": gtfs_flags_2(FLAG_BIKES),
              "gtfs_bikes_3": gtfs_flags_3(FLAG_BIKES),
              "gtfs_reservation_1": gtfs_flags_1(FLAG_RESERVATION_NOT_REQUIRED),
              "gtfs_reservation_2": gtfs_flags_2(FLAG_RESERVATION_NOT_REQUIRED),
              "gtfs_reservation_3": gtfs_flags_3(FLAG_RESERVATION_NOT_REQUIRED)}

# ----------------------------------------------------------------------------
# Golden printout parser (journey::print, src/routing/journey.cc)
# ----------------------------------------------------------------------------
_TIME = r"(\d{4}-\d{2}-\d{2} \d{2}:\d{2})"
_LOC = r"\(([^,]*), ([^)]*)\)"
HEADER = re.compile(r"^\[" + _TIME + r", " + _TIME + r"\]$")
LEG = re.compile(r"^leg (\d+): " + _LOC + r" \[" + _TIME + r"\] -> " + _LOC +
                 r" \[" + _TIME + r"\]$")
FOOTPATH = re.compile(r"^\s+FOOTPATH \(duration=(\d+)\)$")
MUMO = re.compile(r"^\s+MUMO \(id=(\d+), duration=(\d+)\)$")
TRIP = re.compile(r"\{name=([^,]*), day=([^,]*), id=([^,]*), src=")
STOPLINE = re.compile(r"^\s+\d+: ")


def gtfs_wheelchair_assistance():
    """test/routing/wheelchair_assistance_test.cc: agency Europe/Berlin
    (UTC+2 on 2024-06-19), service S on 2024-06-19 only, route type 101
    (high speed: clasz 1), every trip wheelchair accessible (the wheelchair
    route flag on every section), no stop with wheelchair_boarding = 2:
      T1 A 00:00 - B1 00:30 - C 01:10   every hour from 00:00 to 23:00
      T2 B2 00:40 - C 00:50             every hour from 00:40 to 23:40
    (frequencies.txt, local times).  For high-speed, long-distance and night
    trips the loader keeps a stop time's wheelchair boarding (alighting) bit
    only while assistance is available at the stop at its local departure
    (arrival) minute (include/nigiri/loader/gtfs/local_to_utc.h:277-340);
    the assistance of a stop is the first entry within 800 m
    (include/nigiri/loader/assistance.h:17-28).  The test's entries A, B
    (at B1 and B2) and C are open 08:00-22:00 local (C's "Th; 08:00-22:00":
    its second rule covers every day).  Trips whose bits differ get routes of
    their own (the route key is the stop sequence with these bits).  The test
    adds the footpath B1 -> B2 (5 min) to profiles 0 and 2 (wheelchair)."""
    def open_at(minute):  # local minutes after 2024-06-19 00:00
        m = minute % 1440
        return 8 * 60 <= m < 22 * 60

    services = []
    for j in range(24):
        d = 60 * j  # local departure at A
        ev = [d, d + 30, d + 30, d + 70]  # A dep, B1 arr, B1 dep, C arr
        wc = [[1 if open_at(ev[0]) else 0, 1], [1 if open_at(ev[2]) else 0, 1 if open_at(ev[1]) else 0],
              [1, 1 if open_at(ev[3]) else 0]]
        services.append(dict(utc_service("RE 1", ["A", "B1", "C"], "2024-06-19", [x - 120 for x in ev]),
                             clasz=1, sections=[1 << FLAG_WHEELCHAIR] * 2, wc=wc))
    for j in range(24):
        d = 40 + 60 * j  # local departure at B2
        ev = [d, d + 10]
        wc = [[1 if open_at(ev[0]) else 0, 1], [1, 1 if open_at(ev[1]) else 0]]
        services.append(dict(utc_service("RE 2", ["B2", "C"], "2024-06-19", [x - 120 for x in ev]),
                             clasz=1, sections=[1 << FLAG_WHEELCHAIR], wc=wc))
    return {
        "date_range": ["2024-06-18", "2024-06-20"],
        "locations": [{"id": x, "name": x, "transfer_time": 2} for x in ("A", "B1", "B2", "C", "D")],
        "footpaths": [["B1", "B2", 5]],
        "profile_footpaths": {"2": [["B1", "B2", 5]]},
        "routes": group_routes(services),
    }


TIMETABLES["gtfs_wheelchair_assistance"] = gtfs_wheelchair_assistance()


def unix_min(s: str) -> int:
    t = dt.datetime.strptime(s, "%Y-%m-%d %H:%M")
    return int((t - dt.datetime(1970, 1, 1)).total_seconds() // 60)


def parse_journeys(text: str):
    out = []
    cur = None
    leg = None
    for line in text.split("\n"):
        m = HEADER.match(line)
        if m:
            cur = {"dep": unix_min(m.group(1)), "arr": unix_min(m.group(2)),
                   "transfers": None, "legs": []}
            out.append(cur)
            continue
        if cur is None:
            continue
        if line.startswith("TRANSFERS: "):
            cur["transfers"] = int(line.split(": ")[1])
            continue
        m = LEG.match(line)
        if m:
            leg = {"from": m.group(3), "to": m.group(6),
                   "dep": unix_min(m.group(4)), "arr": unix_min(m.group(7)),
                   "kind": None}
            cur["legs"].append(leg)
            continue
        if leg is None:
            continue
        m = FOOTPATH.match(line)
        if m:
            leg["kind"] = "footpath"
            leg["duration"] = int(m.group(1))
            continue
        m = MUMO.match(line)
        if m:
            leg["kind"] = "offset"
            leg["mode_id"] = int(m.group(1))
            leg["duration"] = int(m.group(2))
            continue
        if STOPLINE.match(line):
            leg["kind"] = "transport"
            leg["n_stops"] = leg.get("n_stops", 0) + 1
            m = TRIP.search(line)
            if m and "trip" not in leg:
                leg["trip"] = m.group(3) if m.group(3) else m.group(1)
                leg["trip_name"] = m.group(1)
    return out


def raw_string(src: str, name: str) -> str:
    """Contents of `constexpr auto const <name> = R"(...)"` in src."""
    m = re.search(r"\b" + re.escape(name) + r"\s*=\s*(?:\n\s*)?R\"(\w*)\(", src)
    if not m:
        raise KeyError(name)
    delim = m.group(1)
    start = m.end()
    end = src.index(")" + delim + '"', start)
    return src[start:end]


# ----------------------------------------------------------------------------
# Cases: query + where its golden printout lives
# ----------------------------------------------------------------------------

def t(s):  # "2020-03-30 05:00" (UTC) -> unix minutes
    return unix_min(s)


def cases():
    c = []
    # test/routing/raptor_test.cc
    iv = [t("2020-03-30 05:00"), t("2020-03-30 06:00")]
    c.append(dict(name="raptor_forward", timetable="hrd_abc",
                  ref="test/routing/raptor_test.cc", golden="fwd_journeys",
                  query=dict(start=[["0000001", 0, 0]], dest=[["0000003", 0, 0]],
                             interval=iv, direction="fwd")))
    c.append(dict(name="raptor_backward", timetable="hrd_abc",
                  ref="test/routing/raptor_test.cc", golden="bwd_journeys",
                  query=dict(start=[["0000003", 0, 0]], dest=[["0000001", 0, 0]],
                             interval=iv, direction="bwd")))
    # test/routing/raptor_intermodal_test.cc
    c.append(dict(name="raptor_intermodal_forward", timetable="hrd_abc",
                  ref="test/routing/raptor_intermodal_test.cc", golden="fwd_journeys",
                  query=dict(start=[["0000001", 10, 99]], dest=[["0000003", 15, 77]],
                             interval=iv, direction="fwd", start_mode="intermodal",
                             dest_mode="intermodal")))
    c.append(dict(name="raptor_intermodal_backward", timetable="hrd_abc",
                  ref="test/routing/raptor_intermodal_test.cc", golden="bwd_journeys",
                  query=dict(start=[["0000003", 15, 99]], dest=[["0000001", 10, 77]],
                             interval=iv, direction="bwd", start_mode="intermodal",
                             dest_mode="intermodal", min_connection_count=3,
                             extend_earlier=True, extend_later=True)))
    # test/routing/transfer_time_settings_test.cc
    day_iv = [t("2019-05-01 00:00"), t("2019-05-02 00:00")]
    tts_variants = [
        ("default", {}, "expected_A_C_default"),
        ("min10", dict(min_transfer_time=10), "expected_A_C_dur10"),
        ("f1.5", dict(factor=1.5), "expected_A_C_dur3"),
        ("f2", dict(factor=2.0), "expected_A_C_dur4"),
        ("min10_f2", dict(min_transfer_time=10, factor=2.0), "expected_A_C_dur10"),
        ("min3_f2", dict(min_transfer_time=3, factor=2.0), "expected_A_C_dur4"),
        ("add2", dict(additional_time=2), "expected_A_C_dur4"),
        ("add1_f1.5", dict(additional_time=1, factor=1.5), "expected_A_C_dur4"),
        ("min3_add1", dict(min_transfer_time=3, additional_time=1), "expected_A_C_dur4"),
        ("min3_add5_f2.5", dict(min_transfer_time=3, additional_time=5, factor=2.5),
         "expected_A_C_dur10"),
    ]
    for d in ("fwd", "bwd"):
        s, e = ("A", "C") if d == "fwd" else ("C", "A")
        for vname, tts, golden in tts_variants:
            q = dict(start=[[s, 0, 0]], dest=[[e, 0, 0]], interval=day_iv, direction=d,
                     max_travel_time=30)
            if vname != "default":
                q["tts"] = dict(default=False, **tts)
            c.append(dict(name=f"transfer_time_{vname}_{d}", timetable="gtfs_transfer_time",
                          ref="test/routing/transfer_time_settings_test.cc",
                          golden=golden, query=q))
        # default max_travel_time: the direct T4 journey joins the results
        c.append(dict(name=f"transfer_time_direct_{d}", timetable="gtfs_transfer_time",
                      ref="test/routing/transfer_time_settings_test.cc",
                      golden=("expected_A_C_direct", "expected_A_C_default")
                      if d == "fwd" else ("expected_A_C_default", "expected_A_C_direct"),
                      query=dict(start=[[s, 0, 0]], dest=[[e, 0, 0]], interval=day_iv,
                                 direction=d)))
    c.append(dict(name="transfer_time_max_travel_29", timetable="gtfs_transfer_time",
                  ref="test/routing/transfer_time_settings_test.cc", golden=None,
                  query=dict(start=[["A", 0, 0]], dest=[["C", 0, 0]], interval=day_iv,
                             direction="fwd", max_travel_time=29,
                             tts=dict(default=False, factor=2.0))))
    c.append(dict(name="transfer_time_invalid_max_travel", timetable="gtfs_transfer_time",
                  ref="test/routing/transfer_time_settings_test.cc",
                  golden=("expected_A_C_direct", "expected_A_C_default"),
                  query=dict(start=[["A", 0, 0]], dest=[["C", 0, 0]], interval=day_iv,
                             direction="fwd", max_travel_time=-1440)))
    c.append(dict(name="transfer_time_max_transfers_0", timetable="gtfs_transfer_time",
                  ref="test/routing/transfer_time_settings_test.cc",
                  golden="expected_A_C_direct",
                  query=dict(start=[["A", 0, 0]], dest=[["C", 0, 0]], interval=day_iv,
                             direction="fwd", max_transfers=0)))
    c.append(dict(name="transfer_time_max_transfers_0_tt35", timetable="gtfs_transfer_time",
                  ref="test/routing/transfer_time_settings_test.cc", golden=None,
                  query=dict(start=[["A", 0, 0]], dest=[["C", 0, 0]], interval=day_iv,
                             direction="fwd", max_transfers=0, max_travel_time=35)))
    # test/routing/clasz_filter_test.cc (forward only, as there)
    clasz_iv = [t("2024-03-01 00:00"), t("2024-03-02 00:00")]
    air, regional, bus, ship = 1 << 0, 1 << 6, 1 << 10, 1 << 11
    for vname, mask, golden in [("all", 0xFFFF, "expected"),
                                ("bus_regional_air", bus | regional | air, "expected"),
                                ("bus_regional", bus | regional, "expected_1"),
                                ("ship", ship, None)]:
        c.append(dict(name=f"clasz_{vname}", timetable="gtfs_clasz",
                      ref="test/routing/clasz_filter_test.cc", golden=golden,
                      query=dict(start=[["A", 0, 0]], dest=[["C", 0, 0]], interval=clasz_iv,
                                 direction="fwd", claszes=mask)))
    # test/routing/pong_minlookahead_test.cc (pong_search called directly)
    la = dict(start=[["S0", 0, 0]], dest=[["S2", 0, 0]], direction="fwd", algorithm="pong",
              start_mode="equivalent", dest_mode="equivalent", max_travel_time=300,
              min_connection_count=1, extend_later=True)
    for name, extra, golden in [
            ("pong_ignores_interval_4h01",
             dict(interval=[t("2026-06-01 00:00"), t("2026-06-01 04:01")]), "kJourneys"),
            ("pong_ignores_interval_4h",
             dict(interval=[t("2026-06-01 00:00"), t("2026-06-01 04:00")]), "kJourneys"),
            ("pong_min_lookahead_5h", dict(start_time=t("2026-06-01 00:00")), "kJourneys"),
            ("pong_min_lookahead_4h59",
             dict(start_time=t("2026-06-01 00:00"), max_travel_time=299), None)]:
        c.append(dict(name=name, timetable="gtfs_pong_lookahead",
                      ref="test/routing/pong_minlookahead_test.cc", golden=golden,
                      query=dict(la, **extra)))
    # test/routing/bike_transport_test.cc, no_compulsory_reservation_test.cc
    flag_iv = [t("2019-05-01 00:00"), t("2019-05-02 00:00")]
    for kind, ref, key, off, on in [
            ("bikes", "test/routing/bike_transport_test.cc", "bikes", "no_bike", "bike"),
            ("reservation", "test/routing/no_compulsory_reservation_test.cc",
             "no_reservation", "compulsory", "no_reservation")]:
        for tt_no, a, b, g_off, g_on in [
                (1, "A", "C", f"expected_A_C_{off}", f"expected_A_C_{on}"),
                (1, "C", "D", "expected_C_D", "expected_C_D"),
                (1, "A", "D", f"expected_A_D_{off}", f"expected_A_D_{on}"),
                (1, "A", "F", f"expected_A_F_{off}", f"expected_A_F_{on}"),
                (2, "A", "D", f"expected2_A_D_{off}", f"expected2_A_D_{on}"),
                (3, "A", "D", f"expected3_A_D_{off}", f"expected3_A_D_{on}")]:
            for d in ("fwd", "bwd"):
                s, e = (a, b) if d == "fwd" else (b, a)
                for req, golden in ((False, g_off), (True, g_on)):
                    q = dict(start=[[s, 0, 0]], dest=[[e, 0, 0]], interval=flag_iv, direction=d)
                    if req:
                        q[key] = True
                    c.append(dict(name=f"{kind}{tt_no}_{a}{b}_{'req' if req else 'any'}_{d}",
                                  timetable=f"gtfs_{kind}_{tt_no}", ref=ref, golden=golden,
                                  query=q))
    return c


# ----------------------------------------------------------------------------
# Known answers of intermediate steps: start labels (start_times_test.cc) and
# lower bounds (dijkstra_test.cc), parsed from the test sources.
# ----------------------------------------------------------------------------
START_LINE = re.compile(r"^\|  \{time_at_start=" + _TIME + r", time_at_stop=" + _TIME +
                        r", stop=([^}]*)\}$")


def parse_starts(text: str):
    out = []
    for line in text.splitlines():
        m = START_LINE.match(line.strip("\n"))
        if m:
            out.append([unix_min(m.group(1)), unix_min(m.group(2)), m.group(3)])
    return out


def known_answers(ref_root: str):
    ka = []
    src = open(os.path.join(ref_root, "test/routing/start_times_test.cc")).read()
    ka.append(dict(name="start_times_interval", kind="starts", timetable="hrd_simple",
                   ref="test/routing/start_times_test.cc",
                   query=dict(start=[["0000001", 15, 0], ["0000002", 30, 0]],
                              dest=[], interval=[t("2020-03-30 00:00"), t("2020-03-31 00:00")],
                              direction="fwd", max_start_offset=32767),
                   expected=parse_starts(raw_string(src, "expected"))))
    src = open(os.path.join(ref_root, "test/routing/dijkstra_test.cc")).read()
    got = re.findall(r"EXPECT_EQ\((\d+)U, dists\[(\w+)_l\.v_\]\)", src)
    names = {"d1": "D1", "d": "D"}
    start = t("2024-06-08 07:00")
    queries = [dict(start=[["D1", 0, 0]], dest=[["C2", 0, 0]], start_time=start),
               dict(start=[["D", 0, 0]], dest=[["C", 0, 0]], start_time=start,
                    start_mode="equivalent", dest_mode="equivalent")]
    for (value, var), q in zip(got, queries):
        ka.append(dict(name=f"dijkstra_{var}", kind="lower_bounds", timetable="gtfs_dijkstra",
                       ref="test/routing/dijkstra_test.cc", query=q,
                       expected=[[names[var], int(value)]]))
    # pong_gap_truncation_test.cc: the departures of range RAPTOR's result
    # (its `expected` vector: day + 10h + 5min, day + 15h); pong must not
    # depart before the interval either (the harness's EXPECT_GE)
    src = open(os.path.join(ref_root, "test/routing/pong_gap_truncation_test.cc")).read()
    assert "day + 10h + 5min, day + 15h" in src
    gq = dict(start=[["A", 0, 0]], dest=[["B", 0, 0]], direction="fwd",
              interval=[t("2024-06-19 10:00"), t("2024-06-19 10:03")],
              start_mode="equivalent", dest_mode="equivalent", min_connection_count=2,
              extend_later=True)
    ka.append(dict(name="pong_gap_truncation_range", kind="departures", timetable="gtfs_pong_gap",
                   ref="test/routing/pong_gap_truncation_test.cc", query=gq,
                   expected=[t("2024-06-19 10:05"), t("2024-06-19 15:00")]))
    ka.append(dict(name="pong_gap_truncation_pong", kind="departures", timetable="gtfs_pong_gap",
                   ref="test/routing/pong_gap_truncation_test.cc",
                   query=dict(gq, algorithm="pong"), not_before=t("2024-06-19 10:00")))
    # wheelchair_assistance_test.cc: A -> C, 05:00-21:00 UTC on 2024-06-19,
    # the first and last departures of the walking (0) and wheelchair (2)
    # profiles' results
    src = open(os.path.join(ref_root, "test/routing/wheelchair_assistance_test.cc")).read()
    assert "sys_days{2024_y / June / 19} + 6_hours" in src and "sys_days{2024_y / June / 19} + 19_hours" in src
    for prf, first, last in ((0, "05:00", "20:00"), (2, "06:00", "19:00")):
        ka.append(dict(name=f"wheelchair_assistance_prf{prf}", kind="departure_range",
                       timetable="gtfs_wheelchair_assistance",
                       ref="test/routing/wheelchair_assistance_test.cc",
                       query=dict(start=[["A", 0, 0]], dest=[["C", 0, 0]], direction="fwd",
                                  interval=[t("2024-06-19 05:00"), t("2024-06-19 21:00")], prf=prf),
                       expected=[t(f"2024-06-19 {first}"), t(f"2024-06-19 {last}")]))
    # pong_get_earliest_alternative_test.cc: A -> C between 06:00 and 12:00
    # UTC on the block transport, found without the flag, not with it
    for tt_name, key in (("gtfs_alternative_bikes", "bikes"), ("gtfs_alternative_cars", "cars")):
        for req in (False, True):
            ka.append(dict(name=f"earliest_alternative_{key}_{'req' if req else 'any'}",
                           kind="earliest_alternative", timetable=tt_name,
                           ref="test/routing/pong_get_earliest_alternative_test.cc",
                           query=dict(start=[["A", 0, 0]], dest=[["C", 0, 0]],
                                      start_time=t("2024-06-19 06:00"), **({key: True} if req else {})),
                           to_dep=t("2024-06-19 12:00"), expected=not req))
    return ka


# ----------------------------------------------------------------------------
# The GTFS feeds of the tests behind the gtfs_* timetables, verbatim (the
# text of their mem_dir::read raw strings), with the loader_config the test
# passes: the GTFS reader must rebuild those timetables from them.
# ----------------------------------------------------------------------------

def raw_after(src: str, marker: str, nth: int = 0) -> str:
    """The raw string literal (R"delim(...)delim") after the nth `marker`."""
    pos = -1
    for _ in range(nth + 1):
        pos = src.index(marker, pos + 1)
    m = re.compile(r'R"(\w*)\(').search(src, pos)
    start = m.end()
    return src[start:src.index(")" + m.group(1) + '"', start)]


ALL_CLASSES = 0xFFFF
GTFS_FEEDS = {
    "gtfs_transfer_time": ("test/routing/transfer_time_settings_test.cc", "test_files =", 0, {}),
    "gtfs_dijkstra": ("test/routing/dijkstra_test.cc", "dijkstra_files()", 0, {}),
    "gtfs_clasz": ("test/routing/clasz_filter_test.cc", "test_files =", 0, {}),
    "gtfs_bikes_1": ("test/routing/bike_transport_test.cc", "test_files_1 =", 0, {}),
    "gtfs_bikes_2": ("test/routing/bike_transport_test.cc", "test_files2 =", 0, {}),
    "gtfs_bikes_3": ("test/routing/bike_transport_test.cc", "test_files3 =", 0, {}),
    "gtfs_reservation_1": ("test/routing/no_compulsory_reservation_test.cc", "test_files_1 =", 0,
                           {"reservation_not_required_default": ALL_CLASSES}),
    "gtfs_reservation_2": ("test/routing/no_compulsory_reservation_test.cc", "test_files2 =", 0,
                           {"reservation_not_required_default": ALL_CLASSES}),
    "gtfs_reservation_3": ("test/routing/no_compulsory_reservation_test.cc", "test_files3 =", 0,
                           {"reservation_not_required_default": ALL_CLASSES}),
    "gtfs_pong_lookahead": ("test/routing/pong_minlookahead_test.cc", "kTimetable =", 0, {}),
    "gtfs_pong_gap": ("test/routing/pong_gap_truncation_test.cc", "test_files()", 0, {}),
    "gtfs_alternative_bikes": ("test/routing/pong_get_earliest_alternative_test.cc", "kGTFS =", 0, {}),
    "gtfs_alternative_cars": ("test/routing/pong_get_earliest_alternative_test.cc", "kGTFS =", 1, {}),
}


# feeds whose timetable only the reader builds (no hand restatement)
GTFS_ONLY_FEEDS = {
    "gtfs_shortest_fp": ("test/routing/shortest_fp_test.cc", "shortest_fp_files()", 0, {},
                         ["2024-06-07", "2024-06-09"]),
    "gtfs_egress_bound": ("test/routing/gpu_intermodal_egress_test.cc", "test_files()", 0, {},
                          ["2024-06-16", "2024-06-19"]),
    "gtfs_max_interval": ("test/routing/max_interval_test.cc", "test_files()", 0, {},
                          ["2019-03-25", "2019-11-01"]),
    "gtfs_rt_routing": ("test/routing/rt_routing_test.cc", "test_files()", 0, {},
                        ["2019-03-25", "2019-11-01"]),
}


RT_ROUTING = "test/routing/rt_routing_test.cc"


def rt_cases():
    """test/routing/rt_routing_test.cc: each test applies one GTFS-RT update
    and runs an ontrip search.  The update is restated as the overlay it
    leaves in rt_timetable (gtfsrt_update.cc), in UTC:
    * rt_raptor_forward / _backward: RE 2 (T_RE2, 00:30 local on 2019-05-03
      = 22:30 UTC on its service day 2019-05-02) is 2 h late from its first
      stop on; the delay carries to the later stops, so the run leaves B
      00:30, passes C 00:45 and reaches D 01:00 UTC on 2019-05-03, and the
      static trip no longer runs on 2019-05-02;
    * rt_raptor_unscheduled: an added trip (NEW) from B 00:30 to D 01:00 UTC
      on 2019-05-03 (stop_time_update times 1556843400 and 1556845200 s)."""
    delayed = {"changed": [{"trip_name": "RE 2", "day": "2019-05-02", "runs": False}],
               "runs": [{"trip_name": "RE 2", "day": "2019-05-02", "stops": ["B", "C", "D"],
                         "times": [t("2019-05-03 00:30"), t("2019-05-03 00:45"), t("2019-05-03 00:45"),
                                   t("2019-05-03 01:00")]}]}
    added = {"changed": [],
             "runs": [{"trip_name": None, "day": None, "stops": ["B", "D"],
                       "times": [t("2019-05-03 00:30"), t("2019-05-03 01:00")]}]}
    return [
        dict(name="rt_raptor_forward", timetable="gtfs_rt_routing", ref=RT_ROUTING, golden="kFwdJourneys",
             rt=delayed, query=dict(start=[["A", 0, 0]], dest=[["D", 0, 0]], start_time=t("2019-05-02 23:00"))),
        dict(name="rt_raptor_backward", timetable="gtfs_rt_routing", ref=RT_ROUTING, golden="kBwdJourneys",
             rt=delayed, query=dict(start=[["D", 0, 0]], dest=[["A", 0, 0]], start_time=t("2019-05-03 02:00"),
                                    direction="bwd")),
        dict(name="rt_raptor_unscheduled", timetable="gtfs_rt_routing", ref=RT_ROUTING,
             golden="unscheduled_journeys", rt=added,
             query=dict(start=[["A", 0, 0]], dest=[["D", 0, 0]], start_time=t("2019-05-02 23:00"))),
    ]


def gtfs_only_cases():
    """test/routing/shortest_fp_test.cc: intermodal searches over transfers.txt
    footpaths, forward over 2024-06-07 and backward over 06-07 .. 06-09;
    test/routing/max_interval_test.cc: interval extension clamped by the
    query's max_interval_."""
    a = [["A0", 3, 23], ["A1", 5, 23], ["A2", 10, 23]]
    c = [["C3", 30, 42], ["C4", 20, 42], ["C5", 10, 42]]
    ref = "test/routing/shortest_fp_test.cc"
    return [
        dict(name="shortest_fp_forward", timetable="gtfs_shortest_fp", ref=ref, golden="exp_fwd_journey",
             query=dict(start=a, dest=c, interval=[t("2024-06-07 00:00"), t("2024-06-08 00:00")],
                        direction="fwd", start_mode="intermodal", dest_mode="intermodal")),
        dict(name="shortest_fp_backward", timetable="gtfs_shortest_fp", ref=ref, golden="exp_bwd_journey",
             query=dict(start=c, dest=a, interval=[t("2024-06-07 00:00"), t("2024-06-09 00:00")],
                        direction="bwd", start_mode="intermodal", dest_mode="intermodal")),
        # test/routing/max_interval_test.cc: three connections wanted, the
        # interval may grow later, but only up to max_interval_ (12:00), so
        # the 12:00 departure stays out
        dict(name="max_interval", timetable="gtfs_max_interval", ref="test/routing/max_interval_test.cc",
             golden="expected_journeys",
             query=dict(start=[["A", 0, 0]], dest=[["B", 0, 0]],
                        interval=[t("2019-05-01 10:00"), t("2019-05-01 11:00")], direction="fwd",
                        min_connection_count=3, extend_later=True,
                        max_interval=[t("2019-05-01 10:00"), t("2019-05-01 12:00")])),
    ]


def gtfs_only_known_answers():
    """test/routing/gpu_intermodal_egress_test.cc: the results contain the
    1-transfer journey leaving the coordinate at 09:55 and arriving 11:00
    (its EXPECT_TRUE(found)); nigiri's harness runs the query through range
    RAPTOR and pong."""
    return [dict(name="intermodal_egress_at_bound", timetable="gtfs_egress_bound",
                 ref="test/routing/gpu_intermodal_egress_test.cc",
                 query=dict(start=[["A", 5, 0], ["A2", 5, 0]], dest=[["C", 0, 0]],
                            interval=[t("2024-06-17 09:45"), t("2024-06-17 10:45")],
                            direction="fwd", start_mode="intermodal", dest_mode="intermodal",
                            min_connection_count=1),
                 contains=[t("2024-06-17 09:55"), t("2024-06-17 11:00"), 1])]


JOIN_SPLIT = "test/routing/join_split_test.cc"
MONTHS = {m: i + 1 for i, m in enumerate(["January", "February", "March", "April", "May", "June", "July",
                                          "August", "September", "October", "November", "December"])}


def join_split_feeds(ref_root: str):
    """test/routing/join_split_test.cc (join_split.complex): the feed with its
    six trips.txt rows in the two orders the test loads (0..5 and 5..0)."""
    src = open(os.path.join(ref_root, JOIN_SPLIT)).read()
    body = raw_after(src, "mem_dir::read(fmt::format(")
    assert "{{" not in body and body.count("{}") == 6
    rows = re.findall(r'"([^"]*)"', re.search(r"kTrips\s*=\s*std::array\{([^}]*)\}", src).group(1))
    out = {}
    for name, order in (("gtfs_join_split", range(6)), ("gtfs_join_split_rev", range(5, -1, -1))):
        text = body
        for i in order:
            text = text.replace("{}", rows[i], 1)
        out[name] = {"ref": JOIN_SPLIT, "text": text, "config": {}, "date_range": ["2025-06-12", "2025-06-22"]}
    return out


def join_split_cases(ref_root: str):
    """join_split.complex's kTests before its real-time update: an ontrip
    search at 00:00 UTC of the date finds journeys, all without a transfer
    (the trips joined by stay-seated transfers are one transport)."""
    src = open(os.path.join(ref_root, JOIN_SPLIT)).read()
    tests = re.findall(r'\{"(\w+)", "(\w+)", (\d+)_y / (\w+) / (\d+), (true|false)\}', src)
    assert len(tests) == 14
    out = []
    for feed in ("gtfs_join_split", "gtfs_join_split_rev"):
        for a, b, y, mon, d, exp in tests:
            out.append(dict(name=f"{feed}_{a}_{b}_{mon[:3].lower()}{d}", timetable=feed, ref=JOIN_SPLIT,
                            query=dict(start=[[a, 0, 0]], dest=[[b, 0, 0]],
                                       start_time=t(f"{y}-{MONTHS[mon]:02d}-{int(d):02d} 00:00")),
                            nonempty=exp == "true", max_transfers_seen=0))
    return out


def gtfs_feeds(ref_root: str):
    out = join_split_feeds(ref_root)
    for name, (path, marker, nth, config, date_range) in GTFS_ONLY_FEEDS.items():
        src = open(os.path.join(ref_root, path)).read()
        out[name] = {"ref": path, "text": raw_after(src, marker, nth), "config": config,
                     "date_range": date_range}
    for name, (path, marker, nth, config) in GTFS_FEEDS.items():
        src = open(os.path.join(ref_root, path)).read()
        if config.get("reservation_not_required_default") == ALL_CLASSES:
            # the test's default_reservation_not_required: all 16 classes true
            m = re.search(r"default_reservation_not_required\s*=\s*std::array<bool, kNumClasses>\{([^}]*)\}", src)
            assert m and [x.strip() for x in m.group(1).split(",")] == ["true"] * 16
        out[name] = {"ref": path, "text": raw_after(src, marker, nth), "config": config}
    return out


def main(ref_root: str):
    out_cases = []
    for case in cases():
        src = open(os.path.join(ref_root, case["ref"])).read()
        g = case["golden"]
        if g is None:
            expected = []
        elif isinstance(g, tuple):
            expected = []
            for name in g:
                expected += parse_journeys(raw_string(src, name))
        else:
            expected = parse_journeys(raw_string(src, g))
        case = dict(case)
        case["golden"] = list(g) if isinstance(g, tuple) else g
        case["expected"] = expected
        out_cases.append(case)
    gtfs_cases = []
    for case in gtfs_only_cases():
        src = open(os.path.join(ref_root, case["ref"])).read()
        gtfs_cases.append(dict(case, expected=parse_journeys(raw_string(src, case["golden"]))))
    rt = []
    for case in rt_cases():
        src = open(os.path.join(ref_root, case["ref"])).read()
        rt.append(dict(case, expected=parse_journeys(raw_string(src, case["golden"]))))
    doc = {"timetables": TIMETABLES, "cases": out_cases, "gtfs_cases": gtfs_cases, "rt_cases": rt,
           "gtfs_known_answers": gtfs_only_known_answers(),
           "gtfs_seated_cases": join_split_cases(ref_root),
           "known_answers": known_answers(ref_root), "gtfs_feeds": gtfs_feeds(ref_root),
           "generated_by": "tests/golden/make_fixtures.py"}
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(doc, f, indent=1, sort_keys=True)
    print(f"wrote {len(out_cases)} cases")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <root of the nigiri source tree>")
    main(sys.argv[1])
