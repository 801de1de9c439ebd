"""Loads tests/golden/cases.json into flattened timetables and b2r queries
(test infrastructure).

A fixture timetable is turned into nigiri's route layout (per route, for
every stop pair: departures of all transports, then arrivals) and handed to
b2r_tt_build, which performs finalize()'s derivations.
"""
from __future__ import annotations

import ctypes as C
import datetime as dt
import json
import os

import numpy as np

from nigiri_b200 import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
N_SPECIAL = 9
SPECIAL_NAMES = ["START", "END", "VIA0", "VIA1", "VIA2", "VIA3", "VIA4", "VIA5", "VIA6"]


def load_cases():
    with open(os.path.join(HERE, "cases.json")) as f:
        return json.load(f)


def _day(s):
    return (dt.date.fromisoformat(s) - dt.date(1970, 1, 1)).days


def _enc(minutes):
    return (minutes // 1440) & 0x1F | ((minutes % 1440) << 5)


class FixtureTimetable:
    """Owns the numpy arrays, the host timetable handle and its desc."""

    def __init__(self, spec, lib):
        self.lib = lib
        self.spec = spec
        d_from, d_to = (_day(x) for x in spec["date_range"])
        self.internal_from = d_from - 5
        ids = [x["id"] for x in spec["locations"]]
        self.loc_idx = {i: N_SPECIAL + k for k, i in enumerate(ids)}
        for k, n in enumerate(SPECIAL_NAMES):
            self.loc_idx[n] = k
        self.loc_name = {v: k for k, v in self.loc_idx.items()}
        n_loc = N_SPECIAL + len(ids)
        tt_ = np.zeros(n_loc, np.uint8)
        for k, x in enumerate(spec["locations"]):
            tt_[N_SPECIAL + k] = x.get("transfer_time", 2)
        parent = np.full(n_loc, 0xFFFFFFFF, np.uint32)
        for k, x in enumerate(spec["locations"]):
            if x.get("parent"):
                parent[N_SPECIAL + k] = self.loc_idx[x["parent"]]
        fps = [[] for _ in range(n_loc)]
        for a, b, dur in spec.get("footpaths", []):
            fps[self.loc_idx[a]].append((self.loc_idx[b] & 0x7FFFFF) | (dur << 23))
        fp_index = np.zeros(n_loc + 1, np.uint32)
        fp_data = []
        for l in range(n_loc):
            lst = sorted(fps[l], key=lambda w: w >> 23)  # stable by duration
            fp_data += lst
            fp_index[l + 1] = len(fp_data)
        # footpaths of profiles 1..4 ("profile_footpaths": {"p": [[a, b, min]]})
        self.profile_fp = {}
        for prf, lst in spec.get("profile_footpaths", {}).items():
            pf = [[] for _ in range(n_loc)]
            for a_, b_, dur in lst:
                pf[self.loc_idx[a_]].append((self.loc_idx[b_] & 0x7FFFFF) | (dur << 23))
            idx = np.zeros(n_loc + 1, np.uint32)
            dat = []
            for l in range(n_loc):
                dat += sorted(pf[l], key=lambda w: w >> 23)
                idx[l + 1] = len(dat)
            self.profile_fp[int(prf)] = (idx, np.array(dat or [0], np.uint32))
        # bitfields: one per distinct traffic day set
        bf_list = [np.zeros(8, np.uint64)]
        bf_of = {}
        route_stop_index = [0]
        route_stops = []
        route_clasz = []
        section_flags = []  # per route stop: flags of the section it starts
        route_n_t = []
        stop_times = []
        transport_bf = []
        self.transport_names = []
        for r in spec["routes"]:
            for k, s in enumerate(r["stops"]):
                w = r.get("stop_flags", {}).get(s, (1, 1))
                wc = r["stop_wc"][k] if "stop_wc" in r else (1, 1)  # wheelchair in / out
                route_stops.append(self.loc_idx[s] | (w[0] << 28) | (w[1] << 29)
                                   | (wc[0] << 30) | (wc[1] << 31))
            route_stop_index.append(len(route_stops))
            route_clasz.append(r.get("clasz", 10))
            section_flags += list(r.get("sections", [0] * (len(r["stops"]) - 1))) + [0]
            trs = r["transports"]  # already in route order (mam-sorted)
            # traffic day of the transport = its day; the times stay relative
            route_n_t.append(len(trs))
            n = len(r["stops"])
            for tr in trs:
                key = (tr["day"],) if isinstance(tr["day"], str) else tuple(tr["day"])
                if key not in bf_of:
                    b = np.zeros(8, np.uint64)
                    for dd in key:
                        bit = _day(dd) - self.internal_from
                        b[bit // 64] |= np.uint64(1) << np.uint64(bit % 64)
                    bf_of[key] = len(bf_list)
                    bf_list.append(b)
                transport_bf.append(bf_of[key])
                self.transport_names.append(tr["name"])
            for s in range(n - 1):
                for tr in trs:
                    stop_times.append(_enc(tr["times"][2 * s]))
                for tr in trs:
                    stop_times.append(_enc(tr["times"][2 * s + 1]))
        self.arrays = dict(
            transfer_time=tt_, parent=parent, fp_index=fp_index, fp_data=np.array(fp_data or [0], np.uint32),
            route_stop_index=np.array(route_stop_index, np.uint32),
            route_stops=np.array(route_stops or [0], np.uint32),
            route_n_t=np.array(route_n_t or [0], np.uint32),
            stop_times=np.array(stop_times or [0], np.uint16),
            transport_bf=np.array(transport_bf or [0], np.uint32),
            bitfields=np.concatenate(bf_list).astype(np.uint64),
            route_clasz=np.array(route_clasz or [0], np.uint8),
            section_flags=np.array(section_flags or [0], np.uint8),
        )
        a = self.arrays
        p = lambda arr, t: arr.ctypes.data_as(C.POINTER(t))
        base = A.TtBase()
        base.n_locations = n_loc
        base.date_range_from = d_from
        base.date_range_to = d_to
        base.transfer_time = p(a["transfer_time"], C.c_uint8)
        if any(x.get("parent") for x in spec["locations"]):
            base.parent = p(a["parent"], C.c_uint32)
        base.footpaths_out_index = p(a["fp_index"], C.c_uint32)
        base.footpaths_out = p(a["fp_data"], C.c_uint32)
        for prf, (idx, dat) in self.profile_fp.items():
            base.profile_footpaths_out_index[prf - 1] = p(idx, C.c_uint32)
            base.profile_footpaths_out[prf - 1] = p(dat, C.c_uint32)
        base.n_routes = len(spec["routes"])
        base.route_stop_index = p(a["route_stop_index"], C.c_uint32)
        base.route_stops = p(a["route_stops"], C.c_uint32)
        base.route_n_transports = p(a["route_n_t"], C.c_uint32)
        base.route_stop_times = p(a["stop_times"], C.c_uint16)
        base.transport_bitfield = p(a["transport_bf"], C.c_uint32)
        base.n_bitfields = len(bf_list)
        base.bitfields = p(a["bitfields"], C.c_uint64)
        base.route_clasz = p(a["route_clasz"], C.c_uint8)
        if any(a["section_flags"]):
            base.route_section_flags = p(a["section_flags"], C.c_uint8)
        self.handle = C.c_void_p()
        rc = lib.b2r_tt_build(C.byref(base), C.byref(self.handle))
        assert rc == 0, rc
        self.desc = A.TimetableDesc()
        lib.b2r_tt_desc(self.handle, C.byref(self.desc))

    def __del__(self):
        try:
            self.lib.b2r_tt_destroy(self.handle)
        except Exception:
            pass


class GtfsFixture:
    """A timetable read by the engine's GTFS reader (b2r_tt_load_gtfs) from
    the feed text of one of nigiri's tests, with the same lookups as
    FixtureTimetable (stop ids, transport names)."""

    def __init__(self, name, lib):
        cases = load_cases()
        feed = cases["gtfs_feeds"][name]
        self.spec = cases["timetables"].get(name, {"date_range": feed.get("date_range"), "locations": []})
        self.lib = lib
        cfg = A.GtfsConfig()
        lib.b2r_gtfs_config_init(C.byref(cfg))
        cfg.date_range_from, cfg.date_range_to = (_day(x) for x in self.spec["date_range"])
        for k, v in feed["config"].items():
            setattr(cfg, k, v)
        self.handle = C.c_void_p()
        rc = lib.b2r_tt_load_gtfs(feed["text"].encode(), 1, C.byref(cfg), C.byref(self.handle))
        assert rc == 0, lib.b2r_last_error()
        self.desc = A.TimetableDesc()
        lib.b2r_tt_desc(self.handle, C.byref(self.desc))
        s = C.c_char_p()
        self.loc_name = {}
        for l in range(self.desc.n_locations):
            assert lib.b2r_tt_location_id(self.handle, l, C.byref(s)) == 0
            self.loc_name[l] = s.value.decode()
        self.loc_idx = {v: k for k, v in self.loc_name.items()}
        self.transport_names = []
        for t in range(self.desc.n_transports):
            assert lib.b2r_tt_transport_name(self.handle, t, C.byref(s)) == 0
            self.transport_names.append(s.value.decode())

    def __del__(self):
        try:
            self.lib.b2r_tt_destroy(self.handle)
        except Exception:
            pass


MODES = {"exact": A.B2R_MATCH_EXACT, "intermodal": A.B2R_MATCH_INTERMODAL,
         "equivalent": A.B2R_MATCH_EQUIVALENT, "only_children": A.B2R_MATCH_ONLY_CHILDREN}


class FixtureQuery:
    """A b2r_query plus the offset arrays it points to."""

    def __init__(self, lib, tt: FixtureTimetable, q):
        self.q = A.Query()
        lib.b2r_query_init(C.byref(self.q))
        qq = self.q
        self.start = (A.Offset * max(1, len(q["start"])))()
        for i, (loc, dur, mode) in enumerate(q["start"]):
            self.start[i].target = tt.loc_idx[loc]
            self.start[i].duration = dur
            self.start[i].transport_mode_id = mode
        self.dest = (A.Offset * max(1, len(q.get("dest", []))))()
        for i, (loc, dur, mode) in enumerate(q.get("dest", [])):
            self.dest[i].target = tt.loc_idx[loc]
            self.dest[i].duration = dur
            self.dest[i].transport_mode_id = mode
        qq.start = self.start
        qq.n_start = len(q["start"])
        qq.destination = self.dest
        qq.n_destination = len(q.get("dest", []))
        qq.direction = A.B2R_FORWARD if q.get("direction", "fwd") == "fwd" else A.B2R_BACKWARD
        if "interval" in q:
            qq.is_interval = 1
            qq.interval_from, qq.interval_to = q["interval"]
        else:
            qq.start_time = q["start_time"]
        qq.start_match_mode = MODES[q.get("start_mode", "exact")]
        qq.dest_match_mode = MODES[q.get("dest_mode", "exact")]
        if "max_travel_time" in q:
            qq.max_travel_time = q["max_travel_time"]
        if "max_transfers" in q:
            qq.max_transfers = q["max_transfers"]
        if "max_start_offset" in q:
            qq.max_start_offset = q["max_start_offset"]
        qq.min_connection_count = q.get("min_connection_count", 0)
        qq.extend_interval_earlier = 1 if q.get("extend_earlier") else 0
        qq.extend_interval_later = 1 if q.get("extend_later") else 0
        if "max_interval" in q:
            qq.has_max_interval = 1
            qq.max_interval_from, qq.max_interval_to = q["max_interval"]
        if q.get("kind") == "one_to_all":
            qq.kind = A.B2R_ONE_TO_ALL
        if q.get("algorithm") == "pong":
            qq.algorithm = A.B2R_ALGO_PONG
        if "claszes" in q:
            qq.allowed_claszes = q["claszes"]
        if "prf" in q:
            qq.prf_idx = q["prf"]
        qq.require_bike_transport = 1 if q.get("bikes") else 0
        qq.require_car_transport = 1 if q.get("cars") else 0
        qq.no_compulsory_reservation = 1 if q.get("no_reservation") else 0
        tts = q.get("tts")
        if tts is not None:
            qq.tts_default = 1 if tts.get("default", True) else 0
            qq.tts_min_transfer_time = tts.get("min_transfer_time", 0)
            qq.tts_additional_time = tts.get("additional_time", 0)
            qq.tts_factor = tts.get("factor", 1.0)


def journeys_to_records(tt: FixtureTimetable, res: A.Result):
    """b2r_result journeys -> the parsed-golden record format."""
    out = []
    for ji in range(res.n_journeys):
        j = res.journeys[ji]
        rec = {"dep": min(j.start_time, j.dest_time), "arr": max(j.start_time, j.dest_time),
               "transfers": j.transfers, "legs": []}
        for li in range(j.first_leg, j.first_leg + j.n_legs):
            L = res.legs[li]
            leg = {"from": tt.loc_name[L.from_], "to": tt.loc_name[L.to],
                   "dep": L.dep_time, "arr": L.arr_time}
            if L.kind == A.B2R_LEG_TRANSPORT:
                leg["kind"] = "transport"
                leg["n_stops"] = L.stop_to - L.stop_from
                # an added real-time trip runs for no static trip
                leg["trip_name"] = None if L.transport == 0xFFFFFFFF else tt.transport_names[L.transport]
            elif L.kind == A.B2R_LEG_FOOTPATH:
                leg["kind"] = "footpath"
                leg["duration"] = L.duration
            else:
                leg["kind"] = "offset"
                leg["duration"] = L.duration
                leg["mode_id"] = L.transport_mode_id
            rec["legs"].append(leg)
        out.append(rec)
    return out


def in_window(q, records):
    """The records whose anchor (departure forward, arrival backward) lies
    in the query's interval -- the window in which nigiri's test harness
    requires pong and range RAPTOR to print the same journeys
    (test/raptor_search.cc:198-237)."""
    lo, hi = q["interval"]
    key = "dep" if q.get("direction", "fwd") == "fwd" else "arr"
    return [r for r in records if lo <= r[key] < hi]


def strip_expected(expected, names_by_trip=None):
    """Golden records restricted to the fields the flattened image carries."""
    out = []
    for j in expected:
        r = {k: j[k] for k in ("dep", "arr", "transfers")}
        r["legs"] = []
        for leg in j["legs"]:
            x = {k: leg[k] for k in ("from", "to", "dep", "arr", "kind")}
            if leg["kind"] == "transport":
                x["n_stops"] = leg["n_stops"]
                x["trip_name"] = leg.get("trip_name")
            elif leg["kind"] == "footpath":
                x["duration"] = leg["duration"]
            else:
                x["duration"] = leg["duration"]
                x["mode_id"] = leg["mode_id"]
            r["legs"].append(x)
        out.append(r)
    return out


class RtOverlay:
    """A b2r_rt_desc and the arrays it points to.  changed: (transport,
    8 uint64 day words) pairs; runs: dicts with stop words, times (minutes
    since the epoch, rt_transport_stop_times_ order), static transport and
    day, and optionally clasz, flags and section flags."""

    def __init__(self, changed, runs):
        import numpy as np
        self.changed_t = np.array([c[0] for c in changed] or [0], np.uint32)
        self.changed_d = np.array([w for c in changed for w in c[1]] or [0], np.uint64)
        idx, stops, times, st, sd, cl, fl, sec = [0], [], [], [], [], [], [], []
        for r in runs:
            assert len(r["times"]) == 2 * (len(r["stops"]) - 1)
            stops += r["stops"]
            idx.append(len(stops))
            times += r["times"]
            st.append(r.get("static_transport", 0xFFFFFFFF))
            sd.append(r.get("static_day", 0))
            cl.append(r.get("clasz", 10))
            fl.append(r.get("flags", 0))
            sec += r.get("section_flags", [0] * len(r["stops"]))
        self.arrays = [np.array(idx, np.uint32), np.array(stops or [0], np.uint32),
                       np.array(times or [0], np.int32), np.array(st or [0], np.uint32),
                       np.array(sd or [0], np.uint16), np.array(cl or [0], np.uint8),
                       np.array(fl or [0], np.uint8), np.array(sec or [0], np.uint8)]
        a = self.arrays
        p = lambda arr, t: arr.ctypes.data_as(C.POINTER(t))
        self.desc = A.RtDesc()
        self.desc.n_changed = len(changed)
        self.desc.changed_transport = p(self.changed_t, C.c_uint32)
        self.desc.changed_days = p(self.changed_d, C.c_uint64)
        self.desc.n_rt_transports = len(runs)
        self.desc.rt_stop_index = p(a[0], C.c_uint32)
        self.desc.rt_stops = p(a[1], C.c_uint32)
        self.desc.rt_event_times = p(a[2], C.c_int32)
        self.desc.rt_static_transport = p(a[3], C.c_uint32)
        self.desc.rt_static_day = p(a[4], C.c_uint16)
        self.desc.rt_clasz = p(a[5], C.c_uint8)
        self.desc.rt_flags = p(a[6], C.c_uint8)
        self.desc.rt_section_flags = p(a[7], C.c_uint8)


def stop_word(loc):
    """A stop word with every in / out bit set (an added run's stops)."""
    return loc | (0xF << 28)


def transport_days(desc, t):
    """The 8 day words of transport t's static traffic days."""
    bf = desc.transport_traffic_days[t]
    return [desc.bitfields[8 * bf + i] for i in range(8)]


def rt_overlay_of_case(tt, spec):
    """The overlay a rt case restates, on the timetable the reader built:
    trips named by route short name, days as UTC dates."""
    d = tt.desc
    first = d.date_range_from - 5

    def day_idx(s):
        return _day(s) - first

    def transport(name):
        xs = [i for i, n in enumerate(tt.transport_names) if n == name]
        assert len(xs) == 1, (name, xs)
        return xs[0]

    changed = []
    for c in spec["changed"]:
        t = transport(c["trip_name"])
        words = transport_days(d, t)
        if not c["runs"]:
            di = day_idx(c["day"])
            words[di // 64] &= ~(1 << (di % 64))
        changed.append((t, words))
    runs = []
    for r in spec["runs"]:
        run = dict(stops=[stop_word(tt.loc_idx[x]) for x in r["stops"]], times=r["times"])
        if r["trip_name"] is not None:
            run["static_transport"] = transport(r["trip_name"])
            run["static_day"] = day_idx(r["day"])
        runs.append(run)
    return RtOverlay(changed, runs)
