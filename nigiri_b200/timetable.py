"""Host timetables and seeded query streams (b2r_tt_* / b2r_queries_*)."""
from __future__ import annotations

import ctypes as C
import os

from . import _abi as A
from .routing import B2RError, Offset, Query, TransferTimeSettings, _check, EXACT, INTERMODAL, FORWARD, BACKWARD

# workload -> (timetable config, timetable seed); workloads 3 / 5 reuse the
# timetables of 2 / 4
TIMETABLE_OF = {1: (1, 1), 2: (2, 2), 3: (2, 2), 4: (4, 4), 5: (4, 4)}


class HostTimetable:
    """Flattened timetable in host memory (nigiri's finalize() applied)."""

    def __init__(self, handle: C.c_void_p):
        self.handle = handle
        self.desc = A.TimetableDesc()
        _check(A.lib().b2r_tt_desc(self.handle, C.byref(self.desc)))

    @classmethod
    def generate(cls, workload: int, cache_dir: str | None = None):
        cfg, seed = TIMETABLE_OF[workload]
        lib = A.lib()
        if cache_dir:
            path = os.path.join(cache_dir, f"tt_config{cfg}_seed{seed}.b2r")
            if os.path.exists(path):
                h = C.c_void_p()
                if lib.b2r_tt_load(path.encode(), C.byref(h)) == 0:
                    return cls(h)
        h = C.c_void_p()
        _check(lib.b2r_tt_generate(cfg, seed, C.byref(h)))
        t = cls(h)
        if cache_dir:
            os.makedirs(cache_dir, exist_ok=True)
            lib.b2r_tt_save(h, os.path.join(cache_dir, f"tt_config{cfg}_seed{seed}.b2r").encode())
        return t

    @classmethod
    def load_gtfs(cls, feed: str, date_range: tuple[int, int], text: bool = False,
                  default_transfer_time: int = 2, bikes_allowed_default: int = 0,
                  cars_allowed_default: int = 0, reservation_not_required_default: int = 0,
                  default_tz: str | None = None, tzdata_dir: str | None = None):
        """A GTFS feed (a directory, or with text=True nigiri's "# file.txt"
        text) read for timetable::date_range_ = date_range (days since the
        epoch, [from, to)); the defaults mirror loader_config (bit c of a
        *_default mask = transport class c)."""
        cfg = A.GtfsConfig()
        A.lib().b2r_gtfs_config_init(C.byref(cfg))
        cfg.date_range_from, cfg.date_range_to = date_range
        cfg.default_transfer_time = default_transfer_time
        cfg.bikes_allowed_default = bikes_allowed_default
        cfg.cars_allowed_default = cars_allowed_default
        cfg.reservation_not_required_default = reservation_not_required_default
        cfg.default_tz = default_tz.encode() if default_tz else None
        cfg.tzdata_dir = tzdata_dir.encode() if tzdata_dir else None
        h = C.c_void_p()
        _check(A.lib().b2r_tt_load_gtfs(feed.encode(), 1 if text else 0, C.byref(cfg), C.byref(h)))
        return cls(h)

    def location_id(self, l: int) -> str:
        s = C.c_char_p()
        _check(A.lib().b2r_tt_location_id(self.handle, l, C.byref(s)))
        return s.value.decode()

    def transport_name(self, t: int) -> str:
        s = C.c_char_p()
        _check(A.lib().b2r_tt_transport_name(self.handle, t, C.byref(s)))
        return s.value.decode()

    def close(self):
        if self.handle:
            A.lib().b2r_tt_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class QuerySet:
    """Seeded synthetic queries of a workload, owned by the library."""

    def __init__(self, tt: HostTimetable, workload: int, n: int, seed: int | None = None):
        self.tt = tt
        self.handle = C.c_void_p()
        seed = 1000 + workload if seed is None else seed
        _check(A.lib().b2r_queries_generate(tt.handle, workload, seed, n, C.byref(self.handle)))
        self.n = A.lib().b2r_queries_count(self.handle)
        # contiguous copy of the structs (offset pointers stay owned by the set)
        self.arr = (A.Query * max(1, self.n))()
        for i in range(self.n):
            self.arr[i] = A.lib().b2r_queries_get(self.handle, i).contents

    def subset(self, idx):
        arr = (A.Query * max(1, len(idx)))()
        for j, i in enumerate(idx):
            arr[j] = self.arr[i]
        return arr

    def to_query(self, i) -> tuple[Query, str, int]:
        """(routing.Query, direction, kind) of query i."""
        x = self.arr[i]
        modes = {A.B2R_MATCH_EXACT: EXACT, A.B2R_MATCH_INTERMODAL: INTERMODAL}
        q = Query(start=[Offset(x.start[j].target, x.start[j].duration, x.start[j].transport_mode_id)
                         for j in range(x.n_start)],
                  destination=[Offset(x.destination[j].target, x.destination[j].duration,
                                      x.destination[j].transport_mode_id)
                               for j in range(x.n_destination)],
                  start_time=(x.interval_from, x.interval_to) if x.is_interval else x.start_time,
                  start_match_mode=modes[x.start_match_mode],
                  dest_match_mode=modes[x.dest_match_mode],
                  max_transfers=x.max_transfers,
                  max_travel_time=x.max_travel_time,
                  transfer_time_settings=TransferTimeSettings(),
                  allowed_claszes=x.allowed_claszes & 0xFFFF,
                  require_bike_transport=bool(x.require_bike_transport),
                  require_car_transport=bool(x.require_car_transport),
                  no_compulsory_reservation=bool(x.no_compulsory_reservation))
        return q, (FORWARD if x.direction == A.B2R_FORWARD else BACKWARD), x.kind

    def close(self):
        if self.handle:
            A.lib().b2r_queries_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
