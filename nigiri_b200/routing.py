"""Python mirror of nigiri's routing interface on top of the B200 engine.

Mirrors, for the static timetable / no-via / no-filter case:
  routing::query                  include/nigiri/routing/query.h:70-100
  routing::raptor_search          src/routing/raptor_search.cc:94-159
  routing::one_to_all             src/routing/one_to_all.cc:52-104
  routing::journey / journey::leg include/nigiri/routing/journey.h:20-118
Every call goes through libb2r.so (include/b2r.h); there is no CPU path.
Errors are raised as B2RError carrying the engine's status code.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _abi as A

FORWARD, BACKWARD = "fwd", "bwd"
EXACT, ONLY_CHILDREN, EQUIVALENT, INTERMODAL = "exact", "only_children", "equivalent", "intermodal"
_MODE = {EXACT: A.B2R_MATCH_EXACT, ONLY_CHILDREN: A.B2R_MATCH_ONLY_CHILDREN,
         EQUIVALENT: A.B2R_MATCH_EQUIVALENT, INTERMODAL: A.B2R_MATCH_INTERMODAL}


class B2RError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"b2r status {status}: {msg}")
        self.status = status


def _check(rc: int):
    if rc != A.B2R_OK:
        raise B2RError(rc, A.lib().b2r_last_error().decode(errors="replace"))


@dataclasses.dataclass
class Offset:  # routing::offset
    target: int
    duration: int
    transport_mode_id: int = 0


@dataclasses.dataclass
class TransferTimeSettings:  # routing::transfer_time_settings
    default: bool = True
    min_transfer_time: int = 0
    additional_time: int = 0
    factor: float = 1.0


@dataclasses.dataclass
class Query:  # routing::query (static subset)
    start: List[Offset]
    destination: List[Offset] = dataclasses.field(default_factory=list)
    start_time: Union[int, Tuple[int, int]] = 0  # unix minutes or [from, to)
    start_match_mode: str = EXACT
    dest_match_mode: str = EXACT
    use_start_footpaths: bool = False
    max_start_offset: int = 7200
    max_transfers: int = 14
    max_travel_time: int = 7200
    min_connection_count: int = 0
    extend_interval_earlier: bool = False
    extend_interval_later: bool = False
    transfer_time_settings: TransferTimeSettings = dataclasses.field(
        default_factory=TransferTimeSettings)
    fastest_direct: Optional[int] = None
    fastest_direct_factor: float = 1.0
    allowed_claszes: int = 0xFFFF  # bit c: transport class c (clasz_mask_t)
    require_bike_transport: bool = False
    require_car_transport: bool = False
    no_compulsory_reservation: bool = False


@dataclasses.dataclass
class Leg:  # journey::leg
    from_: int
    to: int
    dep_time: int
    arr_time: int
    kind: str  # "transport" | "footpath" | "offset"
    transport: int = 0
    day: int = 0
    stop_range: Tuple[int, int] = (0, 0)
    target: int = 0
    duration: int = 0
    transport_mode_id: int = 0


@dataclasses.dataclass
class Journey:  # journey
    legs: List[Leg]
    start_time: int
    dest_time: int
    dest: int
    transfers: int

    def departure_time(self):
        return min(self.start_time, self.dest_time)

    def arrival_time(self):
        return max(self.start_time, self.dest_time)


@dataclasses.dataclass
class RoutingResult:  # routing_result
    journeys: List[Journey]
    interval: Tuple[int, int]
    status: int
    n_rounds: int = 0
    n_start_times: int = 0


@dataclasses.dataclass
class OneToAllResult:  # raptor_state rows of one_to_all
    round_times: np.ndarray  # [rows, n_locations] int16 deltas
    base_day: int            # days since epoch
    direction: str


class _QueryBuffer:
    """Owns the b2r_query structs and offset arrays of a batch."""

    def __init__(self, queries: Sequence[Tuple[Query, str, int]], algorithm: int = A.B2R_ALGO_RAPTOR):
        n = len(queries)
        self.arr = (A.Query * max(1, n))()
        self.keep = []
        lib = A.lib()
        for i, (q, direction, kind) in enumerate(queries):
            x = self.arr[i]
            lib.b2r_query_init(C.byref(x))
            x.algorithm = algorithm
            st = (A.Offset * max(1, len(q.start)))()
            for j, o in enumerate(q.start):
                st[j].target, st[j].duration, st[j].transport_mode_id = o.target, o.duration, o.transport_mode_id
            de = (A.Offset * max(1, len(q.destination)))()
            for j, o in enumerate(q.destination):
                de[j].target, de[j].duration, de[j].transport_mode_id = o.target, o.duration, o.transport_mode_id
            self.keep += [st, de]
            x.start, x.n_start = st, len(q.start)
            x.destination, x.n_destination = de, len(q.destination)
            x.kind = kind
            x.direction = A.B2R_FORWARD if direction == FORWARD else A.B2R_BACKWARD
            if isinstance(q.start_time, tuple):
                x.is_interval = 1
                x.interval_from, x.interval_to = q.start_time
            else:
                x.start_time = q.start_time
            x.start_match_mode = _MODE[q.start_match_mode]
            x.dest_match_mode = _MODE[q.dest_match_mode]
            x.use_start_footpaths = int(q.use_start_footpaths)
            x.max_start_offset = q.max_start_offset
            x.max_transfers = q.max_transfers
            x.max_travel_time = q.max_travel_time
            x.min_connection_count = q.min_connection_count
            x.extend_interval_earlier = int(q.extend_interval_earlier)
            x.extend_interval_later = int(q.extend_interval_later)
            tts = q.transfer_time_settings
            x.tts_default = int(tts.default)
            x.tts_min_transfer_time = tts.min_transfer_time
            x.tts_additional_time = tts.additional_time
            x.tts_factor = tts.factor
            x.allowed_claszes = q.allowed_claszes
            x.require_bike_transport = int(q.require_bike_transport)
            x.require_car_transport = int(q.require_car_transport)
            x.no_compulsory_reservation = int(q.no_compulsory_reservation)
            if q.fastest_direct is not None:
                x.has_fastest_direct = 1
                x.fastest_direct = q.fastest_direct
            x.fastest_direct_factor = q.fastest_direct_factor


class Timetable:
    """Device-resident timetable image (b2r_timetable_upload)."""

    def __init__(self, desc: A.TimetableDesc, device: int = 0, owner=None):
        self._owner = owner  # keeps host arrays alive while desc is used
        self.desc = desc
        self.handle = C.c_void_p()
        _check(A.lib().b2r_timetable_upload(C.byref(desc), device, C.byref(self.handle)))

    @property
    def n_locations(self):
        return self.desc.n_locations

    def device_bytes(self):
        return A.lib().b2r_timetable_device_bytes(self.handle)

    def close(self):
        if self.handle:
            A.lib().b2r_timetable_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """Resident query slots on one GPU (b2r_engine_create)."""

    def __init__(self, tt: Timetable, max_slots=1024, hbm_budget=64 << 30, max_journeys=128,
                 use_lower_bounds=True, use_graphs=True, host_threads=0, steps_per_sync=4,
                 max_starts=4096, profile=False):
        cfg = A.EngineConfig()
        A.lib().b2r_engine_config_init(C.byref(cfg))
        cfg.max_slots = max_slots
        cfg.hbm_budget = hbm_budget
        cfg.max_journeys = max_journeys
        # True / "table" -> all-pairs tables on the device when they fit, else
        # host Dijkstra (3); "host" -> 1; "device" -> device solver (2);
        # False -> none (0)
        cfg.use_lower_bounds = {True: 3, "table": 3, "host": 1, "device": 2,
                                False: 0}[use_lower_bounds]
        cfg.use_graphs = int(use_graphs)
        cfg.host_threads = host_threads
        cfg.max_starts = max_starts
        cfg.steps_per_sync = steps_per_sync
        cfg.profile = int(profile)
        self.tt = tt
        self.handle = C.c_void_p()
        _check(A.lib().b2r_engine_create(tt.handle, C.byref(cfg), C.byref(self.handle)))

    @property
    def slots(self):
        return A.lib().b2r_engine_slots(self.handle)

    def bytes_per_slot(self):
        return A.lib().b2r_engine_bytes_per_slot(self.handle)

    def close(self):
        if self.handle:
            A.lib().b2r_engine_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- runs
    def run(self, qbuf: _QueryBuffer, n: int, convert, plain=False):
        """Runs n queries; `convert` turns each b2r_result into Python
        objects before the engine-owned memory is reused."""
        out = (A.Result * max(1, n))()
        lib = A.lib()
        if plain:
            res = []
            for i in range(n):
                _check(lib.b2r_search_plain(self.handle, C.byref(qbuf.arr[i]), C.byref(out[i])))
                res.append(convert(i, out[i]))
            return res
        _check(lib.b2r_search_batch(self.handle, qbuf.arr, n, out))
        return [convert(i, out[i]) for i in range(n)]

    def stats(self):
        s = A.BatchStats()
        _check(A.lib().b2r_last_batch_stats(self.handle, C.byref(s)))
        return s

    @property
    def shape(self) -> A.LaunchShape:
        sh = A.LaunchShape()
        _check(A.lib().b2r_engine_get_shape(self.handle, C.byref(sh)))
        return sh

    @shape.setter
    def shape(self, sh: A.LaunchShape):
        _check(A.lib().b2r_engine_set_shape(self.handle, C.byref(sh)))

    def autotune(self, qarr, n: int) -> A.TuneReport:
        """Picks the launch shape with the shortest batch time on a sample
        (b2r_engine_autotune); results do not depend on the shape."""
        rep = A.TuneReport()
        _check(A.lib().b2r_engine_autotune(self.handle, qarr, n, C.byref(rep)))
        return rep

    def scan_profile(self, cap: int = 4096):
        """Per route-scan launch of the last batch (profiling engines):
        [(milliseconds, marked entries, stop visits)]."""
        ms = (C.c_double * cap)()
        ent = (C.c_uint64 * cap)()
        vis = (C.c_uint64 * cap)()
        n = C.c_uint32()
        _check(A.lib().b2r_last_batch_scan_profile(self.handle, ms, ent, vis, cap, C.byref(n)))
        return [(ms[i], ent[i], vis[i]) for i in range(min(cap, n.value))]


def _journeys(res: A.Result) -> List[Journey]:
    out = []
    for i in range(res.n_journeys):
        j = res.journeys[i]
        legs = []
        for li in range(j.first_leg, j.first_leg + j.n_legs):
            L = res.legs[li]
            kind = {A.B2R_LEG_TRANSPORT: "transport", A.B2R_LEG_FOOTPATH: "footpath",
                    A.B2R_LEG_OFFSET: "offset"}[L.kind]
            leg = Leg(L.from_, L.to, L.dep_time, L.arr_time, kind)
            if kind == "transport":
                leg.transport, leg.day, leg.stop_range = L.transport, L.day, (L.stop_from, L.stop_to)
            else:
                leg.target, leg.duration, leg.transport_mode_id = L.transport, L.duration, L.transport_mode_id
            legs.append(leg)
        out.append(Journey(legs, j.start_time, j.dest_time, j.dest, j.transfers))
    return out


def raptor_search(engine: Engine, queries: Sequence[Query], direction=FORWARD,
                  plain: bool = False) -> List[RoutingResult]:
    """routing::raptor_search for a batch of queries (one direction, or a
    list of per-query directions)."""
    dirs = direction if isinstance(direction, (list, tuple)) else [direction] * len(queries)
    qb = _QueryBuffer([(q, d, A.B2R_ONE_TO_ONE) for q, d in zip(queries, dirs)])

    def conv(_, r):
        return RoutingResult(_journeys(r), (r.interval_from, r.interval_to), r.status,
                             r.n_rounds, r.n_start_times)
    return engine.run(qb, len(queries), conv, plain=plain)


def pong_search(engine: Engine, queries: Sequence[Query], direction=FORWARD,
                plain: bool = False) -> List[RoutingResult]:
    """routing::pong_search (src/routing/raptor/pong.cc): the range search
    by alternating forward and backward searches; same results as
    raptor_search on the intersection of their search intervals.  A query
    whose sweep fails as the reference's would ("no pong", "no pong
    progress") comes back with status B2R_ERR_INTERNAL."""
    dirs = direction if isinstance(direction, (list, tuple)) else [direction] * len(queries)
    qb = _QueryBuffer([(q, d, A.B2R_ONE_TO_ONE) for q, d in zip(queries, dirs)], A.B2R_ALGO_PONG)

    def conv(_, r):
        return RoutingResult(_journeys(r), (r.interval_from, r.interval_to), r.status,
                             r.n_rounds, r.n_start_times)
    return engine.run(qb, len(queries), conv, plain=plain)


def one_to_all(engine: Engine, queries: Sequence[Query], direction=FORWARD,
               plain: bool = False) -> List[OneToAllResult]:
    """routing::one_to_all: the round times of every location."""
    dirs = direction if isinstance(direction, (list, tuple)) else [direction] * len(queries)
    qb = _QueryBuffer([(q, d, A.B2R_ONE_TO_ALL) for q, d in zip(queries, dirs)])
    n = engine.tt.n_locations

    def conv(i, r):
        if r.status != A.B2R_OK:
            raise B2RError(r.status, "one_to_all failed")
        rows = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n,)).reshape(r.n_rows, n).copy()
        return OneToAllResult(rows, r.base_day, dirs[i])
    return engine.run(qb, len(queries), conv, plain=plain)


class Server:
    """Continuous-batching request loop on an engine (b2r_serve_start):
    queries submitted from any thread are admitted into free slots while
    earlier ones are still running; each ticket's result stays readable
    until it is released."""

    def __init__(self, engine: Engine):
        self.engine = engine
        _check(A.lib().b2r_serve_start(engine.handle))

    def submit_raw(self, q: A.Query) -> int:
        """Submits a b2r_query (offsets are copied by the engine)."""
        t = C.c_uint64()
        _check(A.lib().b2r_submit(self.engine.handle, C.byref(q), C.byref(t)))
        return t.value

    def poll(self, ticket: int):
        """The b2r_result of a finished ticket, or None while it runs."""
        r = A.Result()
        rc = A.lib().b2r_poll(self.engine.handle, ticket, C.byref(r))
        if rc == A.B2R_ERR_NOT_READY:
            return None
        _check(rc)
        return r

    def wait(self, ticket: int) -> A.Result:
        r = A.Result()
        _check(A.lib().b2r_wait(self.engine.handle, ticket, C.byref(r)))
        return r

    def stats(self) -> A.BatchStats:
        """Counters of the serving loop since start (b2r_serve_stats)."""
        s = A.BatchStats()
        _check(A.lib().b2r_serve_stats(self.engine.handle, C.byref(s)))
        return s

    def release(self, ticket: int):
        _check(A.lib().b2r_release(self.engine.handle, ticket))

    def stop(self):
        """Finishes every submitted query, then stops the loop."""
        if self.engine.handle:
            _check(A.lib().b2r_serve_stop(self.engine.handle))
