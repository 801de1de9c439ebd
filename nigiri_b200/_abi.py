"""ctypes mirror of include/b2r.h (the engine's C ABI).

Only layout definitions and library loading live here; the user-facing
wrapper is nigiri_b200.routing.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb2r.so")

B2R_OK = 0
B2R_ERR_INVALID_ARGUMENT = -1
B2R_ERR_CAPACITY = -4
B2R_ERR_NOT_READY = -5
B2R_K = 16
B2R_MAX_TRANSFERS = 14
# limits of b2r_one_to_all_noalloc's fixed scratch array
B2R_NOALLOC_MAX_LOCATIONS = 65536
B2R_NOALLOC_MAX_ROUTES = 65536
B2R_NOALLOC_MAX_OFFSETS = 64
B2R_NOALLOC_SCRATCH_BYTES = 8388608 + 256
B2R_FORWARD, B2R_BACKWARD = 0, 1
B2R_MATCH_EXACT, B2R_MATCH_ONLY_CHILDREN, B2R_MATCH_EQUIVALENT, B2R_MATCH_INTERMODAL = 0, 1, 2, 3
B2R_ONE_TO_ONE, B2R_ONE_TO_ALL = 0, 1
B2R_FLAG_BIKES, B2R_FLAG_CARS, B2R_FLAG_WHEELCHAIR, B2R_FLAG_RESERVATION_NOT_REQUIRED = 0, 1, 2, 3
B2R_ALL_CLASZ = 0xFFFFFFFF
B2R_ALGO_RAPTOR, B2R_ALGO_PONG = 0, 1
B2R_N_PROFILES, B2R_PROFILE_WHEELCHAIR = 5, 2
B2R_LEG_TRANSPORT, B2R_LEG_FOOTPATH, B2R_LEG_OFFSET = 0, 1, 2

_u8p, _u16p, _u32p, _u64p = (C.POINTER(C.c_uint8), C.POINTER(C.c_uint16),
                             C.POINTER(C.c_uint32), C.POINTER(C.c_uint64))


class TimetableDesc(C.Structure):
    _fields_ = [
        ("n_locations", C.c_uint32), ("n_routes", C.c_uint32),
        ("n_transports", C.c_uint32), ("n_bitfields", C.c_uint32),
        ("date_range_from", C.c_int32), ("date_range_to", C.c_int32),
        ("transfer_time", _u8p), ("parent", _u32p), ("location_type", _u8p),
        ("children_index", _u32p), ("children", _u32p),
        ("importance", _u32p), ("max_importance", C.c_uint32),
        ("footpaths_out_index", _u32p), ("footpaths_out", _u32p),
        ("footpaths_in_index", _u32p), ("footpaths_in", _u32p),
        ("route_stop_index", _u32p), ("route_stops", _u32p),
        ("route_transport_from", _u32p), ("route_transport_to", _u32p),
        ("route_stop_time_from", _u32p), ("route_stop_times", _u16p),
        ("n_route_stop_times", C.c_uint64),
        ("route_traffic_days", _u32p), ("transport_traffic_days", _u32p),
        ("transport_route", _u32p), ("bitfields", _u64p),
        ("location_routes_index", _u32p), ("location_routes", _u32p),
        ("lb_fwd_index", _u32p), ("lb_fwd", _u32p),
        ("lb_bwd_index", _u32p), ("lb_bwd", _u32p),
        ("route_clasz", _u8p), ("route_flags", _u8p), ("route_section_flags", _u8p),
        ("profile_footpaths_out_index", _u32p * 4), ("profile_footpaths_out", _u32p * 4),
        ("profile_footpaths_in_index", _u32p * 4), ("profile_footpaths_in", _u32p * 4),
        ("profile_lb_fwd_index", _u32p * 4), ("profile_lb_fwd", _u32p * 4),
        ("profile_lb_bwd_index", _u32p * 4), ("profile_lb_bwd", _u32p * 4),
    ]


class GtfsConfig(C.Structure):
    _fields_ = [
        ("date_range_from", C.c_int32), ("date_range_to", C.c_int32),
        ("default_transfer_time", C.c_uint32),
        ("bikes_allowed_default", C.c_uint16), ("cars_allowed_default", C.c_uint16),
        ("reservation_not_required_default", C.c_uint16), ("link_stop_distance", C.c_uint16),
        ("default_tz", C.c_char_p), ("tzdata_dir", C.c_char_p),
    ]


class Offset(C.Structure):
    _fields_ = [("target", C.c_uint32), ("duration", C.c_int16),
                ("pad_", C.c_int16), ("transport_mode_id", C.c_int32)]


class Query(C.Structure):
    _fields_ = [
        ("kind", C.c_uint8), ("direction", C.c_uint8), ("is_interval", C.c_uint8),
        ("start_match_mode", C.c_uint8), ("dest_match_mode", C.c_uint8),
        ("use_start_footpaths", C.c_uint8), ("extend_interval_earlier", C.c_uint8),
        ("extend_interval_later", C.c_uint8),
        ("start_time", C.c_int32), ("interval_from", C.c_int32), ("interval_to", C.c_int32),
        ("start", C.POINTER(Offset)), ("n_start", C.c_uint32),
        ("destination", C.POINTER(Offset)), ("n_destination", C.c_uint32),
        ("max_start_offset", C.c_int16), ("max_transfers", C.c_uint8),
        ("has_fastest_direct", C.c_uint8), ("max_travel_time", C.c_int16),
        ("fastest_direct", C.c_int16), ("min_connection_count", C.c_uint32),
        ("fastest_direct_factor", C.c_double),
        ("tts_default", C.c_uint8), ("pad_", C.c_uint8 * 3),
        ("tts_min_transfer_time", C.c_int16), ("tts_additional_time", C.c_int16),
        ("tts_factor", C.c_float),
        ("allowed_claszes", C.c_uint32), ("require_bike_transport", C.c_uint8),
        ("require_car_transport", C.c_uint8), ("no_compulsory_reservation", C.c_uint8),
        ("algorithm", C.c_uint8),
        ("has_max_interval", C.c_uint8), ("prf_idx", C.c_uint8), ("pad2_", C.c_uint8 * 2),
        ("max_interval_from", C.c_int32), ("max_interval_to", C.c_int32),
    ]


class Leg(C.Structure):
    _fields_ = [
        ("from_", C.c_uint32), ("to", C.c_uint32), ("dep_time", C.c_int32),
        ("arr_time", C.c_int32), ("kind", C.c_uint8), ("pad_", C.c_uint8),
        ("day", C.c_uint16), ("transport", C.c_uint32), ("stop_from", C.c_uint16),
        ("stop_to", C.c_uint16), ("duration", C.c_int16), ("pad2_", C.c_int16),
        ("transport_mode_id", C.c_int32), ("rt_transport", C.c_uint32),
    ]


class RtDesc(C.Structure):  # b2r_rt_desc
    _fields_ = [
        ("n_changed", C.c_uint32), ("changed_transport", C.POINTER(C.c_uint32)),
        ("changed_days", C.POINTER(C.c_uint64)), ("n_rt_transports", C.c_uint32),
        ("rt_stop_index", C.POINTER(C.c_uint32)), ("rt_stops", C.POINTER(C.c_uint32)),
        ("rt_event_times", C.POINTER(C.c_int32)), ("rt_static_transport", C.POINTER(C.c_uint32)),
        ("rt_static_day", C.POINTER(C.c_uint16)), ("rt_clasz", C.POINTER(C.c_uint8)),
        ("rt_flags", C.POINTER(C.c_uint8)), ("rt_section_flags", C.POINTER(C.c_uint8)),
    ]


class Journey(C.Structure):
    _fields_ = [("start_time", C.c_int32), ("dest_time", C.c_int32),
                ("dest", C.c_uint32), ("transfers", C.c_uint8), ("error", C.c_uint8),
                ("n_legs", C.c_uint16), ("first_leg", C.c_uint32)]


class Result(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("n_journeys", C.c_uint32),
        ("journeys", C.POINTER(Journey)), ("legs", C.POINTER(Leg)),
        ("interval_from", C.c_int32), ("interval_to", C.c_int32),
        ("n_rows", C.c_uint32), ("base_day", C.c_int32),
        ("round_times", C.POINTER(C.c_int16)),
        ("n_rounds", C.c_uint64), ("n_start_times", C.c_uint64),
        ("latency_ms", C.c_double),
    ]


class EngineConfig(C.Structure):
    _fields_ = [
        ("max_slots", C.c_uint32), ("hbm_budget", C.c_uint64),
        ("max_journeys", C.c_uint32), ("host_threads", C.c_uint32),
        ("use_lower_bounds", C.c_uint32), ("use_graphs", C.c_uint32),
        ("route_block", C.c_uint32), ("max_starts", C.c_uint32),
        ("steps_per_sync", C.c_uint32), ("profile", C.c_uint32), ("reserved", C.c_uint32 * 4),
    ]


class BatchStats(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("host_prep_ms", C.c_double),
                ("kernel_launches", C.c_uint64), ("super_steps", C.c_uint64),
                ("route_scan_launches", C.c_uint64), ("route_scan_ms", C.c_double),
                ("route_stop_visits", C.c_uint64), ("et_events", C.c_uint64),
                ("et_days", C.c_uint64), ("label_writes", C.c_uint64),
                ("route_scan_bytes", C.c_uint64), ("lb_ms", C.c_double),
                ("lb_iterations", C.c_uint64), ("lb_relaxations", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
                ("route_warp_steps", C.c_uint64), ("recon_ms", C.c_double),
                ("recon_max_journey_us", C.c_double), ("recon_journeys", C.c_uint64),
                ("host_prep_cpu_ms", C.c_double), ("host_admit_ms", C.c_double),
                ("host_export_ms", C.c_double), ("host_idle_ms", C.c_double)]


class LaunchShape(C.Structure):
    _fields_ = [("scan_blocks_per_sm", C.c_uint32), ("scan_threads", C.c_uint32),
                ("pair_blocks_per_sm", C.c_uint32), ("recon_blocks_per_sm", C.c_uint32),
                ("steps_per_sync", C.c_uint32), ("scan_occupancy", C.c_uint32)]


class TuneReport(C.Structure):
    _fields_ = [("n_tried", C.c_uint32), ("start", LaunchShape), ("best", LaunchShape),
                ("start_ms", C.c_double), ("best_ms", C.c_double)]


class TtBase(C.Structure):
    _fields_ = [
        ("n_locations", C.c_uint32), ("date_range_from", C.c_int32),
        ("date_range_to", C.c_int32), ("transfer_time", _u8p), ("parent", _u32p),
        ("location_type", _u8p), ("footpaths_out_index", _u32p),
        ("footpaths_out", _u32p), ("n_routes", C.c_uint32),
        ("route_stop_index", _u32p), ("route_stops", _u32p),
        ("route_clasz", _u8p), ("route_n_transports", _u32p),
        ("route_stop_times", _u16p), ("transport_bitfield", _u32p),
        ("n_bitfields", C.c_uint32), ("bitfields", _u64p),
        ("route_flags", _u8p), ("route_section_flags", _u8p),
        ("profile_footpaths_out_index", _u32p * 4), ("profile_footpaths_out", _u32p * 4),
    ]


# Every entry point include/b2r.h declares (checked by the CPU test suite).
EXPORTS = [
    "b2r_last_error", "b2r_query_init", "b2r_timetable_upload",
    "b2r_timetable_destroy", "b2r_timetable_device_bytes",
    "b2r_engine_config_init", "b2r_engine_create", "b2r_engine_destroy",
    "b2r_engine_bytes_per_slot", "b2r_engine_slots", "b2r_search_batch",
    "b2r_search_plain", "b2r_serve_start", "b2r_serve_stop", "b2r_submit",
    "b2r_poll", "b2r_wait", "b2r_release", "b2r_serve_stats", "b2r_last_batch_stats",
    "b2r_tt_generate", "b2r_tt_build", "b2r_tt_save", "b2r_tt_load",
    "b2r_tt_desc", "b2r_tt_destroy", "b2r_gtfs_config_init", "b2r_tt_load_gtfs",
    "b2r_tt_location_id", "b2r_tt_transport_name", "b2r_queries_generate",
    "b2r_queries_count", "b2r_queries_get", "b2r_queries_destroy",
    "b2r_one_to_all_noalloc", "b2r_last_batch_scan_profile",
    "b2r_engine_get_shape", "b2r_engine_set_shape", "b2r_engine_autotune",
    "b2r_search_prepare", "b2r_search_extend", "b2r_search_plan_free", "b2r_raptor_create",
    "b2r_raptor_destroy", "b2r_raptor_reset_arrivals", "b2r_raptor_next_start_time",
    "b2r_raptor_add_start", "b2r_raptor_execute", "b2r_raptor_reconstruct", "b2r_raptor_rounds",
    "b2r_rt_upload", "b2r_rt_destroy", "b2r_engine_set_rt",
]


def _declare(lib):
    vp = C.c_void_p
    sig = {
        "b2r_last_error": (C.c_char_p, []),
        "b2r_query_init": (None, [C.POINTER(Query)]),
        "b2r_timetable_upload": (C.c_int, [C.POINTER(TimetableDesc), C.c_int, C.POINTER(vp)]),
        "b2r_timetable_destroy": (C.c_int, [vp]),
        "b2r_timetable_device_bytes": (C.c_uint64, [vp]),
        "b2r_engine_config_init": (None, [C.POINTER(EngineConfig)]),
        "b2r_engine_create": (C.c_int, [vp, C.POINTER(EngineConfig), C.POINTER(vp)]),
        "b2r_engine_destroy": (C.c_int, [vp]),
        "b2r_engine_bytes_per_slot": (C.c_uint64, [vp]),
        "b2r_engine_slots": (C.c_uint32, [vp]),
        "b2r_search_batch": (C.c_int, [vp, C.POINTER(Query), C.c_uint32, C.POINTER(Result)]),
        "b2r_search_plain": (C.c_int, [vp, C.POINTER(Query), C.POINTER(Result)]),
        "b2r_serve_start": (C.c_int, [vp]),
        "b2r_serve_stop": (C.c_int, [vp]),
        "b2r_submit": (C.c_int, [vp, C.POINTER(Query), C.POINTER(C.c_uint64)]),
        "b2r_poll": (C.c_int, [vp, C.c_uint64, C.POINTER(Result)]),
        "b2r_wait": (C.c_int, [vp, C.c_uint64, C.POINTER(Result)]),
        "b2r_release": (C.c_int, [vp, C.c_uint64]),
        "b2r_last_batch_stats": (C.c_int, [vp, C.POINTER(BatchStats)]),
        "b2r_serve_stats": (C.c_int, [vp, C.POINTER(BatchStats)]),
        "b2r_tt_generate": (C.c_int, [C.c_uint32, C.c_uint64, C.POINTER(vp)]),
        "b2r_tt_build": (C.c_int, [C.POINTER(TtBase), C.POINTER(vp)]),
        "b2r_tt_save": (C.c_int, [vp, C.c_char_p]),
        "b2r_tt_load": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
        "b2r_tt_desc": (C.c_int, [vp, C.POINTER(TimetableDesc)]),
        "b2r_tt_destroy": (C.c_int, [vp]),
        "b2r_gtfs_config_init": (None, [C.POINTER(GtfsConfig)]),
        "b2r_tt_load_gtfs": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(GtfsConfig), C.POINTER(vp)]),
        "b2r_tt_location_id": (C.c_int, [vp, C.c_uint32, C.POINTER(C.c_char_p)]),
        "b2r_tt_transport_name": (C.c_int, [vp, C.c_uint32, C.POINTER(C.c_char_p)]),
        "b2r_queries_generate": (C.c_int, [vp, C.c_uint32, C.c_uint64, C.c_uint32, C.POINTER(vp)]),
        "b2r_queries_count": (C.c_uint32, [vp]),
        "b2r_queries_get": (C.POINTER(Query), [vp, C.c_uint32]),
        "b2r_queries_destroy": (C.c_int, [vp]),
        "b2r_engine_get_shape": (C.c_int, [vp, C.POINTER(LaunchShape)]),
        "b2r_engine_set_shape": (C.c_int, [vp, C.POINTER(LaunchShape)]),
        "b2r_engine_autotune": (C.c_int, [vp, C.POINTER(Query), C.c_uint32, C.POINTER(TuneReport)]),
        "b2r_last_batch_scan_profile": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                                  C.POINTER(C.c_uint64), C.c_uint32,
                                                  C.POINTER(C.c_uint32)]),
        "b2r_one_to_all_noalloc": (C.c_int, [vp, C.POINTER(Query), C.POINTER(C.c_int16), C.c_uint64,
                                             C.POINTER(C.c_uint32), C.POINTER(C.c_int32), vp]),
        # the Algo concept (search::init's preparation and one raptor state)
        "b2r_search_prepare": (C.c_int, [vp, C.POINTER(Query), C.POINTER(vp)]),
        "b2r_search_extend": (C.c_int, [vp, vp, C.c_uint32, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8)]),
        "b2r_search_plan_free": (None, [vp]),
        "b2r_raptor_create": (C.c_int, [vp, vp, C.POINTER(vp)]),
        "b2r_raptor_destroy": (C.c_int, [vp]),
        "b2r_raptor_reset_arrivals": (C.c_int, [vp]),
        "b2r_raptor_next_start_time": (C.c_int, [vp]),
        "b2r_raptor_add_start": (C.c_int, [vp, C.c_uint32, C.c_int32]),
        "b2r_raptor_execute": (C.c_int, [vp, C.c_int32, C.c_uint8, C.c_int32, C.POINTER(Journey), C.c_uint32,
                                         C.POINTER(C.c_uint32)]),
        "b2r_raptor_reconstruct": (C.c_int, [vp, C.POINTER(Query), C.POINTER(Journey), C.POINTER(Leg),
                                             C.c_uint32]),
        "b2r_raptor_rounds": (C.c_uint64, [vp]),
        # the real-time overlay
        "b2r_rt_upload": (C.c_int, [vp, C.POINTER(RtDesc), C.POINTER(vp)]),
        "b2r_rt_destroy": (C.c_int, [vp]),
        "b2r_engine_set_rt": (C.c_int, [vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib():
    """Load the engine library (fails loudly if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m nigiri_b200.build`")
        _lib = _declare(C.CDLL(LIB_PATH))
    return _lib
