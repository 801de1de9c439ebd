"""ctypes access to the CPU oracle (test infrastructure only)."""
from __future__ import annotations

import ctypes as C
import os

from nigiri_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")


class OrStats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "n_rounds", "n_start_times", "n_routes_visited", "n_route_stops_visited", "n_et_calls",
        "n_et_days", "n_et_events", "n_label_writes", "n_marked_stations",
        "n_location_routes_read", "n_fp_stations", "n_footpaths_visited", "n_sweep_locations",
        "algorithmic_bytes")]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            from nigiri_b200.build import build_oracle
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        vp = C.c_void_p
        L.or_search.argtypes = [C.POINTER(A.TimetableDesc), C.POINTER(A.Query), C.POINTER(vp)]
        L.or_search.restype = C.c_int
        L.or_search_rt.argtypes = [C.POINTER(A.TimetableDesc), C.POINTER(A.RtDesc), C.POINTER(A.Query),
                                   C.POINTER(vp)]
        L.or_search_rt.restype = C.c_int
        L.or_result_view.argtypes = [vp, C.POINTER(A.Result), C.POINTER(OrStats)]
        L.or_result_state.argtypes = [vp, C.POINTER(C.POINTER(C.c_int16)),
                                      C.POINTER(C.POINTER(C.c_int16)), C.POINTER(C.c_int32)]
        L.or_result_free.argtypes = [vp]
        L.or_result_free.restype = None
        L.or_lower_bounds.argtypes = [C.POINTER(A.TimetableDesc), C.POINTER(A.Query),
                                      C.POINTER(C.c_uint16)]
        L.or_get_starts.argtypes = [C.POINTER(A.TimetableDesc), C.POINTER(A.Query),
                                    C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_uint32), C.c_uint32, C.POINTER(C.c_uint32)]
        L.or_run_many.argtypes = [C.POINTER(A.TimetableDesc), C.POINTER(A.Query), C.c_uint32,
                                  C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_uint64),
                                  C.POINTER(C.c_double)]
        L.or_earliest_alternative.argtypes = [C.POINTER(A.TimetableDesc), C.POINTER(A.Query),
                                              C.c_uint32, C.c_uint32, C.c_int32, C.c_int32,
                                              C.POINTER(A.Leg)]
        L.or_last_error.restype = C.c_char_p
        _lib = L
    return _lib


class OracleResult:
    def __init__(self, desc, q, rt=None):
        """rt: a b2r_rt_desc (the real-time overlay) or None."""
        self.h = C.c_void_p()
        if rt is None:
            rc = lib().or_search(C.byref(desc), C.byref(q), C.byref(self.h))
        else:
            rc = lib().or_search_rt(C.byref(desc), C.byref(rt), C.byref(q), C.byref(self.h))
        if rc != 0:
            raise RuntimeError(f"oracle failed: {rc} {lib().or_last_error().decode()}")
        self.view = A.Result()
        self.stats = OrStats()
        lib().or_result_view(self.h, C.byref(self.view), C.byref(self.stats))
        self.n_loc = desc.n_locations

    def records(self):
        """Journey records, read while this result (which owns the journey
        arrays the view points into) is alive."""
        from journeys import records
        return records(self.view)

    def state(self):
        import numpy as np
        rt = C.POINTER(C.c_int16)()
        best = C.POINTER(C.c_int16)()
        bd = C.c_int32()
        lib().or_result_state(self.h, C.byref(rt), C.byref(best), C.byref(bd))
        rows = np.ctypeslib.as_array(rt, shape=(16 * self.n_loc,)).reshape(16, self.n_loc).copy()
        b = np.ctypeslib.as_array(best, shape=(self.n_loc,)).copy()
        return rows, b, bd.value

    def __del__(self):
        try:
            lib().or_result_free(self.h)
        except Exception:
            pass


def answers(desc, qarr, idx, threads=None, rt=None):
    """The oracle's complete answers for queries qarr[i], i in idx, computed
    on host threads (the oracle's calls release the interpreter lock):
    i -> ("journeys", records) or, for one-to-all queries, ("rows", base day,
    round-time rows)."""
    from concurrent.futures import ThreadPoolExecutor
    lib()
    threads = threads or max(1, min(32, len(os.sched_getaffinity(0))))

    def one(i):
        q = qarr[i]
        o = OracleResult(desc, q, rt)
        if q.kind == A.B2R_ONE_TO_ALL:
            rows, _, base_day = o.state()
            return i, ("rows", base_day, rows)
        return i, ("journeys", o.records())

    with ThreadPoolExecutor(threads) as ex:
        return dict(ex.map(one, list(idx)))
