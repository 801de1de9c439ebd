"""b2r_one_to_all_noalloc (one-to-all search of one query in a fixed device
array, no allocation) returns exactly the rows of b2r_search_batch for the
same one-to-all queries, on two calls in a row, and rejects inputs beyond
its stated limits.  It serves callers that cannot allocate device memory
while they answer a query (their HBM belongs to another allocator, or
cudaFree's device-wide synchronisation would stall their other streams), so
the device's free memory must not change over repeated calls.  Collected
last so that it also runs after every other GPU test in the same process."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import fixture as F  # noqa: E402
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

pytestmark = pytest.mark.gpu


# (allowed classes, bikes, no reservation): not bus; bikes; tram or bus
# without compulsory reservation
FILTERS = [(0xFFFF & ~(1 << 10), 0, 0), (0xFFFF, 1, 0), ((1 << 10) | (1 << 9), 0, 1)]


def one_to_all_queries(h, n, seed, filters=False):
    qs = QuerySet(h, 1, n, seed=seed)
    arr = (A.Query * qs.n)()
    for i in range(qs.n):
        arr[i] = qs.arr[i]
        arr[i].kind = A.B2R_ONE_TO_ALL
        arr[i].n_destination = 0
        arr[i].direction = i % 2
        if filters:
            mask, bikes, resv = FILTERS[i % len(FILTERS)]
            arr[i].allowed_claszes = mask
            arr[i].require_bike_transport = bikes
            arr[i].no_compulsory_reservation = resv
    return qs, arr


def one_to_all_profile_queries(h, n, seed, prf):
    qs, arr = one_to_all_queries(h, n, seed)
    for i in range(qs.n):
        arr[i].prf_idx = prf
    return qs, arr


def noalloc_rows(lib, tt, q, n_loc):
    n_rows_max = A.B2R_MAX_TRANSFERS + 2
    buf = np.full(n_rows_max * n_loc, 12345, dtype=np.int16)
    n_rows = C.c_uint32()
    base_day = C.c_int32()
    rc = lib.b2r_one_to_all_noalloc(tt.handle, C.byref(q),
                                    buf.ctypes.data_as(C.POINTER(C.c_int16)), buf.size,
                                    C.byref(n_rows), C.byref(base_day), None)
    assert rc == A.B2R_OK, lib.b2r_last_error()
    return buf[: n_rows.value * n_loc].reshape(n_rows.value, n_loc), base_day.value


def compare_with_batched(lib, tt, eng, arr, n_q, n):
    """Rows of two no-allocation calls in a row against b2r_search_batch's;
    returns the number of labels beyond the starts."""
    out = (A.Result * n_q)()
    assert lib.b2r_search_batch(eng.handle, arr, n_q, out) == A.B2R_OK, lib.b2r_last_error()
    reached = 0
    for i in range(n_q):
        r = out[i]
        want = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n,)).reshape(r.n_rows, n)
        for call in range(2):
            got, base_day = noalloc_rows(lib, tt, arr[i], n)
            assert base_day == r.base_day, (i, call)
            assert got.shape == want.shape, (i, call)
            assert np.array_equal(got, want), (i, call)
        invalid = 32767 if arr[i].direction == A.B2R_FORWARD else -32768
        reached += int((want[1:] != invalid).sum())
    return reached


@pytest.mark.parametrize("workload,filters", [(1, False), (2, False), (2, True)],
                         ids=["w1", "w2", "w2_filters"])
def test_noalloc_rows_equal_batched_rows_on_two_calls_in_a_row(workload, filters):
    lib = A.lib()
    h = HostTimetable.generate(workload)
    tt = R.Timetable(h.desc, owner=h)
    eng = R.Engine(tt, max_slots=64)
    qs, arr = one_to_all_queries(h, 6, seed=40 + workload, filters=filters)
    out = (A.Result * qs.n)()
    assert lib.b2r_search_batch(eng.handle, arr, qs.n, out) == A.B2R_OK, lib.b2r_last_error()
    n = h.desc.n_locations
    reached = 0
    for i in range(qs.n):
        r = out[i]
        want = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n,)).reshape(r.n_rows, n)
        for call in range(2):
            got, base_day = noalloc_rows(lib, tt, arr[i], n)
            assert base_day == r.base_day, (i, call)
            assert got.shape == want.shape, (i, call)
            assert np.array_equal(got, want), (i, call)
        invalid = 32767 if arr[i].direction == A.B2R_FORWARD else -32768
        reached += int((want[1:] != invalid).sum())
    assert reached > 0  # the rows hold labels beyond the starts


def test_noalloc_rejects_inputs_beyond_its_limits():
    lib = A.lib()
    h = HostTimetable.generate(1)
    tt = R.Timetable(h.desc, owner=h)
    qs, arr = one_to_all_queries(h, 1, seed=3)
    q = arr[0]
    n = h.desc.n_locations
    n_rows = C.c_uint32()
    small = np.zeros(n, dtype=np.int16)  # one row: too small
    rc = lib.b2r_one_to_all_noalloc(tt.handle, C.byref(q), small.ctypes.data_as(C.POINTER(C.c_int16)),
                                    small.size, C.byref(n_rows), None, None)
    assert rc == A.B2R_ERR_CAPACITY
    assert b"round_times holds" in lib.b2r_last_error()
    offs = (A.Offset * (A.B2R_NOALLOC_MAX_OFFSETS + 1))()
    for i in range(len(offs)):
        offs[i].target = q.start[0].target
    q.start = offs
    q.n_start = len(offs)
    buf = np.zeros((A.B2R_MAX_TRANSFERS + 2) * n, dtype=np.int16)
    rc = lib.b2r_one_to_all_noalloc(tt.handle, C.byref(q), buf.ctypes.data_as(C.POINTER(C.c_int16)),
                                    buf.size, C.byref(n_rows), None, None)
    assert rc == A.B2R_ERR_CAPACITY
    assert b"start offsets" in lib.b2r_last_error()
    q.kind = A.B2R_ONE_TO_ONE
    q.n_start = 1
    rc = lib.b2r_one_to_all_noalloc(tt.handle, C.byref(q), buf.ctypes.data_as(C.POINTER(C.c_int16)),
                                    buf.size, C.byref(n_rows), None, None)
    assert rc == A.B2R_ERR_INVALID_ARGUMENT


def test_noalloc_wheelchair_profile_rows_equal_batched_rows():
    """The wheelchair profile (its footpaths, stop bits and route filter)."""
    lib = A.lib()
    h = HostTimetable.generate(1)
    tt = R.Timetable(h.desc, owner=h)
    eng = R.Engine(tt, max_slots=64)
    qs, arr = one_to_all_profile_queries(h, 6, 77, A.B2R_PROFILE_WHEELCHAIR)
    assert compare_with_batched(lib, tt, eng, arr, qs.n, h.desc.n_locations) > 0


@pytest.mark.parametrize("mode", ["exact", "only_children", "equivalent"])
def test_noalloc_match_modes_on_parent_stations(mode):
    """Starts at parent stations (the feed of nigiri's dijkstra test: C and D
    have two tracks each) in every start match mode, both directions."""
    lib = A.lib()
    ftt = F.FixtureTimetable(F.load_cases()["timetables"]["gtfs_dijkstra"], lib)
    tt = R.Timetable(ftt.desc, owner=ftt)
    eng = R.Engine(tt, max_slots=32)
    specs = [(["D"], "fwd", 28630500), (["C"], "bwd", 28630800), (["D", "A"], "fwd", 28630400),
             (["C1"], "bwd", 28630800)]
    qs = []
    for starts, direction, t in specs:
        qs.append(F.FixtureQuery(lib, ftt, {"start": [[x, 0, 0] for x in starts], "start_time": t,
                                            "direction": direction, "start_mode": mode,
                                            "kind": "one_to_all"}))
    arr = (A.Query * len(qs))()
    for i, q in enumerate(qs):
        arr[i] = q.q
    n = ftt.desc.n_locations
    assert compare_with_batched(lib, tt, eng, arr, len(qs), n) > 0


def test_noalloc_calls_allocate_no_device_memory():
    """After a first call (the per-device set-up), repeated calls leave the
    device's free memory where it was: no allocation and no leak."""
    import torch
    lib = A.lib()
    h = HostTimetable.generate(2)
    tt = R.Timetable(h.desc, owner=h)
    qs, arr = one_to_all_queries(h, 8, seed=91)
    n = h.desc.n_locations
    noalloc_rows(lib, tt, arr[0], n)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for rep in range(3):
        for i in range(qs.n):
            noalloc_rows(lib, tt, arr[i], n)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
