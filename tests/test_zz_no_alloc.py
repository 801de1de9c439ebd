"""b2r_one_to_all_noalloc (one-to-all search of one query in a fixed device
array, no allocation) returns exactly the rows of b2r_search_batch for the
same one-to-all queries, on two calls in a row, and rejects inputs beyond
its stated limits.  Collected last so that it also runs after every other
GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

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
