"""Served request loop (b2r_serve_start / b2r_submit / b2r_wait): queries of
mixed kinds submitted from several threads while others run are admitted
into free slots (continuous batching), and every result equals the result
of the same query run alone."""
import ctypes as C
import random
import threading
import time

import numpy as np
import pytest

from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

pytestmark = pytest.mark.gpu


def result_key(r, n_loc):
    if r.round_times:
        rows = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n_loc,))
        return ("rows", r.status, r.base_day, rows.tobytes())
    return ("journeys", r.status, records(r), r.interval_from, r.interval_to)


def mixed_queries(h):
    one = QuerySet(h, 1, 48, seed=901)   # one-to-one forward
    rng = QuerySet(h, 3, 16, seed=902)   # range, forward and backward
    ota = QuerySet(h, 1, 8, seed=903)    # one-to-all
    arr = (A.Query * (one.n + rng.n + ota.n))()
    keep = [one, rng, ota]
    i = 0
    for qs, kind in ((one, A.B2R_ONE_TO_ONE), (rng, A.B2R_ONE_TO_ONE), (ota, A.B2R_ONE_TO_ALL)):
        for j in range(qs.n):
            arr[i] = qs.arr[j]
            if kind == A.B2R_ONE_TO_ALL:
                arr[i].kind = kind
                arr[i].n_destination = 0
                arr[i].direction = j % 2
            i += 1
    return arr, keep


def test_served_results_equal_results_alone():
    lib = A.lib()
    h = HostTimetable.generate(1)
    tt = R.Timetable(h.desc, owner=h)
    n_loc = h.desc.n_locations
    arr, _keep = mixed_queries(h)
    n = len(arr)
    alone = R.Engine(tt, max_slots=32)
    want = []
    for i in range(n):
        out = A.Result()
        assert lib.b2r_search_batch(alone.handle, C.byref(arr[i]), 1, C.byref(out)) == 0, \
            lib.b2r_last_error()
        want.append(result_key(out, n_loc))
    del alone

    eng = R.Engine(tt, max_slots=32, steps_per_sync=1)  # fewer slots than queries
    srv = R.Server(eng)
    tickets = [None] * n
    order = list(range(n))
    random.Random(7).shuffle(order)

    def client(part):
        rnd = random.Random(part)
        for i in order[part::4]:
            time.sleep(rnd.random() * 0.004)
            tickets[i] = srv.submit_raw(arr[i])

    threads = [threading.Thread(target=client, args=(p,)) for p in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    got = []
    for i in range(n):
        r = srv.wait(tickets[i])
        got.append(result_key(r, n_loc))
        assert r.latency_ms > 0
        srv.release(tickets[i])
    srv.stop()
    st = srv.stats()  # the loop's counters stay readable after the stop
    assert st.super_steps > 0 and st.kernel_launches >= st.super_steps
    assert st.host_export_ms > 0 and st.host_prep_cpu_ms > 0
    for i in range(n):
        assert got[i] == want[i], i
    assert sum(1 for w in want if w[0] == "journeys" and w[2]) > 10


def test_serving_rejects_misuse():
    lib = A.lib()
    h = HostTimetable.generate(1)
    tt = R.Timetable(h.desc, owner=h)
    eng = R.Engine(tt, max_slots=32)
    t = C.c_uint64()
    q = QuerySet(h, 1, 1, seed=5)
    assert lib.b2r_submit(eng.handle, C.byref(q.arr[0]), C.byref(t)) == A.B2R_ERR_INVALID_ARGUMENT
    srv = R.Server(eng)
    assert lib.b2r_serve_start(eng.handle) == A.B2R_ERR_INVALID_ARGUMENT  # already serving
    out = (A.Result * 1)()
    assert lib.b2r_search_batch(eng.handle, q.arr, 1, out) == A.B2R_ERR_INVALID_ARGUMENT
    tk = srv.submit_raw(q.arr[0])
    srv.wait(tk)
    srv.release(tk)
    assert lib.b2r_release(eng.handle, tk) == A.B2R_ERR_INVALID_ARGUMENT  # unknown now
    srv.stop()
    # batch mode works again after the loop stopped
    assert lib.b2r_search_batch(eng.handle, q.arr, 1, out) == A.B2R_OK
