"""Synthetic timetable invariants and finalize() derivations, recomputed
independently with numpy on workload 1."""
import ctypes as C

import numpy as np
import pytest

from nigiri_b200 import _abi as A
from nigiri_b200.timetable import HostTimetable, QuerySet


def arr(ptr, n, dtype):
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype).copy() if n else np.zeros(0, dtype)


@pytest.fixture(scope="module")
def tt1():
    return HostTimetable.generate(1)


def test_generation_is_deterministic(tt1):
    other = HostTimetable.generate(1)
    a, b = tt1.desc, other.desc
    assert (a.n_locations, a.n_routes, a.n_transports, a.n_route_stop_times) == \
           (b.n_locations, b.n_routes, b.n_transports, b.n_route_stop_times)
    st_a = arr(a.route_stop_times, a.n_route_stop_times, np.uint16)
    st_b = arr(b.route_stop_times, b.n_route_stop_times, np.uint16)
    assert np.array_equal(st_a, st_b)


def test_event_columns_ordered_by_minutes_after_midnight(tt1):
    """nigiri's route rule (loader/get_index.h): at every stop the transports
    of a route are ordered by minutes after midnight."""
    d = tt1.desc
    rsi = arr(d.route_stop_index, d.n_routes + 1, np.int64)
    tf = arr(d.route_transport_from, d.n_routes, np.int64)
    tt_ = arr(d.route_transport_to, d.n_routes, np.int64)
    sf = arr(d.route_stop_time_from, d.n_routes, np.int64)
    st = arr(d.route_stop_times, d.n_route_stop_times, np.int64)
    crossing = 0
    for r in range(d.n_routes):
        n_t, n_s = tt_[r] - tf[r], rsi[r + 1] - rsi[r]
        block = st[sf[r]: sf[r] + n_t * 2 * (n_s - 1)].reshape(2 * (n_s - 1), n_t)
        mam = block >> 5
        assert np.all(np.diff(mam, axis=1) >= 0)
        crossing += int(np.any((block & 31) > 0))
    assert crossing > 0  # some trips run past midnight


def test_footpaths_in_is_transpose_of_out(tt1):
    d = tt1.desc
    n = d.n_locations
    oi = arr(d.footpaths_out_index, n + 1, np.int64)
    od = arr(d.footpaths_out, oi[-1], np.uint32)
    ii = arr(d.footpaths_in_index, n + 1, np.int64)
    idd = arr(d.footpaths_in, ii[-1], np.uint32)
    out_edges = sorted((l, int(w & 0x7FFFFF), int(w >> 23)) for l in range(n) for w in od[oi[l]:oi[l + 1]])
    in_edges = sorted((int(w & 0x7FFFFF), l, int(w >> 23)) for l in range(n) for w in idd[ii[l]:ii[l + 1]])
    assert out_edges == in_edges
    for l in range(n):
        durs = idd[ii[l]:ii[l + 1]] >> 23
        assert np.all(np.diff(durs.astype(np.int64)) >= 0)


def test_location_routes_and_route_days(tt1):
    d = tt1.desc
    n = d.n_locations
    rsi = arr(d.route_stop_index, d.n_routes + 1, np.int64)
    rs = arr(d.route_stops, rsi[-1], np.uint32)
    lri = arr(d.location_routes_index, n + 1, np.int64)
    lr = arr(d.location_routes, lri[-1], np.uint32)
    expect = [set() for _ in range(n)]
    for r in range(d.n_routes):
        for w in rs[rsi[r]:rsi[r + 1]]:
            expect[int(w & 0x0FFFFFFF)].add(r)
    for l in range(n):
        assert list(lr[lri[l]:lri[l + 1]]) == sorted(expect[l])
    # route traffic days = union of transport days shifted by their day offsets
    bf = arr(d.bitfields, 8 * d.n_bitfields, np.uint64).reshape(-1, 8)
    tf = arr(d.route_transport_from, d.n_routes, np.int64)
    tt_ = arr(d.route_transport_to, d.n_routes, np.int64)
    sf = arr(d.route_stop_time_from, d.n_routes, np.int64)
    st = arr(d.route_stop_times, d.n_route_stop_times, np.int64)
    tbf = arr(d.transport_traffic_days, d.n_transports, np.int64)
    rbf = arr(d.route_traffic_days, d.n_routes, np.int64)

    def bits(b):
        return {w * 64 + i for w in range(8) for i in range(64) if (int(b[w]) >> i) & 1}
    for r in range(0, d.n_routes, 7):
        n_t, n_s = tt_[r] - tf[r], rsi[r + 1] - rsi[r]
        block = st[sf[r]: sf[r] + n_t * 2 * (n_s - 1)].reshape(2 * (n_s - 1), n_t)
        want = set()
        for j in range(n_t):
            md = int((block[:, j] & 31).max())
            for x in bits(bf[tbf[tf[r] + j]]):
                want |= {x + dd for dd in range(md + 1) if x + dd < 512}
        assert bits(bf[rbf[r]]) == want


def test_query_streams(tt1):
    qs = QuerySet(tt1, 1, 50)
    assert qs.n == 50
    for i in range(qs.n):
        q, direction, kind = qs.to_query(i)
        assert direction == "fwd" and kind == 0 and q.max_transfers == 7
        assert q.start[0].target != q.destination[0].target
