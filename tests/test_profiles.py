"""Footpath profiles (query::prf_idx_, routing/query.h:90): per-profile
footpaths and lower-bound graphs (timetable.h:97-98, 421-422), and for the
wheelchair profile the stops' wheelchair bits in the route scan, start
times and direct journeys plus the wheelchair-accessible route filter
(raptor.h:251-257, 1252, 1304; start_times.cc:155-160; direct.cc:440-450,
503-513).  Reconstruction reads the plain bits for every profile, as
reconstruct.cc:252-253 does.

CPU: the generated wheelchair data, the oracle's wheelchair journeys, and
the rejected profile index.  GPU: the engine against the oracle for profile
2 (one-to-one both directions, intermodal, ranges, pong, one-to-all, the
no-allocation path) and for a profile without footpaths."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200.timetable import HostTimetable, QuerySet

WC = A.B2R_PROFILE_WHEELCHAIR


def with_profile(arr, n, prf, kind=None):
    out = (A.Query * n)()
    for i in range(n):
        out[i] = arr[i]
        out[i].prf_idx = prf
        if kind is not None:
            out[i].kind = kind
    return out


@pytest.fixture(scope="module")
def tt1():
    return HostTimetable.generate(1)


def test_generated_wheelchair_data(tt1):
    """About a fifth of the stops lack the wheelchair bits, and the
    wheelchair profile has its own footpaths and lower-bound graphs."""
    d = tt1.desc
    rsi = np.ctypeslib.as_array(d.route_stop_index, shape=(d.n_routes + 1,))
    words = np.ctypeslib.as_array(d.route_stops, shape=(int(rsi[-1]),)).astype(np.uint64)
    plain_in = (words >> 28) & 1
    wc_in = (words >> 30) & 1
    assert plain_in.all()
    share = 1.0 - wc_in.mean()
    assert 0.1 < share < 0.3, share
    p = WC - 1
    assert bool(d.profile_footpaths_out_index[p]) and bool(d.profile_footpaths_in_index[p])
    assert bool(d.profile_lb_fwd_index[p]) and bool(d.profile_lb_bwd_index[p])
    n = d.n_locations
    n0 = int(d.footpaths_out_index[n])
    n2 = int(d.profile_footpaths_out_index[p][n])
    assert 0 < n2 < n0
    for prf in (1, 3, 4):  # no footpaths in the other profiles
        assert not bool(d.profile_footpaths_out_index[prf - 1])


def test_oracle_wheelchair_journeys_differ_from_default(tt1):
    """Wheelchair searches find journeys, and not the same ones as the
    default profile for every query."""
    qs = QuerySet(tt1, 1, 40, seed=808)
    wc = with_profile(qs.arr, qs.n, WC)
    found = differ = 0
    for i in range(qs.n):
        r0 = oracle_lib.OracleResult(tt1.desc, qs.arr[i]).records()
        r2 = oracle_lib.OracleResult(tt1.desc, wc[i]).records()
        found += len(r2) > 0
        differ += r0 != r2
    assert found >= 8 and differ > 5, (found, differ)


def test_oracle_rejects_profile_out_of_range(tt1):
    qs = QuerySet(tt1, 1, 1, seed=1)
    q = with_profile(qs.arr, 1, A.B2R_N_PROFILES)[0]
    h = C.c_void_p()
    assert oracle_lib.lib().or_search(C.byref(tt1.desc), C.byref(q), C.byref(h)) == A.B2R_ERR_INVALID_ARGUMENT


# ------------------------------------------------------------------ GPU

@pytest.fixture(scope="module")
def engines():
    from nigiri_b200 import routing as R
    out = {}
    for w in (1, 2):
        h = HostTimetable.generate(w)
        dtt = R.Timetable(h.desc, owner=h)
        out[w] = (h, dtt, R.Engine(dtt, max_slots=128))
    return out


def batch(eng, qarr, n):
    out = (A.Result * n)()
    assert A.lib().b2r_search_batch(eng.handle, qarr, n, out) == 0, A.lib().b2r_last_error()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("workload,kind", [(1, 1), (2, 2), (1, 3)], ids=["w1_station", "w2_intermodal", "w1_range"])
def test_wheelchair_queries_match_oracle(engines, workload, kind):
    h, _, eng = engines[workload]
    qs = QuerySet(h, kind, 48, seed=900 + workload + kind)
    arr = with_profile(qs.arr, qs.n, WC)
    for i in range(qs.n):
        arr[i].direction = i % 2
    out = batch(eng, arr, qs.n)
    n_j = 0
    for i in range(qs.n):
        exp = oracle_lib.OracleResult(h.desc, arr[i])
        assert out[i].status == A.B2R_OK, i
        assert records(out[i]) == exp.records(), i
        n_j += out[i].n_journeys
    assert n_j > 8


@pytest.mark.gpu
def test_wheelchair_pong_matches_oracle(engines):
    h, _, eng = engines[1]
    qs = QuerySet(h, 3, 24, seed=931)
    arr = with_profile(qs.arr, qs.n, WC)
    for i in range(qs.n):
        arr[i].algorithm = A.B2R_ALGO_PONG
        arr[i].use_start_footpaths = 1
    out = batch(eng, arr, qs.n)
    for i in range(qs.n):
        exp = oracle_lib.OracleResult(h.desc, arr[i])
        assert out[i].status == A.B2R_OK, i
        assert records(out[i]) == exp.records(), i


@pytest.mark.gpu
def test_wheelchair_one_to_all_rows_match_oracle(engines):
    """Batched one-to-all and the no-allocation path give the oracle's
    round-time rows for the wheelchair profile."""
    h, dtt, eng = engines[1]
    qs = QuerySet(h, 1, 6, seed=944)
    arr = with_profile(qs.arr, qs.n, WC, kind=A.B2R_ONE_TO_ALL)
    for i in range(qs.n):
        arr[i].n_destination = 0
        arr[i].direction = i % 2
    out = batch(eng, arr, qs.n)
    n = h.desc.n_locations
    lib = A.lib()
    for i in range(qs.n):
        r = out[i]
        got = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n,)).reshape(r.n_rows, n)
        rows, _, _ = oracle_lib.OracleResult(h.desc, arr[i]).state()
        assert np.array_equal(got, rows[: r.n_rows]), i
        buf = np.full(got.size, 12345, dtype=np.int16)
        n_rows, base_day = C.c_uint32(), C.c_int32()
        rc = lib.b2r_one_to_all_noalloc(dtt.handle, C.byref(arr[i]), buf.ctypes.data_as(C.POINTER(C.c_int16)),
                                        buf.size, C.byref(n_rows), C.byref(base_day), None)
        assert rc == A.B2R_OK, lib.b2r_last_error()
        assert np.array_equal(buf.reshape(r.n_rows, n), got), i


@pytest.mark.gpu
def test_profile_without_footpaths_and_bad_profile(engines):
    """A profile with no footpaths and no lower-bound graph (the foot
    profile here) gives the oracle's answers; an index past the last profile
    is an invalid argument."""
    h, _, eng = engines[1]
    qs = QuerySet(h, 1, 8, seed=955)
    arr = with_profile(qs.arr, qs.n, A.B2R_PROFILE_WHEELCHAIR - 1)
    arr[qs.n - 1].prf_idx = A.B2R_N_PROFILES
    out = batch(eng, arr, qs.n)
    for i in range(qs.n - 1):
        assert records(out[i]) == oracle_lib.OracleResult(h.desc, arr[i]).records(), i
    assert out[qs.n - 1].status == A.B2R_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
@pytest.mark.parametrize("prf", [0, WC])
def test_wheelchair_assistance_golden_on_gpu(prf):
    """nigiri's wheelchair_assistance_test.cc restated as a fixture (the
    assistance hours turned into the stop times' wheelchair bits): the
    engine's first and last departures are the test's, and every journey is
    the oracle's."""
    import fixture as F
    from nigiri_b200 import routing as R
    cases = F.load_cases()
    ka = next(k for k in cases["known_answers"] if k["name"] == f"wheelchair_assistance_prf{prf}")
    ftt = F.FixtureTimetable(cases["timetables"][ka["timetable"]], A.lib())
    tt = R.Timetable(ftt.desc, owner=ftt)
    eng = R.Engine(tt, max_slots=32)
    q = F.FixtureQuery(A.lib(), ftt, ka["query"])
    out = A.Result()
    assert A.lib().b2r_search_batch(eng.handle, C.byref(q.q), 1, C.byref(out)) == 0
    got = F.journeys_to_records(ftt, out)
    deps = sorted(j["dep"] for j in got)
    assert deps and [deps[0], deps[-1]] == ka["expected"]
    ref = oracle_lib.OracleResult(ftt.desc, q.q)  # owns the records its view points to
    assert got == F.journeys_to_records(ftt, ref.view)
