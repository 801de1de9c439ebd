"""The Algo concept of nigiri's routing::search<Dir, Algo> over the engine
(include/b2r.hpp: b2r_algo over the C ABI's b2r_raptor, and search<Dir,
Algo> restated from search.h:78-505 over b2r_search_prepare /
b2r_search_extend).  The golden cases of nigiri's routing tests and
generated queries go through search<Dir, b2r_algo> and must give the same
journeys as the golden printouts and as b2r_search_batch (which runs the
whole search on the device)."""
import ctypes as C
import os
import subprocess

import pytest

import fixture as F
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "nigiri_b200")
CASES = F.load_cases()


def build_helper(out_dir):
    so = os.path.join(out_dir, "libalgo_search.so")
    subprocess.check_call([
        "g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-shared", "-fPIC",
        "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "algo_search.cc"),
        "-L" + LIBDIR, "-lb2r", "-Wl,-rpath," + LIBDIR, "-o", so])
    return so


def helper(out_dir):
    A.lib()  # the engine library first, so the helper binds to the same copy
    L = C.CDLL(build_helper(out_dir))
    L.algo_search.argtypes = [C.c_void_p, C.POINTER(A.TimetableDesc), C.POINTER(A.Query), C.POINTER(A.Result)]
    L.algo_search.restype = C.c_int
    return L


def test_algo_helper_builds(tmp_path):
    build_helper(str(tmp_path))


def test_algo_symbols_exported():
    lib = A.lib()
    for name in ("b2r_search_prepare", "b2r_search_extend", "b2r_search_plan_free", "b2r_raptor_create",
                 "b2r_raptor_destroy", "b2r_raptor_reset_arrivals", "b2r_raptor_next_start_time",
                 "b2r_raptor_add_start", "b2r_raptor_execute", "b2r_raptor_reconstruct", "b2r_raptor_rounds"):
        assert hasattr(lib, name), name


@pytest.mark.gpu
def test_golden_cases_through_search_with_b2r_algo(tmp_path):
    """Every golden raptor case (one-to-one, interval and ontrip, both
    directions, intermodal, transfer-time settings, filters, the interval
    extension of the intermodal backward case) through search<Dir,
    b2r_algo>."""
    L = helper(str(tmp_path))
    lib = A.lib()
    n = 0
    for name, spec in CASES["timetables"].items():
        cases = [c for c in CASES["cases"] if c["timetable"] == name
                 and c["query"].get("algorithm", "raptor") == "raptor" and c["query"].get("kind") != "one_to_all"]
        if not cases:
            continue
        ftt = F.FixtureTimetable(spec, lib)
        tt = R.Timetable(ftt.desc, owner=ftt)
        for c in cases:
            q = F.FixtureQuery(lib, ftt, c["query"])
            res = A.Result()
            rc = L.algo_search(tt.handle, C.byref(ftt.desc), C.byref(q.q), C.byref(res))
            assert rc == 0, (c["name"], rc, lib.b2r_last_error())
            assert res.status == 0, c["name"]
            assert F.journeys_to_records(ftt, res) == F.strip_expected(c["expected"]), c["name"]
            n += 1
    assert n >= 80


@pytest.mark.gpu
@pytest.mark.parametrize("workload,n", [(1, 40), (2, 16), (3, 16)])
def test_generated_queries_through_search_with_b2r_algo(tmp_path, workload, n):
    """Generated one-to-one (city, regional intermodal) and range queries:
    search<Dir, b2r_algo> gives the journeys b2r_search_batch gives."""
    L = helper(str(tmp_path))
    lib = A.lib()
    h = HostTimetable.generate(workload)
    tt = R.Timetable(h.desc, owner=h)
    eng = R.Engine(tt, max_slots=64)
    qs = QuerySet(h, workload, n, seed=600 + workload)
    out = (A.Result * qs.n)()
    assert lib.b2r_search_batch(eng.handle, qs.arr, qs.n, out) == 0, lib.b2r_last_error()
    want = [records(out[i]) for i in range(qs.n)]
    n_j = 0
    for i in range(qs.n):
        res = A.Result()
        assert L.algo_search(tt.handle, C.byref(h.desc), C.byref(qs.arr[i]), C.byref(res)) == 0, \
            lib.b2r_last_error()
        assert records(res) == want[i], i
        n_j += len(want[i])
    assert n_j > 0
