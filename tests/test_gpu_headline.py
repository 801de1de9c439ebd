"""Parity at the benchmarked sizes: the configuration the throughput is
quoted on (the regional 40k-stop timetable, 1,024 resident slots, the
autotuned launch shape, two batches through one engine so that every slot
is reused), 256 range queries of mixed direction and window, and the
200-query national sample, each compared query by query with the CPU
oracle (departure, arrival, transfers and every leg; one-to-all: every
round-time row).  The pattern is nigiri's own CPU-against-GPU gate
(exe/benchmark.cc:702-713, test/raptor_search.cc:49-80)."""
import numpy as np
import pytest

import oracle_lib
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

pytestmark = pytest.mark.gpu


def compare(h, qarr, out, idx):
    """Engine results out[j] for queries qarr[i] (j-th of idx) against the
    oracle; returns (mismatching query indices, journeys seen)."""
    want = oracle_lib.answers(h.desc, qarr, idx)
    n_loc = h.desc.n_locations
    bad, n_j = [], 0
    for j, i in enumerate(idx):
        r = out[j]
        w = want[i]
        if w[0] == "rows":
            got = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n_loc,)).reshape(r.n_rows, n_loc)
            ok = r.base_day == w[1] and np.array_equal(got, w[2][: r.n_rows])
        else:
            ok = r.status == 0 and records(r) == w[1]
            n_j += len(w[1])
        if not ok:
            bad.append(i)
    return bad, n_j


@pytest.fixture(scope="module")
def regional():
    h = HostTimetable.generate(2)
    return h, R.Timetable(h.desc, owner=h)


def test_regional_1024_slots_tuned_shape_two_batches_match_oracle(regional):
    """The benchmarked configuration: queries from the bench's generator
    seed, the shape the autotuner picks on a separate sample, two batches
    of 1,024 through the same 1,024-slot engine."""
    h, tt = regional
    lib = A.lib()
    eng = R.Engine(tt, max_slots=1024)
    tune_qs = QuerySet(h, 2, 1024, seed=9002)
    eng.autotune(tune_qs.arr, tune_qs.n)
    qs = QuerySet(h, 2, 2048, seed=1002)
    n_j = 0
    for b in range(2):
        idx = list(range(b * 1024, (b + 1) * 1024))
        arr = qs.subset(idx)
        out = (A.Result * 1024)()
        assert lib.b2r_search_batch(eng.handle, arr, 1024, out) == 0, lib.b2r_last_error()
        bad, nj = compare(h, qs.arr, out, idx)
        assert bad == [], f"batch {b}: {len(bad)} queries differ, first {bad[:5]}"
        n_j += nj
    assert n_j > 2048


def test_regional_range_256_mixed_match_oracle(regional):
    """256 range queries: windows of 30-240 minutes, both directions, in one
    batch."""
    h, tt = regional
    lib = A.lib()
    eng = R.Engine(tt, max_slots=256)
    qs = QuerySet(h, 3, 256, seed=1003)
    out = (A.Result * qs.n)()
    assert lib.b2r_search_batch(eng.handle, qs.arr, qs.n, out) == 0, lib.b2r_last_error()
    bad, n_j = compare(h, qs.arr, out, list(range(qs.n)))
    assert bad == [], f"{len(bad)} range queries differ, first {bad[:5]}"
    assert {qs.arr[i].direction for i in range(qs.n)} == {0, 1}
    assert n_j > 256


def test_national_200_sample_matches_oracle():
    """The national timetable's 200-query sample of the mixed batches
    (one-to-one, 1 h range, one-to-all) on a 256-slot engine."""
    h = HostTimetable.generate(4)
    tt = R.Timetable(h.desc, owner=h)
    lib = A.lib()
    eng = R.Engine(tt, max_slots=256)
    qs = QuerySet(h, 4, 200, seed=2004)
    out = (A.Result * qs.n)()
    assert lib.b2r_search_batch(eng.handle, qs.arr, qs.n, out) == 0, lib.b2r_last_error()
    bad, n_j = compare(h, qs.arr, out, list(range(qs.n)))
    assert bad == [], f"{len(bad)} national queries differ, first {bad[:5]}"
    kinds = {(qs.arr[i].kind, qs.arr[i].is_interval) for i in range(qs.n)}
    assert len(kinds) == 3
    assert n_j > 50
