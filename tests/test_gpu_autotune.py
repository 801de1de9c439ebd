"""The launch-shape autotuner: it tries several shapes on a sample, keeps
the fastest, and the journeys do not depend on the shape."""
import ctypes as C

import pytest

from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

pytestmark = pytest.mark.gpu


def run(eng, qs):
    out = (A.Result * qs.n)()
    assert A.lib().b2r_search_batch(eng.handle, qs.arr, qs.n, out) == 0, A.lib().b2r_last_error()
    return [records(out[i]) for i in range(qs.n)]


def test_autotune_keeps_results_and_reports_its_trials():
    h = HostTimetable.generate(1)
    tt = R.Timetable(h.desc, owner=h)
    eng = R.Engine(tt, max_slots=64)
    qs = QuerySet(h, 1, 64, seed=123)
    before = run(eng, qs)
    sample = QuerySet(h, 1, 64, seed=124)
    rep = eng.autotune(sample.arr, sample.n)
    assert rep.n_tried >= 10
    assert rep.best_ms <= rep.start_ms
    sh = eng.shape
    for f, _ in A.LaunchShape._fields_:
        assert getattr(sh, f) == getattr(rep.best, f)
    assert run(eng, qs) == before
    # an odd shape (small blocks, one step per sync) gives the same journeys
    odd = A.LaunchShape(1, 64, 1, 1, 1)
    eng.shape = odd
    assert run(eng, qs) == before
    bad = A.LaunchShape(8, 100, 8, 4, 4)  # not a multiple of 32
    assert A.lib().b2r_engine_set_shape(eng.handle, C.byref(bad)) == A.B2R_ERR_INVALID_ARGUMENT
