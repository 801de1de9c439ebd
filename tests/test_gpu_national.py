"""National-scale timetable (300k stops, 2.7M transports, stay-seated chain
routes): a mixed batch of one-to-one, range and one-to-all queries matches
the CPU oracle.  The all-pairs lower-bound tables do not fit at this size,
so the engine runs without bounds while the oracle prunes with the
reference's Dijkstra; the journeys must still be identical."""
import numpy as np
import pytest

import oracle_lib
from journeys import records
from nigiri_b200 import _abi as A
from nigiri_b200 import routing as R
from nigiri_b200.timetable import HostTimetable, QuerySet

pytestmark = pytest.mark.gpu


def test_national_sample_matches_oracle():
    lib = A.lib()
    h = HostTimetable.generate(4)
    tt = R.Timetable(h.desc, owner=h)
    eng = R.Engine(tt, max_slots=64)
    qs = QuerySet(h, 4, 40, seed=1004)
    out = (A.Result * qs.n)()
    assert lib.b2r_search_batch(eng.handle, qs.arr, qs.n, out) == 0, lib.b2r_last_error()
    n_loc = h.desc.n_locations
    kinds = set()
    n_j = 0
    for i in range(qs.n):
        q = qs.arr[i]
        o = oracle_lib.OracleResult(h.desc, q)
        if q.kind == A.B2R_ONE_TO_ALL:
            rows, _, base_day = o.state()
            r = out[i]
            got = np.ctypeslib.as_array(r.round_times, shape=(r.n_rows * n_loc,)).reshape(r.n_rows, n_loc)
            assert r.base_day == base_day, i
            assert np.array_equal(got, rows[: r.n_rows]), i
            kinds.add("one_to_all")
        else:
            exp = o.records()
            assert records(out[i]) == exp, i
            n_j += len(exp)
            kinds.add("range" if q.is_interval else "one_to_one")
    assert kinds == {"one_to_one", "range", "one_to_all"}
    assert n_j > 10
