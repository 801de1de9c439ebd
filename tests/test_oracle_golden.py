"""The CPU oracle against the golden journey printouts of nigiri's own
routing tests (tests/golden/cases.json, made by make_fixtures.py)."""
import ctypes as C

import pytest

import fixture as F
import oracle_lib
from nigiri_b200 import _abi as A

CASES = F.load_cases()


@pytest.fixture(scope="module")
def timetables():
    lib = A.lib()
    return {k: F.FixtureTimetable(v, lib) for k, v in CASES["timetables"].items()}


@pytest.mark.parametrize("case", CASES["cases"], ids=[c["name"] for c in CASES["cases"]])
def test_oracle_matches_golden(case, timetables):
    tt = timetables[case["timetable"]]
    q = F.FixtureQuery(A.lib(), tt, case["query"])
    r = oracle_lib.OracleResult(tt.desc, q.q)
    assert F.journeys_to_records(tt, r.view) == F.strip_expected(case["expected"])


def test_golden_cases_cover_both_directions_and_intermodal():
    names = [c["name"] for c in CASES["cases"]]
    assert any("backward" in n or n.endswith("_bwd") for n in names)
    assert any("intermodal" in n for n in names)
    assert sum(len(c["expected"]) for c in CASES["cases"]) >= 40
