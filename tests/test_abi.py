"""The C ABI library loads without a GPU and exports every entry point that
include/b2r.h declares; the ctypes mirror matches the C struct layouts."""
import ctypes as C
import os
import re
import subprocess
import tempfile

from nigiri_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "b2r.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(b2r_[a-z0-9_]+)\s*\(", src)) - {"b2r_"})


def test_library_exports_every_declared_entry_point():
    lib = C.CDLL(A.LIB_PATH)
    missing = [f for f in declared_functions() if not hasattr(lib, f)]
    assert not missing, missing
    assert set(declared_functions()) == set(A.EXPORTS)


def test_struct_layouts_match_c():
    code = r'''
#include <stdio.h>
#include <stddef.h>
#include "b2r.h"
int main() {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(b2r_timetable_desc), sizeof(b2r_offset),
         sizeof(b2r_query), sizeof(b2r_leg), sizeof(b2r_journey), sizeof(b2r_result),
         sizeof(b2r_engine_config), sizeof(b2r_batch_stats), sizeof(b2r_tt_base),
         sizeof(b2r_launch_shape), sizeof(b2r_tune_report), sizeof(b2r_gtfs_config));
  printf("%zu %zu\n", sizeof(b2r_rt_desc), offsetof(b2r_leg, rt_transport));
  printf("%zu %zu %zu\n", offsetof(b2r_query, tts_factor), offsetof(b2r_leg, transport_mode_id),
         offsetof(b2r_result, n_start_times));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(src, "w").write(code)
        subprocess.check_call(["gcc", "-I" + os.path.join(ROOT, "include"), src, "-o", exe])
        out = subprocess.check_output([exe]).decode().split("\n")
    sizes = [int(x) for x in out[0].split()]
    assert sizes == [C.sizeof(A.TimetableDesc), C.sizeof(A.Offset), C.sizeof(A.Query),
                     C.sizeof(A.Leg), C.sizeof(A.Journey), C.sizeof(A.Result),
                     C.sizeof(A.EngineConfig), C.sizeof(A.BatchStats), C.sizeof(A.TtBase),
                     C.sizeof(A.LaunchShape), C.sizeof(A.TuneReport), C.sizeof(A.GtfsConfig)]
    rt = [int(x) for x in out[1].split()]
    assert rt == [C.sizeof(A.RtDesc), A.Leg.rt_transport.offset]
    offs = [int(x) for x in out[2].split()]
    assert offs == [A.Query.tts_factor.offset, A.Leg.transport_mode_id.offset,
                    A.Result.n_start_times.offset]


def test_errors_without_gpu_are_status_codes():
    lib = A.lib()
    assert lib.b2r_engine_create(None, None, None) == -1
    assert b"null" in lib.b2r_last_error()
    assert lib.b2r_search_batch(None, None, 0, None) == -1


def test_noalloc_limits_match_header_and_null_arguments_are_rejected():
    code = r'''
#include <stdio.h>
#include "b2r.h"
int main() {
  printf("%u %u %u %u\n", B2R_NOALLOC_MAX_LOCATIONS, B2R_NOALLOC_MAX_ROUTES,
         B2R_NOALLOC_MAX_OFFSETS, B2R_NOALLOC_SCRATCH_BYTES);
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(src, "w").write(code)
        subprocess.check_call(["gcc", "-I" + os.path.join(ROOT, "include"), src, "-o", exe])
        got = [int(x) for x in subprocess.check_output([exe]).split()]
    assert got == [A.B2R_NOALLOC_MAX_LOCATIONS, A.B2R_NOALLOC_MAX_ROUTES,
                   A.B2R_NOALLOC_MAX_OFFSETS, A.B2R_NOALLOC_SCRATCH_BYTES]
    lib = A.lib()
    n_rows = C.c_uint32()
    assert lib.b2r_one_to_all_noalloc(None, None, None, 0, C.byref(n_rows), None, None) == \
        A.B2R_ERR_INVALID_ARGUMENT
    assert b"null" in lib.b2r_last_error()


def test_serving_entry_points_reject_null_engine():
    lib = A.lib()
    t = C.c_uint64()
    r = A.Result()
    assert lib.b2r_serve_start(None) == A.B2R_ERR_INVALID_ARGUMENT
    assert lib.b2r_serve_stop(None) == A.B2R_ERR_INVALID_ARGUMENT
    assert lib.b2r_submit(None, None, C.byref(t)) == A.B2R_ERR_INVALID_ARGUMENT
    assert lib.b2r_poll(None, 1, C.byref(r)) == A.B2R_ERR_INVALID_ARGUMENT
    assert lib.b2r_wait(None, 1, C.byref(r)) == A.B2R_ERR_INVALID_ARGUMENT
    assert lib.b2r_release(None, 1) == A.B2R_ERR_INVALID_ARGUMENT


def test_launch_shape_entry_points_reject_null():
    lib = A.lib()
    sh = A.LaunchShape()
    assert lib.b2r_engine_get_shape(None, C.byref(sh)) == A.B2R_ERR_INVALID_ARGUMENT
    assert lib.b2r_engine_set_shape(None, C.byref(sh)) == A.B2R_ERR_INVALID_ARGUMENT
    assert lib.b2r_engine_autotune(None, None, 0, None) == A.B2R_ERR_INVALID_ARGUMENT
