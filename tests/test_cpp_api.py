"""The C++ mirror of nigiri's routing interface (include/b2r.hpp) compiles
and links against the engine library, and its parity harness
(tests/cpp/raptor_search_test.cc) matches the CPU oracle on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "nigiri_b200")
ORACLE = os.path.join(ROOT, "oracle")


def build_harness(out_dir):
    exe = os.path.join(out_dir, "raptor_search_test")
    subprocess.check_call([
        "g++", "-std=c++20", "-O2", "-Wall", "-Wextra",
        "-I" + os.path.join(ROOT, "include"), "-I" + ORACLE,
        os.path.join(ROOT, "tests", "cpp", "raptor_search_test.cc"),
        "-L" + LIBDIR, "-lb2r", "-L" + ORACLE, "-loracle",
        "-Wl,-rpath," + LIBDIR, "-Wl,-rpath," + ORACLE, "-o", exe])
    return exe


def test_header_and_harness_build(tmp_path):
    build_harness(str(tmp_path))


@pytest.mark.gpu
def test_cpp_harness_matches_oracle(tmp_path):
    exe = build_harness(str(tmp_path))
    out = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout[-4000:] + out.stderr[-2000:]
    assert out.stdout.strip().endswith("ok")
