"""The C ABI from C++ without Python: tests/c_abi/coupler_table.cpp binds the
five couplers through one function-pointer table in the style of the
reference's research harness (bench_compare_all.cpp:50-70). It is compiled
and linked against include/bm_mpm.h and basements_b200/libbm_mpm.so here
(CPU) and run on a GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "basements_b200")


def build(tmpdir):
    exe = os.path.join(str(tmpdir), "coupler_table")
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "c_abi", "coupler_table.cpp"), "-L" + LIBDIR, "-lbm_mpm",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_c_program_builds_and_links(tmp_path):
    if not os.path.exists(os.path.join(LIBDIR, "libbm_mpm.so")):
        pytest.skip("libbm_mpm.so not built")
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_c_program_runs_every_coupler(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("nodes inside") == 5
