"""The C ABI library loads and exports every symbol the headers declare (CPU)."""
import ctypes
import glob
import os
import re
import subprocess

import basements_b200 as bm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    txt = open(header).read()
    return re.findall(r"BM_API\s+[\w\s\*]+?\b(bm_\w+)\s*\(", txt)


def test_headers_declare_functions():
    names = [n for h in glob.glob(os.path.join(ROOT, "include", "*.h")) for n in declared(h)]
    assert "bm_solver_step" in names and "bm_coupler_m1_apply" in names


def test_library_exports_every_declared_symbol():
    L = bm.lib()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        for name in declared(h):
            assert hasattr(L, name), f"{name} declared in {os.path.basename(h)} but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", bm.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert all(n.startswith("bm_") for n in exported), sorted(n for n in exported if not n.startswith("bm_"))


def test_python_bindings_cover_header():
    names = {n for h in glob.glob(os.path.join(ROOT, "include", "*.h")) for n in declared(h)}
    assert names <= set(bm.declared_symbols()) | set(getattr(bm, "EXTRA_SYMBOLS", ())), \
        sorted(names - set(bm.declared_symbols()))


def test_version_and_status_strings():
    L = bm.lib()
    assert L.bm_get_version() == 2
    for code in range(10):
        assert L.bm_status_string(code)
    assert L.bm_status_string(999) == b"unknown status"


def test_argument_validation_without_compute():
    L = bm.lib()
    h = ctypes.c_void_p()
    assert L.bm_solver_create(-1.0, None, ctypes.byref(h)) == 1
    assert L.bm_solver_create(0.1, None, None) == 1
    assert L.bm_solver_step(None, 0.1) == 1
    assert L.bm_solver_destroy(None) == 1
    assert b"dx" in L.bm_last_error() or b"NULL" in L.bm_last_error()


def test_launch_variant_table_pairs_each_shape_with_its_interleaved_twin():
    """The fused kernel's launch variants (host-side table, no device call):
    the shapes, then the same shapes with interleaved lanes ("/i2"); the
    plain solver's default 128x7 is among the first half."""
    names = bm.launch_variants()
    half = len(names) // 2
    assert len(names) == 2 * half and half > 0
    assert all(re.fullmatch(r"\d+x\d+", n) for n in names[:half])
    assert names[half:] == [n + "/i2" for n in names[:half]]
    assert "128x7" in names[:half]
