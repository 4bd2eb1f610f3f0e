"""C ABI: the library loads and exports every entry point the header declares
(no GPU needed; only functions that do no device work are called)."""
import ctypes
import os
import re

import numpy as np

import dmhm_b200 as D
from dmhm_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "dmhm_b200.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"HM_API\s+[\w\s\*]+?\b(hm_\w+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) >= 10
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared()) == set(_lib.SIGNATURES)


def test_map_matches_oracle():
    from oracle import dmhm_oracle as O
    for sizes, L in [((32, 32), 4), ((24, 20), 3), ((16, 16, 16), 3), ((6, 10, 4), 2),
                     ((1, 7), 2), ((48, 48), 5)]:
        a = D.natural_to_hierarchical_map(sizes, L)
        b = O.natural_to_hierarchical_map(sizes, L)
        assert (a == b).all(), sizes


def test_errors_are_reported():
    sizes = (ctypes.c_int * 2)(4, 4)
    out = (ctypes.c_int * 16)()
    st = _lib.lib().hm_natural_to_hierarchical_map(5, sizes, 2, out)
    assert st == 1
    assert b"dim" in _lib.lib().hm_last_error()


def test_stencil_operator_matches_oracle():
    from oracle import dmhm_oracle as O
    for sizes, L in [((32, 32), 4), ((8, 6, 4), 2)]:
        c = D.operators.uniform_coefficients(sizes, 3)
        S = D.operators.stencil(sizes, c, L)
        r, cc, v, _ = O.stencil_csr(sizes, c, L)
        assert (S.rowOffsets == r).all() and (S.columnIndices == cc).all()
        assert np.array_equal(S.nonzeros, v)


def test_cpp_facade_builds_against_the_library(tmp_path):
    """The header-only C++ facade (include/dmhm_b200.hpp) and the C header
    compile in a C++17 program that uses the whole facade (the GPU test's
    driver, tests/cpp/facade_check.cpp) and link against the built library:
    every entry point the facade calls resolves."""
    import shutil
    import subprocess
    import pytest
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.dirname(_lib.LIB_PATH)
    exe = tmp_path / "facade_check"
    r = subprocess.run(["g++", "-O0", "-std=c++17", "-Wall", "-I", os.path.join(root, "include"),
                        os.path.join(root, "tests", "cpp", "facade_check.cpp"), "-o", str(exe),
                        "-L", libdir, "-ldmhm_b200", f"-Wl,-rpath,{libdir}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_workloads_module_imports_and_rejects_unknown_cases():
    """The profiling workloads (dmhm_b200/workloads.py, named by the
    commands in profiles/) import without a GPU and refuse unknown names."""
    import pytest
    from dmhm_b200 import workloads
    with pytest.raises(SystemExit):
        workloads.main(["no_such_workload"])
