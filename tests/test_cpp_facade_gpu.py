"""The header-only C++ facade (include/dmhm_b200.hpp) compiled against
libdmhm_b200.so, driven like the reference's C++ test drivers, against the
reference fixtures."""
import os
import subprocess

import numpy as np
import pytest

from helpers import load, relerr

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_facade(tmp_path):
    exe = tmp_path / "facade_check"
    libdir = os.path.join(ROOT, "dmhm_b200")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_check.cpp"), "-o", str(exe),
                    "-L", libdir, "-ldmhm_b200", f"-Wl,-rpath,{libdir}"], check=True)
    fx = load("c1")
    N, k = 1024, fx["probes"].shape[1]
    fx["coef"].tofile(tmp_path / "coef.bin")
    np.asfortranarray(fx["probes"]).T.copy().tofile(tmp_path / "probes.bin")
    subprocess.run([str(exe), str(tmp_path), "32", "32", "4", "8", str(k)], check=True,
                   timeout=600)

    def rd(name):
        return np.fromfile(tmp_path / name).reshape(k, N).T

    assert relerr(np.fromfile(tmp_path / "matvec1.bin"), fx["matvec1"]) < 1e-13
    assert relerr(rd("matvec.bin"), fx["matvec"]) < 1e-13
    assert relerr(rd("hh.bin"), fx["hh_AA"]) < 1e-12
    assert relerr(rd("schulz3.bin"), fx["schulz3"]) < 1e-8
