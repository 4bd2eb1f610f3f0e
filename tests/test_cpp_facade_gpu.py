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
    cx = load("cplx")
    N, k = 1024, fx["probes"].shape[1]
    n, ck = int(np.prod(cx["sizes"])), cx["probes"].shape[1]
    fx["coef"].tofile(tmp_path / "coef.bin")
    np.asfortranarray(fx["probes"]).T.copy().tofile(tmp_path / "probes.bin")
    np.asfortranarray(cx["probes"]).T.copy().view(np.float64).tofile(tmp_path / "cprobes.bin")
    subprocess.run([str(exe), str(tmp_path), "32", "32", "4", "8", str(k),
                    str(int(cx["sizes"][0])), str(int(cx["levels"])), str(int(cx["rank"])),
                    repr(float(cx["kwave"])), str(ck)], check=True, timeout=600)

    def rd(name):
        return np.fromfile(tmp_path / name).reshape(k, N).T

    assert relerr(np.fromfile(tmp_path / "matvec1.bin"), fx["matvec1"]) < 1e-13
    assert relerr(rd("matvec.bin"), fx["matvec"]) < 1e-13
    view = np.fromfile(tmp_path / "matvec_view.bin").reshape(k - 1, N).T
    assert relerr(view, fx["matvec"][:, 1:]) < 1e-13
    # the AbstractHMat norm estimate equals the reference's first estimate
    est = np.fromfile(tmp_path / "norm.bin")[0]
    assert abs(est - fx["schulz3_trace"][0]) < 1e-12 * est
    # HMat2d<std::complex<double>>: Multiply against the reference's complex
    # run, AdjointMultiply against 0.5 - 0.25i times A^H by dense algebra
    cm = np.fromfile(tmp_path / "cmatvec.bin").view(np.complex128).reshape(ck, n).T
    assert relerr(cm, cx["matvec"]) < 1e-13
    import dmhm_b200 as D
    from dmhm_b200 import operators as O
    sizes = [int(s) for s in cx["sizes"]]
    Ad = O.dense_from_sparse(O.helmholtz(sizes, float(cx["kwave"]), int(cx["levels"])))
    ca = np.fromfile(tmp_path / "cmatvec_adj.bin").view(np.complex128).reshape(ck, n).T
    assert relerr(ca, (0.5 - 0.25j) * (Ad.conj().T @ cx["probes"])) < 1e-13
    assert relerr(rd("hh.bin"), fx["hh_AA"]) < 1e-12
    assert relerr(rd("schulz3.bin"), fx["schulz3"]) < 1e-8
