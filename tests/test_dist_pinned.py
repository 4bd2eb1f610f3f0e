"""The reference's own single-rank DistHMat2d / DistHMat3d, pinned (CPU).

Fixtures d2s, d2w and d3s hold what the reference's distributed classes
(src/DistHMat2d, src/DistHMat3d), run as one process over a serial MPI
stand-in, compute on three stencil operators: H*H products with multType 0
and 2 (src/DistHMat2d/MultiplyHMat-incl.hpp:28-53), a fixed-count
SchulzInvert and the stop-test SchulzInvert (src/DistHMat2d/Invert-incl.hpp
:14-105), all under CompressionTolerance 1e-8, beside the serial HMat2d /
HMat3d results on the same operator (tests/golden/make_golden.py).

The distributed classes compress each block of a product once, from two-sided
sketches of all its contributions and Gram eigendecompositions
(MultiplyHMatCompress-incl.hpp); the serial classes, and the oracle and the
GPU engine that follow them, round after each contribution.  Both are
approximations of the same product, so these tests compare them at the
approximation's own scale: each against exact dense algebra, and with each
other within that error."""
import pytest

from helpers import load, relerr, stencil_exact as exact
from oracle import dmhm_oracle as O

CASES = ["d2s", "d2w", "d3s"]


@pytest.mark.parametrize("case", CASES)
def test_reference_dist_and_serial_agree(case):
    """The reference's two implementations agree with each other to within
    their own errors; sparse-built strongly admissible products are exact in
    both, and the choice of multType changes nothing beyond that error."""
    fx = load(case)
    ex = exact(fx)
    if int(fx["strong"]):
        for k in ("dist_hh_AA_m0", "dist_hh_AA_m2", "serial_hh_AA"):
            assert relerr(fx[k], ex["AA"]) < 1e-14, k
        assert relerr(fx["dist_hh_AB_m2"], ex["AB"]) < 1e-14
    else:
        e = relerr(fx["dist_hh_AA_m2"], ex["AA"])
        assert 1e-3 < e < 0.1                      # weak admissibility at rank 8 is lossy
        assert relerr(fx["serial_hh_AA"], ex["AA"]) < 1.1 * e
        assert relerr(fx["dist_hh_AA_m0"], fx["dist_hh_AA_m2"]) < e
    for key in ("schulz", "schulz_stop"):
        ed = relerr(fx["dist_" + key], ex["inv"])
        es = relerr(fx["serial_" + key], ex["inv"])
        assert ed < 0.1 and es < 0.1, (key, ed, es)
        assert relerr(fx["dist_" + key], fx["serial_" + key]) < 1.5 * max(ed, es), key


def test_oracle_products_against_reference_dist():
    """The oracle's H*H (the serial algorithm with the global tolerance's
    truncation, which the DistHMat facade runs) against the reference's
    DistHMat2d product on the weakly admissible case, where rank 8 loses
    about 5 %: no less accurate, and within the reference's own error of it."""
    fx = load("d2w")
    ex = exact(fx)
    sizes = [int(s) for s in fx["sizes"]]
    L, r = int(fx["levels"]), int(fx["rank"])
    try:
        O.set_compression_tolerance(float(fx["tol"]))
        HA = O.build_stencil_hmat(2, sizes, L, r, fx["coef"], strong=False)
        HB = O.build_stencil_hmat(2, sizes, L, r, fx["coefB"], strong=False)
        for key, Hb, alpha, ref in (("dist_hh_AA_m2", HA, 1.0, ex["AA"]),
                                    ("dist_hh_AB_m2", HB, -0.5, ex["AB"])):
            C = O.hh_multiply(HA, alpha, Hb, O.Rng(int(fx["oversample"])))
            Y = O.multiply_dense(C, 1.0, fx["probes"])
            ed = relerr(fx[key], ref)
            assert relerr(Y, ref) < 1.1 * ed, key
            assert relerr(Y, fx[key]) < 0.5 * ed, key
    finally:
        O.set_compression_tolerance(0.0)


def test_oracle_schulz_against_reference_dist():
    """The oracle's SchulzInvert under CompressionTolerance 1e-8 against the
    reference's DistHMat2d SchulzInvert (16 iterations, multType 2) on the
    strongly admissible 32 x 32 case: both reach about 1e-8 of the exact
    inverse and agree to 1e-7."""
    fx = load("d2s")
    ex = exact(fx)
    sizes = [int(s) for s in fx["sizes"]]
    try:
        O.set_compression_tolerance(float(fx["tol"]))
        H = O.build_stencil_hmat(2, sizes, int(fx["levels"]), int(fx["rank"]), fx["coef"])
        X, its, _ = O.schulz_invert(H, int(fx["iters"]), O.Rng(int(fx["oversample"])))
        assert its == int(fx["iters"])
        Y = O.multiply_dense(X, 1.0, fx["probes"])
        ed = relerr(fx["dist_schulz"], ex["inv"])
        assert ed < 1e-7
        assert relerr(Y, ex["inv"]) < 1.5 * ed
        assert relerr(Y, fx["dist_schulz"]) < 1e-7
    finally:
        O.set_compression_tolerance(0.0)
