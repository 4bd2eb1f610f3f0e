"""Pins the numpy oracle (oracle/dmhm_oracle.py) to the reference itself.

The fixtures in tests/golden/ hold outputs of the unmodified reference library
(tests/golden/make_golden.py).  Integer work (generator states and uniforms)
must match bit for bit; floating-point results to rounding (matvec, exact H*H)
or, where fixed-rank truncation amplifies rounding, to the stated tolerance.
"""
import numpy as np
import pytest

from helpers import load, relerr
from oracle import dmhm_oracle as O


def oracle_hmat(fx, coef_key="coef"):
    sizes = tuple(int(s) for s in fx["sizes"])
    return O.build_stencil_hmat(len(sizes), sizes, int(fx["levels"]), int(fx["rank"]),
                                fx[coef_key], strong=bool(fx["strong"]))


def test_lcg_bit_exact():
    fx = load("lcg")
    k = int(fx["count"])
    d = fx["draws"]
    r = O.Rng()
    assert np.array_equal(r.serial.uniforms(k), d[:k])
    assert np.array_equal(r.serial.gaussian_vector(k), d[k:2 * k])
    assert np.array_equal(r.serial.gaussian_vectors(k, 3).T.ravel(), d[2 * k:5 * k])
    assert np.array_equal(r.parallel.gaussian_vectors(k, 3).T.ravel(), d[5 * k:8 * k])


def test_lcg_skip_ahead():
    a = O.Lcg()
    s = a.states(5000)
    b = O.Lcg()
    b.state = (O.lcg_jump(4321)[0] * O.LCG_SEED + O.lcg_jump(4321)[1]) & O.MASK64
    assert int(s[4321]) == b.state


@pytest.mark.parametrize("case", ["c1", "ragged", "weak", "c3d"])
def test_matvec(case):
    fx = load(case)
    H = oracle_hmat(fx)
    P = fx["probes"]
    assert relerr(O.multiply_dense(H, 1.0, P), fx["matvec"]) < 1e-14
    assert relerr(O.multiply_dense(H, 1.0, P[:, 0]), fx["matvec1"]) < 1e-14
    assert relerr(O.transpose_multiply_dense(H, 1.0, P), fx["matvec_T"]) < 1e-14


@pytest.mark.parametrize("case", ["c1", "ragged", "weak", "c3d"])
def test_random_matvec(case):
    fx = load(case)
    H = oracle_hmat(fx)
    O.set_to_random(H, O.Rng())
    P = fx["probes"]
    assert relerr(O.multiply_dense(H, 1.0, P), fx["random"]) < 1e-13
    assert relerr(O.transpose_multiply_dense(H, 1.0, P), fx["random_T"]) < 1e-13


@pytest.mark.parametrize("case", ["c1", "ragged", "weak"])
def test_hh_square(case):
    fx = load(case)
    A = oracle_hmat(fx)
    C = O.hh_multiply(A, 1.0, A, O.Rng(int(fx["oversample"])))
    assert relerr(O.multiply_dense(C, 1.0, fx["probes"]), fx["hh_AA"]) < 1e-12


@pytest.mark.parametrize("case", ["c1", "ragged"])
def test_hh_general(case):
    fx = load(case)
    A = oracle_hmat(fx)
    B = oracle_hmat(fx, "coefB")
    C = O.hh_multiply(A, -0.5, B, O.Rng(int(fx["oversample"])))
    assert relerr(O.multiply_dense(C, 1.0, fx["probes"]), fx["hh_AB"]) < 1e-12


@pytest.mark.parametrize("case,its", [("ragged", 3), ("weak", 3)])
def test_schulz_iterations(case, its):
    fx = load(case)
    A = oracle_hmat(fx)
    X, k, trace = O.schulz_invert(A, its, O.Rng(int(fx["oversample"])))
    key = f"schulz{its}"
    assert k == its
    assert abs(trace[0] - fx[key + "_trace"][0]) < 1e-13 * trace[0]
    # fixed-rank truncation inside each H*H amplifies rounding differences
    assert relerr(O.multiply_dense(X, 1.0, fx["probes"]), fx[key]) < 1e-8


@pytest.mark.parametrize("case,bound", [("c1", 1e-5), ("ragged", 1e-5), ("weak", 0.1),
                                        ("c3d", 1e-4)])
def test_direct_invert(case, bound):
    """DirectInvert (recursive Schur complements) equals the reference's to
    rounding: the oracle draws the generator in the reference's order, and
    the result is the inverse to the accuracy of its fixed-rank products."""
    fx = load(case)
    A = oracle_hmat(fx)
    O.direct_invert(A, O.Rng(int(fx["oversample"])))
    Y = O.multiply_dense(A, 1.0, fx["probes"])
    assert relerr(Y, fx["direct"]) < 1e-12
    # against the exact inverse: weak admissibility at rank 4 is lossy
    Ad = O.to_dense(oracle_hmat(fx))              # A itself is exact (dense leaves)
    assert relerr(fx["direct"], np.linalg.solve(Ad, fx["probes"])) < bound


@pytest.mark.parametrize("case", ["c1", "ragged"])
def test_low_rank_products(case):
    """hmat_tools::Multiply / TransposeMultiply (F := alpha A B, alpha A^T B
    as one low-rank matrix, sample rank maxRank + Oversample()): the
    restatement reproduces the reference's F on probe vectors."""
    fx = load(case)
    for tag, fn in (("lr_AB", O.randomized_product), ("lr_AtB", O.randomized_transpose_product)):
        rng = O.Rng(int(fx["oversample"]))
        A = oracle_hmat(fx)
        O.set_to_random(A, rng)
        B = oracle_hmat(fx, "coefB")
        F = fn(int(fx["rank"]) + int(fx["oversample"]), 0.75, A, B, rng)
        assert F.U.shape[1] == int(fx[tag + "_rank"])
        P = fx["probes"]
        assert relerr(F.U @ (F.V.T @ P), fx[tag]) < 1e-10


def test_complex_fixture_against_dense():
    """The reference's complex-double results (tests/golden/cplx.npz) against
    dense complex algebra of the same operator: products exact, the Schulz
    inverse within 1e-8 of the dense inverse on the probes."""
    import numpy as np
    from dmhm_b200 import operators as O
    fx = load("cplx")
    sizes = tuple(int(s) for s in fx["sizes"])
    S = O.helmholtz(sizes, float(fx["kwave"]), int(fx["levels"]))
    A = O.dense_from_sparse(S)
    P = fx["probes"]
    assert relerr(fx["matvec"], A @ P) < 1e-14
    assert relerr(fx["hh_AA"], A @ (A @ P)) < 1e-14
    assert relerr(fx["schulz_stop"], np.linalg.solve(A, P)) < 1e-8


def _walk_pack(raw, pos, H):
    """Parses one block of the reference's Pack layout
    (src/HMat2d/Pack-incl.hpp:183-240) against the oracle's block tree and
    returns the position after it."""
    import struct
    t = struct.unpack_from("<i", raw, pos)[0]
    pos += 4
    if H.kind == O.NODE:
        assert t == 0
        for c in H.children:
            pos = _walk_pack(raw, pos, c)
    elif H.kind == O.LOW_RANK:
        assert t == 2
        r = struct.unpack_from("<i", raw, pos)[0]
        pos += 4 + 8 * (H.height + H.width) * r
    else:
        assert t == 3
        assert struct.unpack_from("<i", raw, pos)[0] == 0      # GENERAL
        pos += 4 + 8 * H.height * H.width
    return pos


@pytest.mark.parametrize("case", ["ragged", "c3d"])
def test_pack_fixture_layout(case):
    """The reference's Pack bytes follow the documented layout over the
    oracle's block tree and are consumed exactly."""
    import struct
    pk = load("pack")
    fx = load(case)
    raw = pk[case + "_pack"].tobytes()
    dim = len(fx["sizes"])
    L, r = struct.unpack_from("<ii", raw, 0)
    assert (L, r) == (int(fx["levels"]), int(fx["rank"]))
    header = 4 * 4 + 2 + 4 * 4 * dim     # 4 ints, 2 bools, per axis 2 sizes + 2 coordinates
    # PackedSize counts one int more than the header holds: 4 zero bytes end
    # the buffer (Pack-incl.hpp:32)
    end = _walk_pack(raw, header, oracle_hmat(fx))
    assert end + 4 == len(raw) and raw[end:] == bytes(4)


def test_tolerance_rule_matches_svdtrunc():
    """The oracle's kept-rank rule against the reference's SVDTrunc loop
    (src/DistHMat2d/Truncation-incl.hpp:51-59) on spectra around the
    thresholds: at least sigma_0 is kept, only sigma_0 below tol^2."""
    def svdtrunc(s, rel_tol, max_rank):
        k = len(s)
        if k == 0:
            return 0
        tolerance = rel_tol * s[0]
        if s[0] < rel_tol * rel_tol:
            cutoff = 0
        else:
            cutoff = min(k, max_rank) - 1
            while cutoff >= 0 and not s[cutoff] > tolerance:
                cutoff -= 1
        return cutoff + 1

    rng = np.random.default_rng(4)
    old = O._COMPRESSION_TOL[0]
    try:
        for tol in (1e-10, 1e-4, 0.3):
            O.set_compression_tolerance(tol)
            for _ in range(200):
                k = int(rng.integers(1, 12))
                s = np.sort(10.0 ** rng.uniform(-25, 2, k))[::-1]
                cap = int(rng.integers(1, 14))
                assert O._kept(s, cap) == svdtrunc(list(s), tol, cap)
            assert O._kept(np.array([1e-30, 1e-31]), 4) == 1
    finally:
        O.set_compression_tolerance(old)
