"""The engine's rounding algorithm (one-sided Jacobi SVD of the core after
QR of the stacked factors), restated on the CPU by oracle/rounding_oracle.py,
against LAPACK: singular values, orthogonality, reconstruction, the
truncation rule, and the all-pairs convergence test that decides whether a
sweep runs."""
import numpy as np
import pytest
import scipy.linalg as sla

from oracle import rounding_oracle as R


def spectrum_matrix(rng, rows, cols, sigma):
    """rows x cols matrix with the given singular values (len = min)."""
    k = min(rows, cols)
    Q1, _ = np.linalg.qr(rng.standard_normal((rows, k)))
    Q2, _ = np.linalg.qr(rng.standard_normal((cols, k)))
    return (Q1 * sigma[:k]) @ Q2.T


SPECTRA = {
    "decaying": lambda k: np.logspace(0, -12, k),
    "clustered": lambda k: 1.0 + 1e-9 * np.arange(k),
    "rank_deficient": lambda k: np.concatenate([np.logspace(0, -3, k // 2),
                                                np.zeros(k - k // 2)]),
    "flat": lambda k: np.ones(k),
}


@pytest.mark.parametrize("shape", [(8, 8), (16, 24), (40, 40), (33, 17), (1, 5)])
@pytest.mark.parametrize("spectrum", sorted(SPECTRA))
def test_jacobi_fp64_against_lapack(shape, spectrum):
    rng = np.random.default_rng(100 * shape[0] + shape[1] + 7 * sorted(SPECTRA).index(spectrum))
    rows, cols = shape
    sig = SPECTRA[spectrum](min(rows, cols))
    M = spectrum_matrix(rng, rows, cols, sig)
    Mo, J, sweeps = R.jacobi(M)
    # a spectrum graded over 12 decades in a random basis takes the most
    # sweeps (about 20 at 40 x 40); the kernel's bound is 40
    assert sweeps <= 25
    assert np.linalg.norm(J.T @ J - np.eye(cols)) < 1e-13 * cols
    assert np.linalg.norm(Mo @ J.T - M) <= 1e-13 * max(1.0, np.linalg.norm(M))
    got = np.sort(np.linalg.norm(Mo, axis=0))[::-1][:min(rows, cols)]
    want = sla.svdvals(M)
    assert np.max(np.abs(got - want)) <= 1e-13 * max(want[0], 1e-300)
    # columns mutually orthogonal to the test's tolerance where they carry weight
    nrm = np.linalg.norm(Mo, axis=0)
    G = Mo.T @ Mo
    big = nrm > 1e-14 * max(nrm.max(), 1e-300)
    off = np.abs(G - np.diag(np.diag(G)))[np.ix_(big, big)]
    assert np.all(off <= 1e-14 * np.outer(nrm, nrm)[np.ix_(big, big)] + 1e-300)


@pytest.mark.parametrize("shape", [(16, 16), (24, 40)])
def test_jacobi_fp32_against_lapack(shape):
    rng = np.random.default_rng(5)
    rows, cols = shape
    M = spectrum_matrix(rng, rows, cols, np.logspace(0, -4, min(rows, cols)))
    Mo, J, sweeps = R.jacobi(M, np.float32)
    assert Mo.dtype == np.float32 and sweeps <= 15
    got = np.sort(np.linalg.norm(Mo.astype(np.float64), axis=0))[::-1][:min(rows, cols)]
    want = sla.svdvals(M)
    assert np.max(np.abs(got - want)) <= 1e-5 * want[0]


@pytest.mark.parametrize("seed", range(4))
def test_all_pairs_test_only_skips_idle_sweeps(seed):
    """With the convergence test the result is the same, bit for bit, as
    without it: it stops only where the next sweep would rotate nothing."""
    rng = np.random.default_rng(seed)
    M = spectrum_matrix(rng, 24, 24, np.logspace(0, -10, 24))
    a = R.jacobi(M, all_pairs_test=True)
    b = R.jacobi(M, all_pairs_test=False)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[2] == b[2] - 1          # the idle sweep is not run


@pytest.mark.parametrize("k,rout", [(12, 8), (32, 16), (6, 8)])
def test_rounding_is_the_best_rank_rout_approximation(k, rout):
    rng = np.random.default_rng(k)
    m, n = 64, 48
    U = rng.standard_normal((m, k)) * np.logspace(0, -6, k)
    V = rng.standard_normal((n, k))
    A = U @ V.T
    Uo, Vo, _ = R.round_factors(U, V, rout)
    s = sla.svdvals(A)
    best = np.sqrt(np.sum(s[rout:] ** 2))
    err = np.linalg.norm(A - Uo @ Vo.T)
    assert err <= best * (1 + 1e-8) + 1e-12 * s[0]
    assert np.linalg.norm(Vo.T @ Vo - np.eye(Vo.shape[1])) < 1e-13
    assert Uo.shape[1] == min(rout, k)


@pytest.mark.parametrize("tol", [1e-10, 1e-4, 0.3])
def test_rounding_tolerance_rule_against_lapack(tol):
    """The kept count under a tolerance equals SVDTrunc's on LAPACK's
    singular values for spectra away from the threshold."""
    rng = np.random.default_rng(11)
    m, n, k = 40, 40, 16
    sig = np.logspace(0, -14, k)
    sig = sig[np.abs(np.log10(sig / tol)) > 0.2]         # away from the cut
    U = spectrum_matrix(rng, m, sig.size, sig)
    V, _ = np.linalg.qr(rng.standard_normal((n, sig.size)))
    Uo, Vo, _ = R.round_factors(U, V, 64, tol)
    want = R.kept(sla.svdvals(U @ V.T) ** 2, 64, tol)
    assert Uo.shape[1] == want == max(1, int(np.sum(sig > tol * sig[0])))


@pytest.mark.parametrize("k,rout", [(24, 16), (40, 32), (12, 8)])
def test_preconditioned_rounding_same_result_fewer_sweeps(k, rout):
    """Jacobi on R_4^T (M^T = Q_4 R_4) returns the same rounding, in the
    same convention (singular values in U, V orthonormal), with fewer
    sweeps on a graded core."""
    rng = np.random.default_rng(k + rout)
    m, n = 64, 64
    U = spectrum_matrix(rng, m, k, np.logspace(0, -12, k))
    V = rng.standard_normal((n, k))
    U1, V1, s1 = R.round_factors(U, V, rout)
    U2, V2, s2 = R.round_factors(U, V, rout, precondition=True)
    A = U @ V.T
    assert np.linalg.norm(U1 @ V1.T - U2 @ V2.T) <= 1e-12 * np.linalg.norm(A)
    assert np.allclose(np.linalg.norm(U1, axis=0), np.linalg.norm(U2, axis=0),
                       rtol=1e-10, atol=1e-13 * np.linalg.norm(A))
    assert np.linalg.norm(V2.T @ V2 - np.eye(V2.shape[1])) < 1e-13
    assert s2 < s1
