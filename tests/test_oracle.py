"""The CPU oracle pinned against LAPACK known answers (CPU only).

The reference's testers accept a result when it agrees with LAPACK within
tol * eps, tol = 50 (test/test_zpotrf.c:124-152, test/test_zposv.c:137-167,
test/test_zcposv.c:139-193).  The oracle must pass the same checks on the
committed fixtures before it is trusted as the checker of the GPU library.
"""
import numpy as np
import pytest

import gen
import oracle
from conftest import EPS, TOL, factor_error, solve_residual

LO, UP = oracle.LOWER, oracle.UPPER


@pytest.mark.parametrize("n", [1, 2, 7, 33, 64, 100])
@pytest.mark.parametrize("nb", [1, 16, 32, 256])
def test_potrf_matches_lapack(golden, n, nb):
    a = golden[f"small{n}_A"]
    for uplo, key in ((LO, "L"), (UP, "U")):
        f = np.asfortranarray(a.copy())
        assert oracle.potrf(uplo, f, nb) == 0
        got = np.tril(f) if uplo == LO else np.triu(f)
        err = factor_error(got, golden[f"small{n}_{key}"], a)
        assert err < TOL * EPS, (uplo, err)


@pytest.mark.parametrize("n", [7, 64, 100])
@pytest.mark.parametrize("nb", [5, 32])
def test_posv_potrs_match_lapack(golden, n, nb):
    a, b = golden[f"small{n}_A"], golden[f"small{n}_B"]
    for uplo in (LO, UP):
        f = np.asfortranarray(a.copy())
        x = np.asfortranarray(b.copy())
        assert oracle.posv(uplo, f, x, nb) == 0
        assert solve_residual(a, x, b) < TOL * EPS
        np.testing.assert_allclose(x, golden[f"small{n}_X"], rtol=1e-12, atol=1e-14)
        # potrs with the factor just computed
        x2 = np.asfortranarray(b.copy())
        assert oracle.potrs(uplo, f, x2, nb) == 0
        np.testing.assert_allclose(x2, x, rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("n", [300, 1000])
def test_ragged_checksums(golden, n):
    a, b = gen.diag_dominant(n, 5, seed=2000 + n)
    f = np.asfortranarray(a.copy())
    assert oracle.potrf(LO, f, 128) == 0
    l = np.tril(f)
    v = gen.probe_vector(n)
    np.testing.assert_allclose(np.diag(l), golden[f"ragged{n}_diagL"], rtol=1e-14)
    np.testing.assert_allclose(l @ v, golden[f"ragged{n}_Lv"], rtol=1e-12)
    x = np.asfortranarray(b.copy())
    assert oracle.posv(LO, np.asfortranarray(a.copy()), x, 128) == 0
    np.testing.assert_allclose(x, golden[f"ragged{n}_X"], rtol=1e-12, atol=1e-15)


def test_cfg1_parity_case(golden):
    """n = 2048, nb = 256, nrhs = 1, seed 42: the CPU parity configuration."""
    a, b = gen.diag_dominant(2048, 1, seed=42)
    f = np.asfortranarray(a.copy())
    assert oracle.potrf(LO, f, 256) == 0
    l = np.tril(f)
    v = gen.probe_vector(2048)
    np.testing.assert_allclose(np.diag(l), golden["cfg1_diagL"], rtol=1e-14)
    np.testing.assert_allclose(l @ v, golden["cfg1_Lv"], rtol=1e-12)
    x = np.asfortranarray(b.copy())
    assert oracle.potrs(LO, f, x, 256) == 0
    assert solve_residual(a, x, b) < TOL * EPS
    np.testing.assert_allclose(x, golden["cfg1_X"], rtol=1e-12)


@pytest.mark.parametrize("n,col", [(100, 37), (300, 0), (300, 299), (513, 256)])
def test_nonspd_info_matches_lapack(golden, n, col):
    a, _ = gen.diag_dominant(n, 1, seed=3000 + n)
    a = gen.zerocol(a, col)
    for uplo, key in ((LO, "lower"), (UP, "upper")):
        for nb in (64, 128):
            f = np.asfortranarray(a.copy())
            info = oracle.potrf(uplo, f, nb)
            assert info == int(golden[f"nonspd{n}_{col}_info_{key}"]), (uplo, nb)


@pytest.mark.parametrize("n", [64, 300])
def test_dsposv_converges_like_reference(n):
    a, b = gen.diag_dominant(n, 2, seed=5000 + n)
    x = np.zeros_like(b, order="F")
    info, it = oracle.dsposv(LO, a, b, x, 64)
    assert info == 0
    assert 0 <= it <= 30
    assert solve_residual(a, x, b) < TOL * EPS


def test_dsposv_fp32_failure_cancels():
    """kappa far beyond 1/eps_fp32: the FP32 factor breaks down, and as in
    the reference's cancelled task sequence the call returns that info with
    iter = -31, no FP64 solve and X untouched (zcposv.c:440-538 with the
    sequence->status test of every core task)."""
    n = 128
    a = gen.spectrum(n, 1e12, seed=11)
    rng = np.random.default_rng(1)
    b = np.asfortranarray(rng.standard_normal((n, 1)))
    x = np.full_like(b, 3.0, order="F")
    info, it = oracle.dsposv(LO, a, b, x, 32)
    assert info > 0
    assert it == -31
    assert np.all(x == 3.0)


def test_dsposv_refinement_exhausted_goes_fp64():
    """The FP32 factor succeeds but 30 refinement steps do not meet the
    stopping rule: the FP64 factorisation answers with iter = -31
    (zcposv.c:522-538).  kappa = 1e8 at n = 256 in upper storage is such a
    case for the oracle's (and the reference's) FP32 rounding."""
    n = 256
    a = gen.spectrum(n, 1e8, seed=11)
    b = np.asfortranarray(a @ np.random.default_rng(12).standard_normal((n, 2)))
    x = np.zeros_like(b, order="F")
    info, it = oracle.dsposv(UP, a, b, x, 256)
    assert info == 0
    assert it == -31
    assert solve_residual(a, x, b) < TOL * EPS


@pytest.mark.parametrize("kappa", [1e2, 1e5])
def test_dsposv_spectrum_against_lapack(golden, kappa):
    n = 256
    a = gen.spectrum(n, kappa, seed=11)
    xt = golden[f"spec{int(np.log10(kappa))}_xtrue"]
    b = np.asfortranarray(a @ xt)
    x = np.zeros_like(b, order="F")
    info, it = oracle.dsposv(LO, a, b, x, 64)
    assert info == 0 and it >= 0
    assert solve_residual(a, x, b) < TOL * EPS
    xl = golden[f"spec{int(np.log10(kappa))}_X"]
    # forward error bounded by kappa * backward error, like LAPACK's answer
    assert np.abs(x - xl).max() / np.abs(xl).max() < kappa * 1e-13


def test_lansy_inf():
    a, _ = gen.diag_dominant(77, 1, seed=9)
    want = np.abs(a).sum(axis=1).max()
    assert abs(oracle.lansy_inf(LO, np.asfortranarray(np.tril(a))) - want) < 1e-12 * want
    assert abs(oracle.lansy_inf(UP, np.asfortranarray(np.triu(a))) - want) < 1e-12 * want


def test_single_precision_potrf():
    a, _ = gen.diag_dominant(100, 1, seed=77)
    f = np.asfortranarray(a.astype(np.float32))
    assert oracle.potrf(LO, f, 32) == 0
    l = np.tril(f).astype(np.float64)
    assert np.linalg.norm(a - l @ l.T) / (100 * np.linalg.norm(a)) < 50 * np.finfo(np.float32).eps


@pytest.mark.parametrize("n", [7, 64, 100])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_potri_against_lapack(golden, n, tag):
    """The oracle's dtrtri + dlauum against LAPACK dpotri: the reference
    tester's check (test/test_zpotri.c:135-155), ||inv - inv_lapack||_F /
    ||inv_lapack||_F < 50 eps on the uplo triangle; the other triangle is
    left as it was."""
    f = np.asfortranarray(golden[f"potri{n}_{tag}_factor"].copy())
    ref = golden[f"potri{n}_{tag}_inv"]
    uplo = oracle.LOWER if tag == "L" else oracle.UPPER
    tri = np.tril if tag == "L" else np.triu
    other = (lambda m: np.triu(m, 1)) if tag == "L" else (lambda m: np.tril(m, -1))
    before = other(f).copy()
    assert oracle.potri(uplo, f) == 0
    assert np.linalg.norm(tri(f) - ref) / np.linalg.norm(ref) < 50 * EPS
    np.testing.assert_array_equal(other(f), before)


def test_potri_zero_diagonal_info():
    """dtrtri's info: the first zero on the diagonal of the factor."""
    a, _ = gen.diag_dominant(50, 1, seed=9)
    f = np.asfortranarray(np.linalg.cholesky(a))
    f[17, 17] = 0.0
    f[30, 30] = 0.0
    keep = f.copy()
    assert oracle.potri(oracle.LOWER, f) == 18
    np.testing.assert_array_equal(f, keep)


BANDS = [(7, 2), (64, 10), (100, 33), (130, 0), (96, 95)]


@pytest.mark.parametrize("n,kd", BANDS)
@pytest.mark.parametrize("tag", ["L", "U"])
@pytest.mark.parametrize("nb", [4, 16, 32])
def test_pbtrf_pbtrs_against_lapack(golden, n, kd, tag, nb):
    """The oracle's band tile Cholesky and band solves against LAPACK dpbtrf
    and dpbtrs: the factor within 50 eps (relative Frobenius), the reference
    tester's residual ||B - A X||_inf / (n ||A||_F ||X||_inf) < 50 eps
    (test/test_zpbsv.c:180-202), and the solution against LAPACK's."""
    a, abl, abu, b = gen.band(n, kd, 2, seed=5000 + n + kd)
    lower = tag == "L"
    ab = np.asfortranarray((abl if lower else abu).copy())
    uplo = LO if lower else UP
    assert oracle.pbtrf(uplo, ab, kd, nb) == 0
    ref = golden[f"band{n}_{kd}_{tag}_factor"]
    assert np.linalg.norm(ab - ref) / np.linalg.norm(ref) < 50 * EPS
    x = np.asfortranarray(b.copy())
    assert oracle.pbtrs(uplo, ab, kd, x, nb) == 0
    r = np.abs(b - a @ x).max() / (n * np.linalg.norm(a) * np.abs(x).max())
    assert r < TOL * EPS
    xr = golden[f"band{n}_{kd}_{tag}_X"]
    assert np.abs(x - xr).max() / np.abs(xr).max() < 1e3 * EPS


@pytest.mark.parametrize("n,kd,col", [(100, 9, 41), (300, 40, 0)])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_pbtrf_info_matches_lapack(golden, n, kd, col, tag):
    """A zeroed row and column: the oracle's info equals LAPACK dpbtrf's and
    the band array is left as it was (test/test_zpbsv.c:108-114, :207-214)."""
    a, _, _, _ = gen.band(n, kd, 1, seed=6000 + n)
    a = gen.zerocol(a, col)
    lower = tag == "L"
    ab = gen.to_band(a, kd, lower=lower)
    keep = ab.copy()
    info = oracle.pbtrf(LO if lower else UP, ab, kd, 16)
    assert info == int(golden[f"bandinfo{n}_{kd}_{tag}"]) > 0
    np.testing.assert_array_equal(ab, keep)


def test_band_storage_round_trip():
    a, abl, abu, _ = gen.band(50, 7, 1, seed=1)
    np.testing.assert_array_equal(gen.from_band(abl, 7, True), np.tril(a))
    np.testing.assert_array_equal(gen.from_band(abu, 7, False), np.triu(a))


@pytest.mark.parametrize("n", [7, 64, 100, 150])
@pytest.mark.parametrize("nb", [1, 16, 32, 256])
def test_getrf_against_lapack(golden, n, nb):
    """The oracle's LU with partial pivoting against LAPACK dgetrf: the same
    pivots, and the reference tester's factor check (test/test_zgetrf.c:
    116-138), ||LU - LU_lapack||_F / ||A||_F / sqrt(n n) < 50 eps."""
    a, b = gen.general(n, 2, seed=9000 + n)
    f = np.asfortranarray(a.copy())
    info, ipiv = oracle.getrf(f, nb)
    assert info == 0
    np.testing.assert_array_equal(ipiv, golden[f"lu{n}_ipiv"])
    err = np.linalg.norm(f - golden[f"lu{n}_LU"]) / np.linalg.norm(a) / n
    assert err < TOL * EPS
    # P A = L U
    lo = np.tril(f, -1) + np.eye(n)
    pa = a.copy()
    for j, p in enumerate(ipiv - 1):
        pa[[j, p]] = pa[[p, j]]
    assert np.linalg.norm(pa - lo @ np.triu(f)) / np.linalg.norm(a) < n * EPS * 10
    # the solve (compute/zgetrs.c) against dgesv, and the tester's residual
    x = np.asfortranarray(b.copy())
    assert oracle.getrs(f, ipiv, x) == 0
    assert solve_residual(a, x, b) < TOL * EPS
    np.testing.assert_allclose(x, golden[f"lu{n}_X"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("n,col", [(64, 20), (100, 0)])
def test_getrf_info_matches_lapack(golden, n, col):
    """A zero column: the first zero pivot, as LAPACK dgetrf reports it."""
    a, _ = gen.general(n, 1, seed=9100 + n)
    a[:, col] = 0.0
    info, _ = oracle.getrf(np.asfortranarray(a), 16)
    assert info == int(golden[f"luinfo{n}_{col}"]) > 0


@pytest.mark.parametrize("kappa,iters", [(1e2, (1, 5)), (1e12, (-31, -31))])
def test_dsgesv_against_lapack(golden, kappa, iters):
    """FP32 LU + FP64 refinement (compute/zcgesv.c:363-532): converges at
    kappa = 1e2, falls back to the FP64 LU at kappa = 1e12; the tester's
    residual (test/test_zcgesv.c:150-170) and the dgesv solution."""
    n = 100
    a = gen.general_spectrum(n, kappa)
    b = np.asfortranarray(np.cos(np.arange(200.0)).reshape(n, 2))
    x = np.zeros((n, 2), order="F")
    a0, b0 = a.copy(), b.copy()
    info, it, _ = oracle.dsgesv(a, b, x, 32)
    assert info == 0
    assert iters[0] <= it <= iters[1]
    np.testing.assert_array_equal(a, a0)
    np.testing.assert_array_equal(b, b0)
    assert solve_residual(a, x, b) < TOL * EPS
    xr = golden[f"gesv_kappa{kappa:.0e}_X"]
    assert np.abs(x - xr).max() / np.abs(xr).max() < 10 * kappa * n * EPS


@pytest.mark.parametrize("kappa", [1e10, 1e12])
def test_dsgesv_diverging_refinement_falls_back(kappa):
    """kappa = 1e10 and 1e12 at n = 400: the FP32-preconditioned iteration
    diverges.  A NaN or infinite iterate must not pass the stopping rule
    (the reference's form, zcgesv.c:265-276, accepts a NaN residual), so the
    oracle ends in the FP64 fallback with a finite solution."""
    n = 400
    a = gen.general_spectrum(n, kappa)
    b = np.asfortranarray(np.cos(np.arange(2.0 * n)).reshape(n, 2))
    x = np.zeros((n, 2), order="F")
    info, it, _ = oracle.dsgesv(np.asfortranarray(a.copy()), b.copy(order="F"), x, 64)
    assert info == 0 and it == -31
    assert np.isfinite(x).all()
    assert solve_residual(a, x, b) < TOL * EPS


def test_dsgesv_fp32_overflow_falls_back():
    n = 50
    a, b = gen.general(n, 1, seed=77)
    a = a * 1e39
    x = np.zeros((n, 1), order="F")
    info, it, _ = oracle.dsgesv(np.asfortranarray(a), b, x, 16)
    assert info == 0 and it == -31
    assert solve_residual(a, x, b) < TOL * EPS
