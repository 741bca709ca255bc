"""The CPU oracle pinned to the reference PLASMA's own outputs (CPU only).

reference_fixtures.npz holds what the reference itself (built from its
sources by oracle/build_ref.sh, run by tests/golden/make_ref_golden.py)
returns on seeded inputs: factor checksums, solutions, dsposv's iter and
info, and its failure semantics; reference_lu_band_fixtures.npz the same
for its LU-based mixed-precision solver (dgetrf, dgetrs, dsgesv) and band
Cholesky (dpbtrf, dpbsv).  The oracle must agree before it is trusted
as the checker of the GPU library.  Where the reference library is present
(oracle/_ref), a few cases are also run live against it, and the library's
argument codes are compared with the reference's.
"""
import ctypes
import os

import numpy as np
import pytest

import gen
import oracle
from conftest import EPS, TOL, solve_residual
from oracle import ref

LO, UP = oracle.LOWER, oracle.UPPER


@pytest.fixture(scope="session")
def rg():
    return np.load(os.path.join(os.path.dirname(__file__), "golden",
                                "reference_fixtures.npz"))


def have_ref():
    return os.path.exists(ref.LIB_PATH) or ref.available()


def F(a):
    return np.asfortranarray(np.array(a, dtype=np.float64))


def close(x, xr, tol=1e-13):
    """Normwise agreement max|x - xr| / max|xr| < tol."""
    assert np.abs(x - xr).max() / np.abs(xr).max() < tol


@pytest.mark.parametrize("key,n,nb,seed", [("cfg1", 2048, 256, 42), ("rag", 1000, 128, 3000)])
def test_oracle_factor_matches_reference(rg, key, n, nb, seed):
    """Config 1 (and a ragged size): the oracle's factor against the
    reference's, through diag(L) and L v, to within the potrf tester's
    50 eps (test/test_zpotrf.c:124-141)."""
    a, _ = gen.diag_dominant(n, 1, seed=seed)
    v = gen.probe_vector(n)
    an = np.linalg.norm(a)
    for uplo, d, p in ((LO, "diagL", "Lv"), (UP, "diagU", "UTv")):
        f = F(a)
        assert oracle.potrf(uplo, f, nb) == 0
        t = np.tril(f) if uplo == LO else np.triu(f).T
        assert np.abs(np.diag(t) - rg[f"{key}_{d}"]).max() / np.abs(np.diag(t)).max() < TOL * EPS
        assert np.linalg.norm(t @ v - rg[f"{key}_{p}"]) / (an * np.linalg.norm(v)) < TOL * EPS


def test_oracle_solves_match_reference(rg):
    a, b = gen.diag_dominant(2048, 1, seed=42)
    x = F(b)
    assert oracle.posv(LO, F(a), x, 256) == 0
    close(x, rg["cfg1_dposv_X"])
    a, b = gen.diag_dominant(1000, 3, seed=3000)
    for uplo, key in ((LO, "rag_dposv_X"), (UP, "rag_dposv_up_X")):
        x = F(b)
        assert oracle.posv(uplo, F(a), x, 128) == 0
        close(x, rg[key])
    a, b = gen.diag_dominant(300, 4, seed=3001)
    f = F(a)
    assert oracle.potrf(LO, f, 64) == 0
    x = F(b)
    assert oracle.potrs(LO, f, x, 64) == 0
    close(x, rg["potrs_X"])


def test_oracle_dsposv_cfg1_matches_reference(rg):
    a, b = gen.diag_dominant(2048, 1, seed=42)
    x = F(np.zeros_like(b))
    info, it = oracle.dsposv(LO, a, b, x, 256)
    assert info == int(rg["cfg1_dsposv_info"]) == 0
    assert it == int(rg["cfg1_dsposv_iter"])
    close(x, rg["cfg1_dsposv_X"])


@pytest.mark.parametrize("n,nb", [(256, 64), (1000, 128)])
@pytest.mark.parametrize("kexp", [2, 5])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_oracle_dsposv_iter_matches_reference(rg, n, nb, kexp, tag):
    """dsposv's refinement count (zcposv.c:474-518) and solution, against the
    reference's on the same bytes."""
    a = gen.spectrum(n, 10.0 ** kexp, seed=11)
    b = F(a @ np.random.default_rng(12).standard_normal((n, 2)))
    x = F(np.zeros_like(b))
    info, it = oracle.dsposv(LO if tag == "L" else UP, a, b, x, nb)
    key = f"spec_n{n}_k{kexp}_{tag}"
    assert info == int(rg[f"{key}_info"]) == 0
    assert it == int(rg[f"{key}_iter"])
    xr = rg[f"{key}_X"]
    assert np.abs(x - xr).max() / np.abs(xr).max() < 10.0 ** kexp * 1e-13
    assert solve_residual(a, x, b) < TOL * EPS


@pytest.mark.parametrize("col", [0, 299, 999])
def test_oracle_zerocol_info_matches_reference(rg, col):
    """--zerocol (test/test_zcposv.c:104-110, :181-192; test_zpotrf.c:97-99,
    :143-151): the same info, iter = -31 and X left as it was."""
    a, b = gen.diag_dominant(1000, 2, seed=6)
    x = F(np.full(b.shape, 7.0))
    info, it = oracle.dsposv(LO, gen.zerocol(a, col), b, x, 128)
    assert info == int(rg[f"fail_zerocol{col}_info"]) == col + 1
    assert it == int(rg[f"fail_zerocol{col}_iter"]) == -31
    assert np.all(x == 7.0) and np.all(rg[f"fail_zerocol{col}_X"] == 7.0)
    f = F(a)
    f[:, col] = 0.0
    assert oracle.potrf(LO, f, 128) == int(rg[f"fail_potrf_zerocol{col}_info"])


@pytest.mark.parametrize("tag", ["L", "U"])
def test_oracle_fp32_failure_matches_reference(rg, tag):
    """kappa = 1e12: the FP32 factorisation breaks down; the reference
    cancels the sequence (info > 0, no FP64 solve).  The failing column
    depends on FP32 rounding, so only its sign is compared."""
    a = gen.spectrum(256, 1e12, seed=11)
    b = F(np.random.default_rng(1).standard_normal((256, 1)))
    x = F(np.full(b.shape, 7.0))
    info, it = oracle.dsposv(LO if tag == "L" else UP, a, b, x, 64)
    assert info > 0 and int(rg[f"fail_k12_{tag}_info"]) > 0
    assert it == int(rg[f"fail_k12_{tag}_iter"]) == -31
    assert np.all(x == 7.0)


def test_oracle_overflow_matches_reference(rg):
    a, b = gen.diag_dominant(1000, 2, seed=6)
    ao = a.copy()
    ao[5, 3] = ao[3, 5] = 1e39
    bo = b.copy()
    bo[4, 1] = -1e39
    for key, aa, bb in (("fail_ovfA", ao, b), ("fail_ovfB", a, bo)):
        x = F(np.full(b.shape, 7.0))
        info, it = oracle.dsposv(LO, F(aa), F(bb), x, 128)
        assert info == int(rg[f"{key}_info"]) == 1
        assert it == int(rg[f"{key}_iter"]) == -31
        assert np.all(x == 7.0)


# ------------------------------------------------------- live reference runs
needs_ref = pytest.mark.skipif(not have_ref(), reason="reference library not built here")


@needs_ref
@pytest.mark.parametrize("n,nb,seed", [(513, 96, 1), (1200, 256, 2)])
def test_oracle_against_live_reference(n, nb, seed):
    """Fresh seeds, run on the reference library and the oracle."""
    a, b = gen.diag_dominant(n, 2, seed=seed)
    xr, xo = F(b), F(b)
    assert ref.dposv(LO, F(a), xr, nb) == 0
    assert oracle.posv(LO, F(a), xo, nb) == 0
    close(xo, xr)
    s = gen.spectrum(n, 1e4, seed=seed)
    bs = F(s @ np.ones((n, 1)))
    xr, xo = F(np.zeros((n, 1))), F(np.zeros((n, 1)))
    ir = ref.dsposv(UP, F(s), bs, xr, nb)
    io = oracle.dsposv(UP, F(s), bs, xo, nb)
    assert ir == io
    assert np.abs(xo - xr).max() / np.abs(xr).max() < 1e-8


@needs_ref
def test_library_argument_codes_match_reference(monkeypatch):
    """The library's LAPACK-layout entry points return the reference's codes
    for each illegal argument and quick return (host-only context)."""
    import plasma_b200 as pb
    monkeypatch.setenv("PLASMA_ALLOW_NO_DEVICE", "1")
    L = pb.lib()
    R = ref.lib()
    if L.plasma_init() != 0:
        pytest.skip("library context unavailable")
    try:
        buf = np.zeros(64 * 4)
        p = buf.ctypes.data
        it1, it2 = ctypes.c_int(5), ctypes.c_int(5)
        cases = [(999, 8, 2, 8, 8, 8), (LO, -1, 2, 8, 8, 8), (LO, 8, -1, 8, 8, 8),
                 (LO, 8, 2, 7, 8, 8), (LO, 8, 2, 8, 7, 8), (LO, 8, 2, 8, 8, 7),
                 (LO, 0, 2, 1, 1, 1), (LO, 8, 0, 8, 8, 8)]
        for uplo, n, nrhs, lda, ldb, ldx in cases:
            got = L.plasma_dsposv(uplo, n, nrhs, p, lda, p, ldb, p, ldx, ctypes.byref(it1))
            want = R.plasma_dsposv(uplo, n, nrhs, ctypes.c_void_p(p), lda, ctypes.c_void_p(p),
                                   ldb, ctypes.c_void_p(p), ldx, ctypes.byref(it2))
            assert got == want, (uplo, n, nrhs, lda, ldb, ldx, got, want)
            if want == 0:
                assert it1.value == it2.value == 0
            # posv / potrs on legal arguments would compute (this context has
            # no device): compared only up to their quick returns
            legal = (uplo in (LO, UP) and n >= 0 and nrhs >= 0 and lda >= max(1, n)
                     and ldb >= max(1, n))
            if not (legal and min(n, nrhs) > 0):
                got = L.plasma_dposv(uplo, n, nrhs, p, lda, p, ldb)
                want = R.plasma_dposv(uplo, n, nrhs, ctypes.c_void_p(p), lda,
                                      ctypes.c_void_p(p), ldb)
                assert got == want
            if not (legal and max(n, nrhs) > 0):
                got = L.plasma_dpotrs(uplo, n, nrhs, p, lda, p, ldb)
                want = R.plasma_dpotrs(uplo, n, nrhs, ctypes.c_void_p(p), lda,
                                       ctypes.c_void_p(p), ldb)
                assert got == want
        for uplo, n, lda in ((999, 8, 8), (LO, -1, 8), (LO, 8, 7), (LO, 0, 1)):
            got = L.plasma_dpotrf(uplo, n, p, lda)
            want = R.plasma_dpotrf(uplo, n, ctypes.c_void_p(p), lda)
            assert got == want, (uplo, n, lda, got, want)
    finally:
        L.plasma_finalize()


@needs_ref
def test_library_argument_codes_match_reference_next_rows(monkeypatch):
    """dsgesv, the band routines and the inverse: the library returns the
    reference's code for each illegal argument and quick return (host-only
    context, so only cases where neither side computes)."""
    import plasma_b200 as pb
    monkeypatch.setenv("PLASMA_ALLOW_NO_DEVICE", "1")
    L = pb.lib()
    R = ref.lib()
    if L.plasma_init() != 0:
        pytest.skip("library context unavailable")
    vp = ctypes.c_void_p
    try:
        buf = np.zeros(64 * 8)
        p = buf.ctypes.data
        piv = np.zeros(64, dtype=np.int32)
        it1, it2 = ctypes.c_int(5), ctypes.c_int(5)
        for n, nrhs, lda, ldb, ldx in ((-1, 2, 8, 8, 8), (8, -1, 8, 8, 8), (8, 2, 7, 8, 8),
                                       (8, 2, 8, 7, 8), (8, 2, 8, 8, 7), (0, 2, 1, 1, 1),
                                       (8, 0, 8, 8, 8)):
            got = L.plasma_dsgesv(n, nrhs, p, lda, piv.ctypes.data, p, ldb, p, ldx,
                                  ctypes.byref(it1))
            want = R.plasma_dsgesv(n, nrhs, vp(p), lda, vp(piv.ctypes.data), vp(p), ldb,
                                   vp(p), ldx, ctypes.byref(it2))
            assert got == want, ("dsgesv", n, nrhs, lda, ldb, ldx, got, want)
        for uplo, n, kd, nrhs, ldab, ldb in ((999, 8, 2, 1, 3, 8), (LO, -1, 2, 1, 3, 8),
                                             (LO, 8, -1, 1, 3, 8), (LO, 8, 2, -1, 3, 8),
                                             (LO, 8, 2, 1, 2, 8), (LO, 8, 2, 1, 3, 7),
                                             (LO, 0, 0, 1, 1, 1), (UP, 8, 2, 0, 3, 8)):
            legal = (uplo in (LO, UP) and n >= 0 and kd >= 0 and nrhs >= 0
                     and ldab >= kd + 1 and ldb >= max(1, n))
            # the quick returns of compute/zpbsv.c:131-133 and zpbtrs.c:120-122;
            # past them both sides go on to build descriptors and compute
            for name, quick in (("plasma_dpbsv", min(n, nrhs) == 0),
                                ("plasma_dpbtrs", max(n, nrhs) == 0)):
                got = getattr(L, name)(uplo, n, kd, nrhs, p, ldab, p, ldb)
                want = getattr(R, name)(uplo, n, kd, nrhs, vp(p), ldab, vp(p), ldb)
                if not legal or quick:
                    assert got == want, (name, uplo, n, kd, nrhs, ldab, ldb, got, want)
        for uplo, n, kd, ldab in ((999, 8, 2, 3), (LO, -1, 2, 3), (LO, 8, -1, 3),
                                  (LO, 8, 2, 2), (LO, 0, 0, 1)):
            got = L.plasma_dpbtrf(uplo, n, kd, p, ldab)
            want = R.plasma_dpbtrf(uplo, n, kd, vp(p), ldab)
            assert got == want, ("dpbtrf", uplo, n, kd, ldab, got, want)
        for uplo, n, lda in ((999, 8, 8), (LO, -1, 8), (LO, 8, 7), (LO, 0, 1)):
            for name in ("plasma_dpotri", "plasma_dpoinv"):
                got = getattr(L, name)(uplo, n, p, lda)
                want = getattr(R, name)(uplo, n, vp(p), lda)
                assert got == want, (name, uplo, n, lda, got, want)
    finally:
        L.plasma_finalize()


@pytest.fixture(scope="session")
def rlb():
    return np.load(os.path.join(os.path.dirname(__file__), "golden",
                                "reference_lu_band_fixtures.npz"))


def normwise(y, yr, t):
    """||y - yr|| / (||T||_F ||v||) for checksums y = T v of a factor T."""
    return np.linalg.norm(y - yr) / (np.linalg.norm(t) * np.linalg.norm(gen.probe_vector(len(y))))


@pytest.mark.parametrize("n,nb", [(300, 64), (1000, 128)])
def test_oracle_getrf_matches_reference(rlb, n, nb):
    """Tile LU with partial pivoting (compute/pzgetrf.c with the panel of
    core_blas/core_zgetrf.c): the reference's pivots exactly, and its factor
    through L v and U v to within the getrf tester's 50 eps
    (test/test_zgetrf.c:116-138); the solve of compute/zgetrs.c."""
    a, b = gen.general(n, 3, seed=9500 + n)
    f = F(a)
    info, ipiv = oracle.getrf(f, nb)
    assert info == 0
    key = f"lu_n{n}_nb{nb}"
    np.testing.assert_array_equal(ipiv, rlb[f"{key}_ipiv"])
    v = gen.probe_vector(n)
    lo, up = np.tril(f, -1) + np.eye(n), np.triu(f)
    assert normwise(lo @ v, rlb[f"{key}_Lv"], lo) < TOL * EPS
    assert normwise(up @ v, rlb[f"{key}_Uv"], up) < TOL * EPS
    d, dr = np.diag(up), rlb[f"{key}_diagU"]
    assert np.abs(d - dr).max() / np.abs(dr).max() < TOL * n * EPS
    if n == 300:
        x = F(b)
        assert oracle.getrs(f, ipiv, x) == 0
        close(x, rlb[f"{key}_getrs_X"], tol=1e-11)


@pytest.mark.parametrize("col", [0, 150, 399])
def test_oracle_getrf_zero_column_matches_reference(rlb, col):
    """A zeroed column: the first zero pivot.  The reference's LAPACK-layout
    plasma_dgetrf returns it offset by min(m, n) (compute/zgetrf.c:101 adds
    imin(m, n) to the tile routine's status, which is LAPACK's index); the
    oracle reports the tile routine's (and LAPACK's) value."""
    a, _ = gen.general(400, 1, seed=9600)
    f = F(a)
    f[:, col] = 0.0
    info, _ = oracle.getrf(f, 64)
    assert info == col + 1 == int(rlb[f"luinfo_{col}"]) - 400


@pytest.mark.parametrize("n,nb,kexp", [(400, 64, 2), (400, 64, 5), (1000, 128, 5)])
def test_oracle_dsgesv_matches_reference(rlb, n, nb, kexp):
    """FP32 LU + FP64 refinement (compute/zcgesv.c:363-532) on
    A = U diag(sigma) V^T, kappa 1e2 and 1e5: the reference's info and
    iteration count, and its solution to within kappa n eps.  (The
    reference's iteration count can move by one with its thread count; the
    fixture ran 8 threads.)"""
    a = gen.general_spectrum(n, 10.0 ** kexp)
    b = F(np.cos(np.arange(2.0 * n)).reshape(n, 2))
    x = F(np.zeros((n, 2)))
    info, it, _ = oracle.dsgesv(F(a), b, x, nb)
    key = f"gesv_n{n}_k{kexp}"
    assert info == int(rlb[f"{key}_info"]) == 0
    assert abs(it - int(rlb[f"{key}_iter"])) <= 1
    xr = rlb[f"{key}_X"]
    assert np.abs(x - xr).max() / np.abs(xr).max() < 10.0 ** kexp * n * EPS


@pytest.mark.parametrize("n,kd,nb", [(500, 40, 64), (1000, 100, 128)])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_oracle_band_matches_reference(rlb, n, kd, nb, tag):
    """Band tile Cholesky and band solves (compute/pzpbtrf.c, pztbsm.c,
    zpbsv.c): the reference's band factor through its diagonal and L v, and
    its dpbsv solution."""
    a, abl, abu, b = gen.band(n, kd, 2, seed=7000 + n)
    uplo, ab = (LO, abl) if tag == "L" else (UP, abu)
    f = F(ab)
    assert oracle.pbtrf(uplo, f, kd, nb) == 0
    x = F(b)
    assert oracle.pbtrs(uplo, f, kd, x, nb) == 0
    t = gen.from_band(f, kd, lower=uplo == LO)
    t = t if uplo == LO else t.T
    key = f"pb_n{n}_kd{kd}_{tag}"
    assert np.abs(np.diag(t) - rlb[f"{key}_diag"]).max() / np.abs(np.diag(t)).max() < TOL * EPS
    assert normwise(t @ gen.probe_vector(n), rlb[f"{key}_Lv"], t) < TOL * EPS
    close(x, rlb[f"{key}_X"])


@pytest.mark.parametrize("col,tag", [(0, "L"), (137, "L"), (137, "U")])
def test_oracle_band_info_matches_reference(rlb, col, tag):
    """A zeroed row and column of a band matrix: dpbtrf's info."""
    a, _, _, _ = gen.band(300, 20, 1, seed=7300)
    a[col, :] = 0.0
    a[:, col] = 0.0
    uplo = LO if tag == "L" else UP
    ab = gen.to_band(a, 20, lower=uplo == LO)
    assert oracle.pbtrf(uplo, F(ab), 20, 64) == int(rlb[f"pbinfo_{col}_{tag}"]) == col + 1


@needs_ref
def test_oracle_lu_band_against_live_reference():
    """Fresh seeds on the reference library and the oracle: LU pivots and
    solve, dsgesv at kappa 1e3, band solve."""
    n, nb = 700, 96
    a, b = gen.general(n, 2, seed=31)
    fr, fo = F(a), F(a)
    ir, pr = ref.dgetrf(fr, nb)
    io, po = oracle.getrf(fo, nb)
    assert ir == io == 0
    np.testing.assert_array_equal(pr, po)
    xr, xo = F(b), F(b)
    assert ref.dgetrs(fr, pr, xr, nb) == 0
    assert oracle.getrs(fo, po, xo) == 0
    close(xo, xr, tol=1e-11)
    s = gen.general_spectrum(n, 1e3, seed=32)
    xr, xo = F(np.zeros((n, 2))), F(np.zeros((n, 2)))
    ir, itr, _ = ref.dsgesv(F(s), F(b), xr, nb)
    io, ito, _ = oracle.dsgesv(F(s), F(b), xo, nb)
    assert ir == io == 0 and abs(itr - ito) <= 1
    assert np.abs(xo - xr).max() / np.abs(xr).max() < 1e3 * n * EPS
    _, abl, _, bb = gen.band(n, 60, 1, seed=33)
    fr, fo = F(abl), F(abl)
    xr, xo = F(bb), F(bb)
    assert ref.dpbsv(LO, fr, 60, xr, nb) == 0
    assert oracle.pbtrf(LO, fo, 60, nb) == 0
    assert oracle.pbtrs(LO, fo, 60, xo, nb) == 0
    close(xo, xr)


@pytest.fixture(scope="session")
def rpi():
    return np.load(os.path.join(os.path.dirname(__file__), "golden",
                                "reference_potri_fixtures.npz"))


@pytest.mark.parametrize("n,nb", [(300, 64), (1000, 128)])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_oracle_potri_matches_reference(rpi, n, nb, tag):
    """The inverse from the factor (compute/zpotri.c: pztrtri then pzlauum):
    the reference's inverse through its diagonal and sym(inv) v, within the
    potri tester's 50 eps (test/test_zpotri.c:135-155) normwise."""
    a, _ = gen.diag_dominant(n, 1, seed=8800 + n)
    uplo = LO if tag == "L" else UP
    f = F(a)
    assert oracle.potrf(uplo, f, nb) == 0
    assert oracle.potri(uplo, f) == 0
    t = np.tril(f) if uplo == LO else np.triu(f)
    full = t + t.T - np.diag(np.diag(t))
    key = f"potri_n{n}_nb{nb}_{tag}"
    d, dr = np.diag(t), rpi[f"{key}_diag"]
    assert np.linalg.norm(d - dr) / np.linalg.norm(dr) < TOL * EPS
    assert normwise(full @ gen.probe_vector(n), rpi[f"{key}_Sv"], full) < TOL * EPS


@pytest.mark.parametrize("col", [0, 137, 299])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_oracle_potri_info_matches_reference(rpi, col, tag):
    """A zero on the factor's diagonal: dpotri's info (dtrtri's index)."""
    a, _ = gen.diag_dominant(300, 1, seed=9100)
    uplo = LO if tag == "L" else UP
    f = F(a)
    assert oracle.potrf(uplo, f, 64) == 0
    f[col, col] = 0.0
    assert oracle.potri(uplo, f) == int(rpi[f"potriinfo_{col}_{tag}"]) == col + 1


@needs_ref
def test_descriptors_match_reference(monkeypatch):
    """plasma_desc_t as the reference builds it (control/descriptor.c): the
    general, triangular and band inits, views and plasma_desc_check give the
    same struct, field for field, and the same codes, on the same arguments
    (host-only context; no storage is allocated)."""
    import plasma_b200 as pb
    monkeypatch.setenv("PLASMA_ALLOW_NO_DEVICE", "1")
    L = pb.lib()
    R = ref.lib()
    if L.plasma_init() != 0:
        pytest.skip("library context unavailable")
    D = pb.plasma_desc_t
    ci, vp = ctypes.c_int, ctypes.c_void_p
    R.plasma_desc_general_init.argtypes = [ci, vp] + [ci] * 8 + [ctypes.POINTER(D)]
    R.plasma_desc_triangular_init.argtypes = [ci, ci, vp] + [ci] * 8 + [ctypes.POINTER(D)]
    R.plasma_desc_general_band_init.argtypes = [ci, ci, vp] + [ci] * 10 + [ctypes.POINTER(D)]
    R.plasma_desc_view.argtypes = [D, ci, ci, ci, ci]
    R.plasma_desc_view.restype = D
    R.plasma_desc_check.argtypes = [D]
    for f in ("plasma_desc_general_init", "plasma_desc_triangular_init",
              "plasma_desc_general_band_init", "plasma_desc_check"):
        getattr(R, f).restype = ci
    mat = vp(0x10000)

    def same(d1, d2, what):
        for name, _ in D._fields_:
            assert getattr(d1, name) == getattr(d2, name), (what, name, getattr(d1, name),
                                                            getattr(d2, name))

    try:
        for prec in (pb.PlasmaRealDouble, pb.PlasmaRealFloat):
            for mb, nb, lm, ln, i, j, m, n in ((256, 256, 1000, 700, 0, 0, 1000, 700),
                                               (64, 64, 512, 512, 64, 128, 300, 200),
                                               (128, 96, 385, 97, 0, 0, 385, 97),
                                               (4, 4, 8, 8, 0, 0, 8, 8)):
                d1, d2 = D(), D()
                r1 = L.plasma_desc_general_init(prec, mat, mb, nb, lm, ln, i, j, m, n,
                                                ctypes.byref(d1))
                r2 = R.plasma_desc_general_init(prec, mat, mb, nb, lm, ln, i, j, m, n,
                                                ctypes.byref(d2))
                assert r1 == r2
                same(d1, d2, ("general", mb, nb, lm, ln, i, j, m, n))
                assert L.plasma_desc_check(d1) == R.plasma_desc_check(d2)
                if m > mb and n > nb:
                    same(L.plasma_desc_view(d1, mb, nb, m - mb, n - nb),
                         R.plasma_desc_view(d2, mb, nb, m - mb, n - nb), "view")
            for uplo in (LO, UP):
                for nb, n in ((256, 1000), (64, 512), (96, 97)):
                    d1, d2 = D(), D()
                    assert (L.plasma_desc_triangular_init(prec, uplo, mat, nb, nb, n, n, 0, 0,
                                                          n, n, ctypes.byref(d1))
                            == R.plasma_desc_triangular_init(prec, uplo, mat, nb, nb, n, n,
                                                             0, 0, n, n, ctypes.byref(d2)))
                    same(d1, d2, ("triangular", uplo, nb, n))
                    assert L.plasma_desc_check(d1) == R.plasma_desc_check(d2)
                for nb, n, kd in ((128, 1000, 100), (64, 300, 200), (256, 2049, 256)):
                    lm = nb * (1 + (kd + nb - 1) // nb)
                    d1, d2 = D(), D()
                    assert (L.plasma_desc_general_band_init(prec, uplo, mat, nb, nb, lm, n, 0,
                                                            0, n, n, kd, kd, ctypes.byref(d1))
                            == R.plasma_desc_general_band_init(prec, uplo, mat, nb, nb, lm, n,
                                                               0, 0, n, n, kd, kd,
                                                               ctypes.byref(d2)))
                    same(d1, d2, ("band", uplo, nb, n, kd))
                    assert L.plasma_desc_check(d1) == R.plasma_desc_check(d2)
        # descriptors plasma_desc_check rejects (mb = 0 is left out: the
        # reference's init divides by it, control/descriptor.c:144, where the
        # library records the descriptor for plasma_desc_check to reject)
        for args in ((pb.PlasmaRealDouble, 4, 4, 8, 8, 2, 0, 4, 8),
                     (pb.PlasmaRealDouble, 4, 4, 8, 8, 4, 0, 8, 8),
                     (99, 4, 4, 8, 8, 0, 0, 8, 8)):
            d1, d2 = D(), D()
            L.plasma_desc_general_init(args[0], mat, *args[1:], ctypes.byref(d1))
            R.plasma_desc_general_init(args[0], mat, *args[1:], ctypes.byref(d2))
            assert L.plasma_desc_check(d1) == R.plasma_desc_check(d2) != 0, args
    finally:
        L.plasma_finalize()


@needs_ref
def test_settings_match_reference(monkeypatch):
    """plasma_set / plasma_get (control/context.c:78-159) on the reference's
    parameters: the same code for every legal and illegal value and for an
    unknown parameter, and plasma_get returning what was set."""
    import plasma_b200 as pb
    monkeypatch.setenv("PLASMA_ALLOW_NO_DEVICE", "1")
    L = pb.lib()
    R = ref.lib()
    if L.plasma_init() != 0:
        pytest.skip("library context unavailable")
    R.plasma_get.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    R.plasma_get.restype = ctypes.c_int
    tuning, nb, ib, inout, threads, householder = range(6)
    cases = [(tuning, v) for v in (0, 1, 2, -1)] + \
            [(nb, v) for v in (1, 96, 256, 0, -5)] + \
            [(ib, v) for v in (1, 32, 0, -1)] + \
            [(inout, v) for v in (0, 1, 5)] + \
            [(threads, v) for v in (1, 4, 0)] + \
            [(householder, v) for v in (0, 1, 2)] + \
            [(77, 1), (-3, 1)]
    saved = {}
    for param in (tuning, nb, ib, threads, householder):
        v = ctypes.c_int()
        assert R.plasma_get(param, ctypes.byref(v)) == 0
        saved[param] = v.value
    try:
        for param, value in cases:
            got, want = L.plasma_set(param, value), R.plasma_set(param, value)
            assert got == want, (param, value, got, want)
            if want == 0:
                g1, g2 = ctypes.c_int(-7), ctypes.c_int(-7)
                assert L.plasma_get(param, ctypes.byref(g1)) == R.plasma_get(
                    param, ctypes.byref(g2)) == 0
                assert g1.value == g2.value == value, (param, value, g1.value, g2.value)
    finally:
        L.plasma_finalize()
        # the reference context is shared by the other tests
        for param, v in saved.items():
            R.plasma_set(param, v)


@needs_ref
def test_lapack_constants_match_reference():
    """plasma_{uplo,trans,side,diag,norm}_const (control/constants.c): the
    reference's enum for every LAPACK character, either case, and for
    characters it does not know."""
    import plasma_b200 as pb
    L = pb.lib()
    R = ref.lib()
    for name in ("plasma_uplo_const", "plasma_trans_const", "plasma_side_const",
                 "plasma_diag_const", "plasma_norm_const"):
        f = getattr(R, name)
        f.argtypes = [ctypes.c_char]
        f.restype = ctypes.c_int
        for ch in b"ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789":
            c = bytes([ch])
            assert getattr(L, name)(c) == f(c), (name, c)
