"""libplasma_core_blas.so: the reference's CPU tile kernels of the
kernel-substitution interface (include/plasma_core_blas_z.h), checked on CPU
against numpy / scipy's LAPACK for every option combination, both
precisions, and against the same kernels of the reference build
(oracle/_ref) on the same inputs (no GPU needed)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import scipy.linalg as sl

import plasma_b200 as pb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "plasma_b200", "libplasma_core_blas.so")
NO, TR = pb.PlasmaNoTrans, pb.PlasmaTrans
UP, LO, GE = pb.PlasmaUpper, pb.PlasmaLower, pb.PlasmaGeneral
LEFT, RIGHT, NONUNIT, UNIT = 141, 142, 131, 132
ONE, FRO, INF, MAX = 171, 174, 175, 177
COLWISE, ROWWISE = 401, 402


@pytest.fixture(scope="module")
def C():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "plasma_b200", "core_blas")],
                       check=True)
    return ctypes.CDLL(LIB)


PRECS = [("d", np.float64, ctypes.c_double, 1e-12), ("s", np.float32, ctypes.c_float, 1e-4)]


def F(a, dt):
    return np.asfortranarray(np.asarray(a, dtype=dt))


def p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def test_exports_every_declared_function(C):
    import re
    src = open(os.path.join(ROOT, "include", "plasma_core_blas.h")).read()
    names = set(re.findall(r"\b(plasma_core_[ds]lag2[sd])\s*\(", src))
    for pfx in ("d", "s"):
        for f in ("potrf", "trsm", "syrk", "gemm", "symm", "lacpy", "geadd", "lange", "lansy"):
            names.add(f"plasma_core_{pfx}{f}")
        names.add(f"plasma_core_omp_{pfx}amax")
    missing = [n for n in sorted(names) if not hasattr(C, n)]
    assert not missing and len(names) == 22


@pytest.mark.parametrize("pfx,dt,ct,tol", PRECS)
@pytest.mark.parametrize("uplo", [LO, UP])
def test_potrf(C, pfx, dt, ct, tol, uplo):
    rng = np.random.default_rng(1)
    n = 37
    g = rng.standard_normal((n, n))
    a = F(g @ g.T + n * np.eye(n), dt)
    f = a.copy(order="F")
    fn = getattr(C, f"plasma_core_{pfx}potrf")
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
    assert fn(uplo, n, p(f), n) == 0
    ref = sl.cholesky(a.astype(np.float64), lower=uplo == LO)
    tri = np.tril if uplo == LO else np.triu
    assert np.abs(tri(f) - ref).max() < tol * np.abs(ref).max()
    other = np.triu(f, 1) if uplo == LO else np.tril(f, -1)
    np.testing.assert_array_equal(other, (np.triu(a, 1) if uplo == LO else np.tril(a, -1)))
    bad = a.copy(order="F")
    bad[5, 5] = -1.0
    assert fn(uplo, n, p(bad), n) > 0
    assert fn(999, n, p(f), n) == -1 and fn(uplo, -1, p(f), n) == -2 and fn(uplo, n, p(f), 1) == -4


@pytest.mark.parametrize("pfx,dt,ct,tol", PRECS)
@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("trans", [NO, TR])
@pytest.mark.parametrize("diag", [NONUNIT, UNIT])
def test_trsm(C, pfx, dt, ct, tol, side, uplo, trans, diag):
    rng = np.random.default_rng(2)
    m, n = 9, 6
    k = m if side == LEFT else n
    a = F(rng.uniform(-1, 1, (k, k)) + 4 * np.eye(k), dt)
    b = F(rng.uniform(-1, 1, (m, n)), dt)
    t = np.tril(a) if uplo == LO else np.triu(a)
    if diag == UNIT:
        t = t - np.diag(np.diag(t)) + np.eye(k)
    op = t.T if trans == TR else t
    x = b.copy(order="F")
    fn = getattr(C, f"plasma_core_{pfx}trsm")
    fn.argtypes = [ctypes.c_int] * 6 + [ct, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_int]
    fn(side, uplo, trans, diag, m, n, 2.0, p(a), k, p(x), m)
    got = (op.astype(np.float64) @ x.astype(np.float64) if side == LEFT
           else x.astype(np.float64) @ op.astype(np.float64))
    assert np.abs(got - 2.0 * b).max() < 10 * tol


@pytest.mark.parametrize("pfx,dt,ct,tol", PRECS)
@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("trans", [NO, TR])
def test_syrk(C, pfx, dt, ct, tol, uplo, trans):
    rng = np.random.default_rng(3)
    n, k = 7, 5
    a = F(rng.uniform(-1, 1, (n, k) if trans == NO else (k, n)), dt)
    c0 = F(rng.uniform(-1, 1, (n, n)), dt)
    c = c0.copy(order="F")
    fn = getattr(C, f"plasma_core_{pfx}syrk")
    fn.argtypes = [ctypes.c_int] * 4 + [ct, ctypes.c_void_p, ctypes.c_int, ct, ctypes.c_void_p,
                                        ctypes.c_int]
    fn(uplo, trans, n, k, -1.5, p(a), a.shape[0], 0.5, p(c), n)
    op = a if trans == NO else a.T
    ref = -1.5 * op.astype(np.float64) @ op.T.astype(np.float64) + 0.5 * c0
    tri = np.tril if uplo == LO else np.triu
    assert np.abs(tri(c) - tri(ref)).max() < tol * 10
    np.testing.assert_array_equal(np.triu(c, 1) if uplo == LO else np.tril(c, -1),
                                  np.triu(c0, 1) if uplo == LO else np.tril(c0, -1))


@pytest.mark.parametrize("pfx,dt,ct,tol", PRECS)
@pytest.mark.parametrize("ta", [NO, TR])
@pytest.mark.parametrize("tb", [NO, TR])
def test_gemm_and_beta_zero(C, pfx, dt, ct, tol, ta, tb):
    rng = np.random.default_rng(4)
    m, n, k = 5, 6, 4
    a = F(rng.uniform(-1, 1, (m, k) if ta == NO else (k, m)), dt)
    b = F(rng.uniform(-1, 1, (k, n) if tb == NO else (n, k)), dt)
    c = F(np.full((m, n), np.nan), dt)     # beta = 0: C is not read
    fn = getattr(C, f"plasma_core_{pfx}gemm")
    fn.argtypes = [ctypes.c_int] * 5 + [ct, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_int, ct, ctypes.c_void_p, ctypes.c_int]
    fn(ta, tb, m, n, k, 1.0, p(a), a.shape[0], p(b), b.shape[0], 0.0, p(c), m)
    ref = (a if ta == NO else a.T).astype(np.float64) @ (b if tb == NO else b.T)
    assert np.abs(c - ref).max() < tol * 10


@pytest.mark.parametrize("pfx,dt,ct,tol", PRECS)
@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("uplo", [LO, UP])
def test_symm(C, pfx, dt, ct, tol, side, uplo):
    rng = np.random.default_rng(5)
    m, n = 6, 4
    k = m if side == LEFT else n
    s = rng.uniform(-1, 1, (k, k))
    s = s + s.T
    stored = F(np.tril(s) if uplo == LO else np.triu(s), dt)   # only uplo is read
    b = F(rng.uniform(-1, 1, (m, n)), dt)
    c0 = F(rng.uniform(-1, 1, (m, n)), dt)
    c = c0.copy(order="F")
    fn = getattr(C, f"plasma_core_{pfx}symm")
    fn.argtypes = [ctypes.c_int] * 4 + [ct, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_int, ct, ctypes.c_void_p, ctypes.c_int]
    fn(side, uplo, m, n, 2.0, p(stored), k, p(b), m, -1.0, p(c), m)
    ref = 2.0 * (s @ b if side == LEFT else b @ s) - c0
    assert np.abs(c - ref).max() < tol * 10


@pytest.mark.parametrize("pfx,dt,ct,tol", PRECS)
@pytest.mark.parametrize("uplo", [GE, LO, UP])
@pytest.mark.parametrize("trans", [NO, TR])
def test_lacpy(C, pfx, dt, ct, tol, uplo, trans):
    rng = np.random.default_rng(6)
    m, n = 7, 5
    a = F(rng.uniform(-1, 1, (m, n)), dt)
    ldb = m if trans == NO else n
    b = F(np.zeros((ldb, n if trans == NO else m)), dt)
    fn = getattr(C, f"plasma_core_{pfx}lacpy")
    fn.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.c_int]
    fn(uplo, trans, m, n, p(a), m, p(b), ldb)
    mask = (np.ones((m, n), bool) if uplo == GE else
            np.tril(np.ones((m, n), bool)) if uplo == LO else np.triu(np.ones((m, n), bool)))
    ref = np.where(mask, a, 0)
    np.testing.assert_array_equal(b, ref if trans == NO else ref.T)


@pytest.mark.parametrize("pfx,dt,ct,tol", PRECS)
def test_geadd_and_codes(C, pfx, dt, ct, tol):
    rng = np.random.default_rng(7)
    m, n = 5, 4
    a = F(rng.uniform(-1, 1, (n, m)), dt)          # transposed operand
    b0 = F(rng.uniform(-1, 1, (m, n)), dt)
    b = b0.copy(order="F")
    fn = getattr(C, f"plasma_core_{pfx}geadd")
    fn.argtypes = [ctypes.c_int] * 3 + [ct, ctypes.c_void_p, ctypes.c_int, ct, ctypes.c_void_p,
                                        ctypes.c_int]
    assert fn(TR, m, n, 2.0, p(a), n, 3.0, p(b), m) == 0
    assert np.abs(b - (3.0 * b0 + 2.0 * a.T)).max() < tol * 10
    assert fn(999, m, n, 1.0, p(a), n, 1.0, p(b), m) == -1
    assert fn(NO, -1, n, 1.0, p(a), n, 1.0, p(b), m) == -2
    assert fn(NO, m, -1, 1.0, p(a), n, 1.0, p(b), m) == -3
    assert fn(NO, m, n, 1.0, None, m, 1.0, p(b), m) == -5
    assert fn(NO, m, n, 1.0, p(a), m - 1, 1.0, p(b), m) == -6
    assert fn(NO, m, n, 1.0, p(a), m, 1.0, None, m) == -8
    assert fn(NO, m, n, 1.0, p(a), m, 1.0, p(b), m - 1) == -9


@pytest.mark.parametrize("pfx,dt,ct,tol", PRECS)
@pytest.mark.parametrize("norm", [ONE, INF, FRO, MAX])
def test_lange_lansy(C, pfx, dt, ct, tol, norm):
    rng = np.random.default_rng(8)
    m, n = 6, 5
    a = F(rng.uniform(-2, 2, (m, n)), dt)
    work = np.zeros(max(m, n))
    val = ctypes.c_double()
    fn = getattr(C, f"plasma_core_{pfx}lange")
    fn.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_double)]
    fn(norm, m, n, p(a), m, p(work), ctypes.byref(val))
    ref = {ONE: np.abs(a).sum(0).max(), INF: np.abs(a).sum(1).max(),
           FRO: np.linalg.norm(a.astype(np.float64)), MAX: np.abs(a).max()}[norm]
    assert abs(val.value - ref) < tol * 10 * ref
    s = rng.uniform(-2, 2, (n, n))
    s = s + s.T
    for uplo in (LO, UP):
        stored = F(np.tril(s) if uplo == LO else np.triu(s), dt)
        fs = getattr(C, f"plasma_core_{pfx}lansy")
        fs.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                            ctypes.POINTER(ctypes.c_double)]
        fs(norm, uplo, n, p(stored), n, p(work), ctypes.byref(val))
        full = s.astype(dt).astype(np.float64)
        ref = {ONE: np.abs(full).sum(0).max(), INF: np.abs(full).sum(1).max(),
               FRO: np.linalg.norm(full), MAX: np.abs(full).max()}[norm]
        assert abs(val.value - ref) < tol * 10 * ref


def test_lag2s_slag2d_and_amax(C):
    a = F([[1.0, -2.5], [3.0, 1e-3]], np.float64)
    s = np.zeros((2, 2), dtype=np.float32, order="F")
    C.plasma_core_dlag2s.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_int]
    assert C.plasma_core_dlag2s(2, 2, p(a), 2, p(s), 2) == 0
    np.testing.assert_array_equal(s, a.astype(np.float32))
    big = F([[1.0, 1e39], [0.0, 1.0]], np.float64)
    assert C.plasma_core_dlag2s(2, 2, p(big), 2, p(s), 2) == 1
    d = np.zeros((2, 2), order="F")
    C.plasma_core_slag2d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_int]
    C.plasma_core_slag2d(2, 2, p(s), 2, p(d), 2)
    np.testing.assert_array_equal(d, s.astype(np.float64))
    x = F([[1.0, -7.0, 2.0], [-3.0, 0.5, 4.0]], np.float64)
    vals = np.zeros(3)
    fn = C.plasma_core_omp_damax
    fn.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    seq, req = pb.plasma_sequence_t(), pb.plasma_request_t()
    fn(COLWISE, 2, 3, p(x), 2, p(vals), ctypes.byref(seq), ctypes.byref(req))
    np.testing.assert_array_equal(vals, np.abs(x).max(0))
    fn(ROWWISE, 2, 3, p(x), 2, p(vals), ctypes.byref(seq), ctypes.byref(req))
    np.testing.assert_array_equal(vals[:2], np.abs(x).max(1))


# ---------------------------------------------- against the reference's own
# The same kernels of the reference build (oracle/_ref/libplasma_ref.so: the
# reference's core_blas sources over OpenBLAS), called on the same inputs.
REF_PRECS = [("d", np.float64, ctypes.c_double, 1e-13), ("s", np.float32, ctypes.c_float, 1e-5)]


@pytest.fixture(scope="module")
def R():
    from oracle import ref
    if not os.path.exists(ref.LIB_PATH):
        pytest.skip("reference library not built here")
    return ref.lib()


def both(C, R, name, argtypes, restype=None):
    out = []
    for lib in (C, R):
        f = getattr(lib, name)
        f.argtypes = argtypes
        f.restype = restype
        out.append(f)
    return out


def agree(x, y, tol):
    x, y = np.asarray(x, np.float64), np.asarray(y, np.float64)
    assert np.abs(x - y).max() <= tol * max(np.abs(y).max(), 1.0)


@pytest.mark.parametrize("pfx,dt,ct,tol", REF_PRECS)
@pytest.mark.parametrize("uplo", [LO, UP])
def test_potrf_matches_reference(C, R, pfx, dt, ct, tol, uplo):
    rng = np.random.default_rng(11)
    n = 40
    g = rng.standard_normal((n, n))
    a = F(g @ g.T + n * np.eye(n), dt)
    ours, theirs = both(C, R, f"plasma_core_{pfx}potrf",
                        [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int], ctypes.c_int)
    f1, f2 = a.copy(order="F"), a.copy(order="F")
    assert ours(uplo, n, p(f1), n) == theirs(uplo, n, p(f2), n) == 0
    agree(f1, f2, tol * n)
    b1, b2 = a.copy(order="F"), a.copy(order="F")
    b1[17, 17] = b2[17, 17] = -1.0
    assert ours(uplo, n, p(b1), n) == theirs(uplo, n, p(b2), n) > 0


@pytest.mark.parametrize("pfx,dt,ct,tol", REF_PRECS)
@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("trans", [NO, TR])
@pytest.mark.parametrize("diag", [NONUNIT, UNIT])
def test_trsm_matches_reference(C, R, pfx, dt, ct, tol, side, uplo, trans, diag):
    rng = np.random.default_rng(12)
    m, n = 23, 17
    k = m if side == LEFT else n
    a = F(rng.uniform(-1, 1, (k, k)) + 4 * np.eye(k), dt)
    b = F(rng.uniform(-1, 1, (m, n)), dt)
    ours, theirs = both(C, R, f"plasma_core_{pfx}trsm",
                        [ctypes.c_int] * 6 + [ct, ctypes.c_void_p, ctypes.c_int,
                                              ctypes.c_void_p, ctypes.c_int])
    x1, x2 = b.copy(order="F"), b.copy(order="F")
    ours(side, uplo, trans, diag, m, n, 0.75, p(a), k, p(x1), m)
    theirs(side, uplo, trans, diag, m, n, 0.75, p(a), k, p(x2), m)
    agree(x1, x2, tol * k)


@pytest.mark.parametrize("pfx,dt,ct,tol", REF_PRECS)
@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("trans", [NO, TR])
def test_syrk_matches_reference(C, R, pfx, dt, ct, tol, uplo, trans):
    rng = np.random.default_rng(13)
    n, k = 19, 11
    a = F(rng.uniform(-1, 1, (n, k) if trans == NO else (k, n)), dt)
    c0 = F(rng.uniform(-1, 1, (n, n)), dt)
    ours, theirs = both(C, R, f"plasma_core_{pfx}syrk",
                        [ctypes.c_int] * 4 + [ct, ctypes.c_void_p, ctypes.c_int, ct,
                                              ctypes.c_void_p, ctypes.c_int])
    c1, c2 = c0.copy(order="F"), c0.copy(order="F")
    ours(uplo, trans, n, k, -1.0, p(a), a.shape[0], 1.0, p(c1), n)
    theirs(uplo, trans, n, k, -1.0, p(a), a.shape[0], 1.0, p(c2), n)
    agree(c1, c2, tol * k)          # the other triangle untouched by both


@pytest.mark.parametrize("pfx,dt,ct,tol", REF_PRECS)
@pytest.mark.parametrize("ta", [NO, TR])
@pytest.mark.parametrize("tb", [NO, TR])
def test_gemm_matches_reference(C, R, pfx, dt, ct, tol, ta, tb):
    rng = np.random.default_rng(14)
    m, n, k = 13, 17, 9
    a = F(rng.uniform(-1, 1, (m, k) if ta == NO else (k, m)), dt)
    b = F(rng.uniform(-1, 1, (k, n) if tb == NO else (n, k)), dt)
    c0 = F(rng.uniform(-1, 1, (m, n)), dt)
    ours, theirs = both(C, R, f"plasma_core_{pfx}gemm",
                        [ctypes.c_int] * 5 + [ct, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_int, ct, ctypes.c_void_p, ctypes.c_int])
    c1, c2 = c0.copy(order="F"), c0.copy(order="F")
    ours(ta, tb, m, n, k, -1.0, p(a), a.shape[0], p(b), b.shape[0], 1.0, p(c1), m)
    theirs(ta, tb, m, n, k, -1.0, p(a), a.shape[0], p(b), b.shape[0], 1.0, p(c2), m)
    agree(c1, c2, tol * k)


@pytest.mark.parametrize("side", [LEFT, RIGHT])
@pytest.mark.parametrize("uplo", [LO, UP])
def test_dsymm_matches_reference(C, R, side, uplo):
    rng = np.random.default_rng(15)
    m, n = 12, 9
    k = m if side == LEFT else n
    a = F(rng.uniform(-1, 1, (k, k)), np.float64)
    b = F(rng.uniform(-1, 1, (m, n)), np.float64)
    c0 = F(rng.uniform(-1, 1, (m, n)), np.float64)
    ours, theirs = both(C, R, "plasma_core_dsymm",
                        [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                                              ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_void_p, ctypes.c_int])
    c1, c2 = c0.copy(order="F"), c0.copy(order="F")
    ours(side, uplo, m, n, -1.0, p(a), k, p(b), m, 1.0, p(c1), m)
    theirs(side, uplo, m, n, -1.0, p(a), k, p(b), m, 1.0, p(c2), m)
    agree(c1, c2, 1e-13 * k)


@pytest.mark.parametrize("pfx,dt,ct,tol", REF_PRECS)
@pytest.mark.parametrize("uplo", [LO, UP, GE])
@pytest.mark.parametrize("trans,m,n", [(NO, 7, 5), (NO, 5, 7), (TR, 5, 7), (TR, 6, 6)])
def test_lacpy_matches_reference(C, R, pfx, dt, ct, tol, uplo, trans, m, n):
    """Exact copies.  Transposed copies with m > n are left out: the
    reference's loop reads a column past A there (core_zlacpy.c:80)."""
    rng = np.random.default_rng(16)
    a = F(rng.uniform(-1, 1, (m, n)), dt)
    shape = (m, n) if trans == NO else (n, m)
    ours, theirs = both(C, R, f"plasma_core_{pfx}lacpy",
                        [ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_int])
    b1, b2 = F(np.full(shape, 9.0), dt), F(np.full(shape, 9.0), dt)
    ours(uplo, trans, m, n, p(a), m, p(b1), shape[0])
    theirs(uplo, trans, m, n, p(a), m, p(b2), shape[0])
    np.testing.assert_array_equal(b1, b2)


@pytest.mark.parametrize("pfx,dt,ct,tol", REF_PRECS)
@pytest.mark.parametrize("trans", [NO, TR])
def test_geadd_matches_reference(C, R, pfx, dt, ct, tol, trans):
    rng = np.random.default_rng(17)
    m, n = 8, 6
    a = F(rng.uniform(-1, 1, (m, n) if trans == NO else (n, m)), dt)
    b0 = F(rng.uniform(-1, 1, (m, n)), dt)
    ours, theirs = both(C, R, f"plasma_core_{pfx}geadd",
                        [ctypes.c_int] * 3 + [ct, ctypes.c_void_p, ctypes.c_int, ct,
                                              ctypes.c_void_p, ctypes.c_int], ctypes.c_int)
    b1, b2 = b0.copy(order="F"), b0.copy(order="F")
    assert (ours(trans, m, n, 1.5, p(a), a.shape[0], -0.5, p(b1), m)
            == theirs(trans, m, n, 1.5, p(a), a.shape[0], -0.5, p(b2), m))
    agree(b1, b2, tol)


@pytest.mark.parametrize("norm", [ONE, INF, FRO, MAX])
def test_dlange_dlansy_match_reference(C, R, norm):
    rng = np.random.default_rng(18)
    m, n = 11, 7
    a = F(rng.uniform(-1, 1, (m, n)), np.float64)
    work = np.zeros(max(m, n))
    v1, v2 = ctypes.c_double(), ctypes.c_double()
    ours, theirs = both(C, R, "plasma_core_dlange",
                        [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p])
    ours(norm, m, n, p(a), m, p(work), ctypes.byref(v1))
    theirs(norm, m, n, p(a), m, p(work), ctypes.byref(v2))
    agree(v1.value, v2.value, 1e-14)
    s = F(rng.uniform(-1, 1, (n, n)), np.float64)
    ours, theirs = both(C, R, "plasma_core_dlansy",
                        [ctypes.c_int] * 3 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p])
    for uplo in (LO, UP):
        ours(norm, uplo, n, p(s), n, p(work), ctypes.byref(v1))
        theirs(norm, uplo, n, p(s), n, p(work), ctypes.byref(v2))
        agree(v1.value, v2.value, 1e-14)


def test_lag2s_slag2d_match_reference(C, R):
    rng = np.random.default_rng(19)
    m, n = 9, 7
    a = F(rng.uniform(-1e3, 1e3, (m, n)), np.float64)
    ours, theirs = both(C, R, "plasma_core_dlag2s",
                        [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                         ctypes.c_void_p, ctypes.c_int], ctypes.c_int)
    s1, s2 = F(np.zeros((m, n)), np.float32), F(np.zeros((m, n)), np.float32)
    assert ours(m, n, p(a), m, p(s1), m) == theirs(m, n, p(a), m, p(s2), m) == 0
    np.testing.assert_array_equal(s1, s2)
    big = a.copy(order="F")
    big[3, 4] = 1e39
    assert (ours(m, n, p(big), m, p(s1), m) == theirs(m, n, p(big), m, p(s2), m)) and \
        ours(m, n, p(big), m, p(s1), m) != 0
    ours, theirs = both(C, R, "plasma_core_slag2d",
                        [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                         ctypes.c_void_p, ctypes.c_int])
    d1, d2 = F(np.zeros((m, n)), np.float64), F(np.zeros((m, n)), np.float64)
    ours(m, n, p(s2), m, p(d1), m)
    theirs(m, n, p(s2), m, p(d2), m)
    np.testing.assert_array_equal(d1, d2)
