"""GPU parity: the library (through its C ABI) against the LAPACK fixtures and
the CPU oracle, with the reference tester's acceptance tests
(test/test_zpotrf.c:124-152, test_zpotrs.c:140-169, test_zposv.c:137-167,
test_zcposv.c:139-193; tol = 50).
"""
import ctypes

import numpy as np
import pytest
import torch

import gen
import oracle
import plasma_b200 as pb
from conftest import EPS, SEPS, TOL, factor_error, factor_residual, solve_residual

pytestmark = pytest.mark.gpu
LO, UP = pb.PlasmaLower, pb.PlasmaUpper


@pytest.fixture(scope="module")
def L():
    import torch
    assert torch.cuda.is_available()
    lib = pb.lib()
    rc = lib.plasma_init()
    assert rc == 0, rc
    yield lib
    lib.plasma_finalize()


def set_nb(L, nb):
    assert L.plasma_set(pb.PlasmaTuning, pb.PlasmaDisabled) == 0
    assert L.plasma_set(pb.PlasmaNb, nb) == 0


def dpotrf(L, uplo, a):
    f = np.asfortranarray(a.copy())
    info = L.plasma_dpotrf(uplo, f.shape[0], f.ctypes.data, f.shape[0])
    return info, f


# ------------------------------------------------------------------ potrf
@pytest.mark.parametrize("n", [1, 2, 7, 33, 64, 100])
@pytest.mark.parametrize("nb", [16, 32, 64, 128])
def test_dpotrf_small_vs_lapack(L, golden, n, nb):
    set_nb(L, nb)
    a = golden[f"small{n}_A"]
    for uplo, key in ((LO, "L"), (UP, "U")):
        info, f = dpotrf(L, uplo, a)
        assert info == 0
        got = np.tril(f) if uplo == LO else np.triu(f)
        assert factor_error(got, golden[f"small{n}_{key}"], a) < TOL * EPS
        # strict other triangle untouched (LAPACK semantics)
        other = np.triu(f, 1) if uplo == LO else np.tril(f, -1)
        ref = np.triu(a, 1) if uplo == LO else np.tril(a, -1)
        np.testing.assert_array_equal(other, ref)


@pytest.mark.parametrize("n,nb", [(300, 128), (1000, 128), (1000, 256), (300, 64)])
def test_dpotrf_ragged_vs_lapack(L, golden, n, nb):
    set_nb(L, nb)
    a, _ = gen.diag_dominant(n, 5, seed=2000 + n)
    info, f = dpotrf(L, LO, a)
    assert info == 0
    l = np.tril(f)
    v = gen.probe_vector(n)
    np.testing.assert_allclose(np.diag(l), golden[f"ragged{n}_diagL"], rtol=1e-13)
    np.testing.assert_allclose(l @ v, golden[f"ragged{n}_Lv"], rtol=1e-12)
    assert factor_residual(l, a) < TOL
    # upper storage on the same matrix
    info, f = dpotrf(L, UP, a)
    assert info == 0
    u = np.triu(f)
    np.testing.assert_allclose(np.diag(u), golden[f"ragged{n}_diagL"], rtol=1e-13)
    assert factor_residual(u, a, lower=False) < TOL


def test_dpotrf_cfg1_vs_lapack_and_oracle(L, golden):
    """n = 2048, nb = 256, seed 42 (the CPU parity configuration)."""
    set_nb(L, 256)
    a, b = gen.diag_dominant(2048, 1, seed=42)
    info, f = dpotrf(L, LO, a)
    assert info == 0
    l = np.tril(f)
    v = gen.probe_vector(2048)
    np.testing.assert_allclose(np.diag(l), golden["cfg1_diagL"], rtol=1e-14)
    np.testing.assert_allclose(l @ v, golden["cfg1_Lv"], rtol=1e-12)
    np.testing.assert_allclose(l.T @ v, golden["cfg1_Ltv"], rtol=1e-12)
    fo = np.asfortranarray(a.copy())
    assert oracle.potrf(oracle.LOWER, fo, 256) == 0
    assert factor_error(l, np.tril(fo), a) < TOL * EPS
    assert factor_residual(l, a) < TOL


@pytest.mark.parametrize("n,col", [(100, 37), (300, 0), (300, 299), (513, 256)])
def test_dpotrf_nonspd_info(L, golden, n, col):
    a, _ = gen.diag_dominant(n, 1, seed=3000 + n)
    a = gen.zerocol(a, col)
    for nb in (64, 128):
        set_nb(L, nb)
        for uplo, key in ((LO, "lower"), (UP, "upper")):
            info, f = dpotrf(L, uplo, a)
            assert info == int(golden[f"nonspd{n}_{col}_info_{key}"])
            np.testing.assert_array_equal(f, a)   # failed call leaves pA alone
    # the context recovers: a good matrix factors next
    good, _ = gen.diag_dominant(64, 1, seed=1)
    assert dpotrf(L, LO, good)[0] == 0


def test_dpotrf_nan_reports_info(L):
    set_nb(L, 32)
    a, _ = gen.diag_dominant(70, 1, seed=4)
    a[40, 40] = np.nan
    info, _ = dpotrf(L, LO, a)
    assert info == 41


def test_dpotrf_lda_padding(L):
    set_nb(L, 32)
    n, lda = 75, 90
    a, _ = gen.diag_dominant(n, 1, seed=8)
    big = np.full((lda, n), 7.0, order="F")
    big[:n, :] = a
    info = L.plasma_dpotrf(LO, n, big.ctypes.data, lda)
    assert info == 0
    assert np.all(big[n:, :] == 7.0)
    assert factor_residual(np.tril(big[:n, :]), a) < TOL


# ------------------------------------------------------------------ solves
@pytest.mark.parametrize("n", [7, 64, 100])
@pytest.mark.parametrize("nb", [16, 32])
def test_dposv_dpotrs_small(L, golden, n, nb):
    set_nb(L, nb)
    a, b = golden[f"small{n}_A"], golden[f"small{n}_B"]
    for uplo in (LO, UP):
        f = np.asfortranarray(a.copy())
        x = np.asfortranarray(b.copy())
        assert L.plasma_dposv(uplo, n, b.shape[1], f.ctypes.data, n, x.ctypes.data, n) == 0
        assert solve_residual(a, x, b) < TOL * EPS
        np.testing.assert_allclose(x, golden[f"small{n}_X"], rtol=1e-12, atol=1e-15)
        x2 = np.asfortranarray(b.copy())
        assert L.plasma_dpotrs(uplo, n, b.shape[1], f.ctypes.data, n, x2.ctypes.data, n) == 0
        np.testing.assert_allclose(x2, x, rtol=1e-13, atol=1e-16)


@pytest.mark.parametrize("n,nb,nrhs", [(300, 128, 5), (1000, 128, 5), (1000, 256, 17)])
def test_dposv_ragged(L, golden, n, nb, nrhs):
    set_nb(L, nb)
    a, b = gen.diag_dominant(n, nrhs, seed=2000 + n)
    x = np.asfortranarray(b.copy())
    f = np.asfortranarray(a.copy())
    assert L.plasma_dposv(LO, n, nrhs, f.ctypes.data, n, x.ctypes.data, n) == 0
    assert solve_residual(a, x, b) < TOL * EPS
    if nrhs == 5:
        np.testing.assert_allclose(x, golden[f"ragged{n}_X"], rtol=1e-12, atol=1e-15)
    xo = np.asfortranarray(b.copy())
    assert oracle.posv(oracle.LOWER, np.asfortranarray(a.copy()), xo, nb) == 0
    np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-15)


def test_dposv_cfg1(L, golden):
    set_nb(L, 256)
    a, b = gen.diag_dominant(2048, 1, seed=42)
    f = np.asfortranarray(a.copy())
    x = np.asfortranarray(b.copy())
    assert L.plasma_dposv(LO, 2048, 1, f.ctypes.data, 2048, x.ctypes.data, 2048) == 0
    assert solve_residual(a, x, b) < TOL * EPS
    np.testing.assert_allclose(x, golden["cfg1_X"], rtol=1e-12)


def test_device_pointer_path(L):
    """LAPACK-layout routines on device memory (no host copies)."""
    import torch
    set_nb(L, 128)
    n, nrhs = 777, 4
    a, b = gen.diag_dominant(n, nrhs, seed=21)
    # column-major device buffers: row-major storage of the transpose
    A = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    B = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    assert L.plasma_dposv(LO, n, nrhs, A.data_ptr(), n, B.data_ptr(), n) == 0
    torch.cuda.synchronize()
    x = B.cpu().numpy().T
    assert solve_residual(a, x, b) < TOL * EPS
    l = np.tril(A.cpu().numpy().T)
    assert factor_residual(l, a) < TOL


# ------------------------------------------------------------------ FP32
@pytest.mark.parametrize("n,nb", [(100, 32), (1000, 256), (513, 128)])
def test_spotrf_sposv(L, n, nb):
    set_nb(L, nb)
    a, b = gen.diag_dominant(n, 3, seed=n)
    a32, b32 = np.asfortranarray(a.astype(np.float32)), np.asfortranarray(b.astype(np.float32))
    for uplo in (LO, UP):
        f = a32.copy(order="F")
        assert L.plasma_spotrf(uplo, n, f.ctypes.data, n) == 0
        fo = a32.copy(order="F")
        assert oracle.potrf(uplo, fo, nb) == 0
        t = np.tril if uplo == LO else np.triu
        err = np.linalg.norm(t(f).astype(np.float64) - t(fo)) / np.linalg.norm(a)
        assert err < TOL * SEPS
        x, af = b32.copy(order="F"), a32.copy(order="F")
        assert L.plasma_sposv(uplo, n, 3, af.ctypes.data, n, x.ctypes.data, n) == 0
        assert solve_residual(a, x.astype(np.float64), b) < TOL * SEPS


# ------------------------------------------------------------------ dsposv
@pytest.mark.parametrize("n,nb,nrhs", [(64, 32, 1), (300, 128, 2), (2048, 256, 1)])
def test_dsposv_diag_dominant(L, n, nb, nrhs):
    set_nb(L, nb)
    a, b = gen.diag_dominant(n, nrhs, seed=5000 + n)
    x = np.zeros((n, nrhs), order="F")
    it = ctypes.c_int(-99)
    a0, b0 = a.copy(), b.copy()
    info = L.plasma_dsposv(LO, n, nrhs, a.ctypes.data, n, b.ctypes.data, n,
                           x.ctypes.data, n, ctypes.byref(it))
    assert info == 0
    assert 0 <= it.value <= 30
    assert solve_residual(a, x, b) < TOL * EPS
    np.testing.assert_array_equal(a, a0)     # A and B are not modified
    np.testing.assert_array_equal(b, b0)
    xo = np.zeros_like(x, order="F")
    info_o, it_o = oracle.dsposv(oracle.LOWER, a, b, xo, nb)
    assert info_o == 0
    np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("kappa", [1e2, 1e5])
def test_dsposv_spectrum(L, golden, kappa):
    set_nb(L, 64)
    n = 256
    a = gen.spectrum(n, kappa, seed=11)
    xt = golden[f"spec{int(np.log10(kappa))}_xtrue"]
    b = np.asfortranarray(a @ xt)
    x = np.zeros_like(b, order="F")
    it = ctypes.c_int()
    assert L.plasma_dsposv(UP, n, 1, a.ctypes.data, n, b.ctypes.data, n,
                           x.ctypes.data, n, ctypes.byref(it)) == 0
    assert solve_residual(a, x, b) < TOL * EPS
    xl = golden[f"spec{int(np.log10(kappa))}_X"]
    assert np.abs(x - xl).max() / np.abs(xl).max() < kappa * 1e-13


def test_dsposv_fp32_failure(L):
    """kappa = 1e12: the FP32 factorisation breaks down.  In the reference's
    configuration (FP32 factor, IR) the call fails with the factorisation's
    info, iter = -31 and X untouched, as the reference's cancelled sequence
    does; the automatic mode escalates and solves through FP64."""
    set_nb(L, 32)
    n = 128
    a = gen.spectrum(n, 1e12, seed=11)
    b = np.asfortranarray(np.random.default_rng(1).standard_normal((n, 1)))
    x = np.full_like(b, 3.0, order="F")
    it = ctypes.c_int()
    info = L.plasma_dsposv(LO, n, 1, a.ctypes.data, n, b.ctypes.data, n,
                           x.ctypes.data, n, ctypes.byref(it))
    assert info > 0
    assert it.value == -31
    assert np.all(x == 3.0)
    xo = np.full_like(b, 3.0, order="F")
    assert oracle.dsposv(oracle.LOWER, a, b, xo, 32)[0] > 0
    L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorAuto)
    try:
        assert L.plasma_dsposv(LO, n, 1, a.ctypes.data, n, b.ctypes.data, n,
                               x.ctypes.data, n, ctypes.byref(it)) == 0
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)
    assert it.value == -31
    assert solve_residual(a, x, b) < TOL * EPS


@pytest.mark.parametrize("n,nb", [(1000, 192), (700, 96)])
def test_dsposv_sweep_block_sizes(L, n, nb):
    """Refinement sweeps with 64-row blocks (nb = 192) and the tile-sweep
    fallback (nb = 96) converge to the FP64 answer."""
    set_nb(L, nb)
    a = gen.spectrum(n, 1e3, seed=1300 + n)
    b = np.asfortranarray(np.random.default_rng(n).standard_normal((n, 1)))
    x = np.zeros((n, 1), order="F")
    it = ctypes.c_int(0)
    af, bf = np.asfortranarray(a.copy()), np.asfortranarray(b.copy())
    assert L.plasma_dsposv(LO, n, 1, af.ctypes.data, n, bf.ctypes.data, n,
                           x.ctypes.data, n, ctypes.byref(it)) == 0
    assert it.value >= 0
    assert solve_residual(a, x, b) < TOL * EPS


def test_dsposv_nonspd(L):
    """Not positive definite (--zerocol): the FP32 factorisation reports the
    reference's info, iter = -31 and X is not written."""
    set_nb(L, 64)
    n = 200
    a, b = gen.diag_dominant(n, 1, seed=6)
    a = gen.zerocol(a, 150)
    x = np.full_like(b, 3.0, order="F")
    it = ctypes.c_int()
    info = L.plasma_dsposv(LO, n, 1, a.ctypes.data, n, b.ctypes.data, n,
                           x.ctypes.data, n, ctypes.byref(it))
    assert info == 151
    assert it.value == -31
    assert np.all(x == 3.0)


# ------------------------------------------------------------------ async API
def test_async_tile_interface(L):
    """plasma_desc_* + plasma_omp_* + plasma_sequence_wait, as a tile-API
    caller of the reference would chain them."""
    set_nb(L, 64)
    n, nrhs = 200, 3
    a, b = gen.diag_dominant(n, nrhs, seed=31)
    A, B = pb.plasma_desc_t(), pb.plasma_desc_t()
    assert L.plasma_desc_triangular_create(pb.PlasmaRealDouble, LO, 64, 64, n, n,
                                           0, 0, n, n, ctypes.byref(A)) == 0
    assert L.plasma_desc_general_create(pb.PlasmaRealDouble, 64, 64, n, nrhs,
                                        0, 0, n, nrhs, ctypes.byref(B)) == 0
    seq, req = pb.new_sequence()
    af, bf = np.asfortranarray(a.copy()), np.asfortranarray(b.copy())
    L.plasma_omp_dtr2desc(af.ctypes.data, n, A, ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_dge2desc(bf.ctypes.data, n, B, ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_dposv(LO, A, B, ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_ddesc2ge(B, bf.ctypes.data, n, ctypes.byref(seq), ctypes.byref(req))
    assert L.plasma_sequence_wait(ctypes.byref(seq)) == 0
    assert solve_residual(a, bf, b) < TOL * EPS
    # a failing factorisation is reported on its own request
    bad = gen.zerocol(a, 100)
    seq2, req2 = pb.new_sequence()
    bad = np.asfortranarray(bad)
    L.plasma_omp_dtr2desc(bad.ctypes.data, n, A, ctypes.byref(seq2), ctypes.byref(req2))
    L.plasma_omp_dpotrf(LO, A, ctypes.byref(seq2), ctypes.byref(req2))
    assert L.plasma_sequence_wait(ctypes.byref(seq2)) == 101
    assert req2.status == 101
    L.plasma_desc_destroy(ctypes.byref(A))
    L.plasma_desc_destroy(ctypes.byref(B))


def test_lookahead_off_matches(L):
    set_nb(L, 128)
    a, _ = gen.diag_dominant(1000, 1, seed=99)
    L.plasma_set(pb.PlasmaLookahead, 0)
    i0, f0 = dpotrf(L, LO, a)
    L.plasma_set(pb.PlasmaLookahead, 1)
    i1, f1 = dpotrf(L, LO, a)
    assert i0 == 0 and i1 == 0
    # same kernels, same order of operations per tile: identical bits
    np.testing.assert_array_equal(f0, f1)


def test_large_dposv_property(L):
    """n = 8192, nrhs = 16 (a benchmark size): tester residual < 50 eps."""
    import torch
    set_nb(L, 256)
    n, nrhs = 8192, 16
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.rand(n, n, generator=g, device="cuda", dtype=torch.float64) - 0.5
    A = torch.tril(A) + torch.tril(A, -1).T
    A.diagonal().add_(n)
    B = torch.rand(n, nrhs, generator=g, device="cuda", dtype=torch.float64) * 2 - 1
    Af = A.clone()          # symmetric: row-major == column-major
    Xf = B.T.contiguous()   # column-major n x nrhs
    assert L.plasma_dposv(LO, n, nrhs, Af.data_ptr(), n, Xf.data_ptr(), n) == 0
    torch.cuda.synchronize()
    X = Xf.T
    R = B - A @ X
    an = A.abs().sum(1).max()
    res = (R.abs().sum(1).max() / (n * an * X.abs().sum(1).max())).item()
    assert res < TOL * EPS


# ------------------------------------------------------------------ tensor-core factors
def dsposv_ex(L, uplo, a, b):
    n, nrhs = b.shape
    x = np.zeros((n, nrhs), order="F")
    it = ctypes.c_int(-99)
    info = pb.plasma_dsposv_info_t()
    rc = L.plasma_dsposv_ex(uplo, n, nrhs, a.ctypes.data, n, b.ctypes.data, n,
                            x.ctypes.data, n, ctypes.byref(it), ctypes.byref(info))
    return rc, it.value, x, info


@pytest.mark.parametrize("mode", [pb.PlasmaFactorTF32, pb.PlasmaFactorBF16])
@pytest.mark.parametrize("n,nb", [(1024, 256), (1000, 256), (640, 128)])
def test_dsposv_tensor_core_factor(L, mode, n, nb):
    """TF32 / BF16 products on tcgen05 with FP32 accumulation, refined to
    FP64 accuracy (ragged n is padded to whole tiles internally)."""
    set_nb(L, nb)
    L.plasma_set(pb.PlasmaMixedPrecisionMode, mode)
    try:
        a, b = gen.diag_dominant(n, 2, seed=700 + n)
        rc, it, x, info = dsposv_ex(L, LO, a, b)
        assert rc == 0
        assert info.factor_mode == mode
        assert 0 <= it <= 30              # diagonally dominant: IR converges
        assert solve_residual(a, x, b) < TOL * EPS
        xo = np.zeros_like(x, order="F")
        assert oracle.dsposv(oracle.LOWER, a, b, xo, nb)[0] == 0
        np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-15)
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)


@pytest.mark.parametrize("mode", [pb.PlasmaFactorFP32, pb.PlasmaFactorTF32,
                                  pb.PlasmaFactorBF16])
@pytest.mark.parametrize("n,nb", [(1024, 256), (1000, 256), (777, 128)])
def test_dsposv_upper_storage(L, mode, n, nb):
    """uplo = Upper: the FP32 copy is built in lower storage from transposed
    upper tiles (only the upper triangle of A is read: the strictly lower
    part holds NaN), so the factor is the one of uplo = Lower; the answer
    matches the oracle and the refinement takes the same number of steps."""
    set_nb(L, nb)
    L.plasma_set(pb.PlasmaMixedPrecisionMode, mode)
    try:
        a, b = gen.diag_dominant(n, 2, seed=900 + n)
        au = np.asfortranarray(np.triu(a) + np.tril(np.full_like(a, np.nan), -1))
        rc, it_up, x, info = dsposv_ex(L, UP, au, b)
        assert rc == 0
        assert info.factor_mode == mode
        assert 0 <= it_up <= 30
        assert solve_residual(a, x, b) < TOL * EPS
        rc, it_lo, xl, _ = dsposv_ex(L, LO, np.asfortranarray(a.copy()), b)
        assert rc == 0 and abs(it_up - it_lo) <= 1
        xo = np.zeros_like(x, order="F")
        assert oracle.dsposv(oracle.UPPER, np.asfortranarray(a.copy()), b, xo, nb)[0] == 0
        np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-15)
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)


@pytest.mark.parametrize("mode", [pb.PlasmaFactorTF32, pb.PlasmaFactorBF16])
def test_tensor_core_factor_quality(L, mode):
    """The low-precision factor itself: ||A - L L^T|| / ||A|| at the level of
    the product precision (checked through one refinement-free solve)."""
    set_nb(L, 256)
    L.plasma_set(pb.PlasmaMixedPrecisionMode, mode)
    try:
        n = 1536
        a = gen.spectrum(n, 1e2, seed=11)
        xt = np.random.default_rng(12).standard_normal((n, 1))
        b = np.asfortranarray(a @ xt)
        rc, it, x, info = dsposv_ex(L, LO, a, b)
        assert rc == 0 and it >= 0
        assert solve_residual(a, x, b) < TOL * EPS
        assert np.abs(x - xt).max() / np.abs(xt).max() < 1e-12
        # convergence speed reflects the product precision
        assert it <= (6 if mode == pb.PlasmaFactorTF32 else 12)
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)


@pytest.mark.parametrize("mode,bound", [(pb.PlasmaFactorFP32, 2e-6),
                                        (pb.PlasmaFactorTF32, 4e-3),
                                        (pb.PlasmaFactorBF16, 3e-2)])
@pytest.mark.parametrize("n,nb", [(1024, 256), (768, 128)])
def test_low_precision_factor_backward_error(L, mode, bound, n, nb):
    """spotrf with the product precision of PlasmaMixedPrecisionMode on a
    matrix whose off-diagonal part matters: ||A - L L^T||_F / ||A||_F is at
    the level of the product precision (a wrong tile or operand gives O(1))."""
    set_nb(L, nb)
    L.plasma_set(pb.PlasmaMixedPrecisionMode, mode)
    try:
        a = gen.spectrum(n, 1e3, seed=11)
        f = np.asfortranarray(a.astype(np.float32))
        assert L.plasma_spotrf(LO, n, f.ctypes.data, n) == 0
        l = np.tril(f).astype(np.float64)
        berr = np.linalg.norm(a - l @ l.T) / np.linalg.norm(a)
        assert berr < bound, berr
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)


@pytest.mark.parametrize("mode", [pb.PlasmaFactorTF32, pb.PlasmaFactorBF16])
@pytest.mark.parametrize("refine", [pb.PlasmaRefineGMRES, pb.PlasmaRefineAuto])
def test_gmres_ir_ill_conditioned(L, mode, refine):
    """kappa = 1e5: classical IR with a TF32/BF16 factor stalls; GMRES-IR
    preconditioned by the same factor reaches the FP64 stopping rule."""
    set_nb(L, 256)
    L.plasma_set(pb.PlasmaMixedPrecisionMode, mode)
    L.plasma_set(pb.PlasmaRefinement, refine)
    try:
        n, kappa = 1536, 1e5
        a = gen.spectrum(n, kappa, seed=11)
        xt = np.random.default_rng(12).standard_normal((n, 1))
        b = np.asfortranarray(a @ xt)
        rc, it, x, info = dsposv_ex(L, LO, a, b)
        assert rc == 0
        assert it >= 0, "fell back to FP64"
        assert info.refinement == pb.PlasmaRefineGMRES
        assert info.gmres_iterations > 0
        assert solve_residual(a, x, b) < TOL * EPS
        assert np.abs(x - xt).max() / np.abs(xt).max() < kappa * 1e-14
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)
        L.plasma_set(pb.PlasmaRefinement, pb.PlasmaRefineIR)


def _errors(a, x, xt):
    """Normwise backward error ||b - A x||_inf / (||A||_inf ||x||_inf) with
    b = A x_true, and forward error ||x - x_true||_inf / ||x_true||_inf."""
    r = a @ xt - a @ x
    be = np.abs(r).max() / (np.abs(a).sum(axis=1).max() * np.abs(x).max())
    fe = np.abs(x - xt).max() / np.abs(xt).max()
    return be, fe


@pytest.mark.parametrize("mode", [pb.PlasmaFactorFP32, pb.PlasmaFactorTF32,
                                  pb.PlasmaFactorBF16, pb.PlasmaFactorAuto])
@pytest.mark.parametrize("refine", [pb.PlasmaRefineGMRES, pb.PlasmaRefineAuto])
def test_gmres_ir_kappa_1e8(L, mode, refine):
    """kappa = 1e8, the condition GMRES-IR is there for: the FP32 factor
    preconditions GMRES to the FP64 stopping rule without the FP64 fallback;
    a TF32 / BF16 factor that cannot get there escalates to FP32 (the report
    says which precision answered).  Backward error <= 50 n eps, forward
    error <= kappa * 1e-14."""
    set_nb(L, 256)
    L.plasma_set(pb.PlasmaMixedPrecisionMode, mode)
    L.plasma_set(pb.PlasmaRefinement, refine)
    try:
        n, kappa = 2048, 1e8
        a = gen.spectrum(n, kappa, seed=11)
        xt = np.random.default_rng(12).standard_normal((n, 1))
        b = np.asfortranarray(a @ xt)
        rc, it, x, info = dsposv_ex(L, LO, a, b)
        assert rc == 0
        assert it >= 0 and info.fallback_fp64 == 0, (it, info.as_dict())
        assert info.refinement == pb.PlasmaRefineGMRES and info.gmres_iterations > 0
        if mode == pb.PlasmaFactorFP32:
            assert info.factor_mode == pb.PlasmaFactorFP32 and info.attempts == 1
        be, fe = _errors(a, x, xt)
        assert be <= 50 * n * EPS, be
        assert fe <= kappa * 1e-14, fe
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)
        L.plasma_set(pb.PlasmaRefinement, pb.PlasmaRefineIR)


def test_gmres_ir_kappa_1e8_fixture(L, golden):
    """n = 256, kappa = 1e8 (the spec8 fixture): FP32 factor + GMRES-IR
    against LAPACK's FP64 dposv answer and x_true."""
    set_nb(L, 64)
    L.plasma_set(pb.PlasmaRefinement, pb.PlasmaRefineGMRES)
    try:
        n, kappa = 256, 1e8
        a = gen.spectrum(n, kappa, seed=11)
        xt = golden["spec8_xtrue"]
        b = np.asfortranarray(a @ xt)
        rc, it, x, info = dsposv_ex(L, LO, a, b)
        assert rc == 0 and it >= 0 and info.fallback_fp64 == 0, (rc, it, info.as_dict())
        be, fe = _errors(a, x, xt)
        assert be <= 50 * n * EPS
        assert fe <= kappa * 1e-14
        xl = golden["spec8_X"]
        assert np.abs(x - xl).max() / np.abs(xl).max() <= kappa * 1e-14
    finally:
        L.plasma_set(pb.PlasmaRefinement, pb.PlasmaRefineIR)


@pytest.mark.parametrize("mode", [pb.PlasmaFactorTF32, pb.PlasmaFactorBF16])
def test_ir_stall_escalates_to_fp32(L, mode):
    """kappa = 1e5 with classical IR: a TF32 / BF16 factor does not contract
    the residual; instead of running out 30 steps and the FP64 fallback the
    solver escalates to the FP32 factor, which refines (iter >= 0)."""
    set_nb(L, 256)
    L.plasma_set(pb.PlasmaMixedPrecisionMode, mode)
    try:
        n, kappa = 2048, 1e5
        a = gen.spectrum(n, kappa, seed=11)
        xt = np.random.default_rng(12).standard_normal((n, 1))
        b = np.asfortranarray(a @ xt)
        rc, it, x, info = dsposv_ex(L, LO, a, b)
        assert rc == 0 and it >= 0 and info.fallback_fp64 == 0
        assert info.factor_mode == pb.PlasmaFactorFP32 and info.attempts >= 2
        assert solve_residual(a, x, b) < TOL * EPS
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)


@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("n,nb", [(1000, 128), (777, 256), (64, 64), (1000, 192),
                                  (500, 96), (4100, 512)])
def test_single_rhs_sweeps(L, uplo, n, nb):
    """nrhs = 1 uses the one-launch block sweeps (ticketed row blocks with
    ready flags) when nb is a multiple of 64 and the tile sweeps otherwise
    (nb = 96); compare with the oracle."""
    set_nb(L, nb)
    a, b = gen.diag_dominant(n, 1, seed=1100 + n)
    x, af = np.asfortranarray(b.copy()), np.asfortranarray(a.copy())
    assert L.plasma_dposv(uplo, n, 1, af.ctypes.data, n, x.ctypes.data, n) == 0
    xo = np.asfortranarray(b.copy())
    assert oracle.posv(uplo, np.asfortranarray(a.copy()), xo, nb) == 0
    np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-15)
    # FP32
    a32 = np.asfortranarray(a.astype(np.float32))
    x32 = np.asfortranarray(b.astype(np.float32))
    assert L.plasma_sposv(uplo, n, 1, a32.ctypes.data, n, x32.ctypes.data, n) == 0
    assert solve_residual(a, x32.astype(np.float64), b) < TOL * SEPS


@pytest.mark.parametrize("n,nb,prec", [(8192, 256, "d"), (3000, 256, "s"), (1000, 128, "d"),
                                       (777, 192, "d"), (1024, 128, "s")])
def test_upper_storage_through_lower_tiles(L, n, nb, prec):
    """uplo = Upper in the LAPACK-layout drivers: the upper triangle goes to
    lower tiles transposed and is factored there (tensor-core updates), then
    comes back transposed.  The factor matches the oracle's upper factor, the
    solution the oracle's, and the strictly lower part of pA (NaN here) is
    neither read nor written -- host and device arrays."""
    set_nb(L, nb)
    a, b = gen.diag_dominant(n, 4, seed=1300 + n)
    dt, eps = (np.float64, EPS) if prec == "d" else (np.float32, SEPS)
    au = np.triu(a) + np.tril(np.full_like(a, np.nan), -1)
    fo = np.asfortranarray(a.copy())
    assert oracle.potrf(oracle.UPPER, fo, nb) == 0
    uo = np.triu(fo)
    # potrf, host array
    f = np.asfortranarray(au.astype(dt))
    assert getattr(L, f"plasma_{prec}potrf")(UP, n, f.ctypes.data, n) == 0
    assert np.isnan(np.tril(f, -1)[np.tril_indices(n, -1)]).all()
    err = np.linalg.norm(np.triu(f).astype(np.float64) - uo) / np.linalg.norm(a)
    assert err < TOL * eps, err
    # posv, device arrays
    A = torch.from_numpy(np.ascontiguousarray(au.astype(dt).T)).cuda()
    B = torch.from_numpy(np.ascontiguousarray(b.astype(dt).T)).cuda()
    assert getattr(L, f"plasma_{prec}posv")(UP, n, 4, A.data_ptr(), n, B.data_ptr(), n) == 0
    fd = A.cpu().numpy().T
    assert np.isnan(fd[np.tril_indices(n, -1)]).all()
    assert np.linalg.norm(np.triu(fd).astype(np.float64) - uo) / np.linalg.norm(a) < TOL * eps
    x = B.cpu().numpy().T.astype(np.float64)
    assert solve_residual(a, x, b) < TOL * eps
    if prec == "d":
        xo = np.asfortranarray(b.copy())
        assert oracle.posv(oracle.UPPER, np.asfortranarray(a.copy()), xo, nb) == 0
        assert np.abs(x - xo).max() / np.abs(xo).max() < 1e-13


@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("n,nb,nrhs", [(1000, 256, 16), (777, 128, 3), (2048, 256, 17),
                                       (1000, 192, 32), (300, 64, 2), (4100, 512, 5)])
def test_multi_rhs_sweeps(L, uplo, n, nb, nrhs):
    """2 <= nrhs <= 32 uses the one-launch multi-column block sweeps (16
    columns per launch; FP64 64-row and FP32 128-row blocks); compare with
    the oracle and the tester's residual, FP64 and FP32, posv and potrs."""
    set_nb(L, nb)
    a, b = gen.diag_dominant(n, nrhs, seed=1200 + n + nrhs)
    x, af = np.asfortranarray(b.copy()), np.asfortranarray(a.copy())
    assert L.plasma_dposv(uplo, n, nrhs, af.ctypes.data, n, x.ctypes.data, n) == 0
    assert solve_residual(a, x, b) < TOL * EPS
    xo = np.asfortranarray(b.copy())
    assert oracle.posv(uplo, np.asfortranarray(a.copy()), xo, nb) == 0
    assert np.abs(x - xo).max() / np.abs(xo).max() < 1e-13
    # potrs with the factor just computed, on new right-hand sides
    b2 = np.asfortranarray(np.random.default_rng(n).standard_normal((n, nrhs)))
    x2 = np.asfortranarray(b2.copy())
    assert L.plasma_dpotrs(uplo, n, nrhs, af.ctypes.data, n, x2.ctypes.data, n) == 0
    assert solve_residual(a, x2, b2) < TOL * EPS
    a32 = np.asfortranarray(a.astype(np.float32))
    x32 = np.asfortranarray(b.astype(np.float32))
    assert L.plasma_sposv(uplo, n, nrhs, a32.ctypes.data, n, x32.ctypes.data, n) == 0
    assert solve_residual(a, x32.astype(np.float64), b) < TOL * SEPS


@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("n,nb", [(1000, 256), (777, 128), (64, 64)])
def test_dsposv_anorm_tile_pass(L, uplo, n, nb):
    """||A||_inf from the one-pass tile kernel (|a| row sums of the stored
    triangle and its mirror) equals the dense row-sum maximum."""
    set_nb(L, nb)
    a, b = gen.diag_dominant(n, 1, seed=1500 + n)
    x = np.zeros_like(b, order="F")
    it = ctypes.c_int()
    info = pb.plasma_dsposv_info_t()
    af, bf = np.asfortranarray(a), np.asfortranarray(b)
    assert L.plasma_dsposv_ex(uplo, n, 1, af.ctypes.data, n, bf.ctypes.data, n,
                              x.ctypes.data, n, ctypes.byref(it), ctypes.byref(info)) == 0
    ref = np.abs(a).sum(axis=1).max()
    assert abs(info.anorm - ref) <= 1e-13 * ref
    assert solve_residual(a, x, b) < TOL * EPS


@pytest.mark.parametrize("uplo", [LO, UP])
def test_dposv_many_rhs(L, uplo):
    """nrhs >= 64: the sweeps' tile updates run as tensor-core GEMMs on views
    of the factor; compare with the oracle and check the tester's residual."""
    set_nb(L, 128)
    n, nrhs = 700, 100
    a, b = gen.diag_dominant(n, nrhs, seed=1700)
    x, af = np.asfortranarray(b.copy()), np.asfortranarray(a.copy())
    assert L.plasma_dposv(uplo, n, nrhs, af.ctypes.data, n, x.ctypes.data, n) == 0
    assert solve_residual(a, x, b) < TOL * EPS
    xo = np.asfortranarray(b.copy())
    assert oracle.posv(uplo, np.asfortranarray(a.copy()), xo, 128) == 0
    np.testing.assert_allclose(x, xo, rtol=1e-11, atol=1e-14)


# ------------------------------------------------------------------ overlapped upload
def _pinned_colmajor(a):
    """A page-locked host copy of `a` in column-major order."""
    a = np.asarray(a)
    t = torch.empty((a.shape[1], a.shape[0]), dtype=torch.float64, pin_memory=True)
    t.copy_(torch.from_numpy(np.ascontiguousarray(a.T)))
    return t


@pytest.mark.parametrize("n,nb,kappa", [(3000, 256, 1e3), (2048, 128, 1e5), (2500, 64, 1e3)])
def test_dsposv_overlapped_upload(L, n, nb, kappa):
    """A lower-stored host matrix in page-locked memory goes up in groups of
    tile columns while the factorization of the groups already in place runs
    (ragged n included; 16 and 32 groups on 13 streams, so streams take on
    later groups): the answer matches the oracle."""
    set_nb(L, nb)
    a = gen.spectrum(n, kappa, seed=2100 + n)
    xt = np.random.default_rng(n).standard_normal((n, 1))
    b = a @ xt
    A, B = _pinned_colmajor(a), _pinned_colmajor(b)
    X = torch.zeros((1, n), dtype=torch.float64, pin_memory=True)
    it = ctypes.c_int(-99)
    info = pb.plasma_dsposv_info_t()
    assert L.plasma_dsposv_ex(LO, n, 1, A.data_ptr(), n, B.data_ptr(), n, X.data_ptr(), n,
                              ctypes.byref(it), ctypes.byref(info)) == 0
    assert it.value >= 0
    x = X.numpy().T.copy()
    assert solve_residual(a, x, b) < TOL * EPS
    assert abs(info.anorm - np.abs(a).sum(axis=1).max()) <= 1e-13 * info.anorm
    xo = np.zeros((n, 1), order="F")
    assert oracle.dsposv(oracle.LOWER, np.asfortranarray(a), np.asfortranarray(b), xo, nb)[0] == 0
    # two FP64-accurate solutions differ by about kappa * eps (normwise)
    assert np.abs(x - xo).max() / np.abs(xo).max() < kappa * 1e-14


@pytest.mark.parametrize("n,nb,lda", [(3000, 256, 3000), (2500, 64, 2519)])
def test_dsposv_pageable_upload_matches_pinned(L, n, nb, lda):
    """A pageable host matrix goes up through the page-locked staging slots
    (host copies on the staging streams, chunks going round them): the same
    bytes reach the device as from page-locked memory, so the iteration
    count and the solution are identical, with lda > n too."""
    set_nb(L, nb)
    a = gen.spectrum(n, 1e4, seed=2300 + n)
    b = a @ np.random.default_rng(n).standard_normal((n, 1))
    ap = np.zeros((lda, n), order="F")
    ap[:n] = a
    A, B = _pinned_colmajor(ap), _pinned_colmajor(b)
    X = torch.zeros((1, n), dtype=torch.float64, pin_memory=True)
    it = ctypes.c_int(-99)
    assert L.plasma_dsposv(LO, n, 1, A.data_ptr(), lda, B.data_ptr(), n, X.data_ptr(), n,
                           ctypes.byref(it)) == 0
    bp = np.asfortranarray(b)
    xp = np.zeros((n, 1), order="F")
    itp = ctypes.c_int(-98)
    assert L.plasma_dsposv(LO, n, 1, ap.ctypes.data, lda, bp.ctypes.data, n, xp.ctypes.data,
                           n, ctypes.byref(itp)) == 0
    assert itp.value == it.value >= 0
    assert np.array_equal(xp, X.numpy().T)
    assert solve_residual(a, xp, b) < TOL * EPS


@pytest.mark.parametrize("uplo", [LO, UP])
def test_dpotrf_pageable_matches_pinned(L, uplo):
    """dpotrf on a pageable array (up and back down through the staging
    slots, chunks of whole columns, a ragged last tile column) returns the
    same factor, bit for bit, as on a page-locked copy of it."""
    set_nb(L, 128)
    n, lda = 1500, 1507
    a, _ = gen.diag_dominant(n, 1, seed=77)
    ap = np.zeros((lda, n), order="F")
    ap[:n] = a
    ap[n:] = 5.0                      # rows below the matrix stay as they are
    A = _pinned_colmajor(ap)
    assert L.plasma_dpotrf(uplo, n, A.data_ptr(), lda) == 0
    assert L.plasma_dpotrf(uplo, n, ap.ctypes.data, lda) == 0
    assert np.array_equal(ap, A.numpy().T)
    assert np.all(ap[n:] == 5.0)


def test_dsposv_overlapped_upload_fallback(L):
    """kappa = 1e12: the FP32 factorization fails while later column groups
    are still on their way.  The reference's configuration fails the call
    (info > 0, iter = -31, X untouched) once the copies are done; in the
    automatic mode the FP64 tiles of A are completed regardless and the
    FP64 fallback solves the system (iter = -31)."""
    set_nb(L, 128)
    n = 2048
    a = gen.spectrum(n, 1e12, seed=11)
    b = np.random.default_rng(1).standard_normal((n, 1))
    A, B = _pinned_colmajor(a), _pinned_colmajor(b)
    X = torch.full((1, n), 3.0, dtype=torch.float64, pin_memory=True)
    it = ctypes.c_int()
    assert L.plasma_dsposv(LO, n, 1, A.data_ptr(), n, B.data_ptr(), n, X.data_ptr(), n,
                           ctypes.byref(it)) > 0
    assert it.value == -31
    assert bool((X == 3.0).all())
    L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorAuto)
    try:
        assert L.plasma_dsposv(LO, n, 1, A.data_ptr(), n, B.data_ptr(), n, X.data_ptr(), n,
                               ctypes.byref(it)) == 0
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)
    assert it.value == -31
    assert solve_residual(a, X.numpy().T.copy(), b) < TOL * EPS


# ------------------------------------------------------------------ potri / poinv
def _factor_with_noise(a, uplo, seed):
    """The Cholesky factor in the uplo triangle, noise in the other one
    (which potri must leave as it is)."""
    n = a.shape[0]
    lf = np.linalg.cholesky(a)
    f = np.asfortranarray(lf if uplo == LO else lf.T)
    mask = (np.triu(np.ones((n, n), bool), 1) if uplo == LO
            else np.tril(np.ones((n, n), bool), -1))
    f[mask] = np.random.default_rng(seed).standard_normal(int(mask.sum()))
    return f, mask


@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("n,nb", [(64, 64), (300, 128), (777, 256), (1024, 256)])
def test_potri_against_oracle(L, uplo, n, nb):
    """plasma_dpotri against the oracle's dtrtri + dlauum with the reference
    tester's check (test/test_zpotri.c:135-155): ||inv - inv_ref||_F /
    ||inv_ref||_F < 50 eps on the uplo triangle; the other triangle of pA
    is not touched."""
    set_nb(L, nb)
    a, _ = gen.diag_dominant(n, 1, seed=4100 + n)
    f, mask = _factor_with_noise(a, uplo, n)
    ref = np.asfortranarray(f.copy())
    assert oracle.potri(uplo, ref) == 0
    got = np.asfortranarray(f.copy())
    assert L.plasma_dpotri(uplo, n, got.ctypes.data, n) == 0
    tri = np.tril if uplo == LO else np.triu
    assert np.linalg.norm(tri(got) - tri(ref)) / np.linalg.norm(tri(ref)) < TOL * EPS
    np.testing.assert_array_equal(got[mask], f[mask])
    # FP32
    f32 = np.asfortranarray(f.astype(np.float32))
    assert L.plasma_spotri(uplo, n, f32.ctypes.data, n) == 0
    assert (np.linalg.norm(tri(f32).astype(np.float64) - tri(ref)) / np.linalg.norm(tri(ref))
            < TOL * SEPS)


@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("n,nb", [(300, 128), (1000, 256)])
def test_poinv_against_oracle(L, uplo, n, nb):
    """plasma_dpoinv = potrf + potri on the matrix itself, against the
    oracle's tile potrf + potri; A inv(A) = I to the tester's tolerance."""
    set_nb(L, nb)
    a, _ = gen.diag_dominant(n, 1, seed=4200 + n)
    ref = np.asfortranarray(a.copy())
    assert oracle.potrf(uplo, ref, nb) == 0
    assert oracle.potri(uplo, ref) == 0
    got = np.asfortranarray(a.copy())
    assert L.plasma_dpoinv(uplo, n, got.ctypes.data, n) == 0
    tri = np.tril if uplo == LO else np.triu
    assert np.linalg.norm(tri(got) - tri(ref)) / np.linalg.norm(tri(ref)) < TOL * EPS
    full = tri(got) + tri(got, -1 if uplo == LO else 1).T
    assert np.abs(a @ full - np.eye(n)).max() < TOL * EPS * n


def test_potri_poinv_info(L):
    """A zero on the factor's diagonal: potri returns its order (dtrtri)
    and leaves pA as it was; poinv of a non-SPD matrix returns potrf's."""
    set_nb(L, 64)
    n = 200
    a, _ = gen.diag_dominant(n, 1, seed=4300)
    f, _ = _factor_with_noise(a, LO, 1)
    f[73, 73] = 0.0
    f[150, 150] = 0.0
    keep = f.copy()
    assert L.plasma_dpotri(LO, n, f.ctypes.data, n) == 74
    np.testing.assert_array_equal(f, keep)
    z = np.asfortranarray(gen.zerocol(a, 120))
    assert L.plasma_dpoinv(LO, n, z.ctypes.data, n) == 121


def _device_colmajor(a, lda):
    """Column-major device copy of a with leading dimension lda."""
    n, m = a.shape
    t = torch.zeros((m, lda), dtype=torch.float64, device="cuda")
    t[:, :n] = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    return t


@pytest.mark.parametrize("n,nb", [(1000, 256), (777, 128)])
def test_dsposv_device_pointer(L, n, nb):
    """A lower-stored device matrix (lda > n) goes to the FP64 and FP32 tile
    copies in one pass inside the solve; the answer matches the oracle."""
    set_nb(L, nb)
    a, b = gen.diag_dominant(n, 2, seed=4400 + n)
    lda = n + 3
    A, B = _device_colmajor(a, lda), _device_colmajor(b, lda)
    X = torch.zeros((2, lda), dtype=torch.float64, device="cuda")
    it = ctypes.c_int(-99)
    assert L.plasma_dsposv(LO, n, 2, A.data_ptr(), lda, B.data_ptr(), lda, X.data_ptr(), lda,
                           ctypes.byref(it)) == 0
    assert 0 <= it.value <= 30
    x = X[:, :n].cpu().numpy().T
    xo = np.zeros((n, 2), order="F")
    assert oracle.dsposv(oracle.LOWER, np.asfortranarray(a), np.asfortranarray(b), xo, nb)[0] == 0
    np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-15)
    # the caller's array is not modified
    np.testing.assert_array_equal(A[:, :n].cpu().numpy().T, a)


def test_dsposv_device_pointer_fp32_overflow(L):
    """Entries beyond the FP32 range: the one-pass conversion reports the
    overflow.  The reference's configuration fails the call with info = 1
    (core_zlag2c.c:60-75), iter = -31 and X untouched; the automatic mode
    goes on to the FP64 fallback, which solves the system from the FP64
    tiles the same pass wrote."""
    set_nb(L, 128)
    n = 600
    a, b = gen.diag_dominant(n, 1, seed=4500)
    a = a * 1e39
    A, B = _device_colmajor(a, n), _device_colmajor(b, n)
    X = torch.full((1, n), 3.0, dtype=torch.float64, device="cuda")
    it = ctypes.c_int()
    assert L.plasma_dsposv(LO, n, 1, A.data_ptr(), n, B.data_ptr(), n, X.data_ptr(), n,
                           ctypes.byref(it)) == 1
    assert it.value == -31
    assert bool((X == 3.0).all())
    L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorAuto)
    try:
        assert L.plasma_dsposv(LO, n, 1, A.data_ptr(), n, B.data_ptr(), n, X.data_ptr(), n,
                               ctypes.byref(it)) == 0
    finally:
        L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorFP32)
    assert it.value == -31
    assert solve_residual(a, X.cpu().numpy().T.copy(), b) < TOL * EPS




# ------------------------------------------------------------------ lifecycle
def test_reinit_and_solve_twice(L):
    """plasma_finalize, plasma_set(PlasmaDevice), plasma_init and a solve, twice:
    the kernels' shared-memory limits are set per device, launch errors are
    checked at every synchronisation, and the answers stay right."""
    n = 1500
    a, b = gen.diag_dominant(n, 2, seed=77)
    for _ in range(2):
        assert L.plasma_finalize() == 0
        assert L.plasma_set(pb.PlasmaDevice, 0) == 0
        assert L.plasma_init() == 0
        set_nb(L, 256)
        x, af = np.asfortranarray(b.copy()), np.asfortranarray(a.copy())
        assert L.plasma_dposv(LO, n, 2, af.ctypes.data, n, x.ctypes.data, n) == 0
        assert solve_residual(a, x, b) < TOL * EPS
        xs = np.zeros_like(b, order="F")
        it = ctypes.c_int()
        assert L.plasma_dsposv(LO, n, 2, a.ctypes.data, n, b.ctypes.data, n, xs.ctypes.data, n,
                               ctypes.byref(it)) == 0
        assert solve_residual(a, xs, b) < TOL * EPS
