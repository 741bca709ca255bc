"""GPU parity of the LU-based mixed-precision solver plasma_dsgesv (FP32 LU
with partial pivoting + FP64 refinement, FP64 LU fallback) through the C ABI,
against the LAPACK dgesv fixtures and the CPU oracle, with the reference
tester's acceptance test (test/test_zcgesv.c:133-182: ||B - A X||_inf /
(n ||A||_inf ||X||_inf) < 50 eps, and LAPACK's info on failure).
"""
import ctypes

import numpy as np
import pytest
import torch

import gen
import oracle
import plasma_b200 as pb
from conftest import EPS, TOL, solve_residual

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    assert torch.cuda.is_available()
    lib = pb.lib()
    rc = lib.plasma_init()
    assert rc == 0, rc
    yield lib
    lib.plasma_finalize()


def set_nb(L, nb):
    assert L.plasma_set(pb.PlasmaTuning, pb.PlasmaDisabled) == 0
    assert L.plasma_set(pb.PlasmaNb, nb) == 0


def dsgesv(L, a, b):
    n, nrhs = b.shape
    af, bf = np.asfortranarray(a.copy()), np.asfortranarray(b.copy())
    x = np.zeros((n, nrhs), order="F")
    piv = np.zeros(max(n, 1), dtype=np.int32)
    it = ctypes.c_int(-99)
    info = L.plasma_dsgesv(n, nrhs, af.ctypes.data, n, piv.ctypes.data, bf.ctypes.data, n,
                           x.ctypes.data, n, ctypes.byref(it))
    # A and B are not modified
    np.testing.assert_array_equal(af, a)
    np.testing.assert_array_equal(bf, b)
    return info, it.value, x, piv[:n]


def valid_pivots(piv, n):
    j = np.arange(n)
    return bool(np.all(piv - 1 >= j) and np.all(piv <= n))


@pytest.mark.parametrize("n", [7, 64, 100, 150])
@pytest.mark.parametrize("nb", [16, 64])
def test_dsgesv_vs_lapack(L, golden, n, nb):
    set_nb(L, nb)
    a, b = gen.general(n, 2, seed=9000 + n)
    info, it, x, piv = dsgesv(L, a, b)
    assert info == 0
    assert 0 <= it <= 10
    assert valid_pivots(piv, n)
    assert solve_residual(a, x, b) < TOL * EPS
    np.testing.assert_allclose(x, golden[f"lu{n}_X"], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("kappa,fallback", [(1e2, False), (1e12, True)])
def test_dsgesv_spectrum(L, golden, kappa, fallback):
    """Refinement at kappa = 1e2; the FP64 LU (iter = -31) at kappa = 1e12."""
    set_nb(L, 32)
    n = 100
    a = gen.general_spectrum(n, kappa)
    b = np.asfortranarray(np.cos(np.arange(200.0)).reshape(n, 2))
    info, it, x, piv = dsgesv(L, a, b)
    assert info == 0
    assert (it == -31) == fallback and (fallback or it >= 0)
    assert valid_pivots(piv, n)
    assert solve_residual(a, x, b) < TOL * EPS
    xr = golden[f"gesv_kappa{kappa:.0e}_X"]
    assert np.abs(x - xr).max() / np.abs(xr).max() < 10 * kappa * n * EPS


@pytest.mark.parametrize("n,col", [(64, 20), (100, 0)])
def test_dsgesv_singular_info(L, golden, n, col):
    """A zero column: the FP32 LU meets the zero pivot, the FP64 LU reports
    LAPACK's info."""
    set_nb(L, 16)
    a, _ = gen.general(n, 1, seed=9100 + n)
    a[:, col] = 0.0
    b = np.asfortranarray(np.ones((n, 1)))
    info, it, _, _ = dsgesv(L, np.asfortranarray(a), b)
    assert info == int(golden[f"luinfo{n}_{col}"]) > 0
    assert it == -31


def test_dsgesv_fp32_overflow(L):
    set_nb(L, 32)
    a, b = gen.general(90, 1, seed=77)
    a = np.asfortranarray(a * 1e39)
    info, it, x, _ = dsgesv(L, a, b)
    assert info == 0 and it == -31
    assert solve_residual(a, x, b) < TOL * EPS


@pytest.mark.parametrize("n,nb,nrhs", [(1000, 128, 3), (777, 64, 1), (2048, 256, 1)])
def test_dsgesv_vs_oracle(L, n, nb, nrhs):
    """Ragged sizes: the solution against the oracle's dsgesv."""
    set_nb(L, nb)
    a, b = gen.general(n, nrhs, seed=9200 + n)
    info, it, x, piv = dsgesv(L, a, b)
    assert info == 0 and it >= 0
    assert valid_pivots(piv, n)
    assert solve_residual(a, x, b) < TOL * EPS
    xo = np.zeros((n, nrhs), order="F")
    oinfo, oit, _ = oracle.dsgesv(np.asfortranarray(a), np.asfortranarray(b), xo, nb)
    assert oinfo == 0 and oit >= 0
    np.testing.assert_allclose(x, xo, rtol=1e-8, atol=1e-12 * np.abs(xo).max())


def test_dsgesv_device_pointers(L):
    set_nb(L, 128)
    n, nrhs = 600, 2
    a, b = gen.general(n, nrhs, seed=9300)
    A = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    B = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    X = torch.zeros((nrhs, n), dtype=torch.float64, device="cuda")
    piv = np.zeros(n, dtype=np.int32)
    it = ctypes.c_int()
    assert L.plasma_dsgesv(n, nrhs, A.data_ptr(), n, piv.ctypes.data, B.data_ptr(), n,
                           X.data_ptr(), n, ctypes.byref(it)) == 0
    assert it.value >= 0
    x = X.cpu().numpy().T
    assert solve_residual(a, x, b) < TOL * EPS
    np.testing.assert_array_equal(A.cpu().numpy().T, a)


def test_omp_dsgesv_tile_interface(L):
    """plasma_omp_dsgesv on caller-made descriptors, as the reference's tile
    API caller would chain it (ge2desc, dsgesv, desc2ge, sequence wait)."""
    set_nb(L, 64)
    n, nrhs, nb = 300, 2, 64
    a, b = gen.general(n, nrhs, seed=9400)
    D = {k: pb.plasma_desc_t() for k in ("A", "B", "X", "R", "As", "Xs")}
    for k in D:
        prec = pb.PlasmaRealFloat if k in ("As", "Xs") else pb.PlasmaRealDouble
        cols = n if k in ("A", "As") else nrhs
        assert L.plasma_desc_general_create(prec, nb, nb, n, cols, 0, 0, n, cols,
                                            ctypes.byref(D[k])) == 0
    seq, req = pb.new_sequence()
    af, bf = np.asfortranarray(a.copy()), np.asfortranarray(b.copy())
    x = np.zeros((n, nrhs), order="F")
    piv = np.zeros(n, dtype=np.int32)
    it = ctypes.c_int(-99)
    L.plasma_omp_dge2desc(af.ctypes.data, n, D["A"], ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_dge2desc(bf.ctypes.data, n, D["B"], ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_dsgesv(D["A"], piv.ctypes.data, D["B"], D["X"], D["As"], D["Xs"], D["R"],
                        None, None, None, ctypes.byref(it), ctypes.byref(seq),
                        ctypes.byref(req))
    L.plasma_omp_ddesc2ge(D["X"], x.ctypes.data, n, ctypes.byref(seq), ctypes.byref(req))
    assert L.plasma_sequence_wait(ctypes.byref(seq)) == 0
    assert it.value >= 0
    assert solve_residual(a, x, b) < TOL * EPS
    for k in D:
        L.plasma_desc_destroy(ctypes.byref(D[k]))


def test_dsgesv_tuned_tiles_cluster_panel(L):
    """Tuning on: dsgesv picks 64-wide tiles and the one-launch cluster panel
    (panels of up to 3000 rows); the solution against the oracle's."""
    assert L.plasma_set(pb.PlasmaTuning, pb.PlasmaEnabled) == 0
    n = 3000
    a, b = gen.general(n, 1, seed=9300)
    info, it, x, piv = dsgesv(L, a, b)
    assert info == 0 and it >= 0
    assert valid_pivots(piv, n)
    assert solve_residual(a, x, b) < TOL * EPS
    xo = np.zeros((n, 1), order="F")
    oinfo, oit, _ = oracle.dsgesv(np.asfortranarray(a), np.asfortranarray(b), xo, 64)
    assert oinfo == 0 and oit >= 0
    np.testing.assert_allclose(x, xo, rtol=1e-8, atol=1e-12 * np.abs(xo).max())


def test_dsgesv_fp64_lu_mixed_panels(L):
    """An FP32 overflow in A sends dsgesv straight to the FP64 LU; with
    64-wide tiles at n = 3500 its first panels are taller than a cluster
    holds in FP64 (the per-column kernels), the later ones take the cluster
    panel: the solution meets the tester's residual bound."""
    set_nb(L, 64)
    n = 3500
    a, b = gen.general(n, 1, seed=9400)
    a = np.asfortranarray(a * 1e39)
    info, it, x, piv = dsgesv(L, a, b)
    assert info == 0 and it == -31
    assert valid_pivots(piv, n)
    assert solve_residual(a, x, b) < TOL * EPS
