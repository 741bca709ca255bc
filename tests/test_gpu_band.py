"""GPU parity of the band Cholesky path (plasma_{d,s}pbtrf / pbtrs / pbsv and
their tile forms) through the C ABI, against the LAPACK fixtures and the CPU
oracle, with the reference tester's acceptance tests (test/test_zpbtrf.c:
155-214, test_zpbsv.c:175-214: ||B - A X||_inf / (n ||A||_F ||X||_inf) < 50
eps, and LAPACK's info when the factorization fails).
"""
import ctypes

import numpy as np
import pytest
import torch

import gen
import oracle
import plasma_b200 as pb
from conftest import EPS, SEPS, TOL

pytestmark = pytest.mark.gpu
LO, UP = pb.PlasmaLower, pb.PlasmaUpper


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


def band_residual(a, x, b):
    """test/test_zpbsv.c:193-199 (Anorm is the Frobenius norm there)."""
    n = a.shape[0]
    r = np.abs(b - a @ x).sum(axis=1).max()
    return r / (n * np.linalg.norm(a) * np.abs(x).sum(axis=1).max())


def band_input(n, kd, nrhs, seed, lower, ldab=None, dtype=np.float64):
    a, _, _, b = gen.band(n, kd, nrhs, seed, dtype)
    ab = gen.to_band(a, kd, lower=lower, ldab=ldab)
    return a, ab, b


def sentinel_positions(ab, kd, lower):
    """Entries of the band array that hold no matrix element: the corner
    positions and the rows past kd+1.  LAPACK never touches them."""
    ldab, n = ab.shape
    mask = np.zeros(ab.shape, dtype=bool)
    mask[kd + 1:, :] = True
    for j in range(n):
        for r in range(kd + 1):
            i = j + r if lower else j - kd + r
            if i < 0 or i >= n:
                mask[r, j] = True
    return mask


# ------------------------------------------------------------------ pbtrf
@pytest.mark.parametrize("n,kd", [(7, 2), (64, 10), (100, 33), (130, 0), (96, 95)])
@pytest.mark.parametrize("nb", [16, 64])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_dpbtrf_vs_lapack_and_oracle(L, golden, n, kd, nb, tag):
    set_nb(L, nb)
    lower = tag == "L"
    a, ab, b = band_input(n, kd, 2, 5000 + n + kd, lower, ldab=kd + 3)
    mask = sentinel_positions(ab, kd, lower)
    ab[mask] = 7.25
    got = np.asfortranarray(ab.copy())
    assert L.plasma_dpbtrf(LO if lower else UP, n, kd, got.ctypes.data, kd + 3) == 0
    ref = golden[f"band{n}_{kd}_{tag}_factor"]
    diff = np.where(mask[:kd + 1], 0.0, got[:kd + 1] - ref)
    assert np.linalg.norm(diff) / np.linalg.norm(a) < TOL * EPS
    # the oracle's tile algorithm on the same tile size
    orc = np.asfortranarray(ab[:kd + 1].copy())
    assert oracle.pbtrf(LO if lower else UP, orc, kd, nb) == 0
    np.testing.assert_allclose(got[:kd + 1], orc, rtol=0, atol=1e-13 * np.abs(orc).max())
    # positions outside the band come back untouched
    np.testing.assert_array_equal(got[mask], ab[mask])
    # the band solve with the factor (test_zpbtrf.c:177-201)
    x = np.asfortranarray(b.copy())
    assert L.plasma_dpbtrs(LO if lower else UP, n, kd, 2, got.ctypes.data, kd + 3,
                           x.ctypes.data, n) == 0
    assert band_residual(a, x, b) < TOL * EPS
    np.testing.assert_allclose(x, golden[f"band{n}_{kd}_{tag}_X"], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("n,kd,col", [(100, 9, 41), (300, 40, 0)])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_dpbtrf_info_and_untouched(L, golden, n, kd, col, tag):
    """A zeroed row and column: LAPACK's info, and AB left as it was."""
    set_nb(L, 32)
    lower = tag == "L"
    a, _, _, _ = gen.band(n, kd, 1, seed=6000 + n)
    a = gen.zerocol(a, col)
    ab = gen.to_band(a, kd, lower=lower)
    keep = ab.copy()
    info = L.plasma_dpbtrf(LO if lower else UP, n, kd, ab.ctypes.data, kd + 1)
    assert info == int(golden[f"bandinfo{n}_{kd}_{tag}"]) > 0
    np.testing.assert_array_equal(ab, keep)
    # pbsv reports the same info and leaves B alone
    b = np.asfortranarray(np.ones((n, 2)))
    assert L.plasma_dpbsv(LO if lower else UP, n, kd, 2, ab.ctypes.data, kd + 1,
                          b.ctypes.data, n) == info
    np.testing.assert_array_equal(b, np.ones((n, 2)))


# ------------------------------------------------------------------ pbsv
@pytest.mark.parametrize("n,kd,nb", [(3000, 100, 128), (3000, 700, 256), (2500, 0, 128),
                                     (2049, 256, 256), (1500, 1499 // 3, 64)])
@pytest.mark.parametrize("nrhs", [1, 70])
@pytest.mark.parametrize("uplo", [LO, UP])
def test_dpbsv_vs_oracle(L, n, kd, nb, nrhs, uplo):
    """Ragged sizes, kd below, at and above the tile size, one right-hand side
    and a block of them (the tensor-core sweep update): the tester's residual
    and the oracle's solution."""
    set_nb(L, nb)
    lower = uplo == LO
    a, ab, b = band_input(n, kd, nrhs, 7000 + n + kd, lower)
    abf, x = np.asfortranarray(ab.copy()), np.asfortranarray(b.copy())
    assert L.plasma_dpbsv(uplo, n, kd, nrhs, abf.ctypes.data, kd + 1, x.ctypes.data, n) == 0
    assert band_residual(a, x, b) < TOL * EPS
    abo, xo = np.asfortranarray(ab.copy()), np.asfortranarray(b.copy())
    assert oracle.pbtrf(oracle.LOWER if lower else oracle.UPPER, abo, kd, nb) == 0
    oracle.pbtrs(oracle.LOWER if lower else oracle.UPPER, abo, kd, xo, nb)
    np.testing.assert_allclose(x, xo, rtol=1e-11, atol=1e-14 * np.abs(xo).max())
    np.testing.assert_allclose(abf, abo, rtol=0, atol=1e-12 * np.abs(abo).max())


@pytest.mark.parametrize("uplo", [LO, UP])
def test_spbsv(L, uplo):
    set_nb(L, 128)
    n, kd = 2000, 300
    lower = uplo == LO
    a, ab, b = band_input(n, kd, 3, 8100, lower, dtype=np.float32)
    abf, x = np.asfortranarray(ab.copy()), np.asfortranarray(b.copy())
    assert L.plasma_spbsv(uplo, n, kd, 3, abf.ctypes.data, kd + 1, x.ctypes.data, n) == 0
    r = band_residual(a.astype(np.float64), x.astype(np.float64), b.astype(np.float64))
    assert r < TOL * SEPS
    abo, xo = np.asfortranarray(ab.copy()), np.asfortranarray(b.copy())
    assert oracle.pbtrf(oracle.LOWER if lower else oracle.UPPER, abo, kd, 128) == 0
    oracle.pbtrs(oracle.LOWER if lower else oracle.UPPER, abo, kd, xo, 128)
    np.testing.assert_allclose(x, xo, rtol=2e-3, atol=1e-4 * np.abs(xo).max())


def test_band_wider_than_matrix(L):
    """kd >= n fails the band descriptor check, as in the reference
    (control/descriptor.c:364-367)."""
    set_nb(L, 16)
    ab = np.asfortranarray(np.ones((10, 8)))
    assert L.plasma_dpbtrf(LO, 8, 9, ab.ctypes.data, 10) == pb.PlasmaErrorIllegalValue


def test_lookahead_off_matches(L):
    set_nb(L, 128)
    a, ab, _ = band_input(1500, 400, 1, 8200, True)
    L.plasma_set(pb.PlasmaLookahead, 0)
    f0 = np.asfortranarray(ab.copy())
    assert L.plasma_dpbtrf(LO, 1500, 400, f0.ctypes.data, 401) == 0
    L.plasma_set(pb.PlasmaLookahead, 1)
    f1 = np.asfortranarray(ab.copy())
    assert L.plasma_dpbtrf(LO, 1500, 400, f1.ctypes.data, 401) == 0
    # same kernels and the same order of operations per tile: identical bits
    np.testing.assert_array_equal(f0, f1)


def test_band_tile_interface_device_pointer(L):
    """plasma_desc_general_band_create + plasma_omp_dpb2desc (from a device
    array) + plasma_omp_dpbsv + plasma_omp_ddesc2pb, chained on one
    sequence as a tile-API caller of the reference would."""
    set_nb(L, 64)
    n, kd, nrhs = 700, 90, 4
    a, ab, b = band_input(n, kd, nrhs, 8300, True)
    lm = 64 * (1 + (kd + 63) // 64)
    AB, B = pb.plasma_desc_t(), pb.plasma_desc_t()
    assert L.plasma_desc_general_band_create(pb.PlasmaRealDouble, LO, 64, 64, lm, n, 0, 0,
                                             n, n, kd, kd, ctypes.byref(AB)) == 0
    assert L.plasma_desc_general_create(pb.PlasmaRealDouble, 64, 64, n, nrhs, 0, 0, n, nrhs,
                                        ctypes.byref(B)) == 0
    abd = torch.from_numpy(np.ascontiguousarray(ab.T)).cuda()      # column-major
    bf = np.asfortranarray(b.copy())
    seq, req = pb.new_sequence()
    L.plasma_omp_dpb2desc(abd.data_ptr(), kd + 1, AB, ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_dge2desc(bf.ctypes.data, n, B, ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_dpbsv(LO, AB, B, ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_ddesc2pb(AB, abd.data_ptr(), kd + 1, ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_ddesc2ge(B, bf.ctypes.data, n, ctypes.byref(seq), ctypes.byref(req))
    assert L.plasma_sequence_wait(ctypes.byref(seq)) == 0
    assert band_residual(a, bf, b) < TOL * EPS
    fac = abd.cpu().numpy().T
    orc = np.asfortranarray(ab.copy())
    assert oracle.pbtrf(oracle.LOWER, orc, kd, 64) == 0
    np.testing.assert_allclose(fac, orc, rtol=0, atol=1e-12 * np.abs(orc).max())
    # a descriptor of the other triangle is refused
    seq2, req2 = pb.new_sequence()
    L.plasma_omp_dpbtrf(UP, AB, ctypes.byref(seq2), ctypes.byref(req2))
    assert L.plasma_sequence_wait(ctypes.byref(seq2)) == pb.PlasmaErrorIllegalValue
    L.plasma_desc_destroy(ctypes.byref(AB))
    L.plasma_desc_destroy(ctypes.byref(B))


def test_large_band_property(L):
    """n = 32768, kd = 1024, nb = 256: the tester residual at a benchmark
    size (the oracle would take minutes here)."""
    set_nb(L, 256)
    n, kd = 32768, 1024
    rng = np.random.default_rng(8400)
    ab = np.asfortranarray(rng.uniform(-0.5, 0.5, size=(kd + 1, n)))
    ab[0, :] += 2 * kd + 1          # diagonally dominant: SPD
    for d in range(1, kd + 1):
        ab[d, n - d:] = 0.0
    b = np.asfortranarray(rng.uniform(-1, 1, size=(n, 2)))
    abf, x = ab.copy(order="F"), b.copy(order="F")
    assert L.plasma_dpbsv(LO, n, kd, 2, abf.ctypes.data, kd + 1, x.ctypes.data, n) == 0
    # A x through the band storage
    ax = ab[0][:, None] * x
    for d in range(1, kd + 1):
        ax[d:] += ab[d, :n - d][:, None] * x[:n - d]
        ax[:n - d] += ab[d, :n - d][:, None] * x[d:]
    anorm = np.sqrt((ab[0] ** 2).sum() + 2 * (ab[1:] ** 2).sum())
    r = np.abs(b - ax).sum(axis=1).max() / (n * anorm * np.abs(x).sum(axis=1).max())
    assert r < TOL * EPS
