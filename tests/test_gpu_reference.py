"""GPU parity against the reference PLASMA itself, on the same bytes.

The library (through its C ABI) against
  * reference_fixtures.npz, the outputs of the reference built from its
    sources (tests/golden/make_ref_golden.py): config 1 factor checksums and
    solutions, dsposv iteration counts and solutions on prescribed spectra,
    and the failure semantics (--zerocol info, FP32 overflow, kappa = 1e12);
  * the reference library itself (oracle/_ref/libplasma_ref.so, built by
    oracle/build_ref.sh), when present: the whole config-1 factor with the
    potrf tester's check (test/test_zpotrf.c:124-141);
  * reference_lu_band_fixtures.npz: the reference's dsgesv (kappa 1e2, 1e5)
    and dpbsv outputs and dpbtrf's info;
  * reference_potri_fixtures.npz: its SPD inverse and dpotri's info.
The iteration count may differ by one: the FP32 factor here comes from
tensor-core tiles (three TF32 products per FP32 product) and a different
summation order than OpenBLAS's sgemm.
"""
import ctypes
import os

import numpy as np
import pytest

import gen
import plasma_b200 as pb
from conftest import EPS, TOL, solve_residual
from oracle import ref

pytestmark = pytest.mark.gpu
LO, UP = pb.PlasmaLower, pb.PlasmaUpper


@pytest.fixture(scope="module")
def L():
    import torch
    assert torch.cuda.is_available()
    lib = pb.lib()
    assert lib.plasma_init() == 0
    yield lib
    lib.plasma_finalize()


@pytest.fixture(scope="module")
def rg():
    return np.load(os.path.join(os.path.dirname(__file__), "golden",
                                "reference_fixtures.npz"))


def set_nb(L, nb):
    assert L.plasma_set(pb.PlasmaTuning, pb.PlasmaDisabled) == 0
    assert L.plasma_set(pb.PlasmaNb, nb) == 0


def F(a):
    return np.asfortranarray(np.array(a, dtype=np.float64))


def close(x, xr, tol):
    assert np.abs(x - xr).max() / np.abs(xr).max() < tol


def dsposv(L, uplo, a, b, fill=7.0):
    n, nrhs = b.shape
    x = F(np.full(b.shape, fill))
    af, bf = F(a), F(b)                  # held until the call returns
    it = ctypes.c_int(-99)
    info = L.plasma_dsposv(uplo, n, nrhs, af.ctypes.data, n, bf.ctypes.data, n,
                           x.ctypes.data, n, ctypes.byref(it))
    return info, it.value, x


@pytest.mark.parametrize("key,n,nb,seed", [("cfg1", 2048, 256, 42), ("rag", 1000, 128, 3000)])
def test_factor_matches_reference(L, rg, key, n, nb, seed):
    set_nb(L, nb)
    a, _ = gen.diag_dominant(n, 1, seed=seed)
    v = gen.probe_vector(n)
    an = np.linalg.norm(a)
    for uplo, d, p in ((LO, "diagL", "Lv"), (UP, "diagU", "UTv")):
        f = F(a)
        assert L.plasma_dpotrf(uplo, n, f.ctypes.data, n) == 0
        t = np.tril(f) if uplo == LO else np.triu(f).T
        assert np.abs(np.diag(t) - rg[f"{key}_{d}"]).max() / np.abs(np.diag(t)).max() < TOL * EPS
        assert np.linalg.norm(t @ v - rg[f"{key}_{p}"]) / (an * np.linalg.norm(v)) < TOL * EPS


def test_solves_match_reference(L, rg):
    set_nb(L, 256)
    a, b = gen.diag_dominant(2048, 1, seed=42)
    x, af = F(b), F(a)
    assert L.plasma_dposv(LO, 2048, 1, af.ctypes.data, 2048, x.ctypes.data, 2048) == 0
    close(x, rg["cfg1_dposv_X"], 1e-13)
    set_nb(L, 128)
    a, b = gen.diag_dominant(1000, 3, seed=3000)
    for uplo, key in ((LO, "rag_dposv_X"), (UP, "rag_dposv_up_X")):
        x, af = F(b), F(a)
        assert L.plasma_dposv(uplo, 1000, 3, af.ctypes.data, 1000, x.ctypes.data, 1000) == 0
        close(x, rg[key], 1e-13)
    set_nb(L, 64)
    a, b = gen.diag_dominant(300, 4, seed=3001)
    f = F(a)
    assert L.plasma_dpotrf(LO, 300, f.ctypes.data, 300) == 0
    x = F(b)
    assert L.plasma_dpotrs(LO, 300, 4, f.ctypes.data, 300, x.ctypes.data, 300) == 0
    close(x, rg["potrs_X"], 1e-13)


def test_dsposv_cfg1_matches_reference(L, rg):
    set_nb(L, 256)
    a, b = gen.diag_dominant(2048, 1, seed=42)
    info, it, x = dsposv(L, LO, a, b)
    assert info == int(rg["cfg1_dsposv_info"]) == 0
    assert abs(it - int(rg["cfg1_dsposv_iter"])) <= 1
    close(x, rg["cfg1_dsposv_X"], 1e-13)


@pytest.mark.parametrize("n,nb", [(256, 64), (1000, 128)])
@pytest.mark.parametrize("kexp", [2, 5])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_dsposv_iter_matches_reference(L, rg, n, nb, kexp, tag):
    """dsposv's refinement count (zcposv.c:474-518) within one of the
    reference's, and the solution to within kappa * 1e-13 of its."""
    set_nb(L, nb)
    a = gen.spectrum(n, 10.0 ** kexp, seed=11)
    b = F(a @ np.random.default_rng(12).standard_normal((n, 2)))
    info, it, x = dsposv(L, LO if tag == "L" else UP, a, b)
    key = f"spec_n{n}_k{kexp}_{tag}"
    assert info == int(rg[f"{key}_info"]) == 0
    assert abs(it - int(rg[f"{key}_iter"])) <= 1, (it, int(rg[f"{key}_iter"]))
    close(x, rg[f"{key}_X"], 10.0 ** kexp * 1e-13)
    assert solve_residual(a, x, b) < TOL * EPS


@pytest.mark.parametrize("col", [0, 299, 999])
def test_zerocol_info_matches_reference(L, rg, col):
    """--zerocol: dsposv's and dpotrf's info equal the reference's
    (test/test_zcposv.c:181-192, test_zpotrf.c:143-151); dsposv leaves X
    as it was and returns iter = -31, as the reference does."""
    set_nb(L, 128)
    a, b = gen.diag_dominant(1000, 2, seed=6)
    info, it, x = dsposv(L, LO, gen.zerocol(a, col), b)
    assert info == int(rg[f"fail_zerocol{col}_info"])
    assert it == int(rg[f"fail_zerocol{col}_iter"]) == -31
    assert np.all(x == 7.0)
    f = F(a)
    f[:, col] = 0.0
    assert L.plasma_dpotrf(LO, 1000, f.ctypes.data, 1000) == int(
        rg[f"fail_potrf_zerocol{col}_info"])


@pytest.mark.parametrize("tag", ["L", "U"])
def test_fp32_breakdown_matches_reference(L, rg, tag):
    """kappa = 1e12: the reference's FP32 factor breaks down and the call
    fails (info > 0, iter = -31); so does the library's.  The failing column
    depends on FP32 rounding and is not compared."""
    set_nb(L, 64)
    a = gen.spectrum(256, 1e12, seed=11)
    b = F(np.random.default_rng(1).standard_normal((256, 1)))
    info, it, x = dsposv(L, LO if tag == "L" else UP, a, b)
    assert info > 0 and int(rg[f"fail_k12_{tag}_info"]) > 0
    assert it == int(rg[f"fail_k12_{tag}_iter"]) == -31
    assert np.all(x == 7.0)


def test_overflow_matches_reference(L, rg):
    """An FP32 overflow in the stored triangle of A or in B: info = 1, as the
    reference's lag2c task reports (core_zlag2c.c:60-75)."""
    set_nb(L, 128)
    a, b = gen.diag_dominant(1000, 2, seed=6)
    ao = a.copy()
    ao[5, 3] = ao[3, 5] = 1e39
    bo = b.copy()
    bo[4, 1] = -1e39
    for key, aa, bb in (("fail_ovfA", ao, b), ("fail_ovfB", a, bo)):
        info, it, x = dsposv(L, LO, aa, bb)
        assert info == int(rg[f"{key}_info"]) == 1
        assert it == int(rg[f"{key}_iter"]) == -31
        assert np.all(x == 7.0)


needs_ref = pytest.mark.skipif(not os.path.exists(ref.LIB_PATH),
                               reason="reference library (oracle/_ref) not built")


@needs_ref
def test_cfg1_whole_factor_against_reference_library(L):
    """Config 1 (n = 2048, nb = 256, seed 42): the whole factor against the
    reference library's on the same bytes, ||L - L_ref||_F / ||A||_F < 50
    eps, lower and upper."""
    ref.set_threads(min(8, os.cpu_count() or 1))
    set_nb(L, 256)
    n = 2048
    a, _ = gen.diag_dominant(n, 1, seed=42)
    for uplo in (LO, UP):
        f, fr = F(a), F(a)
        assert L.plasma_dpotrf(uplo, n, f.ctypes.data, n) == 0
        assert ref.dpotrf(uplo, fr, 256) == 0
        t = np.tril if uplo == LO else np.triu
        assert np.linalg.norm(t(f) - t(fr)) / np.linalg.norm(a) < TOL * EPS


@needs_ref
@pytest.mark.parametrize("n,nb,kappa", [(1536, 256, 1e3), (4096, 256, 1e5)])
def test_dsposv_against_reference_library(L, n, nb, kappa):
    """Fresh spectra at sizes the fixtures do not hold: info equal, iter
    within one, solutions within kappa * 1e-13."""
    ref.set_threads(min(8, os.cpu_count() or 1))
    set_nb(L, nb)
    a = gen.spectrum(n, kappa, seed=n)
    b = F(a @ np.random.default_rng(n + 1).standard_normal((n, 1)))
    info, it, x = dsposv(L, LO, a, b)
    xr = F(np.zeros_like(b))
    info_r, it_r = ref.dsposv(LO, F(a), b, xr, nb)
    assert info == info_r == 0
    assert abs(it - it_r) <= 1, (it, it_r)
    close(x, xr, kappa * 1e-13)


@pytest.fixture(scope="module")
def rlb():
    return np.load(os.path.join(os.path.dirname(__file__), "golden",
                                "reference_lu_band_fixtures.npz"))


@pytest.mark.parametrize("n,nb,kexp", [(400, 64, 2), (400, 64, 5), (1000, 128, 5)])
def test_dsgesv_matches_reference(L, rlb, n, nb, kexp):
    """dsgesv (compute/zcgesv.c:363-532) on the reference's fixture: its
    info, refinement without the FP64 fallback in about as many steps (the
    FP32 LU here is tensor-core tiles in another summation order than
    OpenBLAS's), the solution within kappa n eps of the reference's, and
    the tester's residual (test/test_zcgesv.c:150-170)."""
    set_nb(L, nb)
    a = gen.general_spectrum(n, 10.0 ** kexp)
    b = F(np.cos(np.arange(2.0 * n)).reshape(n, 2))
    af, bf = F(a), F(b)
    x = F(np.zeros((n, 2)))
    piv = np.zeros(n, dtype=np.int32)
    it = ctypes.c_int(-99)
    info = L.plasma_dsgesv(n, 2, af.ctypes.data, n, piv.ctypes.data, bf.ctypes.data, n,
                           x.ctypes.data, n, ctypes.byref(it))
    key = f"gesv_n{n}_k{kexp}"
    assert info == int(rlb[f"{key}_info"]) == 0
    assert it.value >= 0 and abs(it.value - int(rlb[f"{key}_iter"])) <= 2, it.value
    close(x, rlb[f"{key}_X"], 10.0 ** kexp * n * EPS)
    assert solve_residual(a, x, b) < TOL * EPS


@pytest.mark.parametrize("n,kd,nb", [(500, 40, 64), (1000, 100, 128)])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_dpbsv_matches_reference(L, rlb, n, kd, nb, tag):
    """Band factor and solve (compute/zpbsv.c) against the reference's
    dpbsv on the same bytes: the factor's diagonal and L v, the solution,
    and the tester's residual."""
    set_nb(L, nb)
    a, abl, abu, b = gen.band(n, kd, 2, seed=7000 + n)
    lower = tag == "L"
    ab, x = F(abl if lower else abu), F(b)
    assert L.plasma_dpbsv(LO if lower else UP, n, kd, 2, ab.ctypes.data, kd + 1,
                          x.ctypes.data, n) == 0
    t = gen.from_band(ab, kd, lower=lower)
    t = t if lower else t.T
    key = f"pb_n{n}_kd{kd}_{tag}"
    close(np.diag(t), rlb[f"{key}_diag"], 1e-12)
    v = gen.probe_vector(n)
    assert np.linalg.norm(t @ v - rlb[f"{key}_Lv"]) / (np.linalg.norm(t) * np.linalg.norm(v)) < 1e-12
    close(x, rlb[f"{key}_X"], 1e-11)
    assert solve_residual(a, x, b) < TOL * EPS


@pytest.mark.parametrize("col,tag", [(0, "L"), (137, "L"), (137, "U")])
def test_dpbtrf_info_matches_reference(L, rlb, col, tag):
    """A zeroed row and column of a band matrix: the reference's dpbtrf info."""
    set_nb(L, 64)
    a, _, _, _ = gen.band(300, 20, 1, seed=7300)
    a[col, :] = 0.0
    a[:, col] = 0.0
    lower = tag == "L"
    ab = F(gen.to_band(a, 20, lower=lower))
    info = L.plasma_dpbtrf(LO if lower else UP, 300, 20, ab.ctypes.data, 21)
    assert info == int(rlb[f"pbinfo_{col}_{tag}"]) == col + 1


@pytest.fixture(scope="module")
def rpi():
    return np.load(os.path.join(os.path.dirname(__file__), "golden",
                                "reference_potri_fixtures.npz"))


@pytest.mark.parametrize("n,nb", [(300, 64), (1000, 128)])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_poinv_matches_reference(L, rpi, n, nb, tag):
    """plasma_dpoinv (factor and inverse, compute/zpoinv.c) against the
    reference's inverse of the same matrix, through the inverse's diagonal
    and sym(inv) v."""
    set_nb(L, nb)
    a, _ = gen.diag_dominant(n, 1, seed=8800 + n)
    lower = tag == "L"
    f = F(a)
    assert L.plasma_dpoinv(LO if lower else UP, n, f.ctypes.data, n) == 0
    t = np.tril(f) if lower else np.triu(f)
    full = t + t.T - np.diag(np.diag(t))
    key = f"potri_n{n}_nb{nb}_{tag}"
    dr = rpi[f"{key}_diag"]
    assert np.linalg.norm(np.diag(t) - dr) / np.linalg.norm(dr) < 1e-12
    v = gen.probe_vector(n)
    assert (np.linalg.norm(full @ v - rpi[f"{key}_Sv"]) / (np.linalg.norm(full) * np.linalg.norm(v))
            < 1e-12)


@pytest.mark.parametrize("col", [0, 137, 299])
@pytest.mark.parametrize("tag", ["L", "U"])
def test_potri_info_matches_reference(L, rpi, col, tag):
    """A zero on the factor's diagonal: the reference's dpotri info."""
    set_nb(L, 64)
    a, _ = gen.diag_dominant(300, 1, seed=9100)
    lower = tag == "L"
    f = F(a)
    assert L.plasma_dpotrf(LO if lower else UP, 300, f.ctypes.data, 300) == 0
    f[col, col] = 0.0
    info = L.plasma_dpotri(LO if lower else UP, 300, f.ctypes.data, 300)
    assert info == int(rpi[f"potriinfo_{col}_{tag}"]) == col + 1
