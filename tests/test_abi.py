"""C-ABI boundary tests that need no GPU.

* the library loads and exports every function include/*.h declares;
* lifecycle and configuration semantics of control/context.c:30-159;
* argument checking of the LAPACK-layout routines (negative codes as in
  compute/zpotrf.c:87-100, zposv.c:103-121, zpotrs.c, zcposv.c:124-147);
* descriptor arithmetic against the reference's formulas
  (control/descriptor.c:134-175, 216-264, include/plasma_descriptor.h:93-151).
Without a GPU the library runs in host-only mode (PLASMA_ALLOW_NO_DEVICE=1):
every call that would touch the device returns PlasmaErrorEnvironment.
"""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import plasma_b200 as pb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(plasma_\w+)\s*\(", src):
            name = m.group(1)
            # skip macros and static inline helpers defined in the headers
            if re.search(r"(#define\s+%s\b)|(PLASMA_HD\s+[\w\s\*]*\b%s\s*\()|"
                         r"(static inline[\w\s\*]*\b%s\s*\()" % (name, name, name), src):
                continue
            names.add(name)
    return sorted(names)


def test_library_exports_every_declared_function():
    L = pb.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert len(declared_functions()) >= 40


def test_python_binding_covers_exports():
    L = pb.lib()
    for name in pb.exported_symbols():
        assert hasattr(L, name), name


@pytest.fixture
def hostonly():
    os.environ["PLASMA_ALLOW_NO_DEVICE"] = "1"
    L = pb.lib()
    rc = L.plasma_init()
    assert rc == 0
    yield L
    L.plasma_finalize()


def test_lifecycle_and_settings(hostonly):
    L = hostonly
    assert L.plasma_init() == pb.PlasmaErrorNotInitialized     # second init
    assert pb.get_param(pb.PlasmaNb) == 256                    # default nb
    assert pb.get_param(pb.PlasmaIb) == 64
    assert pb.get_param(pb.PlasmaTuning) == pb.PlasmaEnabled
    assert L.plasma_set(pb.PlasmaNb, 0) == pb.PlasmaErrorIllegalValue
    assert L.plasma_set(pb.PlasmaNb, -4) == pb.PlasmaErrorIllegalValue
    assert L.plasma_set(pb.PlasmaNb, 384) == 0
    assert pb.get_param(pb.PlasmaNb) == 384
    assert L.plasma_set(pb.PlasmaTuning, 7) == pb.PlasmaErrorIllegalValue
    assert L.plasma_set(pb.PlasmaMixedPrecisionMode, pb.PlasmaFactorBF16) == 0
    assert pb.get_param(pb.PlasmaMixedPrecisionMode) == pb.PlasmaFactorBF16
    assert L.plasma_set(pb.PlasmaMixedPrecisionMode, 9) == pb.PlasmaErrorIllegalValue
    assert L.plasma_set(12345, 1) == pb.PlasmaErrorIllegalValue
    v = ctypes.c_int()
    assert L.plasma_get(12345, ctypes.byref(v)) == pb.PlasmaErrorIllegalValue
    maj, mi, pa = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    L.plasma_version(ctypes.byref(maj), ctypes.byref(mi), ctypes.byref(pa))
    assert (maj.value, mi.value, pa.value) == (25, 5, 27)


def test_not_initialized():
    L = pb.lib()
    L.plasma_finalize()
    assert L.plasma_finalize() == pb.PlasmaErrorNotInitialized
    assert L.plasma_set(pb.PlasmaNb, 128) == pb.PlasmaErrorNotInitialized
    a = np.eye(4, order="F")
    assert L.plasma_dpotrf(pb.PlasmaLower, 4, a.ctypes.data, 4) == pb.PlasmaErrorNotInitialized
    b = np.ones((4, 1), order="F")
    assert L.plasma_dposv(pb.PlasmaLower, 4, 1, a.ctypes.data, 4, b.ctypes.data, 4) == \
        pb.PlasmaErrorNotInitialized


def test_argument_codes(hostonly):
    L = hostonly
    a = np.eye(8, order="F")
    b = np.ones((8, 2), order="F")
    x = np.zeros((8, 2), order="F")
    p, q, r = a.ctypes.data, b.ctypes.data, x.ctypes.data
    lo = pb.PlasmaLower
    # potrf: -1 uplo, -2 n, -4 lda
    assert L.plasma_dpotrf(999, 8, p, 8) == -1
    assert L.plasma_dpotrf(lo, -1, p, 8) == -2
    assert L.plasma_dpotrf(lo, 8, p, 7) == -4
    assert L.plasma_dpotrf(lo, 0, p, 1) == 0
    assert L.plasma_spotrf(999, 8, p, 8) == -1
    # posv / potrs: -1, -2, -3, -5, -7
    for fn in (L.plasma_dposv, L.plasma_dpotrs, L.plasma_sposv, L.plasma_spotrs):
        assert fn(999, 8, 2, p, 8, q, 8) == -1
        assert fn(lo, -1, 2, p, 8, q, 8) == -2
        assert fn(lo, 8, -1, p, 8, q, 8) == -3
        assert fn(lo, 8, 2, p, 7, q, 8) == -5
        assert fn(lo, 8, 2, p, 8, q, 7) == -7
    # quick returns
    assert L.plasma_dposv(lo, 8, 0, p, 8, q, 8) == 0
    assert L.plasma_dpotrs(lo, 0, 0, p, 1, q, 1) == 0
    # dsposv adds -9 and sets iter = 0 on quick return
    it = ctypes.c_int(5)
    assert L.plasma_dsposv(lo, 8, 2, p, 8, q, 8, r, 7, ctypes.byref(it)) == -9
    assert L.plasma_dsposv(999, 8, 2, p, 8, q, 8, r, 8, ctypes.byref(it)) == -1
    assert L.plasma_dsposv(lo, 8, 0, p, 8, q, 8, r, 8, ctypes.byref(it)) == 0
    assert it.value == 0
    # a real call without a device reports the environment error
    assert L.plasma_dpotrf(lo, 8, p, 8) == pb.PlasmaErrorEnvironment


def ref_general_offsets(lm, ln, mb, nb):
    a21 = (lm - lm % mb) * (ln - ln % nb)
    a12 = (lm % mb) * (ln - ln % nb) + a21
    a22 = (lm - lm % mb) * (ln % nb) + a12
    return a21, a12, a22


@pytest.mark.parametrize("lm,ln,mb,nb", [(10, 10, 4, 4), (256, 300, 128, 128),
                                         (1000, 16, 256, 256), (7, 7, 7, 7)])
def test_descriptor_arithmetic(hostonly, lm, ln, mb, nb):
    L = hostonly
    d = pb.plasma_desc_t()
    assert L.plasma_desc_general_init(pb.PlasmaRealDouble, None, mb, nb, lm, ln,
                                      0, 0, lm, ln, ctypes.byref(d)) == 0
    assert (d.A21, d.A12, d.A22) == ref_general_offsets(lm, ln, mb, nb)
    assert d.mt == -(-lm // mb) and d.nt == -(-ln // nb)
    assert d.gmt == -(-lm // mb) and d.gnt == -(-ln // nb)
    assert L.plasma_desc_check(d) == 0
    # a view starting at a tile boundary
    if lm > mb:
        v = L.plasma_desc_view(d, mb, 0, lm - mb, ln)
        assert v.i == mb and v.m == lm - mb and v.mt == -(-(lm - mb) // mb)
    # storage of a general descriptor is gm * gn elements
    assert L.plasma_desc_storage_bytes(d) == lm * ln * 8


@pytest.mark.parametrize("n,nb", [(10, 4), (300, 128), (256, 256), (1000, 96)])
def test_triangular_descriptor(hostonly, n, nb):
    L = hostonly
    d = pb.plasma_desc_t()
    assert L.plasma_desc_triangular_init(pb.PlasmaRealDouble, pb.PlasmaLower, None,
                                         nb, nb, n, n, 0, 0, n, n, ctypes.byref(d)) == 0
    lm1 = n // nb
    mnt = (lm1 * (1 + lm1)) // 2
    assert d.A21 == nb * nb * mnt and d.A12 == nb * nb * mnt
    assert d.A22 == (n - n % nb) * (n % nb) + d.A12
    assert d.type == pb.PlasmaLower
    assert L.plasma_desc_storage_bytes(d) == (mnt * nb * nb + n * (n % nb)) * 8


def test_descriptor_check_errors(hostonly):
    L = hostonly
    d = pb.plasma_desc_t()
    L.plasma_desc_general_init(pb.PlasmaRealDouble, None, 0, 4, 8, 8, 0, 0, 8, 8,
                               ctypes.byref(d))
    assert L.plasma_desc_check(d) == pb.PlasmaErrorIllegalValue      # mb <= 0
    L.plasma_desc_general_init(pb.PlasmaRealDouble, None, 4, 4, 8, 8, 2, 0, 4, 8,
                               ctypes.byref(d))
    assert L.plasma_desc_check(d) == pb.PlasmaErrorIllegalValue      # not aligned
    L.plasma_desc_general_init(pb.PlasmaRealDouble, None, 4, 4, 8, 8, 4, 0, 8, 8,
                               ctypes.byref(d))
    assert L.plasma_desc_check(d) == pb.PlasmaErrorIllegalValue      # out of bounds
    L.plasma_desc_general_init(99, None, 4, 4, 8, 8, 0, 0, 8, 8, ctypes.byref(d))
    assert L.plasma_desc_check(d) == pb.PlasmaErrorIllegalValue      # precision


def test_sequence_request(hostonly):
    L = hostonly
    seq, req = pb.new_sequence()
    assert seq.status == 0 and req.status == 0
    assert L.plasma_request_fail(ctypes.byref(seq), ctypes.byref(req), 7) == 7
    assert seq.status == 7 and req.status == 7


def test_lapack_constants():
    L = pb.lib()
    assert L.plasma_uplo_const(b"L") == pb.PlasmaLower
    assert L.plasma_uplo_const(b"u") == pb.PlasmaUpper
    assert L.plasma_uplo_const(b"G") == pb.PlasmaGeneral
    assert L.plasma_trans_const(b"T") == pb.PlasmaTrans
    assert L.plasma_norm_const(b"I") == 175
    assert L.plasma_side_const(b"R") == 142
    assert L.plasma_diag_const(b"U") == 132


def test_adjoint_argument_codes(hostonly):
    """Illegal arguments of the adjoint entry points are rejected before any
    device work, with LAPACK-style negative codes."""
    L = hostonly
    assert L.plasma_dpotrf_adjoint(0, 4, None, 4, None, 4) == -1
    assert L.plasma_dpotrf_adjoint(pb.PlasmaLower, -1, None, 4, None, 4) == -2
    assert L.plasma_dpotrf_adjoint(pb.PlasmaLower, 4, None, 3, None, 4) == -4
    assert L.plasma_dpotrf_adjoint(pb.PlasmaLower, 4, None, 4, None, 3) == -6
    assert L.plasma_dpotrf_adjoint(pb.PlasmaLower, 0, None, 1, None, 1) == 0
    assert L.plasma_spotrs_adjoint(7, 4, 1, None, 4, None, 4, None, 4, None, 4) == -1
    assert L.plasma_dpotrs_adjoint(pb.PlasmaUpper, 4, -2, None, 4, None, 4, None, 4, None, 4) == -3
    assert L.plasma_dpotrs_adjoint(pb.PlasmaUpper, 4, 1, None, 4, None, 2, None, 4, None, 4) == -7
    assert L.plasma_dpotrs_adjoint(pb.PlasmaUpper, 4, 1, None, 4, None, 4, None, 4, None, 1) == -11


def test_autotune_argument_codes(hostonly):
    L = hostonly
    assert L.plasma_autotune_potrf(0, 100, None) == -1
    assert L.plasma_autotune_potrf(pb.PlasmaRealDouble, 0, None) == -2
    assert L.plasma_autotune_batched(pb.PlasmaRealFloat, 0) == -2
    assert L.plasma_autotune_potrf(pb.PlasmaRealDouble, 100, None) == pb.PlasmaErrorEnvironment


def test_dsposv_descriptor_triangles(hostonly):
    """plasma_omp_dsposv checks that packed triangles hold what the solve
    reads: A the uplo triangle, As lower (for either uplo) or upper (for
    uplo = Upper only); a mismatch fails the sequence with IllegalValue
    before any device work, a match reaches the device check."""
    L = hostonly
    n, nb = 64, 32
    buf = np.zeros(4 * n * n)
    p = buf.ctypes.data

    def tri(prec, uplo):
        d = pb.plasma_desc_t()
        assert L.plasma_desc_triangular_init(prec, uplo, p, nb, nb, n, n, 0, 0, n, n,
                                             ctypes.byref(d)) == 0
        return d

    def gen(prec, m):
        d = pb.plasma_desc_t()
        assert L.plasma_desc_general_init(prec, p, nb, nb, n, m, 0, 0, n, m,
                                          ctypes.byref(d)) == 0
        return d

    B, X, R = gen(pb.PlasmaRealDouble, 1), gen(pb.PlasmaRealDouble, 1), gen(pb.PlasmaRealDouble, 1)
    Xs = gen(pb.PlasmaRealFloat, 1)
    D, S = pb.PlasmaRealDouble, pb.PlasmaRealFloat
    cases = [
        (pb.PlasmaLower, tri(D, pb.PlasmaLower), tri(S, pb.PlasmaUpper), pb.PlasmaErrorIllegalValue),
        (pb.PlasmaUpper, tri(D, pb.PlasmaLower), tri(S, pb.PlasmaLower), pb.PlasmaErrorIllegalValue),
        (pb.PlasmaUpper, tri(D, pb.PlasmaUpper), tri(S, pb.PlasmaLower), pb.PlasmaErrorEnvironment),
        (pb.PlasmaUpper, tri(D, pb.PlasmaUpper), tri(S, pb.PlasmaUpper), pb.PlasmaErrorEnvironment),
        (pb.PlasmaLower, gen(D, n), gen(S, n), pb.PlasmaErrorEnvironment),
    ]
    for uplo, A, As, want in cases:
        seq, req = pb.new_sequence()
        it = ctypes.c_int(-5)
        L.plasma_omp_dsposv(uplo, A, B, X, As, Xs, R, None, None, None, ctypes.byref(it),
                            ctypes.byref(seq), ctypes.byref(req))
        assert seq.status == want, (uplo, A.type, As.type)
        assert it.value == 0


def test_potri_poinv_argument_codes(hostonly):
    """plasma_{d,s}{potri,poinv}: -1 uplo, -2 n, -4 lda (compute/zpotri.c:76-90,
    zpoinv.c:78-92), quick return for n = 0, no device -> Environment."""
    L = hostonly
    for f in ("plasma_dpotri", "plasma_spotri", "plasma_dpoinv", "plasma_spoinv"):
        fn = getattr(L, f)
        assert fn(0, 4, None, 4) == -1
        assert fn(pb.PlasmaLower, -1, None, 4) == -2
        assert fn(pb.PlasmaUpper, 4, None, 3) == -4
        assert fn(pb.PlasmaLower, 0, None, 1) == 0
        assert fn(pb.PlasmaLower, 4, None, 4) == pb.PlasmaErrorEnvironment
