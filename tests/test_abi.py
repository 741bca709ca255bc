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
import subprocess

import numpy as np
import pytest

import plasma_b200 as pb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(headers=None):
    names = set()
    if headers is None:
        # plasma_core_blas.h belongs to libplasma_core_blas.so
        headers = [h for h in glob.glob(os.path.join(ROOT, "include", "*.h"))
                   if not h.endswith("plasma_core_blas.h")]
    for h in headers:
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


def test_batched_plan_argument_codes(hostonly):
    """Batched plans: the argument checks run before any device work, so a
    host-only context reports them; a valid plan needs the device."""
    L = hostonly
    plan = ctypes.c_void_p()
    n = (ctypes.c_int * 3)(16, 512, 0)
    assert L.plasma_batch_create(0, 3, n, ctypes.byref(plan)) == -1
    assert L.plasma_batch_create(pb.PlasmaRealDouble, -1, n, ctypes.byref(plan)) == -2
    assert L.plasma_batch_create(pb.PlasmaRealDouble, 3, None, ctypes.byref(plan)) == -3
    big = (ctypes.c_int * 2)(16, 513)
    assert L.plasma_batch_create(pb.PlasmaRealFloat, 2, big, ctypes.byref(plan)) == -3
    neg = (ctypes.c_int * 1)(-1,)
    assert L.plasma_batch_create(pb.PlasmaRealFloat, 1, neg, ctypes.byref(plan)) == -3
    assert L.plasma_batch_create(pb.PlasmaRealDouble, 3, n, None) == -4
    assert L.plasma_batch_create(pb.PlasmaRealDouble, 3, n,
                                 ctypes.byref(plan)) == pb.PlasmaErrorEnvironment
    assert L.plasma_dposv_batched(None, None, None, None) == -1
    assert L.plasma_batch_offsets(None, None, None) == -1
    assert L.plasma_batch_set_graph(None, 1) == -1
    assert L.plasma_batch_matrix_elems(None) == 0
    assert L.plasma_batch_vector_elems(None) == 0


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


def test_band_argument_codes(hostonly):
    """plasma_{d,s}pbtrf: -1 uplo, -2 n, -3 kd, -5 ldab (compute/zpbtrf.c:86-105);
    pbtrs: -1, -2, kd -4, nrhs -5, ldab -7, ldb -10 (compute/zpbtrs.c:94-118);
    pbsv: -1, -2, -3, -4, ldab -6, ldb -8 (compute/zpbsv.c:105-129); the
    quick returns; no device -> Environment."""
    L = hostonly
    lo = pb.PlasmaLower
    for p in ("d", "s"):
        trf = getattr(L, f"plasma_{p}pbtrf")
        trs = getattr(L, f"plasma_{p}pbtrs")
        sv = getattr(L, f"plasma_{p}pbsv")
        assert trf(0, 8, 2, None, 3) == -1
        assert trf(lo, -1, 2, None, 3) == -2
        assert trf(lo, 8, -1, None, 3) == -3
        assert trf(lo, 8, 2, None, 2) == -5
        assert trf(lo, 0, 2, None, 3) == 0
        assert trf(lo, 8, 2, None, 3) == pb.PlasmaErrorEnvironment
        assert trs(0, 8, 2, 1, None, 3, None, 8) == -1
        assert trs(lo, -1, 2, 1, None, 3, None, 8) == -2
        assert trs(lo, 8, -1, 1, None, 3, None, 8) == -4
        assert trs(lo, 8, 2, -1, None, 3, None, 8) == -5
        assert trs(lo, 8, 2, 1, None, 2, None, 8) == -7
        assert trs(lo, 8, 2, 1, None, 3, None, 7) == -10
        assert trs(lo, 0, 2, 0, None, 3, None, 1) == 0
        assert sv(0, 8, 2, 1, None, 3, None, 8) == -1
        assert sv(lo, -1, 2, 1, None, 3, None, 8) == -2
        assert sv(lo, 8, -1, 1, None, 3, None, 8) == -3
        assert sv(lo, 8, 2, -1, None, 3, None, 8) == -4
        assert sv(lo, 8, 2, 1, None, 2, None, 8) == -6
        assert sv(lo, 8, 2, 1, None, 3, None, 7) == -8
        assert sv(lo, 8, 2, 0, None, 3, None, 8) == 0


def band_desc(L, uplo, n, kd, nb):
    """The band descriptor the LAPACK-layout band routines build
    (compute/zpbtrf.c:117-124)."""
    d = pb.plasma_desc_t()
    lm = nb * (1 + (kd + nb - 1) // nb)
    rc = L.plasma_desc_general_band_init(pb.PlasmaRealDouble, uplo, None, nb, nb, lm, n,
                                         0, 0, n, n, kd, kd, ctypes.byref(d))
    assert rc == 0
    return d


def band_offset(d, m, n):
    """plasma_tile_offset of a band descriptor (include/plasma_descriptor.h),
    restated: the general formula at stored tile row (kut-1) + m - n."""
    row, col = d.kut - 1 + m - n, n + d.j // d.nb
    lm1, ln1 = d.gm // d.mb, d.gn // d.nb
    assert 0 <= row < lm1
    return d.mb * d.nb * (row + lm1 * col) if col < ln1 else d.A12 + d.mb * (d.gn % d.nb) * row


@pytest.mark.parametrize("n,kd,nb", [(1000, 300, 128), (1000, 0, 128), (300, 299, 64),
                                     (4096, 256, 256), (777, 1, 32)])
@pytest.mark.parametrize("uplo", [pb.PlasmaLower, pb.PlasmaUpper])
def test_band_descriptor_covers_the_walk(hostonly, n, kd, nb, uplo):
    """The band descriptor's tile counts (control/descriptor.c:199-211) and,
    for every tile the band factorization and solves touch (tile rows
    [k, k+kt) of column k, the window [k+1, k+kt)^2), a stored location
    inside the allocation, distinct per tile."""
    L = hostonly
    d = band_desc(L, uplo, n, kd, nb)
    assert d.type == pb.PlasmaGeneralBand and d.uplo == uplo
    kt = 1 + -(-kd // nb)
    assert (d.klt, d.kut) == ((kt, 1) if uplo == pb.PlasmaLower else (1, kt))
    assert L.plasma_desc_check(d) == 0
    assert L.plasma_desc_general_band_check(d) == 0
    size = L.plasma_desc_storage_bytes(d) // 8
    assert size == d.gm * d.gn
    seen = {}
    for k in range(d.mt):
        r = min(d.mt, k + kt)
        for m in range(k, r):
            for c in range(k, m + 1):
                # logical lower tile (m, c) is stored at (m, c) or (c, m)
                t = (m, c) if uplo == pb.PlasmaLower else (c, m)
                off = band_offset(d, *t)
                rows = d.mb
                cols = nb if t[1] < d.gn // nb else d.gn % nb
                assert 0 <= off and off + rows * cols <= size, (t, off, size)
                assert seen.setdefault(off, t) == t
    # views cut at r tiles keep the stored tiles where they were
    assert len(seen) == sum(min(kt, d.mt - k) for k in range(d.mt))


def test_band_descriptor_check_errors(hostonly):
    L = hostonly
    d = band_desc(L, pb.PlasmaLower, 100, 10, 16)
    assert L.plasma_desc_check(d) == 0
    # a band wider than the matrix (the reference rejects kd >= n)
    assert L.plasma_desc_general_band_init(pb.PlasmaRealDouble, pb.PlasmaLower, None, 16,
                                           16, 32, 10, 0, 0, 10, 10, 10, 10,
                                           ctypes.byref(d)) == 0
    assert L.plasma_desc_check(d) == pb.PlasmaErrorIllegalValue
    # too few stored tile rows for the band
    assert L.plasma_desc_general_band_init(pb.PlasmaRealDouble, pb.PlasmaLower, None, 16,
                                           16, 16, 100, 0, 0, 100, 100, 10, 10,
                                           ctypes.byref(d)) == 0
    assert L.plasma_desc_check(d) == pb.PlasmaErrorIllegalValue
    # stored rows not a multiple of the tile height
    assert L.plasma_desc_general_band_init(pb.PlasmaRealDouble, pb.PlasmaLower, None, 16,
                                           16, 40, 100, 0, 0, 100, 100, 10, 10,
                                           ctypes.byref(d)) == 0
    assert L.plasma_desc_check(d) == pb.PlasmaErrorIllegalValue


def test_dsgesv_argument_codes(hostonly):
    """plasma_dsgesv: -1 n, -2 nrhs, -4 lda, -7 ldb, -9 ldx (compute/zcgesv.c:
    119-138), iter = 0 and success on quick return, no device -> Environment."""
    L = hostonly
    it = ctypes.c_int(5)
    piv = (ctypes.c_int * 8)()
    assert L.plasma_dsgesv(-1, 1, None, 1, piv, None, 1, None, 1, ctypes.byref(it)) == -1
    assert L.plasma_dsgesv(8, -1, None, 8, piv, None, 8, None, 8, ctypes.byref(it)) == -2
    assert L.plasma_dsgesv(8, 1, None, 7, piv, None, 8, None, 8, ctypes.byref(it)) == -4
    assert L.plasma_dsgesv(8, 1, None, 8, piv, None, 7, None, 8, ctypes.byref(it)) == -7
    assert L.plasma_dsgesv(8, 1, None, 8, piv, None, 8, None, 7, ctypes.byref(it)) == -9
    it.value = 5
    assert L.plasma_dsgesv(8, 0, None, 8, piv, None, 8, None, 8, ctypes.byref(it)) == 0
    assert it.value == 0
    assert L.plasma_dsgesv(8, 1, None, 8, piv, None, 8, None, 8,
                           ctypes.byref(it)) == pb.PlasmaErrorEnvironment


def _general(L, prec, m, n, nb=16):
    d = pb.plasma_desc_t()
    assert L.plasma_desc_general_init(prec, None, nb, nb, m, n, 0, 0, m, n,
                                      ctypes.byref(d)) == 0
    return d


def test_omp_dsgesv_descriptor_checks(hostonly):
    """plasma_omp_dsgesv refuses descriptors of the wrong precision, shape or
    tiling before touching the device (IllegalValue in the sequence)."""
    L = hostonly
    D, S = pb.PlasmaRealDouble, pb.PlasmaRealFloat
    n, nrhs = 40, 2
    ok = dict(A=_general(L, D, n, n), B=_general(L, D, n, nrhs), X=_general(L, D, n, nrhs),
              As=_general(L, S, n, n), Xs=_general(L, S, n, nrhs), R=_general(L, D, n, nrhs))
    bad = [("As", _general(L, D, n, n)),            # FP64 where FP32 is expected
           ("X", _general(L, D, n, nrhs + 1)),      # X wider than B
           ("A", _general(L, D, n, n - 1)),         # A not square
           ("R", _general(L, D, n, nrhs, nb=8))]    # another tiling
    piv = (ctypes.c_int * n)()
    for name, d in bad:
        args = dict(ok)
        args[name] = d
        seq, req = pb.new_sequence()
        it = ctypes.c_int(7)
        L.plasma_omp_dsgesv(args["A"], piv, args["B"], args["X"], args["As"], args["Xs"],
                            args["R"], None, None, None, ctypes.byref(it), ctypes.byref(seq),
                            ctypes.byref(req))
        assert seq.status == pb.PlasmaErrorIllegalValue, name
        assert it.value == 0
    # well-formed descriptors reach the device check
    seq, req = pb.new_sequence()
    it = ctypes.c_int(7)
    L.plasma_omp_dsgesv(ok["A"], piv, ok["B"], ok["X"], ok["As"], ok["Xs"], ok["R"], None,
                        None, None, ctypes.byref(it), ctypes.byref(seq), ctypes.byref(req))
    assert seq.status == pb.PlasmaErrorEnvironment


def test_omp_band_descriptor_checks(hostonly):
    """The async band routines take band descriptors of the uplo triangle (or
    general band storage) only; the layout converters refuse general band
    storage and a too small ldab."""
    L = hostonly
    lo, up = pb.PlasmaLower, pb.PlasmaUpper
    ab = band_desc(L, lo, 100, 10, 16)
    ge = _general(L, pb.PlasmaRealDouble, 100, 100)
    for fn, args in (("plasma_omp_dpbtrf", (up, ab)), ("plasma_omp_dpbtrf", (lo, ge)),
                     ("plasma_omp_dpbsv", (up, ab, ge)), ("plasma_omp_dpbtrs", (lo, ge, ge))):
        seq, req = pb.new_sequence()
        getattr(L, fn)(*args, ctypes.byref(seq), ctypes.byref(req))
        assert seq.status == pb.PlasmaErrorIllegalValue, (fn, args)
    # the matching triangle gets as far as the device check
    seq, req = pb.new_sequence()
    L.plasma_omp_dpbtrf(lo, ab, ctypes.byref(seq), ctypes.byref(req))
    assert seq.status == pb.PlasmaErrorEnvironment
    buf = np.zeros((11, 100), order="F")
    seq, req = pb.new_sequence()
    L.plasma_omp_dpb2desc(buf.ctypes.data, 10, ab, ctypes.byref(seq), ctypes.byref(req))
    assert seq.status == pb.PlasmaErrorIllegalValue              # ldab < kd + 1
    gband = pb.plasma_desc_t()
    assert L.plasma_desc_general_band_init(pb.PlasmaRealDouble, pb.PlasmaGeneral, None, 16, 16,
                                           64, 100, 0, 0, 100, 100, 10, 10,
                                           ctypes.byref(gband)) == 0
    seq, req = pb.new_sequence()
    L.plasma_omp_dpb2desc(buf.ctypes.data, 11, gband, ctypes.byref(seq), ctypes.byref(req))
    assert seq.status == pb.PlasmaErrorNotSupported
    # band storage cannot be allocated without a device
    d = pb.plasma_desc_t()
    assert L.plasma_desc_general_band_create(pb.PlasmaRealDouble, lo, 16, 16, 32, 100, 0, 0,
                                             100, 100, 10, 10,
                                             ctypes.byref(d)) == pb.PlasmaErrorEnvironment


C_CALLER = r"""
#include "plasma.h"
#include <stdio.h>
#include <stdlib.h>

int main(void)
{
    /* the reference's calling sequence, host-only (no device): argument
     * codes come back before any device work */
    if (plasma_init() != 0) return 10;
    double A[16] = {4, 1, 0, 0, 1, 4, 1, 0, 0, 1, 4, 1, 0, 0, 1, 4};
    double B[4] = {1, 2, 3, 4}, X[4];
    int iter = 5, ipiv[4];
    int rc = 0;
    rc |= plasma_dposv(999, 4, 1, A, 4, B, 4) != -1;
    rc |= plasma_dpotrf(PlasmaLower, 4, A, 3) != -4;
    rc |= plasma_dsposv(PlasmaLower, 4, 1, A, 4, B, 4, X, 3, &iter) != -9;
    rc |= plasma_dsgesv(4, 1, A, 4, ipiv, B, 4, X, 4, &iter) != PlasmaErrorEnvironment;
    rc |= plasma_dpbsv(PlasmaLower, 4, 1, 1, A, 1, B, 4) != -6;
    plasma_desc_t D;
    rc |= plasma_desc_general_init(PlasmaRealDouble, NULL, 2, 2, 4, 4, 0, 0, 4, 4, &D) != 0;
    rc |= plasma_desc_check(D) != 0;
    rc |= plasma_finalize() != 0;
    printf("%s\n", rc ? "FAIL" : "ok");
    return rc;
}
"""


@pytest.mark.parametrize("compiler,ext", [("gcc", "c"), ("g++", "cpp")])
def test_c_and_cxx_callers_compile_link_and_run(tmp_path, compiler, ext):
    """A caller written against plasma.h compiles as C and as C++, links with
    -lplasma_b200 (the INTEGRATION recipe) and gets the reference's argument
    codes back (host-only mode, no device)."""
    import shutil
    if shutil.which(compiler) is None:
        pytest.skip(f"{compiler} not available")
    pb.lib()                      # the library is built
    src = tmp_path / f"caller.{ext}"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    libdir = os.path.join(ROOT, "plasma_b200")
    cmd = [compiler, str(src), "-I", os.path.join(ROOT, "include"), "-L", libdir,
           "-lplasma_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    if ext == "c":
        cmd[1:1] = ["-std=c99", "-Wall", "-Werror"]
    else:
        cmd[1:1] = ["-Wall", "-Werror"]
    subprocess.run(cmd, check=True)
    env = dict(os.environ, PLASMA_ALLOW_NO_DEVICE="1")
    out = subprocess.run([str(exe)], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", (out.stdout, out.stderr)
