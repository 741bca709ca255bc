"""ctypes binding of the CPU oracle (test infrastructure only).

Loaded by tests/, __graft_entry__.smoke() and the CPU-baseline leg of
bench.py to check or time against; the product library never uses it.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")
UPPER, LOWER = 121, 122
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, ci = ctypes.c_void_p, ctypes.c_int
        for p in ("d", "s"):
            getattr(L, f"{p}oracle_potrf").argtypes = [ci, ci, vp, ci, ci]
            getattr(L, f"{p}oracle_potrs").argtypes = [ci, ci, ci, vp, ci, vp, ci, ci]
            getattr(L, f"{p}oracle_posv").argtypes = [ci, ci, ci, vp, ci, vp, ci, ci]
            getattr(L, f"{p}oracle_potri").argtypes = [ci, ci, vp, ci]
            getattr(L, f"{p}oracle_pbtrf").argtypes = [ci, ci, ci, vp, ci, ci]
            getattr(L, f"{p}oracle_pbtrs").argtypes = [ci, ci, ci, ci, vp, ci, vp, ci, ci]
            for f in ("potrf", "potrs", "posv", "potri", "pbtrf", "pbtrs"):
                getattr(L, f"{p}oracle_{f}").restype = ci
        for p in ("d", "s"):
            getattr(L, f"{p}oracle_getrf").argtypes = [ci, vp, ci, vp, ci]
            getattr(L, f"{p}oracle_getrs").argtypes = [ci, ci, vp, ci, vp, vp, ci]
            getattr(L, f"{p}oracle_gesv").argtypes = [ci, ci, vp, ci, vp, vp, ci, ci]
            for f in ("getrf", "getrs", "gesv"):
                getattr(L, f"{p}oracle_{f}").restype = ci
        L.oracle_dsgesv.argtypes = [ci, ci, vp, ci, vp, vp, ci, vp, ci,
                                    ctypes.POINTER(ci), ci]
        L.oracle_dsgesv.restype = ci
        L.oracle_dlange_inf.argtypes = [ci, vp, ci]
        L.oracle_dlange_inf.restype = ctypes.c_double
        L.oracle_dsposv.argtypes = [ci, ci, ci, vp, ci, vp, ci, vp, ci,
                                    ctypes.POINTER(ci), ci]
        L.oracle_dsposv.restype = ci
        L.oracle_dlansy_inf.argtypes = [ci, ci, vp, ci]
        L.oracle_dlansy_inf.restype = ctypes.c_double
        L.oracle_set_threads.argtypes = [ci]
        L.oracle_get_threads.restype = ci
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _prefix(a):
    import numpy as np
    return "d" if a.dtype == np.float64 else "s"


def potrf(uplo, a, nb):
    """In-place tile Cholesky of the Fortran-ordered array a; returns info."""
    n = a.shape[0]
    return getattr(lib(), f"{_prefix(a)}oracle_potrf")(uplo, n, _p(a), a.shape[0], nb)


def potri(uplo, a):
    """In-place inverse from the Cholesky factor in the uplo triangle of the
    Fortran-ordered array a (dtrtri + dlauum); returns info."""
    n = a.shape[0]
    return getattr(lib(), f"{_prefix(a)}oracle_potri")(uplo, n, _p(a), a.shape[0])


def potrs(uplo, a, b, nb):
    n, nrhs = b.shape
    return getattr(lib(), f"{_prefix(a)}oracle_potrs")(uplo, n, nrhs, _p(a),
                                                       a.shape[0], _p(b), b.shape[0], nb)


def posv(uplo, a, b, nb):
    n, nrhs = b.shape
    return getattr(lib(), f"{_prefix(a)}oracle_posv")(uplo, n, nrhs, _p(a),
                                                      a.shape[0], _p(b), b.shape[0], nb)


def pbtrf(uplo, ab, kd, nb):
    """In-place band tile Cholesky of the Fortran-ordered LAPACK band array ab
    ((ldab >= kd+1) x n); returns info (ab unchanged when info > 0)."""
    return getattr(lib(), f"{_prefix(ab)}oracle_pbtrf")(uplo, ab.shape[1], kd, _p(ab),
                                                        ab.shape[0], nb)


def pbtrs(uplo, ab, kd, b, nb):
    """Solves with the band factor held in ab; b (n x nrhs, Fortran order) is
    overwritten with the solution."""
    n, nrhs = b.shape
    return getattr(lib(), f"{_prefix(ab)}oracle_pbtrs")(uplo, n, kd, nrhs, _p(ab),
                                                        ab.shape[0], _p(b), b.shape[0], nb)


def dsposv(uplo, a, b, x, nb):
    it = ctypes.c_int(0)
    n, nrhs = b.shape
    info = lib().oracle_dsposv(uplo, n, nrhs, _p(a), a.shape[0], _p(b), b.shape[0],
                               _p(x), x.shape[0], ctypes.byref(it), nb)
    return info, it.value


def getrf(a, nb):
    """In-place LU with partial pivoting of the Fortran-ordered square a;
    returns (info, ipiv) with LAPACK's 1-based pivots."""
    import numpy as np
    n = a.shape[0]
    ipiv = np.zeros(max(n, 1), dtype=np.int32)
    info = getattr(lib(), f"{_prefix(a)}oracle_getrf")(n, _p(a), a.shape[0], _p(ipiv), nb)
    return info, ipiv[:n]


def getrs(a, ipiv, b):
    import numpy as np
    n, nrhs = b.shape
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int32)
    return getattr(lib(), f"{_prefix(a)}oracle_getrs")(n, nrhs, _p(a), a.shape[0],
                                                       _p(ipiv), _p(b), b.shape[0])


def dsgesv(a, b, x, nb):
    """FP32 LU + FP64 refinement (FP64 LU fallback); returns (info, iter, ipiv)."""
    import numpy as np
    n, nrhs = b.shape
    it = ctypes.c_int(0)
    ipiv = np.zeros(max(n, 1), dtype=np.int32)
    info = lib().oracle_dsgesv(n, nrhs, _p(a), a.shape[0], _p(ipiv), _p(b), b.shape[0],
                               _p(x), x.shape[0], ctypes.byref(it), nb)
    return info, it.value, ipiv[:n]


def lange_inf(a):
    return lib().oracle_dlange_inf(a.shape[0], _p(a), a.shape[0])


def lansy_inf(uplo, a):
    return lib().oracle_dlansy_inf(uplo, a.shape[0], _p(a), a.shape[0])


def set_threads(n):
    lib().oracle_set_threads(n)


def get_threads():
    return lib().oracle_get_threads()
