"""ctypes binding of the reference PLASMA itself (test infrastructure only).

oracle/_ref/libplasma_ref.so is the reference's own SPD path, LU-based
mixed-precision solver, band Cholesky and SPD inverse, built from its sources by
oracle/build_ref.sh against the image's OpenBLAS 0.3.15.  Tests
use it to pin the oracle and this library to the reference's outputs on the
same bytes, and bench.py's CPU legs time it on the host cores.  The product
library never loads it.

Threading follows the reference's documented setup (README.md:77-82):
OpenBLAS single-threaded, PLASMA's OpenMP tasks on the host cores.  The
library exports the reference's public names (plasma_init, plasma_dsposv,
...); it is loaded with RTLD_LOCAL and linked -Bsymbolic, so it neither
sees nor shadows this package's libplasma_b200.so of the same API.
"""
import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libplasma_ref.so")
REFERENCE_DIR = os.environ.get("PLASMA_REFERENCE_DIR", "/root/reference")
UPPER, LOWER = 121, 122
NOTRANS = 111
# include/plasma_types.h of the reference
PlasmaTuning, PlasmaNb = 0, 1
PlasmaDisabled, PlasmaEnabled = 0, 1
_lib = None
_omp = None


def available():
    """True when the reference library is built (or can be built here)."""
    return os.path.exists(LIB_PATH) or os.path.isdir(os.path.join(REFERENCE_DIR, "tools"))


def build():
    subprocess.run(["bash", os.path.join(_HERE, "build_ref.sh"), REFERENCE_DIR], check=True,
                   stdout=subprocess.DEVNULL)


def lib():
    """Loads the reference library (building it first when the reference
    sources are present and the library is not), initialises PLASMA with
    tuning off, and pins OpenBLAS to one thread."""
    global _lib, _omp
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    L = ctypes.CDLL(LIB_PATH, mode=os.RTLD_LOCAL)
    vp, ci = ctypes.c_void_p, ctypes.c_int
    L.plasma_init.restype = ci
    L.plasma_set.argtypes = [ci, ci]
    L.plasma_dpotrf.argtypes = [ci, ci, vp, ci]
    L.plasma_dpotrs.argtypes = [ci, ci, ci, vp, ci, vp, ci]
    L.plasma_dposv.argtypes = [ci, ci, ci, vp, ci, vp, ci]
    L.plasma_spotrf.argtypes = [ci, ci, vp, ci]
    L.plasma_dsposv.argtypes = [ci, ci, ci, vp, ci, vp, ci, vp, ci, ctypes.POINTER(ci)]
    L.plasma_dgetrf.argtypes = [ci, ci, vp, ci, vp]
    L.plasma_dgetrs.argtypes = [ci, ci, ci, vp, ci, vp, vp, ci]
    L.plasma_dgesv.argtypes = [ci, ci, vp, ci, vp, vp, ci]
    L.plasma_dsgesv.argtypes = [ci, ci, vp, ci, vp, vp, ci, vp, ci, ctypes.POINTER(ci)]
    L.plasma_dpbtrf.argtypes = [ci, ci, ci, vp, ci]
    L.plasma_dpbtrs.argtypes = [ci, ci, ci, ci, vp, ci, vp, ci]
    L.plasma_dpbsv.argtypes = [ci, ci, ci, ci, vp, ci, vp, ci]
    L.plasma_dpotri.argtypes = [ci, ci, vp, ci]
    L.plasma_dpoinv.argtypes = [ci, ci, vp, ci]
    for f in ("plasma_dpotrf", "plasma_dpotrs", "plasma_dposv", "plasma_spotrf",
              "plasma_dsposv", "plasma_dgetrf", "plasma_dgetrs", "plasma_dgesv",
              "plasma_dsgesv", "plasma_dpbtrf", "plasma_dpbtrs", "plasma_dpbsv",
              "plasma_dpotri", "plasma_dpoinv"):
        getattr(L, f).restype = ci
    # the OpenBLAS the library links: one thread, whatever the environment said
    for name in ("openblas_set_num_threads",):
        try:
            blas = ctypes.CDLL(_openblas_path(), mode=os.RTLD_LOCAL)
            getattr(blas, name).argtypes = [ci]
            getattr(blas, name)(1)
        except (OSError, AttributeError):
            pass
    # libgomp's ICVs, to set the task threads
    _omp = ctypes.CDLL("libgomp.so.1", mode=os.RTLD_LOCAL)
    rc = L.plasma_init()
    if rc != 0:
        raise RuntimeError(f"reference plasma_init failed: {rc}")
    L.plasma_set(PlasmaTuning, PlasmaDisabled)
    _lib = L
    return L


def _openblas_path():
    with open(f"/proc/{os.getpid()}/maps") as f:
        for line in f:
            if "libopenblas" in line:
                return line.split()[-1]
    raise OSError("OpenBLAS not mapped")


def set_threads(n):
    """OpenMP threads for the reference's task DAG (OpenBLAS stays at one)."""
    lib()
    _omp.omp_set_num_threads(int(n))


def get_threads():
    lib()
    return _omp.omp_get_max_threads()


def set_nb(nb):
    lib().plasma_set(PlasmaNb, int(nb))


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def dpotrf(uplo, a, nb=256):
    """In-place factor of the Fortran-ordered array a; returns info."""
    set_nb(nb)
    return lib().plasma_dpotrf(uplo, a.shape[0], _p(a), a.shape[0])


def spotrf(uplo, a, nb=256):
    set_nb(nb)
    return lib().plasma_spotrf(uplo, a.shape[0], _p(a), a.shape[0])


def dpotrs(uplo, a, b, nb=256):
    set_nb(nb)
    n, nrhs = b.shape
    return lib().plasma_dpotrs(uplo, n, nrhs, _p(a), a.shape[0], _p(b), b.shape[0])


def dposv(uplo, a, b, nb=256):
    """a is overwritten by the factor, b by the solution; returns info."""
    set_nb(nb)
    n, nrhs = b.shape
    return lib().plasma_dposv(uplo, n, nrhs, _p(a), a.shape[0], _p(b), b.shape[0])


def dsposv(uplo, a, b, x, nb=256):
    """The reference's mixed-precision solve; returns (info, iter).  a and b
    are left as they were; x receives the solution (left untouched when the
    reference fails the call)."""
    set_nb(nb)
    n, nrhs = b.shape
    it = ctypes.c_int(0)
    info = lib().plasma_dsposv(uplo, n, nrhs, _p(a), a.shape[0], _p(b), b.shape[0], _p(x),
                               x.shape[0], ctypes.byref(it))
    return info, it.value


def dgetrf(a, nb=256):
    """In-place LU with partial pivoting of the Fortran-ordered square a;
    returns (info, ipiv) with 1-based pivots."""
    import numpy as np
    set_nb(nb)
    n = a.shape[0]
    ipiv = np.zeros(max(n, 1), dtype=np.int32)
    info = lib().plasma_dgetrf(n, n, _p(a), a.shape[0], _p(ipiv))
    return info, ipiv[:n]


def dgetrs(a, ipiv, b, nb=256):
    """b <- A^-1 b with the factor and pivots of dgetrf."""
    import numpy as np
    set_nb(nb)
    n, nrhs = b.shape
    ipiv = np.ascontiguousarray(ipiv, dtype=np.int32)
    return lib().plasma_dgetrs(NOTRANS, n, nrhs, _p(a), a.shape[0], _p(ipiv), _p(b),
                               b.shape[0])


def dsgesv(a, b, x, nb=256):
    """The reference's LU-based mixed-precision solve; returns (info, iter,
    ipiv).  a and b are left as they were, x receives the solution."""
    import numpy as np
    set_nb(nb)
    n, nrhs = b.shape
    it = ctypes.c_int(0)
    ipiv = np.zeros(max(n, 1), dtype=np.int32)
    info = lib().plasma_dsgesv(n, nrhs, _p(a), a.shape[0], _p(ipiv), _p(b), b.shape[0],
                               _p(x), x.shape[0], ctypes.byref(it))
    return info, it.value, ipiv[:n]


def dpbtrf(uplo, ab, kd, nb=256):
    """In-place band Cholesky of the LAPACK band array ab ((kd+1) x n)."""
    set_nb(nb)
    return lib().plasma_dpbtrf(uplo, ab.shape[1], kd, _p(ab), ab.shape[0])


def dpbtrs(uplo, ab, kd, b, nb=256):
    set_nb(nb)
    n, nrhs = b.shape
    return lib().plasma_dpbtrs(uplo, n, kd, nrhs, _p(ab), ab.shape[0], _p(b), b.shape[0])


def dpbsv(uplo, ab, kd, b, nb=256):
    """ab is overwritten by the band factor, b by the solution; returns info."""
    set_nb(nb)
    n, nrhs = b.shape
    return lib().plasma_dpbsv(uplo, n, kd, nrhs, _p(ab), ab.shape[0], _p(b), b.shape[0])


def dpotri(uplo, a, nb=256):
    """The inverse from the Cholesky factor in the uplo triangle of a (in
    place, that triangle only); returns info."""
    set_nb(nb)
    return lib().plasma_dpotri(uplo, a.shape[0], _p(a), a.shape[0])


def dpoinv(uplo, a, nb=256):
    """Factor and inverse in one call (in place, the uplo triangle)."""
    set_nb(nb)
    return lib().plasma_dpoinv(uplo, a.shape[0], _p(a), a.shape[0])
