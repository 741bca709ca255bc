"""Seeded input generators shared by the fixture script, the tests and bench.py.

The workloads are the synthetic SPD systems of the benchmark configurations:
  * diagonally dominant: A = sym(U[-0.5, 0.5]) + n I, b ~ U[-1, 1]
    (seed 42 for the CPU parity case n = 2048, seed 7 for n in {8192 .. 32768});
  * prescribed spectrum: A = Q diag(lambda) Q^T, Q from Householder QR of an
    N(0,1) matrix, lambda log-spaced from 1 to 1/kappa (seed 11);
  * Gaussian likelihood: A = G G^T / n + I (seed 3);
  * band: the diagonally dominant matrix cut to the band |i - j| <= kd, the
    reference tester's band inputs (test/test_zpbsv.c:90-106), with its
    LAPACK band storage;
  * general (LU): A = U[-0.5, 0.5] with no diagonal boost, so that partial
    pivoting interchanges rows, or U diag(sigma) V^T with sigma log-spaced
    1 .. 1/kappa (the mixed-precision LU inputs).
numpy's PCG64 streams are stable across numpy versions, so the same seed
gives the same bytes on every machine.
"""
import numpy as np


def diag_dominant(n, nrhs, seed, dtype=np.float64):
    """Column-major (Fortran-ordered) A (full symmetric) and B."""
    rng = np.random.default_rng(seed)
    g = rng.uniform(-0.5, 0.5, size=(n, n))
    a = np.tril(g) + np.tril(g, -1).T
    a[np.diag_indices(n)] += n
    b = rng.uniform(-1.0, 1.0, size=(n, nrhs))
    return np.asfortranarray(a.astype(dtype)), np.asfortranarray(b.astype(dtype))


def zerocol(a, col):
    """The reference tester's --zerocol: zero one column (test_zpotrf.c:97-99)
    or, for the solvers, one row and column (test_zcposv.c:104-110)."""
    a = a.copy(order="F")
    a[:, col] = 0.0
    a[col, :] = 0.0
    return a


def spectrum(n, kappa, seed=11):
    """A = Q diag(lambda) Q^T with lambda log-spaced 1 .. 1/kappa (numpy, for
    small n; the GPU-sized version lives in bench.py)."""
    rng = np.random.default_rng(seed)
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.logspace(0.0, -np.log10(kappa), n)
    a = (q * lam) @ q.T
    a = 0.5 * (a + a.T)
    return np.asfortranarray(a)


def likelihood(n, nrhs, seed=3):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, n))
    a = g @ g.T / n + np.eye(n)
    b = rng.standard_normal((n, nrhs))
    return np.asfortranarray(a), np.asfortranarray(b)


def probe_vector(n):
    """Fixed vector used for checksums L @ v of large factors."""
    return np.cos(np.arange(n, dtype=np.float64) * 0.37) + 0.5


def band(n, kd, nrhs, seed, dtype=np.float64):
    """Symmetric positive definite band matrix of bandwidth kd: A (full,
    Fortran order), its LAPACK band storage for lower (AB(i-j, j)) and upper
    (AB(kd+i-j, j)) triangles, both (kd+1) x n, and B."""
    a, b = diag_dominant(n, nrhs, seed, dtype)
    i, j = np.indices((n, n))
    a = np.asfortranarray(np.where(np.abs(i - j) <= kd, a, 0).astype(dtype))
    return a, to_band(a, kd, lower=True), to_band(a, kd, lower=False), b


def to_band(a, kd, lower, ldab=None):
    """LAPACK band storage of the lower or upper band of a (ldab x n,
    Fortran order; rows past kd+1 and the corner positions are zero)."""
    n = a.shape[0]
    ldab = kd + 1 if ldab is None else ldab
    ab = np.zeros((ldab, n), dtype=a.dtype, order="F")
    for d in range(kd + 1):
        if lower:
            ab[d, :n - d] = np.diagonal(a, -d)
        else:
            ab[kd - d, d:] = np.diagonal(a, d)
    return ab


def from_band(ab, kd, lower):
    """The triangle of a band matrix from its LAPACK band storage."""
    n = ab.shape[1]
    a = np.zeros((n, n), dtype=ab.dtype)
    for d in range(kd + 1):
        if lower:
            a += np.diag(ab[d, :n - d], -d)
        else:
            a += np.diag(ab[kd - d, d:], d)
    return a


def general(n, nrhs, seed, dtype=np.float64):
    """Nonsymmetric A ~ U[-0.5, 0.5] and B ~ U[-1, 1] (Fortran order)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-0.5, 0.5, size=(n, n))
    b = rng.uniform(-1.0, 1.0, size=(n, nrhs))
    return np.asfortranarray(a.astype(dtype)), np.asfortranarray(b.astype(dtype))


def general_spectrum(n, kappa, seed=13):
    """A = U diag(sigma) V^T with sigma log-spaced 1 .. 1/kappa."""
    rng = np.random.default_rng(seed)
    u, _ = np.linalg.qr(rng.standard_normal((n, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    sig = np.logspace(0.0, -np.log10(kappa), n)
    return np.asfortranarray((u * sig) @ v.T)
