"""plasma_omp_dpotrs_noalloc (no reference counterpart): the single
right-hand-side FP64 potrs for callers that cannot allocate device memory
while they solve (memory owned by another allocator, or a latency-bound loop
that must not synchronise the device through cudaMalloc).  Its scratch is a
static device array; it is checked against plasma_omp_dpotrs on the same
factor, on two calls in a row.
Collected last: the static array must hold no state that a later call
depends on, whatever ran before."""
import ctypes

import numpy as np
import pytest

import gen
import plasma_b200 as pb
from conftest import EPS, TOL, solve_residual

pytestmark = pytest.mark.gpu
LO, UP = pb.PlasmaLower, pb.PlasmaUpper
MAX_N = 8192


@pytest.fixture(scope="module")
def L():
    import torch
    assert torch.cuda.is_available()
    lib = pb.lib()
    assert lib.plasma_init() == 0
    yield lib
    lib.plasma_finalize()


def general_desc(L, n, ncols, nb):
    d = pb.plasma_desc_t()
    assert L.plasma_desc_general_create(pb.PlasmaRealDouble, nb, nb, n, ncols,
                                        0, 0, n, ncols, ctypes.byref(d)) == 0
    return d


def solve(L, fn, uplo, A, n, nb, b):
    """Loads b into a fresh n x 1 descriptor, solves with fn, returns x."""
    B = general_desc(L, n, 1, nb)
    x = np.asfortranarray(b.copy())
    seq, req = pb.new_sequence()
    L.plasma_omp_dge2desc(x.ctypes.data, n, B, ctypes.byref(seq), ctypes.byref(req))
    fn(uplo, A, B, ctypes.byref(seq), ctypes.byref(req))
    L.plasma_omp_ddesc2ge(B, x.ctypes.data, n, ctypes.byref(seq), ctypes.byref(req))
    rc = L.plasma_sequence_wait(ctypes.byref(seq))
    L.plasma_desc_destroy(ctypes.byref(B))
    return rc, x


@pytest.mark.parametrize("uplo", [LO, UP])
@pytest.mark.parametrize("n,nb", [(1000, 128), (MAX_N, 256)])
def test_noalloc_matches_potrs(L, uplo, n, nb):
    assert L.plasma_set(pb.PlasmaNb, nb) == 0
    a, b = gen.diag_dominant(n, 2, seed=4000 + n)
    f = np.asfortranarray(a.copy())
    assert L.plasma_dpotrf(uplo, n, f.ctypes.data, n) == 0
    A = general_desc(L, n, n, nb)
    seq, req = pb.new_sequence()
    L.plasma_omp_dge2desc(f.ctypes.data, n, A, ctypes.byref(seq), ctypes.byref(req))
    assert L.plasma_sequence_wait(ctypes.byref(seq)) == 0
    try:
        for j in range(2):                  # two calls in a row
            bj = b[:, j:j + 1]
            rc0, x0 = solve(L, L.plasma_omp_dpotrs, uplo, A, n, nb, bj)
            rc1, x1 = solve(L, L.plasma_omp_dpotrs_noalloc, uplo, A, n, nb, bj)
            assert rc0 == 0 and rc1 == 0
            np.testing.assert_allclose(x1, x0, rtol=1e-12, atol=1e-14)
            assert solve_residual(a, x1, bj) < TOL * EPS
    finally:
        L.plasma_desc_destroy(ctypes.byref(A))


def test_noalloc_rejects_beyond_max(L):
    """n above the static limit fails the request before any launch."""
    nb = 64
    n = MAX_N + nb
    A, B = general_desc(L, n, n, nb), general_desc(L, n, 1, nb)
    before = L.plasma_kernel_launches()
    seq, req = pb.new_sequence()
    L.plasma_omp_dpotrs_noalloc(LO, A, B, ctypes.byref(seq), ctypes.byref(req))
    assert seq.status == pb.PlasmaErrorIllegalValue
    assert L.plasma_kernel_launches() == before
    L.plasma_desc_destroy(ctypes.byref(A))
    L.plasma_desc_destroy(ctypes.byref(B))


def test_noalloc_rejects_shapes(L):
    nb, n = 96, 500                  # nb not a multiple of 64
    A, B = general_desc(L, n, n, nb), general_desc(L, n, 1, nb)
    seq, req = pb.new_sequence()
    L.plasma_omp_dpotrs_noalloc(LO, A, B, ctypes.byref(seq), ctypes.byref(req))
    assert seq.status == pb.PlasmaErrorNotSupported
    L.plasma_desc_destroy(ctypes.byref(A))
    L.plasma_desc_destroy(ctypes.byref(B))
    nb = 64                          # two right-hand sides
    A, B = general_desc(L, n, n, nb), general_desc(L, n, 2, nb)
    seq, req = pb.new_sequence()
    L.plasma_omp_dpotrs_noalloc(LO, A, B, ctypes.byref(seq), ctypes.byref(req))
    assert seq.status == pb.PlasmaErrorNotSupported
    L.plasma_desc_destroy(ctypes.byref(A))
    L.plasma_desc_destroy(ctypes.byref(B))


def test_noalloc_allocates_nothing(L):
    """The point of the entry point: the library's allocation counter does not
    move across its calls, the first one at a size no call here has used
    included (plasma_omp_dpotrs grows its workspace there)."""
    n, nb = 2496, 192
    assert L.plasma_set(pb.PlasmaNb, nb) == 0
    a, b = gen.diag_dominant(n, 1, seed=4100)
    f = np.asfortranarray(a.copy())
    assert L.plasma_dpotrf(LO, n, f.ctypes.data, n) == 0
    A, B = general_desc(L, n, n, nb), general_desc(L, n, 1, nb)
    x = np.asfortranarray(b.copy())
    seq, req = pb.new_sequence()
    L.plasma_omp_dge2desc(f.ctypes.data, n, A, ctypes.byref(seq), ctypes.byref(req))
    assert L.plasma_sequence_wait(ctypes.byref(seq)) == 0
    try:
        for _ in range(2):
            seq, req = pb.new_sequence()
            L.plasma_omp_dge2desc(x.ctypes.data, n, B, ctypes.byref(seq), ctypes.byref(req))
            assert L.plasma_sequence_wait(ctypes.byref(seq)) == 0
            before = L.plasma_device_allocations()
            seq, req = pb.new_sequence()
            L.plasma_omp_dpotrs_noalloc(LO, A, B, ctypes.byref(seq), ctypes.byref(req))
            assert L.plasma_sequence_wait(ctypes.byref(seq)) == 0
            assert L.plasma_device_allocations() == before
            y = np.asfortranarray(np.zeros_like(b))
            seq, req = pb.new_sequence()
            L.plasma_omp_ddesc2ge(B, y.ctypes.data, n, ctypes.byref(seq), ctypes.byref(req))
            assert L.plasma_sequence_wait(ctypes.byref(seq)) == 0
            assert solve_residual(a, y, b) < TOL * EPS
    finally:
        L.plasma_desc_destroy(ctypes.byref(A))
        L.plasma_desc_destroy(ctypes.byref(B))
