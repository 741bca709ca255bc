"""torch.autograd binding of the library's Cholesky factor and solve.

Forward passes run plasma_?potrf / plasma_?potrs on the GPU; backward passes
run the hand-written adjoints plasma_?potrf_adjoint / plasma_?potrs_adjoint
(include/plasma_b200.h).  No reference counterpart: PLASMA computes no
derivatives.  Tensors are CUDA float64 or float32; the library works on
column-major arrays, so a contiguous row-major tensor T is handed over as the
column-major array T^T.

    L = cholesky(A)                 # A symmetric positive definite
    X = cholesky_solve(L, B)        # X = A^-1 B
    f = logdet_from_factor(L) + (B * X).sum()

Gradients of A come back symmetric: the cotangent of the symmetric matrix,
sym(L^-T Phi(L^T Lbar) L^-1).  Errors of the library (a non-positive-definite
A, an illegal argument) raise RuntimeError; there is no CPU fallback.
"""
import ctypes

import torch

from . import PlasmaErrorNotInitialized, PlasmaLower, lib

_owned = False


def _ensure_init():
    """plasma_init() once, unless the caller already initialised the library."""
    global _owned
    L = lib()
    rc = L.plasma_init()
    if rc == 0:
        _owned = True
    elif rc != PlasmaErrorNotInitialized:
        raise RuntimeError(f"plasma_init failed: {rc}")
    return L


def _check(A):
    if not A.is_cuda:
        raise RuntimeError("plasma_b200.autograd needs CUDA tensors")
    if A.dtype not in (torch.float64, torch.float32):
        raise RuntimeError("float64 or float32 tensors only")


def _fn(dtype, name):
    L = _ensure_init()
    return getattr(L, ("plasma_d" if dtype == torch.float64 else "plasma_s") + name)


def _colmajor(t):
    """A contiguous tensor whose column-major reading is t."""
    return t.t().contiguous()


class _Potrf(torch.autograd.Function):
    @staticmethod
    def forward(ctx, A):
        _check(A)
        n = A.shape[-1]
        work = _colmajor(A)
        torch.cuda.synchronize(A.device)
        rc = _fn(A.dtype, "potrf")(PlasmaLower, n, work.data_ptr(), n)
        if rc != 0:
            raise RuntimeError(f"plasma potrf failed: {rc}"
                               + (" (not positive definite)" if rc > 0 else ""))
        Lf = torch.tril(work.t())
        ctx.save_for_backward(Lf)
        return Lf

    @staticmethod
    def backward(ctx, Lbar):
        (Lf,) = ctx.saved_tensors
        n = Lf.shape[-1]
        pL = _colmajor(Lf)
        pLbar = _colmajor(torch.tril(Lbar))
        torch.cuda.synchronize(Lf.device)
        rc = _fn(Lf.dtype, "potrf_adjoint")(PlasmaLower, n, pL.data_ptr(), n,
                                              pLbar.data_ptr(), n)
        if rc != 0:
            raise RuntimeError(f"plasma potrf_adjoint failed: {rc}")
        return pLbar.t()            # symmetric


class _Potrs(torch.autograd.Function):
    @staticmethod
    def forward(ctx, Lf, B):
        _check(Lf)
        if B.dtype != Lf.dtype or B.device != Lf.device:
            raise RuntimeError("L and B must share dtype and device")
        n, k = B.shape
        pL = _colmajor(Lf)
        pX = _colmajor(B)
        torch.cuda.synchronize(B.device)
        rc = _fn(B.dtype, "potrs")(PlasmaLower, n, k, pL.data_ptr(), n, pX.data_ptr(), n)
        if rc != 0:
            raise RuntimeError(f"plasma potrs failed: {rc}")
        X = pX.t()
        ctx.save_for_backward(pL, pX)
        return X

    @staticmethod
    def backward(ctx, Xbar):
        pL, pX = ctx.saved_tensors
        n, k = pX.shape[1], pX.shape[0]
        pXbar = _colmajor(Xbar)
        pLbar = torch.zeros_like(pL)
        torch.cuda.synchronize(pL.device)
        rc = _fn(pL.dtype, "potrs_adjoint")(PlasmaLower, n, k, pL.data_ptr(), n,
                                              pX.data_ptr(), n, pXbar.data_ptr(), n,
                                              pLbar.data_ptr(), n)
        if rc != 0:
            raise RuntimeError(f"plasma potrs_adjoint failed: {rc}")
        return pLbar.t(), pXbar.t()


def cholesky(A):
    """Lower Cholesky factor of the symmetric positive definite A."""
    return _Potrf.apply(A)


def cholesky_solve(Lf, B):
    """X = A^-1 B with A = Lf Lf^T (Lf from cholesky)."""
    return _Potrs.apply(Lf, B)


def logdet_from_factor(Lf):
    """log det A = 2 sum log diag(L)."""
    return 2.0 * torch.log(torch.diagonal(Lf)).sum()


def gaussian_nll(A, B):
    """logdet(A) + trace(B^T A^-1 B), the Gaussian-likelihood form."""
    Lf = cholesky(A)
    X = cholesky_solve(Lf, B)
    return logdet_from_factor(Lf) + (B * X).sum()
