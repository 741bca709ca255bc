"""Reverse mode of the Cholesky factor and solve (no reference counterpart:
PLASMA has no derivatives).  Oracles: FP64 finite differences of the loss
computed with numpy, the analytic gradient of the Gaussian-likelihood form,
and the closed form of the factor adjoint, sym(L^-T Phi(L^T Lbar) L^-1).
"""
import ctypes

import numpy as np
import pytest

import plasma_b200 as pb

pytestmark = pytest.mark.gpu
LO, UP = pb.PlasmaLower, pb.PlasmaUpper


@pytest.fixture(scope="module")
def torch_ag():
    import torch
    assert torch.cuda.is_available()
    L = pb.lib()
    assert L.plasma_init() == 0
    import plasma_b200.autograd as ag
    yield torch, ag, L
    L.plasma_finalize()


def likelihood_system(n, nrhs, seed=3):
    """A = G G^T / n + I, G ~ N(0,1); B ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, n))
    a = g @ g.T / n + np.eye(n)
    b = rng.standard_normal((n, nrhs))
    return a, b


def loss_np(a, b):
    sign, logdet = np.linalg.slogdet(a)
    assert sign > 0
    return logdet + np.sum(b * np.linalg.solve(a, b))


def fd4(f, x, e, h):
    """Fourth-order central difference of f along e."""
    return (8 * (f(x + h * e) - f(x - h * e)) - (f(x + 2 * h * e) - f(x - 2 * h * e))) / (12 * h)


def phi_formula(lf, lbar):
    p = lf.T @ np.tril(lbar)
    phi = np.tril(p) - 0.5 * np.diag(np.diag(p))
    li = np.linalg.inv(lf)
    m = li.T @ phi @ li
    return 0.5 * (m + m.T)


def test_finite_differences_fp64(torch_ag):
    """n = 256, nrhs = 8: directional derivatives of logdet(A) + tr(B^T A^-1 B)
    along random symmetric directions agree with FP64 finite differences to
    1e-8 relative."""
    torch, ag, _ = torch_ag
    n, nrhs = 256, 8
    a, b = likelihood_system(n, nrhs)
    A = torch.tensor(a, device="cuda", requires_grad=True)
    B = torch.tensor(b, device="cuda", requires_grad=True)
    f = ag.gaussian_nll(A, B)
    f.backward()
    assert abs(f.item() - loss_np(a, b)) <= 1e-12 * abs(loss_np(a, b))
    ga, gb = A.grad.cpu().numpy(), B.grad.cpu().numpy()
    rng = np.random.default_rng(7)
    for _ in range(4):
        e = rng.standard_normal((n, n))
        e = 0.5 * (e + e.T)
        fd = fd4(lambda x: loss_np(x, b), a, e, 1e-4)
        an = np.sum(ga * e)
        assert abs(an - fd) <= 1e-8 * abs(fd), (an, fd)
        eb = rng.standard_normal((n, nrhs))
        fdb = fd4(lambda x: loss_np(a, x), b, eb, 1e-4)
        anb = np.sum(gb * eb)
        assert abs(anb - fdb) <= 1e-8 * abs(fdb), (anb, fdb)


@pytest.mark.parametrize("n,nb", [(256, 64), (1000, 256), (777, 128)])
def test_analytic_gradient_fp64(torch_ag, n, nb):
    """Against dA = A^-1 - A^-1 B B^T A^-1 and dB = 2 A^-1 B (ragged n too)."""
    torch, ag, L = torch_ag
    assert L.plasma_set(pb.PlasmaNb, nb) == 0
    a, b = likelihood_system(n, 8, seed=30 + n)
    A = torch.tensor(a, device="cuda", requires_grad=True)
    B = torch.tensor(b, device="cuda", requires_grad=True)
    ag.gaussian_nll(A, B).backward()
    ai = np.linalg.inv(a)
    x = ai @ b
    ga_ref = ai - x @ x.T
    gb_ref = 2 * x
    ga, gb = A.grad.cpu().numpy(), B.grad.cpu().numpy()
    assert np.abs(ga - ga_ref).max() <= 1e-10 * np.abs(ga_ref).max()
    assert np.abs(gb - gb_ref).max() <= 1e-10 * np.abs(gb_ref).max()
    assert np.array_equal(ga, ga.T)


def test_factor_adjoint_closed_form(torch_ag):
    """potrf adjoint alone, random lower cotangent, through the C ABI, lower
    and upper storage (upper: U = L^T, Ubar = Lbar^T)."""
    torch, ag, L = torch_ag
    L.plasma_set(pb.PlasmaNb, 128)
    n = 500
    a, _ = likelihood_system(n, 1, seed=5)
    lf = np.linalg.cholesky(a)
    rng = np.random.default_rng(9)
    lbar = np.tril(rng.standard_normal((n, n)))
    ref = phi_formula(lf, lbar)
    for uplo in (LO, UP):
        fac = lf if uplo == LO else lf.T
        cot = lbar if uplo == LO else lbar.T
        pl = np.asfortranarray(fac)
        pbar = np.asfortranarray(cot.copy())
        assert L.plasma_dpotrf_adjoint(uplo, n, pl.ctypes.data, n, pbar.ctypes.data, n) == 0
        assert np.abs(pbar - ref).max() <= 1e-11 * np.abs(ref).max(), uplo


def test_solve_adjoint_closed_form(torch_ag):
    """potrs adjoint through the C ABI: Bbar = A^-1 Xbar and
    Lbar -= tril((Bbar X^T + X Bbar^T) L), lower and upper storage."""
    torch, ag, L = torch_ag
    L.plasma_set(pb.PlasmaNb, 64)
    n, k = 300, 5
    a, b = likelihood_system(n, k, seed=6)
    lf = np.linalg.cholesky(a)
    x = np.linalg.solve(a, b)
    rng = np.random.default_rng(10)
    xbar = rng.standard_normal((n, k))
    lbar0 = np.tril(rng.standard_normal((n, n)))
    bbar_ref = np.linalg.solve(a, xbar)
    lbar_ref = lbar0 - np.tril((bbar_ref @ x.T + x @ bbar_ref.T) @ lf)
    for uplo in (LO, UP):
        fac = np.asfortranarray(lf if uplo == LO else lf.T)
        px = np.asfortranarray(x)
        pxbar = np.asfortranarray(xbar.copy())
        plbar = np.asfortranarray((lbar0 if uplo == LO else lbar0.T).copy())
        assert L.plasma_dpotrs_adjoint(uplo, n, k, fac.ctypes.data, n, px.ctypes.data, n,
                                       pxbar.ctypes.data, n, plbar.ctypes.data, n) == 0
        got = plbar if uplo == LO else plbar.T
        mask = np.tril(np.ones((n, n), bool))
        assert np.abs(pxbar - bbar_ref).max() <= 1e-11 * np.abs(bbar_ref).max()
        assert np.abs(got[mask] - lbar_ref[mask]).max() <= 1e-11 * np.abs(lbar_ref).max()


def test_fp32(torch_ag):
    """FP32 forward and backward (three-product TF32 GEMMs): relative error of
    the gradient against the FP64 analytic one at FP32 level."""
    torch, ag, L = torch_ag
    L.plasma_set(pb.PlasmaNb, 128)
    n = 512
    a, b = likelihood_system(n, 8, seed=8)
    A = torch.tensor(a, device="cuda", dtype=torch.float32, requires_grad=True)
    B = torch.tensor(b, device="cuda", dtype=torch.float32, requires_grad=True)
    ag.gaussian_nll(A, B).backward()
    ai = np.linalg.inv(a)
    x = ai @ b
    ga_ref = ai - x @ x.T
    ga = A.grad.double().cpu().numpy()
    assert np.abs(ga - ga_ref).max() <= 2e-4 * np.abs(ga_ref).max()


def test_not_positive_definite_raises(torch_ag):
    torch, ag, _ = torch_ag
    a = -np.eye(16)
    with pytest.raises(RuntimeError):
        ag.cholesky(torch.tensor(a, device="cuda"))
