"""Batched SPD systems of uneven order in one launch (no reference
counterpart: PLASMA solves one matrix at a time).  Oracles: LAPACK through
numpy per matrix (factor, solve, info), the closed forms of the adjoints, the
tester's scaled residual < 50 eps, and the single-matrix path of this library.
"""
import numpy as np
import pytest

import plasma_b200 as pb
from conftest import EPS, SEPS, TOL, solve_residual

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    assert torch.cuda.is_available()
    L = pb.lib()
    assert L.plasma_init() == 0
    from plasma_b200.batched import Batch
    yield torch, Batch, L
    L.plasma_finalize()


EDGE = [1, 2, 7, 15, 16, 17, 31, 32, 33, 48, 63, 64, 65, 100, 128, 129, 200, 255, 256,
        257, 300, 383, 384, 450, 511, 512, 0]


def systems(sizes, seed, shift=0.1):
    """A = G G^T / n + shift I, b ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    mats, vecs = [], []
    for n in sizes:
        g = rng.standard_normal((n, n))
        mats.append(g @ g.T / max(n, 1) + shift * np.eye(n))
        vecs.append(rng.standard_normal(n))
    return mats, vecs


@pytest.mark.parametrize("dtype_name", ["f64", "f32"])
def test_posv_uneven_edges(env, dtype_name):
    torch, Batch, _ = env
    dt = torch.float64 if dtype_name == "f64" else torch.float32
    eps = EPS if dtype_name == "f64" else SEPS
    rng = np.random.default_rng(1)
    sizes = EDGE + list(rng.integers(16, 513, 40))
    mats, vecs = systems(sizes, seed=2)
    b = Batch(sizes, dt)
    A, B, info = b.pack_matrices(mats), b.pack_vectors(vecs), b.info_buffer()
    b.posv(A, B, info)
    torch.cuda.synchronize()
    assert not info.any()
    for i, n in enumerate(sizes):
        if n == 0:
            continue
        x = b.vector(B, i)
        assert solve_residual(mats[i], x[:, None], vecs[i][:, None]) < TOL * eps, (i, n)
        lf = np.tril(b.matrix(A, i))
        lref = np.linalg.cholesky(mats[i])
        assert np.abs(lf - lref).max() <= 50 * n * eps * np.abs(lref).max(), (i, n)
    b.close()


def test_info_not_positive_definite(env):
    """A matrix with a zero column k reports info = k + 1 (LAPACK dpotrf) and
    its neighbours are solved."""
    torch, Batch, _ = env
    sizes = [40, 100, 300, 64]
    mats, vecs = systems(sizes, seed=3)
    bad = {1: 57, 2: 0, 3: 63}
    for i, k in bad.items():
        mats[i][:, k] = 0.0
        mats[i][k, :] = 0.0
    b = Batch(sizes)
    A, B, info = b.pack_matrices(mats), b.pack_vectors(vecs), b.info_buffer()
    b.posv(A, B, info)
    got = info.cpu().numpy()
    assert got[0] == 0
    for i, k in bad.items():
        assert got[i] == k + 1, (i, got[i])
    assert solve_residual(mats[0], b.vector(B, 0)[:, None], vecs[0][:, None]) < TOL * EPS
    b.close()


def test_potrf_then_potrs_and_block_widths(env):
    """potrf + potrs equal posv; block widths 16 and 32 agree."""
    torch, Batch, L = env
    sizes = [33, 64, 150, 257, 512]
    mats, vecs = systems(sizes, seed=4)
    saved = [L.plasma_tuning_get_batched_nb(pb.PlasmaRealDouble, n) for n in sizes]
    results = []
    for nb in (16, 32):
        for n in sizes:
            assert L.plasma_tuning_set_batched_nb(pb.PlasmaRealDouble, n, nb) == 0
        b = Batch(sizes)
        A, B, info = b.pack_matrices(mats), b.pack_vectors(vecs), b.info_buffer()
        b.potrf(A, info)
        b.potrs(A, B)
        torch.cuda.synchronize()
        assert not info.any()
        results.append([b.vector(B, i) for i in range(len(sizes))])
        b.close()
    for i, n in enumerate(sizes):
        assert solve_residual(mats[i], results[0][i][:, None], vecs[i][:, None]) < TOL * EPS
        assert np.abs(results[0][i] - results[1][i]).max() <= 1e-9 * np.abs(results[0][i]).max()
    for n, nb in zip(sizes, saved):
        L.plasma_tuning_set_batched_nb(pb.PlasmaRealDouble, n, nb)


def test_graph_replay(env):
    """A plan in graph mode replays one captured launch; results equal the
    direct launch on fresh copies, twice."""
    torch, Batch, _ = env
    sizes = [20, 90, 333, 512, 5]
    mats, vecs = systems(sizes, seed=5)
    ref = Batch(sizes)
    A0, B0 = ref.pack_matrices(mats), ref.pack_vectors(vecs)
    A, B, info = A0.clone(), B0.clone(), ref.info_buffer()
    ref.posv(A, B, info)
    g = Batch(sizes, graph=True)
    for _ in range(2):
        A1, B1 = A0.clone(), B0.clone()
        Ag, Bg, infog = A1, B1, g.info_buffer()
        g.posv(Ag, Bg, infog)
        torch.cuda.synchronize()
        assert torch.equal(Bg, B) and torch.equal(Ag, A)
    ref.close()
    g.close()


def phi_formula(lf, lbar):
    p = lf.T @ np.tril(lbar)
    phi = np.tril(p) - 0.5 * np.diag(np.diag(p))
    li = np.linalg.inv(lf)
    m = li.T @ phi @ li
    return 0.5 * (m + m.T)


def test_adjoints_closed_form(env):
    torch, Batch, _ = env
    sizes = [1, 17, 32, 33, 90, 200, 301]
    mats, vecs = systems(sizes, seed=6, shift=1.0)
    rng = np.random.default_rng(7)
    lfs = [np.linalg.cholesky(a) for a in mats]
    lbars = [np.tril(rng.standard_normal(a.shape)) for a in mats]
    xs = [np.linalg.solve(a, v) for a, v in zip(mats, vecs)]
    xbars = [rng.standard_normal(len(v)) for v in vecs]
    b = Batch(sizes)
    Lf = b.pack_matrices(lfs)
    # factor adjoint
    Lbar = b.pack_matrices(lbars)
    b.potrf_adjoint(Lf, Lbar)
    for i, n in enumerate(sizes):
        ref = phi_formula(lfs[i], lbars[i])
        got = b.matrix(Lbar, i)
        assert np.abs(got - ref).max() <= 1e-11 * max(1.0, np.abs(ref).max()), (i, n)
    # solve adjoint
    Lbar = b.pack_matrices(lbars)
    X, Xbar = b.pack_vectors(xs), b.pack_vectors(xbars)
    b.potrs_adjoint(Lf, X, Xbar, Lbar)
    for i, n in enumerate(sizes):
        bbar = np.linalg.solve(mats[i], xbars[i])
        lref = lbars[i] - np.tril(np.outer(bbar, xs[i]) @ lfs[i] + np.outer(xs[i], bbar) @ lfs[i])
        assert np.abs(b.vector(Xbar, i) - bbar).max() <= 1e-11 * np.abs(bbar).max()
        got = np.tril(b.matrix(Lbar, i))
        assert np.abs(got - lref).max() <= 1e-11 * np.abs(lref).max(), (i, n)
    b.close()


def test_likelihood_batch_gradient(env):
    """Config-shaped batch (n uniform in [16, 512], A = G G^T/n + 0.1 I,
    seed 5), smaller count: the gradient of logdet(A) + b^T A^-1 b from the
    batched factor, solve and both adjoints equals A^-1 - x x^T."""
    torch, Batch, _ = env
    rng = np.random.default_rng(5)
    sizes = list(rng.integers(16, 513, 24))
    mats, vecs = systems(sizes, seed=5)
    b = Batch(sizes)
    A, B, info = b.pack_matrices(mats), b.pack_vectors(vecs), b.info_buffer()
    Bx = B.clone()
    b.posv(A, Bx, info)                      # A <- L, Bx <- x
    assert not info.any()
    # cotangents: d/dL logdet = diag(2 / L_ii); d/dx (b^T x) = b
    lb = []
    for i, n in enumerate(sizes):
        lf = np.tril(b.matrix(A, i))
        lb.append(np.diag(2.0 / np.diag(lf)))
    Lbar = b.pack_matrices(lb)
    Xbar = B.clone()
    b.potrs_adjoint(A, Bx, Xbar, Lbar)       # Xbar <- bbar = A^-1 b = x
    b.potrf_adjoint(A, Lbar)                 # Lbar <- dA
    for i, n in enumerate(sizes):
        ai = np.linalg.inv(mats[i])
        x = ai @ vecs[i]
        ref = ai - np.outer(x, x)
        got = b.matrix(Lbar, i)
        assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max(), (i, n)
    b.close()


def test_plan_rejects_large_orders(env):
    torch, Batch, L = env
    with pytest.raises(RuntimeError):
        Batch([10, 513])
