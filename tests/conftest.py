import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

EPS = np.finfo(np.float64).eps * 0.5   # LAPACK dlamch('E')
SEPS = np.finfo(np.float32).eps * 0.5
TOL = 50.0                              # reference tester default (test/test.c:920)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "lapack_fixtures.npz"))


def solve_residual(a_full, x, b):
    """Reference tester residual ||B - A X||_inf / (n ||A||_inf ||X||_inf)."""
    n = a_full.shape[0]
    r = b - a_full @ x
    an = np.abs(a_full).sum(axis=1).max()
    xn = np.abs(x).sum(axis=1).max()
    rn = np.abs(r).sum(axis=1).max()
    return rn / (n * an * xn) if an * xn > 0 else rn


def factor_error(l, l_ref, a_full):
    """Reference potrf tester error ||L - L_lapack||_F / ||A||_F."""
    an = np.linalg.norm(a_full)
    return np.linalg.norm(l - l_ref) / an if an > 0 else np.linalg.norm(l - l_ref)


def factor_residual(l, a_full, lower=True):
    """||A - L L^T||_F / (n ||A||_F eps)."""
    n = a_full.shape[0]
    r = a_full - (l @ l.T if lower else l.T @ l)
    return np.linalg.norm(r) / (n * np.linalg.norm(a_full) * EPS)
