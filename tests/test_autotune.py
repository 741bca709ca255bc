"""Measured autotuner of the tile-shape tables (no reference counterpart:
the reference reads nb from a Lua script).  The tuned tables must hold
candidate values, be what the library then uses, and leave results correct."""
import numpy as np
import pytest

import gen
import plasma_b200 as pb
from conftest import EPS, TOL, solve_residual

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def L():
    import torch
    assert torch.cuda.is_available()
    lib = pb.lib()
    assert lib.plasma_init() == 0
    yield lib
    lib.plasma_finalize()


def test_autotune_potrf_sets_table(L, tmp_path):
    import plasma_b200.autotune as at
    t = at.tune(potrf_sizes=(600, 2048), batched_count=64, precisions=("f64",))
    for n in (600, 2048):
        nb = t["potrf_nb"]["f64"][str(n)]
        assert nb in (128, 256, 384, 512)
        assert L.plasma_tuning_get_potrf_nb(pb.PlasmaRealDouble, n) == nb
        assert t["potrf_ms"]["f64"][str(n)] > 0
    for n, nb in t["batched_nb"]["f64"].items():
        assert nb in (16, 32)
    # round trip through the saved tables
    p = tmp_path / "tables.json"
    at.save(t, p)
    L.plasma_tuning_set_potrf_nb(pb.PlasmaRealDouble, 2048, 128)
    at.load(p)
    assert L.plasma_tuning_get_potrf_nb(pb.PlasmaRealDouble, 2048) == t["potrf_nb"]["f64"]["2048"]
    # the LAPACK-layout solve uses the tuned nb and stays correct
    n = 2048
    a, b = gen.diag_dominant(n, 3, seed=77)
    x, af = np.asfortranarray(b.copy()), np.asfortranarray(a.copy())
    assert L.plasma_dposv(pb.PlasmaLower, n, 3, af.ctypes.data, n, x.ctypes.data, n) == 0
    assert solve_residual(a, x, b) < TOL * EPS
