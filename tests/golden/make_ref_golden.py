"""Writes reference_fixtures.npz: outputs of the reference PLASMA itself.

The reference's SPD path is built from its own sources by oracle/build_ref.sh
(oracle/_ref/libplasma_ref.so, OpenBLAS 0.3.15 single-threaded) and run here
on the seeded inputs of gen.py.  The fixtures pin the oracle (tests/
test_reference_pin.py) and the GPU library (tests/test_gpu_reference.py) to
the reference's own answers where the reference itself cannot travel:
  cfg1_*   config 1: n = 2048, nb = 256, nrhs = 1, diagonally dominant,
           seed 42 -- factor checksums (diagonal, L v, U^T v), the dposv
           solution, the dsposv solution, iter and info;
  rag_*    n = 1000, nb = 128: factor checksums, dposv with 3 right-hand sides;
  potrs_*  dpotrs on the reference's own factor, n = 300, nrhs = 4;
  spec_*   dsposv on A = Q diag(lambda) Q^T (kappa 1e2, 1e5), n 256 / 1000,
           nb 64 / 128, both triangles, nrhs 2: iter, info, X;
  fail_*   the failure semantics: --zerocol inputs (dpotrf and dsposv info),
           kappa = 1e12 (the FP32 factor fails), FP32 overflow in A or B.
Factors are stored as checksums (diag(L), L v with gen.probe_vector) rather
than whole, to keep the file small.

Run: python tests/golden/make_ref_golden.py   (builds oracle/_ref if needed)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import gen  # noqa: E402
from oracle import ref  # noqa: E402

LO, UP = ref.LOWER, ref.UPPER


def F(a):
    return np.asfortranarray(np.array(a, dtype=np.float64))


def factor_checksums(out, key, a, nb):
    n = a.shape[0]
    v = gen.probe_vector(n)
    f = F(a)
    assert ref.dpotrf(LO, f, nb) == 0
    lo = np.tril(f)
    out[f"{key}_diagL"] = np.diag(lo).copy()
    out[f"{key}_Lv"] = lo @ v
    f = F(a)
    assert ref.dpotrf(UP, f, nb) == 0
    up = np.triu(f)
    out[f"{key}_diagU"] = np.diag(up).copy()
    out[f"{key}_UTv"] = up.T @ v


def dsposv_case(out, key, uplo, a, b, nb):
    x = F(np.full(b.shape, 7.0))
    info, it = ref.dsposv(uplo, F(a), F(b), x, nb)
    out[f"{key}_info"] = np.int64(info)
    out[f"{key}_iter"] = np.int64(it)
    out[f"{key}_X"] = x
    return info, it


def main():
    ref.set_threads(min(8, os.cpu_count() or 1))
    out = {}

    # config 1
    n, nb = 2048, 256
    a, b = gen.diag_dominant(n, 1, seed=42)
    factor_checksums(out, "cfg1", a, nb)
    x = F(b)
    assert ref.dposv(LO, F(a), x, nb) == 0
    out["cfg1_dposv_X"] = x
    dsposv_case(out, "cfg1_dsposv", LO, a, b, nb)

    # ragged size, several right-hand sides
    n, nb = 1000, 128
    a, b = gen.diag_dominant(n, 3, seed=3000)
    factor_checksums(out, "rag", a, nb)
    x = F(b)
    assert ref.dposv(LO, F(a), x, nb) == 0
    out["rag_dposv_X"] = x
    x = F(b)
    assert ref.dposv(UP, F(a), x, nb) == 0
    out["rag_dposv_up_X"] = x

    # dpotrs with the reference's factor
    n, nb = 300, 64
    a, b = gen.diag_dominant(n, 4, seed=3001)
    f = F(a)
    assert ref.dpotrf(LO, f, nb) == 0
    x = F(b)
    assert ref.dpotrs(LO, f, x, nb) == 0
    out["potrs_X"] = x

    # mixed precision on prescribed spectra
    for n, nb in ((256, 64), (1000, 128)):
        for kexp in (2, 5):
            a = gen.spectrum(n, 10.0 ** kexp, seed=11)
            xt = np.random.default_rng(12).standard_normal((n, 2))
            b = F(a @ xt)
            for uplo, tag in ((LO, "L"), (UP, "U")):
                info, it = dsposv_case(out, f"spec_n{n}_k{kexp}_{tag}", uplo, a, b, nb)
                assert info == 0 and it >= 0, (n, kexp, tag, info, it)

    # failure semantics
    n, nb = 1000, 128
    a, b = gen.diag_dominant(n, 2, seed=6)
    for col in (0, 299, 999):
        za = gen.zerocol(a, col)
        dsposv_case(out, f"fail_zerocol{col}", LO, za, b, nb)
        f = F(a)
        f[:, col] = 0.0                    # test_zpotrf.c zeroes the column only
        out[f"fail_potrf_zerocol{col}_info"] = np.int64(ref.dpotrf(LO, f, nb))
    a12 = gen.spectrum(256, 1e12, seed=11)
    b12 = F(np.random.default_rng(1).standard_normal((256, 1)))
    for uplo, tag in ((LO, "L"), (UP, "U")):
        dsposv_case(out, f"fail_k12_{tag}", uplo, a12, b12, 64)
    ao = a.copy()
    ao[5, 3] = ao[3, 5] = 1e39
    dsposv_case(out, "fail_ovfA", LO, ao, b, nb)
    bo = b.copy()
    bo[4, 1] = -1e39
    dsposv_case(out, "fail_ovfB", LO, a, bo, nb)

    path = os.path.join(HERE, "reference_fixtures.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays")
    for k in sorted(out):
        if k.endswith("_info") or k.endswith("_iter"):
            print(f"  {k} = {int(out[k])}")


if __name__ == "__main__":
    main()
