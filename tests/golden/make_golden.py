"""Writes tests/golden/lapack_fixtures.npz: LAPACK (scipy) answers for seeded
SPD inputs.  The reference's own tester defines correctness against LAPACK
(test/test_zpotrf.c:124-141 compares with LAPACKE_dpotrf; the posv/dsposv
testers check the scaled residual), so these are the known answers the
oracle and the GPU library are pinned to.

Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np
import scipy
import scipy.linalg.lapack as lapack

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import gen  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lapack_fixtures.npz")


def main():
    d = {"scipy_version": np.array(scipy.__version__)}
    # small cases: full outputs
    for n in (1, 2, 7, 33, 64, 100):
        a, b = gen.diag_dominant(n, 3, seed=1000 + n)
        lo, info_l = lapack.dpotrf(a, lower=1, clean=1)
        up, info_u = lapack.dpotrf(a, lower=0, clean=1)
        _, x, info_x = lapack.dposv(a, b, lower=1)
        assert info_l == 0 and info_u == 0 and info_x == 0
        d[f"small{n}_A"] = a
        d[f"small{n}_B"] = b
        d[f"small{n}_L"] = np.tril(lo)
        d[f"small{n}_U"] = np.triu(up)
        d[f"small{n}_X"] = x
    # ragged sizes (n not a multiple of the tile size): checksums only
    for n in (300, 1000):
        a, b = gen.diag_dominant(n, 5, seed=2000 + n)
        lo, info = lapack.dpotrf(a, lower=1, clean=1)
        _, x, _ = lapack.dposv(a, b, lower=1)
        v = gen.probe_vector(n)
        d[f"ragged{n}_diagL"] = np.diag(lo).copy()
        d[f"ragged{n}_Lv"] = np.tril(lo) @ v
        d[f"ragged{n}_X"] = x
    # the CPU parity configuration: n = 2048, nrhs = 1, seed 42
    n = 2048
    a, b = gen.diag_dominant(n, 1, seed=42)
    lo, info = lapack.dpotrf(a, lower=1, clean=1)
    _, x, _ = lapack.dposv(a, b, lower=1)
    v = gen.probe_vector(n)
    d["cfg1_diagL"] = np.diag(lo).copy()
    d["cfg1_Lv"] = np.tril(lo) @ v
    d["cfg1_Ltv"] = np.tril(lo).T @ v
    d["cfg1_X"] = x
    d["cfg1_normL"] = np.array(np.linalg.norm(np.tril(lo)))
    # non positive definite: LAPACK's info for a zeroed row/column
    for n, col in ((100, 37), (300, 0), (300, 299), (513, 256)):
        a, _ = gen.diag_dominant(n, 1, seed=3000 + n)
        a = gen.zerocol(a, col)
        _, info_l = lapack.dpotrf(a, lower=1)
        _, info_u = lapack.dpotrf(a, lower=0)
        d[f"nonspd{n}_{col}_info_lower"] = np.array(info_l)
        d[f"nonspd{n}_{col}_info_upper"] = np.array(info_u)
    # prescribed spectrum (mixed-precision cases), n = 256
    for kappa in (1e2, 1e5, 1e8):
        a = gen.spectrum(256, kappa, seed=11)
        rng = np.random.default_rng(12)
        xt = rng.standard_normal((256, 1))
        bb = a @ xt
        _, x, info = lapack.dposv(a, bb, lower=1)
        d[f"spec{int(np.log10(kappa))}_X"] = x
        d[f"spec{int(np.log10(kappa))}_xtrue"] = xt
    # inverse from the Cholesky factor (dpotri; the reference tester
    # test/test_zpotri.c:135-155 compares plasma_zpotri with LAPACKE_zpotri)
    for n in (7, 64, 100):
        a, _ = gen.diag_dominant(n, 1, seed=4000 + n)
        for lower, tag in ((1, "L"), (0, "U")):
            c, info = lapack.dpotrf(a, lower=lower, clean=1)
            inv, info_i = lapack.dpotri(c, lower=lower)
            assert info == 0 and info_i == 0
            tri = np.tril if lower else np.triu
            d[f"potri{n}_{tag}_factor"] = tri(c)
            d[f"potri{n}_{tag}_inv"] = tri(inv)
    # band Cholesky (dpbtrf) and band solve (dpbtrs): the reference tester
    # test/test_zpbsv.c:167-214 and test_zpbtrf.c:155-214 check the residual
    # and, on failure, LAPACKE_zpbsv's info
    # (inputs are rebuilt from gen.band with the same seed)
    for n, kd in ((7, 2), (64, 10), (100, 33), (130, 0), (96, 95)):
        a, abl, abu, b = gen.band(n, kd, 2, seed=5000 + n + kd)
        for lower, tag, ab in ((1, "L", abl), (0, "U", abu)):
            c, info = lapack.dpbtrf(ab, lower=lower)
            x, info_x = lapack.dpbtrs(c, b, lower=lower)
            assert info == 0 and info_x == 0
            d[f"band{n}_{kd}_{tag}_factor"] = c
            d[f"band{n}_{kd}_{tag}_X"] = x
    for n, kd, col in ((100, 9, 41), (300, 40, 0)):
        a, abl, abu, _ = gen.band(n, kd, 1, seed=6000 + n)
        a = gen.zerocol(a, col)
        for lower, tag in ((1, "L"), (0, "U")):
            _, info = lapack.dpbtrf(gen.to_band(a, kd, lower=bool(lower)), lower=lower)
            d[f"bandinfo{n}_{kd}_{tag}"] = np.array(info)
    # LU with partial pivoting (dgetrf, 1-based pivots), dgesv solutions,
    # dgetrf's info for a zero column; the reference's getrf tester compares
    # with LAPACKE_zgetrf (test/test_zgetrf.c:116-138), gesv and dcgesv check
    # the residual (test_zgesv.c, test_zcgesv.c:133-170)
    for n in (7, 64, 100, 150):
        a, b = gen.general(n, 2, seed=9000 + n)
        lu, piv, info = lapack.dgetrf(a)
        _, _, x, info_x = lapack.dgesv(a, b)
        assert info == 0 and info_x == 0
        d[f"lu{n}_LU"] = lu
        d[f"lu{n}_ipiv"] = (piv + 1).astype(np.int32)
        d[f"lu{n}_X"] = x
    for n, col in ((64, 20), (100, 0)):
        a, _ = gen.general(n, 1, seed=9100 + n)
        a[:, col] = 0.0
        _, _, info = lapack.dgetrf(a)
        d[f"luinfo{n}_{col}"] = np.array(info)
    for kappa in (1e2, 1e12):
        a = gen.general_spectrum(100, kappa)
        b = np.asfortranarray(np.cos(np.arange(200.0)).reshape(100, 2))
        _, _, x, info = lapack.dgesv(a, b)
        d[f"gesv_kappa{kappa:.0e}_X"] = x
    np.savez_compressed(OUT, **d)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
