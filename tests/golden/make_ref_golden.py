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

reference_lu_band_fixtures.npz holds the same for the LU-based
mixed-precision solver and the band Cholesky:
  lu_n{n}_nb{nb}_*   dgetrf of gen.general (seed 9500 + n): the pivots, diag(U),
                     L v and U v (L unit lower); getrs_X with 3 right-hand
                     sides on that factor (n = 300);
  luinfo_{col}       dgetrf's info for a zeroed column (n = 400, nb = 64);
  gesv_n{n}_k{e}_*   dsgesv on gen.general_spectrum (kappa 1e2, 1e5): info,
                     iter, X.  Only kappa <= 1e5: above about 1e10 the
                     reference's dsgesv is not reproducible (its iteration
                     count and whether X holds NaN change with the thread
                     count and from run to run, since its convergence test
                     passes a NaN residual);
  pb_n{n}_kd{kd}_{L,U}_*  dpbsv of gen.band: the factor's diagonal, its
                     L v (or U^T v) and the solution; pbinfo_* dpbtrf's info
                     for a zeroed row and column.

reference_potri_fixtures.npz holds its SPD inverse:
  potri_n{n}_nb{nb}_{L,U}_*  dpotri on its own dpotrf factor of
                     gen.diag_dominant (seed 8800 + n): the inverse's
                     diagonal and sym(inv) v; poinv gives the same bytes;
  potriinfo_{col}_{L,U}  dpotri's info for a zero on the factor's diagonal
                     (n = 300, nb = 64).

Run: python tests/golden/make_ref_golden.py [spd|lu_band|potri]  (default
all; builds oracle/_ref if needed)
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


def lu_band():
    ref.set_threads(min(8, os.cpu_count() or 1))
    out = {}
    for n, nb in ((300, 64), (1000, 128)):
        a, b = gen.general(n, 3, seed=9500 + n)
        f = F(a)
        info, ipiv = ref.dgetrf(f, nb)
        assert info == 0
        v = gen.probe_vector(n)
        key = f"lu_n{n}_nb{nb}"
        out[f"{key}_ipiv"] = ipiv.astype(np.int32)
        out[f"{key}_diagU"] = np.diag(f).copy()
        out[f"{key}_Lv"] = (np.tril(f, -1) + np.eye(n)) @ v
        out[f"{key}_Uv"] = np.triu(f) @ v
        if n == 300:
            x = F(b)
            assert ref.dgetrs(f, ipiv, x, nb) == 0
            out[f"{key}_getrs_X"] = x
    a, _ = gen.general(400, 1, seed=9600)
    for col in (0, 150, 399):
        f = F(a)
        f[:, col] = 0.0
        out[f"luinfo_{col}"] = np.int64(ref.dgetrf(f, 64)[0])
    for n, nb in ((400, 64), (1000, 128)):
        for kexp in (2, 5):
            if n == 1000 and kexp == 2:
                continue
            a = gen.general_spectrum(n, 10.0 ** kexp)
            b = F(np.cos(np.arange(2.0 * n)).reshape(n, 2))
            x = F(np.zeros((n, 2)))
            info, it, _ = ref.dsgesv(F(a), F(b), x, nb)
            assert info == 0 and it >= 0, (n, kexp, info, it)
            key = f"gesv_n{n}_k{kexp}"
            out[f"{key}_info"] = np.int64(info)
            out[f"{key}_iter"] = np.int64(it)
            out[f"{key}_X"] = x
    for n, kd, nb in ((500, 40, 64), (1000, 100, 128)):
        a, abl, abu, b = gen.band(n, kd, 2, seed=7000 + n)
        v = gen.probe_vector(n)
        for uplo, ab, tag in ((LO, abl, "L"), (UP, abu, "U")):
            f = F(ab)
            x = F(b)
            assert ref.dpbsv(uplo, f, kd, x, nb) == 0
            t = gen.from_band(f, kd, lower=uplo == LO)
            t = t if uplo == LO else t.T
            key = f"pb_n{n}_kd{kd}_{tag}"
            out[f"{key}_diag"] = np.diag(t).copy()
            out[f"{key}_Lv"] = t @ v
            out[f"{key}_X"] = x
    a, _, _, _ = gen.band(300, 20, 1, seed=7300)
    for col, tag, uplo in ((0, "L", LO), (137, "L", LO), (137, "U", UP)):
        z = a.copy()
        z[col, :] = 0.0
        z[:, col] = 0.0
        ab = gen.to_band(z, 20, lower=uplo == LO)
        out[f"pbinfo_{col}_{tag}"] = np.int64(ref.dpbtrf(uplo, F(ab), 20, 64))
    path = os.path.join(HERE, "reference_lu_band_fixtures.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays")
    for k in sorted(out):
        if k.endswith("_info") or k.endswith("_iter") or "info_" in k:
            print(f"  {k} = {int(out[k])}")


def potri():
    ref.set_threads(min(8, os.cpu_count() or 1))
    out = {}
    for n, nb in ((300, 64), (1000, 128)):
        a, _ = gen.diag_dominant(n, 1, seed=8800 + n)
        v = gen.probe_vector(n)
        for uplo, tag in ((LO, "L"), (UP, "U")):
            f = F(a)
            assert ref.dpotrf(uplo, f, nb) == 0
            assert ref.dpotri(uplo, f, nb) == 0
            t = np.tril(f) if uplo == LO else np.triu(f)
            full = t + t.T - np.diag(np.diag(t))
            g = F(a)
            assert ref.dpoinv(uplo, g, nb) == 0
            tg = np.tril(g) if uplo == LO else np.triu(g)
            assert np.array_equal(tg, t)
            key = f"potri_n{n}_nb{nb}_{tag}"
            out[f"{key}_diag"] = np.diag(t).copy()
            out[f"{key}_Sv"] = full @ v
    a, _ = gen.diag_dominant(300, 1, seed=9100)
    for col in (0, 137, 299):
        for uplo, tag in ((LO, "L"), (UP, "U")):
            f = F(a)
            assert ref.dpotrf(uplo, f, 64) == 0
            f[col, col] = 0.0
            out[f"potriinfo_{col}_{tag}"] = np.int64(ref.dpotri(uplo, f, 64))
    path = os.path.join(HERE, "reference_potri_fixtures.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}: {len(out)} arrays")


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    if which in ("spd", "all"):
        main()
    if which in ("lu_band", "all"):
        lu_band()
    if which in ("potri", "all"):
        potri()
