#!/usr/bin/env bash
# Build the reference PLASMA's SPD path (dpotrf, dpotrs, dposv, dsposv and
# what they call), its LU-based mixed-precision solver (dsgesv with dgetrf,
# dgetrs), its band Cholesky (dpbtrf, dpbtrs, dpbsv) and its SPD inverse
# (dpotri, dpoinv) as a shared library,
# oracle/_ref/libplasma_ref.so, for the parity tests and for the CPU
# reference arm of bench.py.  Test infrastructure: the product never loads
# it.
#
# What it does:
#   1. copies the reference sources to a scratch directory (the source tree
#      is read-only and its precision generator writes next to its inputs);
#   2. runs the reference's precision generator (tools/codegen.py) on the
#      complex-double templates of the path, producing the d / s / ds files;
#   3. compiles the control layer and the generated files with gcc -fopenmp
#      against oracle/ref_shim (self-written CBLAS / LAPACKE declarations
#      and a plasma_config.h selecting OpenBLAS) and links the OpenBLAS
#      0.3.15 that the image's opencv wheel ships (unprefixed cblas_* /
#      LAPACKE_* symbols), with an rpath to it.
# Only the shared library lands in the repository tree (oracle/_ref/, which
# git ignores); no reference source is copied into the repository.
#
# Usage: oracle/build_ref.sh [REFERENCE_DIR]   (default /root/reference)
# Run OpenBLAS single-threaded: OPENBLAS_NUM_THREADS=1, OMP_NUM_THREADS=cores.
set -euo pipefail

REF=${1:-/root/reference}
HERE=$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)
OUT="$HERE/_ref"
SCRATCH=$(mktemp -d /tmp/plasma_ref_build.XXXXXX)
trap 'rm -rf "$SCRATCH"' EXIT

PY=${PYTHON:-python3}
if [ -z "${OPENBLAS_DIR:-}" ]; then
    OPENBLAS_DIR=$("$PY" - <<'EOF'
import glob, os, site, sys
for d in site.getsitepackages() + [os.path.dirname(os.__file__)]:
    hits = glob.glob(os.path.join(d, "opencv_python_headless.libs", "libopenblas*.so"))
    if hits:
        print(os.path.dirname(hits[0]))
        sys.exit(0)
sys.exit(1)
EOF
) || { echo "build_ref.sh: no OpenBLAS shared library found" >&2; exit 1; }
fi
OPENBLAS_SO=$(ls "$OPENBLAS_DIR"/libopenblas*.so | head -1)

[ -f "$REF/tools/codegen.py" ] || { echo "build_ref.sh: $REF is not the reference tree" >&2; exit 1; }
cp -r "$REF"/. "$SCRATCH/src"
cd "$SCRATCH/src"

COMPUTE_Z="zpotrf zpotrs zposv zcposv pzpotrf pztrsm pzsymm pzlansy pzlacpy
           pzgeadd pzlag2c pclag2z zge2desc zdesc2ge ztr2desc zdesc2tr pzge2desc
           pzdesc2ge pztr2desc pzdesc2tr pdzamax
           zgetrf zgetrs zgesv zcgesv pzgetrf pzgeswp pzgemm pzlange
           zpbtrf zpbtrs zpbsv pzpbtrf pztbsm zpb2desc zdesc2pb pzpb2desc pzdesc2pb
           zpotri zpoinv pztrtri pzlauum"
CORE_Z="core_zpotrf core_ztrsm core_zsyrk core_zgemm core_zsymm core_zlacpy
        core_zgeadd core_zlansy core_zlange core_zsyssq core_zgessq core_zlag2c
        core_clag2z core_dzamax core_zgetrf core_zgeswp core_zlacpy_band
        core_ztrmm core_ztrtri core_zlauum"
HDR_Z="plasma_z plasma_zc plasma_internal_z plasma_internal_zc plasma_core_blas_z
       plasma_core_blas_zc core_lapack_z plasma_zlaebz2_work"

"$PY" tools/codegen.py -p d -p s -p ds \
    $(for f in $COMPUTE_Z; do echo compute/$f.c; done) \
    $(for f in $CORE_Z; do echo core_blas/$f.c; done) >/dev/null
"$PY" tools/codegen.py $(for f in $HDR_Z; do echo include/$f.h; done) >/dev/null

SRC="control/async.c control/barrier.c control/constants.c control/context.c
     control/descriptor.c control/tuning.c control/version.c control/workspace.c"
for f in dpotrf dpotrs dposv dsposv spotrf spotrs sposv pdpotrf pspotrf pdtrsm \
         pstrsm pdlacpy pslacpy pdgeadd psgeadd pdsymm pdlansy pdamax pdlag2s \
         pslag2d dge2desc ddesc2ge dtr2desc ddesc2tr sge2desc sdesc2ge str2desc \
         sdesc2tr pdge2desc pddesc2ge pdtr2desc pddesc2tr psge2desc psdesc2ge \
         pstr2desc psdesc2tr \
         dgetrf dgetrs dgesv dsgesv pdgetrf psgetrf pdgeswp psgeswp pdgemm pdlange \
         dpbtrf dpbtrs dpbsv pdpbtrf pdtbsm dpb2desc ddesc2pb pdpb2desc pddesc2pb \
         dpotri dpoinv pdtrtri pdlauum; do
    SRC="$SRC compute/$f.c"
done
for f in core_dpotrf core_spotrf core_dtrsm core_strsm core_dsyrk core_ssyrk \
         core_dgemm core_sgemm core_dlacpy core_slacpy core_dsymm core_dgeadd \
         core_dlag2s core_slag2d core_dlansy core_dlange core_dsyssq core_dgessq core_sgeadd \
         core_dcabs1 core_damax core_dgetrf core_sgetrf core_dgeswp core_sgeswp \
         core_dlacpy_band core_dtrmm core_dtrtri core_dlauum; do
    SRC="$SRC core_blas/$f.c"
done

mkdir -p "$OUT"
gcc -O3 -std=gnu99 -fopenmp -fPIC -shared -Werror=implicit-function-declaration \
    -I"$HERE/ref_shim" -Iinclude \
    $SRC -o "$OUT/libplasma_ref.so" \
    -L"$OPENBLAS_DIR" -l:"$(basename "$OPENBLAS_SO")" -Wl,--disable-new-dtags,-rpath,"$OPENBLAS_DIR" -Wl,-Bsymbolic \
    -Wl,--no-undefined -lm
echo "built $OUT/libplasma_ref.so (OpenBLAS: $OPENBLAS_SO)"
