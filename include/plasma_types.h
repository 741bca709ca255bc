/*
 * plasma_types.h -- enumerations and scalar types of the PLASMA C API.
 *
 * Every numeric value below is part of the binary interface: callers pass raw
 * ints (PlasmaLower == 122 ...) and the reference casts them straight to the
 * CBLAS enumerations, so the values equal the reference's
 * include/plasma_types.h:49-165 one for one.  Only the declarations needed by
 * the SPD path (potrf / potrs / posv / dsposv) and its descriptors are kept.
 */
#ifndef PLASMA_TYPES_H
#define PLASMA_TYPES_H

#include <limits.h>

#define PLASMA_VERSION_MAJOR 25
#define PLASMA_VERSION_MINOR 5
#define PLASMA_VERSION_PATCH 27

#ifdef __cplusplus
extern "C" {
#endif

/* Element types of a descriptor (reference include/plasma_types.h:49-57). */
enum {
    PlasmaByte            = 0,
    PlasmaInteger         = 1,
    PlasmaRealFloat       = 2,
    PlasmaRealDouble      = 3,
    PlasmaComplexFloat    = 4,
    PlasmaComplexDouble   = 5,
    PlasmaDatatypeUnknown = INT_MIN
};

/* CBLAS/LAPACK-compatible constants (reference include/plasma_types.h:71-121). */
enum {
    PlasmaInvalid       = -1,

    PlasmaNoTrans       = 111,
    PlasmaTrans         = 112,
    PlasmaConjTrans     = 113,
    Plasma_ConjTrans    = PlasmaConjTrans,

    PlasmaUpper         = 121,
    PlasmaLower         = 122,
    PlasmaGeneral       = 123,
    PlasmaGeneralBand   = 124,

    PlasmaNonUnit       = 131,
    PlasmaUnit          = 132,

    PlasmaLeft          = 141,
    PlasmaRight         = 142,

    PlasmaOneNorm       = 171,
    PlasmaRealOneNorm   = 172,
    PlasmaTwoNorm       = 173,
    PlasmaFrobeniusNorm = 174,
    PlasmaInfNorm       = 175,
    PlasmaRealInfNorm   = 176,
    PlasmaMaxNorm       = 177,
    PlasmaRealMaxNorm   = 178,

    PlasmaNoVec         = 301,
    PlasmaVec           = 302,
    PlasmaCount         = 303,
    PlasmaIVec          = 304,
    PlasmaAllVec        = 305,
    PlasmaSomeVec       = 306,

    PlasmaRangeAll      = 351,
    PlasmaRangeV        = 352,
    PlasmaRangeI        = 353,

    PlasmaForward       = 391,
    PlasmaBackward      = 392,

    PlasmaColumnwise    = 401,
    PlasmaRowwise       = 402,

    PlasmaW             = 501,
    PlasmaA2            = 502,
    Plasma_Const_Limit,

    PlasmaConstUnknown  = INT_MIN
};

/* Return codes (reference include/plasma_types.h:123-137). */
enum {
    PlasmaSuccess             = 0,
    PlasmaErrorNotInitialized = -101,
    PlasmaErrorNotSupported   = -102,
    PlasmaErrorIllegalValue   = -103,
    PlasmaErrorOutOfMemory    = -104,
    PlasmaErrorNullParameter  = -105,
    PlasmaErrorInternal       = -106,
    PlasmaErrorSequence       = -107,
    PlasmaErrorComponent      = -108,
    PlasmaErrorEnvironment    = -109,
    PlasmaErrorUnknown        = INT_MIN
};

enum {
    PlasmaInplace,
    PlasmaOutplace,
    PlasmaInoutUnknown = INT_MAX
};

enum {
    PlasmaFlatHouseholder,
    PlasmaTreeHouseholder,
    PlasmaHouseholderUnknown = INT_MAX
};

enum {
    PlasmaDisabled     = 0,
    PlasmaEnabled      = 1,
    PlasmaAbledUnknown = INT_MAX
};

/*
 * plasma_set / plasma_get parameters.  The first six keep the reference's
 * values (include/plasma_types.h:157-165).  The GPU build adds its own
 * parameters in a separate range starting at 1000 so that no existing value
 * moves.
 */
enum {
    PlasmaTuning,
    PlasmaNb,
    PlasmaIb,
    PlasmaInplaceOutplace,
    PlasmaNumPanelThreads,
    PlasmaHouseholderMode,

    /* GPU-build extensions. */
    PlasmaMixedPrecisionMode = 1000, /* factor precision used by dsposv  */
    PlasmaRefinement         = 1001, /* IR, GMRES-IR or automatic choice  */
    PlasmaDevice             = 1002, /* CUDA device ordinal               */
    PlasmaLookahead          = 1003, /* panels factored ahead of update   */

    PlasmaParamUnknown = INT_MAX
};

/* Values of PlasmaMixedPrecisionMode (GPU-build extension). */
enum {
    PlasmaFactorFP32 = 0,   /* FP32 factor on CUDA cores                     */
    PlasmaFactorTF32 = 1,   /* TF32 tensor-core update, FP32 accumulation    */
    PlasmaFactorBF16 = 2,   /* BF16 tensor-core update, FP32 accumulation    */
    PlasmaFactorAuto = 3    /* BF16 first, escalate on failure or stagnation */
};

/* Values of PlasmaRefinement (GPU-build extension). */
enum {
    PlasmaRefineIR     = 0, /* classical iterative refinement (reference)  */
    PlasmaRefineGMRES  = 1, /* GMRES-IR preconditioned by the factor       */
    PlasmaRefineAuto   = 2  /* IR, switching to GMRES-IR on stagnation     */
};

typedef int plasma_enum_t;

typedef double plasma_time_t;

plasma_enum_t plasma_uplo_const(char lapack_char);
plasma_enum_t plasma_trans_const(char lapack_char);
plasma_enum_t plasma_side_const(char lapack_char);
plasma_enum_t plasma_diag_const(char lapack_char);
plasma_enum_t plasma_norm_const(char lapack_char);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_TYPES_H */
