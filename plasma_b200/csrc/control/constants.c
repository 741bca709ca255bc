/*
 * constants.c -- LAPACK character to PLASMA constant mapping, the same
 * mapping as the reference's control/constants.c (plasma_uplo_const :124-131
 * and siblings).
 */
#include "plasma_types.h"

plasma_enum_t plasma_uplo_const(char c)
{
    switch (c) {
    case 'U': case 'u': return PlasmaUpper;
    case 'L': case 'l': return PlasmaLower;
    default:            return PlasmaGeneral;
    }
}

plasma_enum_t plasma_trans_const(char c)
{
    switch (c) {
    case 'N': case 'n': return PlasmaNoTrans;
    case 'T': case 't': return PlasmaTrans;
    case 'C': case 'c': return PlasmaConjTrans;
    default:            return PlasmaInvalid;
    }
}

plasma_enum_t plasma_side_const(char c)
{
    switch (c) {
    case 'L': case 'l': return PlasmaLeft;
    case 'R': case 'r': return PlasmaRight;
    default:            return PlasmaInvalid;
    }
}

plasma_enum_t plasma_diag_const(char c)
{
    switch (c) {
    case 'N': case 'n': return PlasmaNonUnit;
    case 'U': case 'u': return PlasmaUnit;
    default:            return PlasmaInvalid;
    }
}

plasma_enum_t plasma_norm_const(char c)
{
    switch (c) {
    case 'M': case 'm': return PlasmaMaxNorm;
    case '1': case 'O': case 'o': return PlasmaOneNorm;
    case '2':           return PlasmaTwoNorm;
    case 'F': case 'f': case 'E': case 'e': return PlasmaFrobeniusNorm;
    case 'I': case 'i': return PlasmaInfNorm;
    default:            return PlasmaInvalid;
    }
}
