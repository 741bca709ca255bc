/* Configuration for building the reference PLASMA's SPD path against
 * OpenBLAS (no MKL, no ESSL, no Lua tuning scripts); test infrastructure
 * only. */
#define PLASMA_WITH_OPENBLAS 1
