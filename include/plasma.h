/*
 * plasma.h -- umbrella header of the B200 build of PLASMA's SPD path.
 * Mirrors the reference's include/plasma.h: one include gives the types,
 * descriptors, the sequence/request model, the context API and the s, d and
 * ds routines.
 */
#ifndef PLASMA_H
#define PLASMA_H

#include "plasma_types.h"
#include "plasma_error.h"
#include "plasma_async.h"
#include "plasma_descriptor.h"

#include "plasma_s.h"
#include "plasma_d.h"
#include "plasma_ds.h"

#ifdef __cplusplus
extern "C" {
#endif

/* reference control/context.c:30-47: PlasmaErrorNotInitialized on a second
 * call.  Also selects the CUDA device (PlasmaDevice, default 0), creates the
 * context streams and the device status word. */
int plasma_init(void);
/* reference control/context.c:54-71 */
int plasma_finalize(void);
/* reference control/context.c:78-127 (PlasmaNb <= 0 -> IllegalValue) */
int plasma_set(plasma_enum_t param, int value);
/* reference control/context.c:133-159 */
int plasma_get(plasma_enum_t param, int *value);
/* reference control/version.c:14-19 */
void plasma_version(int *major, int *minor, int *micro);

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_H */
