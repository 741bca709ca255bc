/*
 * plasma_error.h -- diagnostics printed by the library.
 *
 * Same observable behaviour as the reference's include/plasma_error.h:21-69:
 * messages go to stderr with the function, line and file, and a fatal error
 * ends the process.
 */
#ifndef PLASMA_ERROR_H
#define PLASMA_ERROR_H

#include <stdio.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

static inline void plasma_report_(const char *kind, const char *func, int line,
                                  const char *file, const char *msg)
{
    fprintf(stderr, "PLASMA %s at %d of %s() in %s: %s\n",
            kind, line, func, file, msg);
}

#define plasma_warning(msg) \
    plasma_report_("WARNING", __func__, __LINE__, __FILE__, msg)

#define plasma_error(msg) \
    plasma_report_("ERROR", __func__, __LINE__, __FILE__, msg)

#define plasma_error_with_code(msg, code) \
    fprintf(stderr, "PLASMA ERROR at %d of %s() in %s: %s %d\n", \
            __LINE__, __func__, __FILE__, msg, (int)(code))

#define plasma_fatal_error(msg) \
    do { plasma_report_("FATAL ERROR", __func__, __LINE__, __FILE__, msg); \
         exit(EXIT_FAILURE); } while (0)

#ifdef __cplusplus
}
#endif

#endif /* PLASMA_ERROR_H */
