/*
 * Helper macros the reference sources expect from H2Pack's utils.h (absent from the
 * reference checkout). Test infrastructure only; see H2Pack.h in this folder.
 */
#ifndef ORACLE_REF_SHIM_UTILS_H
#define ORACLE_REF_SHIM_UTILS_H

#include <math.h>
#include <stdio.h>

#define DABS(x)   fabs(x)
#define DCEIL(x)  ceil(x)
#define DLOG2(x)  log2(x)
#define DPOW(x, y) pow((x), (y))
#ifndef MAX
#define MAX(a, b) ((a) > (b) ? (a) : (b))
#endif
#ifndef MIN
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#endif

double get_wtime_sec(void);

#endif
