/*
 * Definitions that sailfish prepends to every kernel source before it
 * compiles it (sailfish/kernel/library.py:26-87): PRIVATE / PUBLIC linkage and
 * the FOR_EACH_2D loop, for the serial (EXEC_MODE 0) and OpenMP (EXEC_MODE 1)
 * CPU builds. Used only to build the reference kernels into oracle/_ref, a
 * test-only checker.
 */
#include <math.h>
#include <stddef.h>
#define PRIVATE static
#define PUBLIC
#if EXEC_MODE == 1
#define FOR_EACH_2D(NI, NJ) _Pragma("omp parallel for") for (int i = 0; i < NI; ++i) for (int j = 0; j < NJ; ++j)
#else
#define FOR_EACH_2D(NI, NJ) for (int i = 0; i < NI; ++i) for (int j = 0; j < NJ; ++j)
#endif
