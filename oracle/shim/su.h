/*
 * su.h -- compatibility shim (TEST INFRASTRUCTURE ONLY).
 *
 * The FWI-EDU C sources include <su.h>, <par.h> and <segy.h> from CWP/Seismic Unix,
 * which is not installed in this image.  This header re-declares, from the public
 * CWP/SU API, exactly the names those sources use (allocators, err/warn, getpar,
 * a few macros) so that the UNMODIFIED reference sources compile in place into the
 * oracle under oracle/_ref/.  Nothing here is linked into the product library.
 */
#ifndef FWI_SHIM_SU_H
#define FWI_SHIM_SU_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <limits.h>

#ifndef PI
#define PI (3.141592653589793)
#endif
#ifndef FSIZE
#define FSIZE ((int)sizeof(float))
#endif
#ifndef DSIZE
#define DSIZE ((int)sizeof(double))
#endif
#ifndef ISIZE
#define ISIZE ((int)sizeof(int))
#endif
#ifndef SQR
#define SQR(x) ((x) * (x))
#endif
#ifndef MAX
#define MAX(x, y) ((x) > (y) ? (x) : (y))
#endif
#ifndef MIN
#define MIN(x, y) ((x) < (y) ? (x) : (y))
#endif
#ifndef ABS
#define ABS(x) ((x) < 0 ? -(x) : (x))
#endif
#ifndef SGN
#define SGN(x) ((x) < 0 ? -1.0 : 1.0)
#endif
#ifndef NINT
#define NINT(x) ((int)((x) > 0.0 ? (x) + 0.5 : (x) - 0.5))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* contiguous allocators: alloc2float(n1,n2) returns n2 row pointers into one n1*n2 block */
void *alloc1(size_t n1, size_t size);
void **alloc2(size_t n1, size_t n2, size_t size);
void ***alloc3(size_t n1, size_t n2, size_t n3, size_t size);
void free1(void *p);
void free2(void **p);
void free3(void ***p);
float *alloc1float(size_t n1);
float **alloc2float(size_t n1, size_t n2);
float ***alloc3float(size_t n1, size_t n2, size_t n3);
double *alloc1double(size_t n1);
double **alloc2double(size_t n1, size_t n2);
int *alloc1int(size_t n1);
int *ealloc1int(size_t n1);
float *ealloc1float(size_t n1);
void free1float(float *p);
void free2float(float **p);
void free3float(float ***p);
void free1double(double *p);
void free2double(double **p);
void free1int(int *p);

void err(const char *fmt, ...);
void warn(const char *fmt, ...);

FILE *efopen(const char *file, const char *mode);
int efclose(FILE *stream);

float sasum(int n, float *sx, int incx);
int CWP_Exit(void);

/* set by the test harness to turn err() into a longjmp instead of exit() */
void fwi_shim_set_err_hook(void (*hook)(const char *msg));

#ifdef __cplusplus
}
#endif

#include "par.h"

#endif
