/*
 * par.h -- compatibility shim (TEST INFRASTRUCTURE ONLY): the CWP "getpar"
 * key=value argument parser names used by the FWI-EDU front-ends.
 */
#ifndef FWI_SHIM_PAR_H
#define FWI_SHIM_PAR_H

#ifdef __cplusplus
extern "C" {
#endif

extern int xargc;
extern char **xargv;

void initargs(int argc, char **argv);
void requestdoc(int flag);
int getparint(const char *name, int *p);
int getparfloat(const char *name, float *p);
int getpardouble(const char *name, double *p);
int getparstring(const char *name, char **p);
int countparval(const char *name);

#ifdef __cplusplus
}
#endif

#endif
