/*
 * Implementation of the minimal MEX stand-in declared in mex.h.
 * TEST INFRASTRUCTURE ONLY (see mex.h).
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include "mex.h"

double *mxGetDoubles(const mxArray *a) { return a->owned ? (double *)&a->scalar : a->data; }
double *mxGetPr(const mxArray *a) { return mxGetDoubles(a); }
size_t mxGetM(const mxArray *a) { return a->m; }
size_t mxGetN(const mxArray *a) { return a->n; }
double mxGetScalar(const mxArray *a) { return mxGetDoubles(a)[0]; }

mxArray *mxCreateDoubleScalar(double v)
{
    mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
    a->owned = 1;
    a->scalar = v;
    a->data = NULL;
    a->m = a->n = 1;
    return a;
}

void mxDestroyArray(mxArray *a) { if (a && a->owned) free(a); }

int mexPrintf(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    int r = vfprintf(stderr, fmt, ap);
    va_end(ap);
    return r;
}

mxArray gputo_shim_wrap(double *data, size_t m, size_t n)
{
    mxArray a;
    a.data = data;
    a.m = m;
    a.n = n;
    a.owned = 0;
    a.scalar = 0.0;
    return a;
}
