/*
 * Minimal stand-in for MATLAB's MEX API, written for this project.
 *
 * TEST INFRASTRUCTURE ONLY.  It lets the reference's own MEX sources
 * (Cantilever/omp/mgcg1.c, Cantilever/TOP3D125MGCGCUDA/mgcg1.cu) and this
 * project's MEX gateway compile and run without MATLAB.  Only the calls those
 * sources make are provided: mxGetDoubles, mxGetM, mxGetN, mxGetScalar,
 * mxCreateDoubleScalar and mexPrintf.
 *
 * An mxArray here is a dense column-major double matrix that does not own
 * its storage (the harness passes caller-owned buffers, exactly as MATLAB
 * passes its arrays to a MEX function by reference).
 */
#ifndef GPUTO_SHIM_MEX_H
#define GPUTO_SHIM_MEX_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag {
    double *data;    /* column-major payload, m*n doubles            */
    size_t m, n;     /* rows, columns                               */
    int owned;       /* 1 when created by mxCreateDoubleScalar      */
    double scalar;   /* storage for scalars created by the shim     */
} mxArray;

double *mxGetDoubles(const mxArray *a);
double *mxGetPr(const mxArray *a);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
double mxGetScalar(const mxArray *a);
mxArray *mxCreateDoubleScalar(double v);
void mxDestroyArray(mxArray *a);
int mexPrintf(const char *fmt, ...);

/* Helper for harnesses: wrap a caller-owned buffer without copying. */
mxArray gputo_shim_wrap(double *data, size_t m, size_t n);

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

#ifdef __cplusplus
}
#endif

#endif
