/*
 * Declarations of the part of MATLAB's MEX API that the gputo gateways call
 * (gpu-to_b200/csrc/mex_gateway.cpp, mex_gateway9.cpp), for building them
 * where MATLAB's own extern/include is absent.
 *
 * Only declarations: mxArray stays an opaque type and the mx / mex symbols
 * stay undefined in the built gateway.  Inside MATLAB they resolve from
 * MATLAB's libmx / libmex when the MEX file is loaded; a harness that runs the
 * gateway without MATLAB links its own implementation of these six calls.
 * With MATLAB_ROOT set, build.py compiles against MATLAB's mex.h instead.
 */
#ifndef GPUTO_MEX_API_H
#define GPUTO_MEX_API_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxArray_tag mxArray;

double *mxGetDoubles(const mxArray *a);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
double mxGetScalar(const mxArray *a);
mxArray *mxCreateDoubleScalar(double v);
int mexPrintf(const char *fmt, ...);

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

#ifdef __cplusplus
}
#endif

#endif
