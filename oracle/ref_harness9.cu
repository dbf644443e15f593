/*
 * C entry point around the reference's CUDA MEX function mgcg9.
 *
 * TEST INFRASTRUCTURE ONLY.  Linked with the reference's own, unmodified
 * Homogenization/QNC/mgcg9.cu (compiled where it lies in the reference tree
 * by oracle/Makefile, for sm_100a) and with the project's MEX stand-in.  It
 * packs plain C buffers into the 18 positional arguments of the MEX
 * (mgcg9.cu:124-187):
 *   [cgres,cgiters] = mgcg9(Ae,F,U,CX,FDofs,nFD,nelx,nely,nelz,nl,tol,maxit,
 *                           nswp,printLev,nu,hx,hy,hz)
 * and reads the two outputs back.  U is written in place.
 *
 * The reference resets the CUDA device at the start of every call and writes
 * mgcg9.log into the current directory: callers run it in a process of its
 * own (no other CUDA user) from a scratch directory.
 */
#include <cstdio>
#include <set>

#include "mex.h"

extern "C" bool utIsInterruptPending() { return false; }   /* MATLAB's Ctrl-C poll */

/* mgcg9() closes its log FILE* once more after the last logging helper has
 * already closed it (mgcg9.cu:191-192 and :304 against :1074-1130), which the
 * Windows runtime it was written for tolerates and glibc aborts on.  The
 * reference file is compiled with fopen/fclose renamed to these two
 * (oracle/Makefile, target ref9), which pass through to the C library and
 * skip a close of a stream that is not open. */
static std::set<FILE *> g_open_streams;

extern "C" FILE *gputo_ref_fopen(const char *name, const char *mode)
{
    FILE *f = std::fopen(name, mode);
    if (f) g_open_streams.insert(f);
    return f;
}

extern "C" int gputo_ref_fclose(FILE *f)
{
    if (!g_open_streams.erase(f)) return 0;
    return std::fclose(f);
}

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);   /* mgcg9.cu:124 */

extern "C" int ref_cuda_mgcg9(const double *Ke0, const double *F, double *U, const double *CX,
                              const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl, double tol,
                              int maxit, int nswp, int printLev, double nu, double hx, double hy, double hz,
                              double *relres, int *nit)
{
    const long ndof = 3L * (nelx + 1) * (nely + 1) * (nelz + 1);
    const long nel = (long)nelx * nely * nelz;
    double s[13] = {(double)nfd, (double)nelx, (double)nely, (double)nelz, (double)nl, tol, (double)maxit,
                    (double)nswp, (double)printLev, nu, hx, hy, hz};
    mxArray a[18];
    a[0] = gputo_shim_wrap((double *)Ke0, 24, 24);
    a[1] = gputo_shim_wrap((double *)F, (size_t)ndof, 1);
    a[2] = gputo_shim_wrap(U, (size_t)ndof, 1);
    a[3] = gputo_shim_wrap((double *)CX, (size_t)nel, 1);
    a[4] = gputo_shim_wrap((double *)fixed1b, 1, (size_t)nfd);
    for (int i = 0; i < 13; ++i) a[5 + i] = gputo_shim_wrap(&s[i], 1, 1);
    const mxArray *prhs[18];
    for (int i = 0; i < 18; ++i) prhs[i] = &a[i];
    mxArray *plhs[2] = {0, 0};
    mexFunction(2, plhs, 18, prhs);
    *relres = mxGetScalar(plhs[0]);
    *nit = (int)mxGetScalar(plhs[1]);
    mxDestroyArray(plhs[0]);
    mxDestroyArray(plhs[1]);
    return *nit < 0 ? 1 : 0;
}
