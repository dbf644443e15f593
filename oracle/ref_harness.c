/*
 * C entry point around the reference's OpenMP MEX function.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is linked with the reference's own,
 * unmodified Cantilever/omp/mgcg1.c (compiled where it lies in the reference
 * tree by oracle/Makefile) and with the project's MEX stand-in
 * (oracle/shim).  It packs plain C buffers into the 13 positional arguments
 * that top3D125mod.m passes (Cantilever/omp/top3D125mod.m:134):
 *   [cgres,cgiters] = mgcg1(Ke0,F1,U,CX,fixed',WRK,nfd,nelx,nely,nelz,nl,cgtol,cgmax)
 * and reads the two outputs back (mgcg1.c:51-105).  U is written in place.
 *
 * The reference writes mgcg1.log into the current directory and calls
 * omp_set_num_threads(16) (mgcg1.c:109,120-121); callers run it from a
 * scratch directory and cap threads with OMP_THREAD_LIMIT.
 */
#include "mex.h"

int estWorkSpace(int nFD0, int nl, int nelx0, int nely0, int nelz0); /* mgcg1.c:181 */

int ref_omp_workspace(int nfd, int nl, int nelx, int nely, int nelz)
{
    return estWorkSpace(nfd, nl, nelx, nely, nelz);
}

int ref_omp_mgcg1(const double *Ke0, const double *F, double *U, const double *CX,
                  const double *fixed1b, double *W, long lenW, int nfd, int nelx,
                  int nely, int nelz, int nl, double tol, int maxit, double *relres,
                  int *nit)
{
    long ndof = 3L * (nelx + 1) * (nely + 1) * (nelz + 1);
    long nel = (long)nelx * nely * nelz;
    double s_nfd = nfd, s_nelx = nelx, s_nely = nely, s_nelz = nelz, s_nl = nl;
    double s_tol = tol, s_maxit = maxit;
    mxArray a[13];
    a[0] = gputo_shim_wrap((double *)Ke0, 24, 24);
    a[1] = gputo_shim_wrap((double *)F, (size_t)ndof, 1);
    a[2] = gputo_shim_wrap(U, (size_t)ndof, 1);
    a[3] = gputo_shim_wrap((double *)CX, (size_t)nel, 1);
    a[4] = gputo_shim_wrap((double *)fixed1b, 1, (size_t)nfd);
    a[5] = gputo_shim_wrap(W, (size_t)lenW, 1);
    a[6] = gputo_shim_wrap(&s_nfd, 1, 1);
    a[7] = gputo_shim_wrap(&s_nelx, 1, 1);
    a[8] = gputo_shim_wrap(&s_nely, 1, 1);
    a[9] = gputo_shim_wrap(&s_nelz, 1, 1);
    a[10] = gputo_shim_wrap(&s_nl, 1, 1);
    a[11] = gputo_shim_wrap(&s_tol, 1, 1);
    a[12] = gputo_shim_wrap(&s_maxit, 1, 1);
    const mxArray *prhs[13];
    for (int i = 0; i < 13; ++i) prhs[i] = &a[i];
    mxArray *plhs[2] = {0, 0};
    mexFunction(2, plhs, 13, prhs);
    *relres = mxGetScalar(plhs[0]);
    *nit = (int)mxGetScalar(plhs[1]);
    mxDestroyArray(plhs[0]);
    mxDestroyArray(plhs[1]);
    return *nit < 0 ? 1 : 0;
}
