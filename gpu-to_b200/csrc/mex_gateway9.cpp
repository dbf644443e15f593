// MATLAB MEX gateway: the drop-in replacement for mgcg9.mexw64
// (Homogenization/QNC/mgcg9.cu:124-187), used by the QNC homogenization and
// CrossWalk drivers.
//
//   [cgres,cgiters] = mgcg9(Ae,F,U,CX,FDofs,nFD,nelx,nely,nelz,nl,tol,maxit,
//                           nswp,printLev,nu,hx,hy,hz)
//
// Same 18 positional arguments as the reference.  U (prhs[2]) is written in
// place.  Where the reference exit()s on a CUDA error, this gateway prints the
// reason and returns cgiters = -1, as the mgcg1 gateway does.
#include "mex.h"
#include "gputo.h"

extern "C" void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs;
    if (nrhs < 18) {
        mexPrintf("mgcg9: expected 18 arguments, got %d\n", nrhs);
        plhs[0] = mxCreateDoubleScalar(0.0);
        plhs[1] = mxCreateDoubleScalar(-1.0);
        return;
    }
    const double *Ae = mxGetDoubles(prhs[0]);
    const double *F = mxGetDoubles(prhs[1]);
    double *U = mxGetDoubles(prhs[2]);
    const double *CX = mxGetDoubles(prhs[3]);
    const double *fixed = mxGetDoubles(prhs[4]);
    const int nfd = (int)mxGetScalar(prhs[5]);
    const int nelx = (int)mxGetScalar(prhs[6]);
    const int nely = (int)mxGetScalar(prhs[7]);
    const int nelz = (int)mxGetScalar(prhs[8]);
    const int nl = (int)mxGetScalar(prhs[9]);
    const double tol = mxGetScalar(prhs[10]);
    const int maxit = (int)mxGetScalar(prhs[11]);
    const int nswp = (int)mxGetScalar(prhs[12]);
    const int printLev = (int)mxGetScalar(prhs[13]);
    const double nu = mxGetScalar(prhs[14]);
    const double hx = mxGetScalar(prhs[15]), hy = mxGetScalar(prhs[16]), hz = mxGetScalar(prhs[17]);

    const size_t ndof = 3 * (size_t)(nelx + 1) * (nely + 1) * (nelz + 1);
    const size_t nel = (size_t)nelx * nely * nelz;
    const bool shapes_ok = mxGetM(prhs[0]) * mxGetN(prhs[0]) == 576 &&
                           mxGetM(prhs[1]) * mxGetN(prhs[1]) == ndof &&
                           mxGetM(prhs[2]) * mxGetN(prhs[2]) == ndof &&
                           mxGetM(prhs[3]) * mxGetN(prhs[3]) == nel &&
                           mxGetM(prhs[4]) * mxGetN(prhs[4]) >= (size_t)(nfd > 0 ? nfd : 0);
    double relres = 0.0;
    int nit = -1;
    int st = GPUTO_ERR_ARG;
    if (shapes_ok)
        st = gputo_mgcg9(Ae, F, U, CX, fixed, nfd, nelx, nely, nelz, nl, tol, maxit, nswp, printLev, nu, hx, hy,
                         hz, &relres, &nit);
    else
        mexPrintf("mgcg9: argument sizes do not match nelx/nely/nelz/nFD\n");
    if (st != GPUTO_OK) {
        if (st == GPUTO_ERR_OOM)
            mexPrintf("\nMGCG - Cuda device has not enough free memory: %s\n", gputo_last_error());
        else if (shapes_ok)
            mexPrintf("mgcg9: %s: %s\n", gputo_status_string(st), gputo_last_error());
        // every failure gives cgiters = -1, which the drivers test to stop
        // their loop (top3D125modCuda.m:135); after a CG breakdown relres
        // keeps the last residual and U the last iterate
        if (st != GPUTO_ERR_BREAKDOWN) relres = 0.0;
        nit = -1;
    }
    plhs[0] = mxCreateDoubleScalar(relres);
    plhs[1] = mxCreateDoubleScalar((double)nit);
}
