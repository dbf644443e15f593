// MATLAB MEX gateway: the drop-in replacement for mgcg1.mexw64 / mgcg1.cu's
// mexFunction (Cantilever/TOP3D125MGCGCUDA/mgcg1.cu:120-182).
//
//   [cgres,cgiters] = mgcg1(Ke0,F1,U,CX,fixed',nfd,nelx,nely,nelz,nl,cgtol,cgmax[,printLev])
//
// Same positional layout as the reference.  The reference reads prhs[12]
// unconditionally (an out-of-bounds read for the 12-argument cantilever call,
// mgcg1.cu:165); here printLev defaults to 1 when it is absent.  U (prhs[2])
// is written in place, exactly as the reference does through
// mxGetDoubles(prhs[2]).  Where the reference exit()s on a CUDA error, this
// gateway prints the reason and returns cgiters = -1, the value the drivers
// already test for (top3D125modCuda.m:135).
#include "mex.h"
#include "gputo.h"

extern "C" void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs;
    if (nrhs < 12) {
        mexPrintf("mgcg1: expected 12 or 13 arguments, got %d\n", nrhs);
        plhs[0] = mxCreateDoubleScalar(0.0);
        plhs[1] = mxCreateDoubleScalar(-1.0);
        return;
    }
    const double *Ke0 = mxGetDoubles(prhs[0]);
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
    const int printLev = nrhs > 12 ? (int)mxGetScalar(prhs[12]) : 1;

    // argument shapes, checked before anything touches the buffers
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
        st = gputo_mgcg1(Ke0, F, U, CX, fixed, nfd, nelx, nely, nelz, nl, tol, maxit, printLev,
                         &relres, &nit);
    else
        mexPrintf("mgcg1: argument sizes do not match nelx/nely/nelz/nfd\n");
    if (st != GPUTO_OK) {
        if (st == GPUTO_ERR_OOM)
            mexPrintf("\nMGCG - Cuda device has not enough free memory: %s\n", gputo_last_error());
        else if (shapes_ok)
            mexPrintf("mgcg1: %s: %s\n", gputo_status_string(st), gputo_last_error());
        // every failure gives cgiters = -1, which the drivers test to stop
        // their loop (top3D125modCuda.m:135); after a CG breakdown relres
        // keeps the last residual and U the last iterate
        if (st != GPUTO_ERR_BREAKDOWN) relres = 0.0;
        nit = -1;
    }
    plhs[0] = mxCreateDoubleScalar(relres);
    plhs[1] = mxCreateDoubleScalar((double)nit);
}
