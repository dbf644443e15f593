/*
 * CPU restatement of GPU-TO's MGCG solver path and the MATLAB-side design
 * steps around it (density filter, SIMP, compliance sensitivity, Heaviside
 * projection, OC update).
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA product is compared
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it; the product never links or calls it.
 *
 * Conventions (shared with the reference, Cantilever/TOP3D125MGCGCUDA/mgcg1.cu):
 *   node  n = (nelz+1)(nely+1)*i + (nely+1)*k + j     (i=x, j=y, k=z; y fastest)  :966
 *   elem  e = nelz*nely*i + nely*k + j                                             :980
 *   dof   3*n + d, d in {x,y,z}
 *   local element node order (x,y,z offsets) 0:(0,0,0) 1:(1,0,0) 2:(1,1,0)
 *   3:(0,1,0) 4:(0,0,1) 5:(1,0,1) 6:(1,1,1) 7:(0,1,1)   (Cantilever/omp/mgcg1.c:621-624)
 */
#ifndef GPUTO_TOPO_ORACLE_H
#define GPUTO_TOPO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Element stiffness of an axis-aligned hex8 of size hx*hy*hz, E=1, Poisson nu,
 * 2x2x2 Gauss quadrature of B^T D B (mgcg1.c:1370-1418 Kem3/defD). */
void or_hex8_stiffness(double nu, double hx, double hy, double hz, double *Ke /*576*/);

/* The eight single-Gauss-point parts of the same integral, g = 4*ix + 2*iz + iy
 * (ix: x-point, iy: y-point, iz: z-point), i.e. Ke = sum_g Kg[g].  These are
 * the level-1 quadrature matrices of mgcg1.cu:2000-2040 (prepAelm). */
void or_hex8_gauss_parts(double nu, double hx, double hy, double hz, double *Kg /*8*576*/);

/* r = K(CX) u on the fine grid (no boundary handling): mgcg1.cu:941-997 multAV0c. */
void or_apply_fine(const double *Ke, const double *CX, const double *u, double *r,
                   int nelx, int nely, int nelz);

/* Solver options that the MEX hard-codes (mgcg1.cu:188,331,1199-1206). */
typedef struct {
    int nswp;          /* Jacobi sweeps per smoothing step            (3)    */
    double omega;      /* damped Jacobi weight                        (0.48) */
    double prerelax;   /* initial relaxation factor U = c F / diag    (0.7)  */
    double nu;         /* Poisson ratio of the level-1 quadrature     (0.3)  */
    int coarse;        /* 0: mgcg1 hierarchy (level-1 quadrature, Galerkin,
                          element penalty); 1: mgcg9 hierarchy
                          (Homogenization/QNC/mgcg9.cu: every level CX_l Ke with
                          CX_l = 2 mean(children), dense coarsest with zero
                          rows/columns and 1e10 on fixed dofs)        (0)    */
} or_opts;

void or_default_opts(or_opts *o);

/* Drop-in restatement of the MEX mgcg1 (mgcg1.cu:184-291).  U is written in
 * place (y components negated on output, as mgcg1.cu:282-283).  Returns 0,
 * or a nonzero status for bad arguments.  nit follows the reference: the
 * 0-based iteration index at which relres < tol first held, else maxit. */
int or_mgcg1(const double *Ke0, const double *F, double *U, const double *CX,
             const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl,
             double tol, int maxit, const or_opts *opts, double *relres, int *nit,
             double *res_history /* optional, maxit+1 entries, may be NULL */);

/* One application of the V-cycle preconditioner z = M r (mgcg1.cu:468-651),
 * after the hierarchy for CX is built.  For tests of the preconditioner alone. */
int or_vcycle_apply(const double *Ke0, const double *CX, const double *fixed1b, int nfd,
                    int nelx, int nely, int nelz, int nl, const or_opts *opts,
                    const double *r, double *z);

/* ce_e = u_e^T Ke u_e for every element (top3D125modCuda.m:139), u in the
 * solver's frame (the y sign does not change ce). */
void or_element_energy(const double *Ke, const double *U, double *ce, int nelx, int nely,
                       int nelz);

/* MATLAB imfilter(A, h, 'symmetric') with h = max(0, rmin - |d|) on the
 * (2*ceil(rmin)-1)^3 stencil, A laid out (nely, nelz, nelx) column-major (y fastest),
 * i.e. in element order (top3D125modCuda.m:95-96,109,140-141).  out = correlation;
 * the caller divides by Hs.  Returns sum(h) (= Hs everywhere under 'symmetric'). */
double or_filter3d(const double *in, double *out, int nelx, int nely, int nelz, double rmin);

#ifdef __cplusplus
}
#endif
#endif
