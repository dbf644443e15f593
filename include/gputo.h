/*
 * gputo: B200 (sm_100a) implementation of GPU-TO's topology-optimization
 * solver path, exposed as a plain C ABI.
 *
 * The drop-in entry point is gputo_mgcg1(), which takes exactly the arguments
 * of the MATLAB MEX function mgcg1 that the top3D125 MGCG drivers call:
 *
 *   [cgres,cgiters] = mgcg1(Ke0,F1,U,CX,fixed',nfd,nelx,nely,nelz,nl,cgtol,cgmax[,printLev])
 *   (Cantilever/TOP3D125MGCGCUDA/top3D125modCuda.m:134; 13-argument form
 *    ArchBridge/1/top3D125modCudaBridge1.m:175; gateway mgcg1.cu:120-182)
 *
 * The MEX gateway in gpu-to_b200/csrc/mex_gateway.cpp calls it; so can ctypes,
 * cgo, JNI or any other FFI.  Everything else here is the device-resident API
 * that the design loop uses to keep its fields in HBM between steps.
 *
 * Grid conventions (identical to the reference):
 *   node n = (nelz+1)(nely+1) i + (nely+1) k + j,  i=x, j=y, k=z, y fastest
 *   element e = nelz nely i + nely k + j;  dof = 3 n + d, d in {x,y,z}
 *
 * All functions return a gputo_status; none of them exits the process or traps
 * the GPU.  Functions whose names end in _dev take device pointers; the rest
 * take host pointers.  Calls are synchronous with respect to the host unless
 * stated otherwise.
 */
#ifndef GPUTO_H
#define GPUTO_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    GPUTO_OK = 0,
    GPUTO_ERR_ARG = 1,          /* bad size, index or option                        */
    GPUTO_ERR_CUDA = 2,         /* a CUDA call failed (message: gputo_last_error)     */
    GPUTO_ERR_OOM = 3,          /* not enough device memory (MEX returns cgiters=-1) */
    GPUTO_ERR_NOT_SPD = 4,      /* coarsest-grid Cholesky met a non-positive pivot   */
    GPUTO_ERR_BREAKDOWN = 5,    /* CG breakdown: p'q <= 0 or a non-finite scalar     */
    GPUTO_ERR_NO_DEVICE = 6,    /* no CUDA device / no sm_100 device                 */
    GPUTO_ERR_TIMEOUT = 7       /* a bounded device wait gave up                     */
} gputo_status;

/* Human-readable name of a status code. */
const char *gputo_status_string(int status);
/* Last error message recorded by this thread (empty string when none). */
const char *gputo_last_error(void);
/* Library version string. */
const char *gputo_version(void);

/* Precision of the preconditioner.  The outer PCG (residual update, dot
 * products, operator apply p -> K p) is always FP64. */
typedef enum {
    GPUTO_PREC_FP64 = 0,   /* everything FP64: the reference's arithmetic        */
    GPUTO_PREC_MIXED = 1   /* V-cycle in FP32 (coarsest Cholesky still FP64),
                              flexible PCG                                       */
} gputo_precision;

/* Coarse operators of the hierarchy. */
typedef enum {
    GPUTO_COARSE_GALERKIN = 0,       /* mgcg1: level 1 by quadrature, Galerkin above   */
    GPUTO_COARSE_REDISCRETIZED = 1   /* mgcg9: every level K_l = sum_e CX_l Ke with
                                        CX_l = 2 mean(children) (no stored matrices)  */
} gputo_coarse;

/* Solver options.  gputo_default_options() gives the constants that the MEX
 * hard-codes (mgcg1.cu:188 nswp=3, :1199-1206 omega=0.48, :1190-1197
 * pre-relaxation 0.7, :331 nu=0.3 for the level-1 quadrature). */
typedef struct {
    int precision;       /* gputo_precision                                      */
    int nswp;            /* Jacobi sweeps per pre/post smoothing step             */
    double omega;        /* damped-Jacobi weight                                  */
    double prerelax;     /* initial smoother guess U = prerelax * F / diag(A)     */
    double nu;           /* Poisson ratio of the level-1 quadrature operator      */
    int check_every;     /* PCG iterations between host convergence checks (>=1) */
    int use_graph;       /* capture the PCG iteration in a CUDA graph (0/1)      */
    int max_coarse_dofs; /* reject hierarchies whose coarsest grid is larger      */
    int tc_parts;        /* GPUTO_PREC_MIXED only: fine-level smoother on the
                            tensor cores, u and Ke each split into this many
                            BF16 parts (1: plain BF16, about 2e-3 relative;
                            2: about 1e-5), FP32 accumulation; 0 = FP32 CUDA
                            cores                                                 */
    int tc_xchunk;       /* node planes per CTA of the tensor-core smoother
                            (0 = 16)                                              */
    int coarse;          /* gputo_coarse                                          */
    int fine_op;         /* fine-level sweeps: 0 = the element matrix in its
                            Hadamard basis when Ke has the structure of an
                            isotropic cube element and nely <= 256 (fewer
                            operations, same results to rounding), else dense
                            element rows; 1 = always dense element rows       */
    int nswp_fine;       /* Jacobi sweeps per smoothing step on the finest level
                            only (0 = nswp, the reference's schedule); the
                            autotuner may pick fewer there, where a sweep costs
                            most                                                  */
    int fuse_prolong;    /* 1: the finest level's first post-smoothing sweep
                            adds the prolonged coarse correction in its own
                            tiles (Hadamard-basis sweep; same results bit for
                            bit); 0 (default): a separate prolongation pass,
                            measured faster                                      */
    int sweep_xchunk;    /* node planes per CTA along x of the Hadamard-basis
                            fine sweeps: 0 = chosen from the device's resident
                            clusters, else 8 .. 32 (the autotuner's tile
                            choice)                                               */
    int sweep_pairs;     /* 1 (default): the FP32 fine sweeps of the mixed
                            V-cycle give each lane two element columns
                            (paired FP32 arithmetic, nely <= 256; same results
                            bit for bit); 0: one column per lane              */
    int nswp_coarse;     /* Jacobi sweeps per smoothing step on levels
                            coarse_from and below (0 = nswp; the levels above
                            keep nswp): an autotuner choice                       */
    int coarse_from;     /* first level of nswp_coarse, >= 2 (0 = 2): the
                            autotuner tries 2, 3 and 4                           */
} gputo_options;

void gputo_default_options(gputo_options *opt);

/* Element stiffness of a unit-modulus hex8 cube of edge h with Poisson ratio
 * nu, 2x2x2 Gauss quadrature, in the reference's element node order; Ke is
 * 576 doubles, row-major and symmetric.  Equals the Ke0 the drivers build
 * (top3D125modCuda.m:50-77) and Kem3 (Cantilever/omp/mgcg1.c:1370).  Host
 * only; needs no GPU. */
int gputo_hex8_stiffness(double nu, double h, double *Ke);

/* The eight constants of Ke in the element's Hadamard basis (S = T Ke T', T
 * the 2x2x2 Hadamard transform over the element's corners): a, b, c, d, e,
 * f, g, h of the 45-entry pattern that the fine sweeps with fine_op = 0 use.
 * Returns GPUTO_OK when Ke has that pattern to 1e-12 relative (every
 * isotropic cube element does), GPUTO_ERR_ARG when it does not; such a Ke
 * runs on the dense element-row sweeps.  Host only; no reference counterpart. */
int gputo_fine_op_constants(const double *Ke, double *c8);

/* ---------------------------------------------------------------------- */
/* Drop-in MEX replacement                                                  */
/* ---------------------------------------------------------------------- */

/*
 * Replaces the MEX mgcg1 (Cantilever/TOP3D125MGCGCUDA/mgcg1.cu:120-291).
 *
 * Ke0     24x24 element stiffness (symmetric; either storage order)
 * F       ndof right-hand side, ndof = 3 (nelx+1)(nely+1)(nelz+1)
 * U       ndof output, written in place; its input values are ignored (the
 *         solve starts from zero, mgcg1.cu:235); y components are negated on
 *         output (mgcg1.cu:282-283), as the MATLAB drivers expect
 * CX      nel element stiffness scale E(x)
 * fixed1b nfd 1-based indices of the fixed dofs (MATLAB's fixed')
 * nl      multigrid levels; nelx, nely, nelz divisible by 2^(nl-1); nelx <= 65534
 * tol     relative residual tolerance on ||r||/||F||
 * maxit   PCG iteration limit
 * printLev  0: silent; >=1: append a summary to ./mgcg1.log as the MEX does
 * relres  output: ||r||/||F|| at exit
 * nit     output: 0-based iteration index at which relres < tol first held,
 *         maxit if it never did, -1 if device memory was insufficient
 *         (mgcg1.cu:166-174)
 * The hierarchy and buffers are cached per device and grid shape, so later
 * calls of the same shape allocate nothing.
 */
int gputo_mgcg1(const double *Ke0, const double *F, double *U, const double *CX,
                const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl,
                double tol, int maxit, int printLev, double *relres, int *nit);

/* gputo_mgcg1 with explicit options (precision, sweeps, ...). */
int gputo_mgcg1_ex(const double *Ke0, const double *F, double *U, const double *CX,
                   const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl,
                   double tol, int maxit, int printLev, const gputo_options *opt,
                   double *relres, int *nit);

/*
 * Replaces the MEX mgcg9 (Homogenization/QNC/mgcg9.cu:124-305), used by the
 * QNC homogenization and CrossWalk drivers: the same PCG with a re-discretised
 * hierarchy (every level K_l = sum_e CX_l Ae with CX_l twice the mean of its
 * eight children, mgcg9.cu:753-781; damped Jacobi with weight 0.33 and
 * pre-relaxation 0.7, nswp sweeps, mgcg9.cu:920-935; dense coarsest solve
 * with zero rows/columns and 1e10 on fixed dofs, mgcg9.cu:1005-1028).  The
 * 18 MEX arguments in order: Ae F U CX FDofs nFD nelx nely nelz nl tol maxit
 * nswp printLev nu hx hy hz; nu and hx/hy/hz are accepted and, as in the
 * reference, not used by the solve.  Outputs and U follow gputo_mgcg1 (y
 * negated, nit the 0-based break index); printLev >= 1 writes mgcg9.log.
 * Coarsest grids of 20,000 dofs or more are rejected (the reference switches
 * to 10 nswp Jacobi sweeps there), and so is nl = 1 (the reference then
 * smooths without a coarse solve).
 */
int gputo_mgcg9(const double *Ae, const double *F, double *U, const double *CX, const double *fixed1b, int nfd,
                int nelx, int nely, int nelz, int nl, double tol, int maxit, int nswp, int printLev, double nu,
                double hx, double hy, double hz, double *relres, int *nit);

/* ---------------------------------------------------------------------- */
/* Device-resident solver (the same solve without host copies)             */
/* ---------------------------------------------------------------------- */

typedef struct gputo_solver gputo_solver;

/* Create a solver for one grid shape on the current CUDA device.  Replaces the
 * allocation half of mgcg1.cu:184-232 and estWorkSpace (mgcg1.cu:293-322),
 * with 64-bit sizes throughout. */
int gputo_solver_create(gputo_solver **out, int nelx, int nely, int nelz, int nl,
                        const gputo_options *opt);
void gputo_solver_destroy(gputo_solver *s);
/* r = K u with the fine-level FP32 operator of the mixed-precision V-cycle
 * (precision GPUTO_PREC_MIXED only): tc_parts = 0 uses the CUDA-core tile
 * kernel, 1 or 2 the tensor-core sweep with u and Ke split into that many
 * BF16 parts.  u
 * and r are ndof doubles on the device (converted to and from FP32). */
int gputo_solver_apply_fp32_dev(gputo_solver *s, const double *u, double *r, int tc_parts, void *stream);
/* Bytes of device memory the solver holds. */
size_t gputo_solver_device_bytes(const gputo_solver *s);

/* Element matrix (host, 24x24) and Dirichlet dofs (host, 1-based doubles, as
 * the MEX receives them).  Must be called before setup. */
int gputo_solver_set_problem(gputo_solver *s, const double *Ke0, const double *fixed1b, int nfd);

/* Build the multigrid hierarchy for the element scales CX (device, nel
 * doubles): diagonal, level-1 quadrature operator, Galerkin levels, coarsest
 * Cholesky (initVcycle, mgcg1.cu:326-466).  Stream-ordered on 'stream'
 * (a cudaStream_t, NULL = the solver's own stream); returns after the
 * coarsest factorisation has been checked. */
int gputo_solver_setup_dev(gputo_solver *s, const double *CX, void *stream);

/* PCG solve K u = f (mgcg1.cu:233-286) on device vectors of ndof doubles.
 * U is in the solver's frame (no y negation).  relres/nit as gputo_mgcg1. */
int gputo_solver_solve_dev(gputo_solver *s, const double *F, double *U, double tol, int maxit,
                           double *relres, int *nit, void *stream);

/* Element energies of the solution of the last gputo_solver_solve_dev call on
 * this solver, from one FP64 operator apply of that U with the energies in
 * its epilogue (the element loop of the driver's sensitivity line,
 * top3D125modCuda.m:139, fused into the operator apply):
 *   ce_e = u_e' Ke u_e,  dc = dsK .* ce  (dsK and dc may be NULL),
 *   *compliance = sum_e CX_e ce_e,
 *   *true_relres = |F - K U| / |F| over the free dofs (the solve itself stops
 *   on the recursively updated residual, mgcg1.cu:254-275).
 * ce, dc, dsK: device arrays of nel in element order; compliance and
 * true_relres: host pointers, either may be NULL.  When the grid runs on the
 * dense-row kernel (nely > 256 or a Ke without the cube element's pattern),
 * ce comes from a separate pass and *true_relres is -1.  GPUTO_ERR_ARG
 * without a successful solve since the last setup (a V-cycle call in between
 * also discards the solve). */
int gputo_solver_energy_dev(gputo_solver *s, const double *dsK, double *ce, double *dc,
                            double *compliance, double *true_relres, void *stream);

/* One V-cycle z = M r on device vectors (the preconditioner alone). */
int gputo_solver_vcycle_dev(gputo_solver *s, const double *r, double *z, void *stream);

/* r = K(CX) u with fixed rows zeroed, on device vectors (multAV0c + ZeroBCc,
 * mgcg1.cu:941-997,1326-1331). */
int gputo_solver_apply_dev(gputo_solver *s, const double *u, double *r, void *stream);

/* Kernel launches this library has issued in this process (for accounting). */
long long gputo_solver_launch_count(const gputo_solver *s);

/* Time 'reps' back-to-back launches of one solver kernel on the current
 * hierarchy with CUDA events on 'stream' and return the mean launch time in
 * milliseconds.  which: 0 fine-level FP64 apply (p -> K p), 1 fine-level FP32
 * Jacobi sweep, 2 level-1 FP32 sweep, 3 level-1 FP64 sweep, 4 fine-level
 * tensor-core Jacobi sweep (tc_parts of the options, 1 if 0), 5 the FP64
 * apply with the element energies (gputo_solver_energy_dev's pass; Hadamard-
 * basis grids only), 6 level-2 FP32 sweep (Galerkin element matrices; nl >=
 * 4).  Inputs are the solver's own work vectors; results are discarded.
 * Needs setup first. */
int gputo_solver_time_kernel(gputo_solver *s, int which, int reps, double *ms_per_launch,
                             void *stream);

/* Test hook of the failure handling; no counterpart in the reference, whose
 * kernels have no bounded waits.  The Hadamard-basis fine sweeps launched
 * after this call leave the tile copies of ring stage 'skip_stage' unissued
 * (its mbarrier armed, nothing in flight), and every wait of their march
 * gives up after 'wait_us' microseconds; the sweep then ends early and the
 * call reports GPUTO_ERR_TIMEOUT, with the context still usable.
 * gputo_debug_set_sweep_fault(-1, 0) restores normal operation (waits give up
 * after 2 s).  Affects launches, not CUDA graphs captured earlier.  Not for
 * production use. */
int gputo_debug_set_sweep_fault(int skip_stage, unsigned wait_us);

/* ---------------------------------------------------------------------- */
/* Periodic homogenization (no reference counterpart)                      */
/* ---------------------------------------------------------------------- */

/* Effective elasticity of a periodic voxel unit cell of nx x ny x nz unit
 * elements (element (i, j, k) at (nz ny) i + ny k + j, as the solver's).  The
 * six unit-strain load cases (Voigt order xx, yy, zz, yz, xz, xy, engineering
 * shear strains) are solved together as six right-hand sides: each operator,
 * smoother and transfer launch serves all six, and one CUDA graph launch runs
 * a PCG iteration of all six.  Method: the MGCG of gputo_mgcg1 on a periodic
 * grid (node 0 held against the rigid translations), coarse levels
 * re-discretised as gputo_mgcg9's (CX_l = 2 mean of the children), FP32
 * V-cycle, flexible FP64 PCG per load case.  nx, ny, nz divisible by
 * 2^(nl-1) with at least 2 coarsest elements per direction; the options'
 * nswp, omega, prerelax, check_every, use_graph and max_coarse_dofs apply. */
typedef struct gputo_homog gputo_homog;
int gputo_homog_create(gputo_homog **out, int nx, int ny, int nz, int nl, const gputo_options *opt);
void gputo_homog_destroy(gputo_homog *h);
size_t gputo_homog_device_bytes(const gputo_homog *h);
/* Ke0: the 24x24 element matrix (host, as for gputo_mgcg1); CX: device array
 * of the element moduli.  Ceff: host 6x6 (row-major, symmetric)
 * C_rs = mean_e CX_e (u0_r + chi_r)_e' Ke0 (u0_s + chi_s)_e, with u0_r the
 * affine field of unit strain r and chi_r its periodic fluctuation; relres[6],
 * nit[6]: per load case (either may be NULL); chi (optional, device,
 * 18 nx ny nz doubles): the fluctuations as [3 node + d][r].  Ke0 goes to
 * constant memory shared by every gputo_homog on the device, so calls with
 * different Ke0 must not overlap on one device.  The call synchronises its
 * stream before it returns. */
int gputo_homog_solve_dev(gputo_homog *h, const double *Ke0, const double *CX, double tol, int maxit,
                          double *Ceff, double *relres, int *nit, double *chi, void *stream);

/* ---------------------------------------------------------------------- */
/* Batched solves and the option autotuner (no reference counterpart)       */
/* ---------------------------------------------------------------------- */

/* Several solvers (any grid sizes, same device) solved together: one PCG
 * iteration of every member is one branch of a single CUDA graph, so each CG
 * step of the batch is one graph launch.  The solvers stay owned by the
 * caller and must outlive the batch. */
typedef struct gputo_batch gputo_batch;
int gputo_batch_create(gputo_batch **out, gputo_solver **solvers, int n);
void gputo_batch_destroy(gputo_batch *b);
/* F[i], U[i]: device vectors (dense layout) of member i; relres[i], nit[i] as
 * gputo_solver_solve_dev returns them.  Results equal the members' own
 * solves; the host checks convergence every check_every CG steps. */
int gputo_batch_solve_dev(gputo_batch *b, const double *const *F, double *const *U, double tol, int maxit,
                          int check_every, double *relres, int *nit);

/* Change the options that need no new hierarchy (nswp, nswp_fine,
 * nswp_coarse, omega, prerelax, check_every, use_graph, tc_parts, tc_xchunk,
 * sweep_xchunk, sweep_pairs) on an existing solver, e.g. to
 * reuse what gputo_autotune_dev chose for another solver of the same shape. */
int gputo_solver_set_options(gputo_solver *s, const gputo_options *opt);

/* Choose the options that change neither the hierarchy nor its buffers
 * (Jacobi sweeps per smoothing step, on all levels, the finest level and
 * levels 2 and below; for GPUTO_PREC_MIXED also the CUDA-core
 * or tensor-core fine smoother and its x-chunk; host check interval) by
 * timing complete solves of this solver's problem (F, U: device vectors as
 * for gputo_solver_solve_dev) with CUDA events.  The fastest candidate that
 * converges is applied to the solver and returned in best (best_ms: its solve
 * time).  table_ms / table_nit (optional, table_cap entries) receive every
 * candidate's time and iteration count (-1: did not converge), ncand the
 * number of candidates. */
int gputo_autotune_dev(gputo_solver *s, const double *F, double *U, double tol, int maxit, gputo_options *best,
                       double *best_ms, double *table_ms, int *table_nit, int table_cap, int *ncand);

/* ---------------------------------------------------------------------- */
/* Learned coarse-grid correction (no reference counterpart)                */
/* ---------------------------------------------------------------------- */

/* A small 3D convolutional network on the level-2 node grid: three 3x3x3
 * convolutions 4 -> 16 -> 32 -> 64 with ReLU and a 1x1x1 convolution 64 -> 3;
 * FP32 master weights used rounded to BF16, FP32 activations.  Tensors are
 * channels-first [C][X][Z][Y] with Y fastest (the solver's node order); the
 * input channels are a density feature and the residual restricted twice in
 * Jacobi-scaled units, the output the level-2 error estimate in those units.
 * Flat parameter layout: per layer w[co][ci][tap] then b[co], tap = 9 (dx+1)
 * + 3 (dz+1) + (dy+1). */
typedef struct gputo_net gputo_net;
long long gputo_net_num_params(void);
int gputo_net_create(gputo_net **out, unsigned long long seed);
void gputo_net_destroy(gputo_net *net);
int gputo_net_get_params(const gputo_net *net, float *host);
/* Replaces the parameters and resets the optimizer state. */
int gputo_net_set_params(gputo_net *net, const float *host);
/* y[3][n] = net(x[4][n]) on device buffers, n = X Z Y. */
int gputo_net_forward_dev(gputo_net *net, const float *x, int X, int Z, int Y, float *y, void *stream);
/* One training step on nsamples samples stored back to back (x: [4][n] each,
 * target t and loss mask m: [3][n] each): the masked mean-square losses and
 * their gradients are summed; if lr > 0 one Adam step with the mean gradient
 * follows.  loss receives the mean loss, grads_out (host, optional) the summed
 * gradient before the step. */
int gputo_net_train_step_dev(gputo_net *net, const float *x, const float *t, const float *m, int nsamples,
                             int X, int Z, int Y, float lr, double *loss, float *grads_out, void *stream);

/* Attach a network to a solver (precision GPUTO_PREC_MIXED, nl >= 3), or
 * detach it (net = NULL).  mode 1 adds z += P P e2 with e2 = net(R R r) after
 * every V-cycle of the flexible PCG; mode 2 (auto) measures solves with and
 * without it and keeps the plain V-cycle whenever the network does not lower
 * the iteration count, re-measuring every 8 solves.  The solution is
 * unchanged: CG still converges to the same tolerance. */
int gputo_solver_set_net(gputo_solver *s, gputo_net *net, int mode);
/* Whether the correction is on for the next solve, and the last measured
 * iteration counts without / with it (-1 if not measured yet). */
int gputo_solver_net_state(const gputo_solver *s, int *on, int *plain_nit, int *net_nit);
/* The network's grid for this solver: level-2 nodes (nelx/4+1, nelz/4+1, nely/4+1). */
int gputo_solver_net_dims(const gputo_solver *s, int *X, int *Z, int *Y);
/* Network input [4][n] for a fine residual r (ndof doubles, device), as the
 * preconditioner builds it: the residual is restricted twice, scaled to
 * D^-1/2 r with the level-2 diagonal D and divided by its RMS s.  m
 * (optional, [3][n]) receives the loss mask (1 on free dofs), dsq (optional,
 * [3][n]) sqrt(D), scale s: a level-2 error e enters the loss as
 * e sqrt(D) / s.  Uses the solver's work buffers: not during a solve. */
int gputo_solver_net_features_dev(gputo_solver *s, const double *r, float *x, float *m, float *dsq,
                                  float *scale, void *stream);
/* Energy-loss data for a post-V-cycle residual w = r - A V(r) (fine dense
 * doubles, device): gt [3][n] = D^-1/2 P'P' w / scale at the level-2 nodes,
 * with scale the value gputo_solver_net_features_dev returned for r. */
int gputo_solver_net_energy_rhs_dev(gputo_solver *s, const double *w, float scale, float *gt, void *stream);
/* One training step on the energy of the error left after the V-cycle and
 * the correction: per sample L = y'A~y - 2 y'g~ (A~ = D^-1/2 A2 D^-1/2 with the
 * solver's Galerkin level-2 operator A2, y the network output for x, g~ = gt),
 * the optimum being the exact two-grid correction and L = 0 the plain V-cycle;
 * summed over nsamples stacked samples (grads_out, host, optional: the summed
 * gradient), then one Adam step (lr > 0).  The solver's hierarchy (setup)
 * must be the one the samples came from. */
int gputo_solver_net_train_step_dev(gputo_solver *s, gputo_net *net, const float *x, const float *gt,
                                    int nsamples, float lr, double *loss, float *grads_out, void *stream);
/* Values of a fine dense vector v at the level-2 nodes, [3][n] floats. */
int gputo_solver_level2_inject_dev(gputo_solver *s, const double *v, float *out, void *stream);

/* ---------------------------------------------------------------------- */
/* Design-loop steps that the MATLAB drivers run around the solve          */
/* ---------------------------------------------------------------------- */

/* Compliance sensitivity (top3D125modCuda.m:139,163) on device data:
 *   ce_e = u_e^T Ke u_e,  dc_e = dsK_e ce_e  (dc may be NULL),
 *   *compliance = sum_e CX_e ce_e (= F'U at equilibrium) when non-NULL.
 * U in the solver's frame. */
int gputo_compliance_sens_dev(const double *Ke0, const double *U, const double *CX,
                              const double *dsK, int nelx, int nely, int nelz, double *ce,
                              double *dc, double *compliance, void *stream);
/* Same with host buffers; U in the MATLAB frame (as gputo_mgcg1 returns it). */
int gputo_compliance_sens(const double *Ke0, const double *U, const double *CX,
                          const double *dsK, int nelx, int nely, int nelz, double *ce,
                          double *dc, double *compliance);

/* gputo_compliance_sens_dev with the element contraction U Ke on the tensor
 * cores: the [n_elem x 24] x [24 x 24] product runs as tcgen05 BF16 MMAs with
 * FP32 accumulation (U and Ke each split into three BF16 parts), then
 * ce = u . (Ke u) in FP64.  About 1e-7 relative accuracy. */
int gputo_compliance_sens_tc_dev(const double *Ke0, const double *U, const double *CX,
                                 const double *dsK, int nelx, int nely, int nelz, double *ce,
                                 double *dc, double *compliance, void *stream);

/* gputo_compliance_sens_dev for callers that cannot allocate device memory.
 * No counterpart in the reference: its sensitivity step is MATLAB code.
 *
 * gputo_compliance_sens_dev creates reduction scratch and a stream the first
 * time it runs.  Hosts whose memory manager owns the whole device (a MATLAB
 * gpuArray workspace, a caching allocator that has reserved the free memory)
 * and real-time loops that must not hit the implicit device synchronisation
 * of cudaMalloc / cudaFree cannot allow that.  This variant takes the same
 * arguments and gives the same results, but keeps its scratch in a fixed
 * device array compiled into the library (about 64 KB, held by every GPU that
 * loads the library until the process exits) and calls no allocator.
 *  - Grids above 16,777,216 elements are rejected with GPUTO_ERR_ARG.
 *  - The first call on a device (and the first after a cudaDeviceReset)
 *    looks up the array's device address; make that first call before any
 *    stream capture.
 *  - Every call shares the array: calls that overlap on the GPU (different
 *    streams, or different host threads on one device) race and must be
 *    serialised by the caller.
 *  - A call whose Ke0 differs from the last one the device saw rewrites the
 *    library's constant-memory copy of Ke, which every gputo kernel on that
 *    device reads: serialise such a call against all other gputo work on the
 *    device (solves, sensitivities) as well.
 * 'stream' may be NULL (the legacy default stream); the call returns after
 * the stream has finished the work, and 'compliance' is a host pointer. */
int gputo_compliance_sens_noalloc_dev(const double *Ke0, const double *U, const double *CX,
                                      const double *dsK, int nelx, int nely, int nelz, double *ce,
                                      double *dc, double *compliance, void *stream);

/* Density filter, the three imfilter calls of the driver
 * (top3D125modCuda.m:95-96,109,140-141):
 *   out = imfilter(reshape(in ./ divisor, nely,nelz,nelx), h, 'symmetric')   [./ Hs]
 * with h = max(0, rmin - |d|) on the (2 ceil(rmin)-1)^3 stencil.  divisor may
 * be NULL (no division).  normalize != 0 divides the result by Hs, which under
 * 'symmetric' padding is sum(h) everywhere (the xTilde form, :109);
 * normalize == 0 with divisor = dHs is the dc / dV0 form (:140-141). */
int gputo_density_filter_dev(const double *in, const double *divisor, double *out, int nelx,
                             int nely, int nelz, double rmin, int normalize, void *stream);
int gputo_density_filter(const double *in, const double *divisor, double *out, int nelx,
                         int nely, int nelz, double rmin, int normalize);
/* Profiling aid (no counterpart in the reference): the mean time of one
 * normalised density-filter launch (no divisor), 'reps' launches back to back
 * on 'stream' cycling through the n input/output pairs (device arrays of nel
 * doubles), CUDA events on that stream, after one warm-up launch per pair.
 * Unlike gputo_density_filter_dev, no synchronisation between launches. */
int gputo_time_filter_dev(const double *const *in, double *const *out, int n, int nelx, int nely, int nelz,
                          double rmin, int reps, double *ms_per_launch, void *stream);

/* SIMP interpolation (top3D125modCuda.m:124,130) on device arrays of n:
 *   CX = Emin + xPhys^penal (E0 - Emin),  dsK = -penal (E0 - Emin) xPhys^(penal-1)
 * dsK may be NULL. */
int gputo_simp_dev(const double *xPhys, long long n, double penal, double E0, double Emin,
                   double *CX, double *dsK, void *stream);
/* The same on host arrays (the MATLAB lines themselves): xPhys in, CX and
 * dsK out (dsK may be NULL). */
int gputo_simp(const double *xPhys, long long n, double penal, double E0, double Emin, double *CX, double *dsK);

/* Optimality-criteria update with bisection on the Lagrange multiplier
 * (top3D125modCuda.m:143-151), all elements active:
 *   ocP = x .* sqrt(-dc ./ dV0);  l = [0, mean(ocP)/volfrac]
 *   while (l2-l1)/(l2+l1) > 1e-4: lmid = (l1+l2)/2;
 *       xnew = max(max(min(min(ocP/lmid, x+move), 1), x-move), 0)
 *       if mean(xnew) > volfrac: l1 = lmid else l2 = lmid
 * xnew must not alias x.  *lmid receives the last multiplier evaluated. */
int gputo_oc_update_dev(const double *x, const double *dc, const double *dV0, long long n,
                        double volfrac, double move, double *xnew, double *lmid, void *stream);
int gputo_oc_update(const double *x, const double *dc, const double *dV0, long long n,
                    double volfrac, double move, double *xnew, double *lmid);

/* Heaviside projection with the volume-preserving threshold (ft = 3,
 * top3D125modCuda.m:60-64,111-119) on device arrays of n elements:
 *   while |mean(prj(xTilde, eta, beta)) - volfrac| > 1e-6:
 *       eta = eta - f / mean(deta(xTilde, eta, beta))
 *   xPhys = prj(xTilde, eta, beta);  dprj (optional) = dprj(xTilde, eta, beta)
 * with prj(v) = (tanh(beta eta) + tanh(beta (v - eta))) / (tanh(beta eta) +
 * tanh(beta (1 - eta))).  eta: the starting threshold in (the previous design
 * iteration's), the final one out.  The sensitivity chain rule of the driver,
 * dc ./ dHs with dHs = Hs ./ dprj, is the filtered dc .* dprj (gputo_mul_dev). */
int gputo_heaviside_dev(const double *xTilde, long long n, double volfrac, double beta, double *eta,
                        double *xPhys, double *dprj, void *stream);
/* out = a .* b on device arrays of n (out may alias a or b). */
int gputo_mul_dev(const double *a, const double *b, double *out, long long n, void *stream);

/* ---------------------------------------------------------------------- */
/* Design-state files (host buffers; no GPU needed)                         */
/* ---------------------------------------------------------------------- */

/* Save / resume a design: the reference's drivers warm-start from a MATLAB
 * file (CrossWalk/crosswalk.m:135, load x46.mat).  Binary file: 64-byte header
 * (magic "GPUTODS1", version 1, nelx, nely, nelz, iteration, nparams), then
 * params[nparams], x[nel], xPhys[nel] as little-endian doubles in element
 * order.  params holds whatever loop state the caller keeps (e.g. volfrac,
 * penal, rmin, eta, beta). */
int gputo_design_save(const char *path, int nelx, int nely, int nelz, int iteration, const double *params,
                      int nparams, const double *x, const double *xPhys);
/* Reads the header; with x, xPhys and params all NULL it only reports the
 * sizes.  *nparams: in, the capacity of params; out, the saved count.
 * Truncated or foreign files give GPUTO_ERR_ARG with a message. */
int gputo_design_load(const char *path, int *nelx, int *nely, int *nelz, int *iteration, double *params,
                      int *nparams, double *x, double *xPhys);
/* xPhys as a volume for external viewers (replaces the drivers' isosurface
 * plot): <base>.raw (float32, y fastest, then z, then x) and <base>.nhdr. */
int gputo_design_export_volume(const char *base, int nelx, int nely, int nelz, const double *xPhys);

#ifdef __cplusplus
}
#endif
#endif
