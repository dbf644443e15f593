// The MGCG solver object behind the C ABI.
#pragma once

#include <cstdio>
#include <vector>

#include "gputo_internal.h"

namespace gputo {

struct Solver {
    gputo_options opt{};
    int nl = 0, device = 0, nc = 0;
    Grid g[kMaxLevels]{};
    Lay lay[kMaxLevels]{};     // padded vector layout per level
    ELay elay{};               // padded element layout of the fine level
    cudaStream_t own_stream = nullptr;

    double Ke[576]{};
    HadamardKe hk{};           // Ke in its Hadamard basis (ok = false: dense sweeps only)
    bool have_problem = false, ready = false;
    std::vector<double> fixed_host;
    double *fixed_dev = nullptr;
    long long fixed_cap = 1;

    // fine-level PCG vectors (FP64, padded layout)
    double *R = nullptr, *P = nullptr, *Q = nullptr, *Z = nullptr, *Zold = nullptr;
    float *Zold32 = nullptr;   // mixed precision: z_old as the FP32 V-cycle output it is
    double *Uw = nullptr, *Fw = nullptr;
    // staging in the reference's dense layout (MEX / device API boundary)
    double *Dn = nullptr;
    // element scales: natural order (setup kernels) and padded (fine sweeps)
    double *CX = nullptr, *CXp = nullptr;
    float *CXpf = nullptr;
    uint8_t *mask[kMaxLevels]{};
    uint8_t *maskp[kMaxLevels]{};   // the same, rows padded to 16 bytes (Hadamard-basis sweeps)
    LevelBuf<double> L[kMaxLevels];
    // FP32 preconditioner copies (mixed precision)
    LevelBuf<float> Lf[kMaxLevels];
    // coarsest grid
    double *AQ = nullptr, *Linv = nullptr, *LinvT = nullptr, *ctmp = nullptr, *Apk0 = nullptr;
    int *info = nullptr;
    int *err = nullptr;        // device error flag (bounded waits)
    // device scalars and reduction scratch
    PcgScalars *sc = nullptr, *h_sc = nullptr;
    double *partial = nullptr;
    int partial_cap = 0;
    unsigned *ticket = nullptr;
    double last_res0 = 0.0;
    bool have_solution = false;   // Uw and Fw hold the last solve's U and F
    double *e2 = nullptr;         // (|F - K U|^2, compliance) of energy()
    int launch_status = GPUTO_OK;   // first failure seen while enqueuing kernels

    cudaGraphExec_t graph_exec = nullptr;     // one PCG iteration
    cudaGraphExec_t graph_exec_n = nullptr;   // graph_n iterations back to back (a host-check interval)
    int graph_n = 0;
    void drop_graphs();
    int capture_iterations(int iters, cudaStream_t st, cudaGraphExec_t *exec);
    cudaStream_t graph_stream = nullptr;

    // learned coarse-grid correction (mixed precision, nl >= 3): z += P P net(R R r)
    Net *net = nullptr;
    int net_mode = 0;          // 0 off, 1 always, 2 auto: kept only while it lowers the iteration count
    bool net_on = false;       // part of the captured iteration
    int ref_plain_nit = -1, ref_net_nit = -1, net_solves = 0;
    float *net_x = nullptr, *net_y = nullptr, *dens2 = nullptr, *net_s = nullptr;
    NetDims nd{};
    int attach_net(Net *n, int mode);
    void learned_correction(double *z, const int *done, cudaStream_t st);
    // FP32 operator of level l >= 2 (packed Galerkin): out = A_l u, padded layout
    void apply_level_f32(int l, const float *u, float *out, cudaStream_t st);
    // One training step of n on the energy loss: x [ns][4][n2], gt [ns][3][n2]
    int net_train_energy(Net *n, const float *x, const float *gt, int ns, float lr, double *loss, float *grads_out,
                         cudaStream_t st);

    size_t bytes = 0;
    std::vector<void *> owned;

    ~Solver();
    int create(int nelx, int nely, int nelz, int nl, const gputo_options *o);
    int set_problem(const double *Ke0, const double *fixed1b, int nfd, cudaStream_t st);
    // CX in natural element order (device).
    int setup(const double *CX_dev, cudaStream_t st);
    // setup() in two parts: the hierarchy's kernels enqueued on st, then the
    // wait for them and the coarsest factor's pivot check (host work such as
    // a right-hand side's upload can run in between)
    int setup_enqueue(const double *CX_dev, cudaStream_t st);
    int setup_finish(cudaStream_t st);
    // F, U in the padded layout (solver-owned or compatible buffers).
    int solve(const double *Fp, double *Up, double tol, int maxit, double *relres, int *nit,
              cudaStream_t st, FILE *log);
    // The same solve in phases, for drivers that interleave several solvers:
    // begin (initial residual and V-cycle), then iteration() steps, poll
    // (device scalars to h_sc), end (result, status).
    int solve_begin(const double *Fp, double tol, int maxit, cudaStream_t st);
    int solve_poll(cudaStream_t st, bool *finished);
    int solve_end(double *Up, double *relres, int *nit, cudaStream_t st);
    void iteration(cudaStream_t st);
    // Element energies of the last solve's U, fused into an FP64 apply (see solver.cu).
    int energy(const double *dsK, double *ce, double *dc, double *out2, cudaStream_t st);
    int set_tunables(const gputo_options &o);
    // Padded-layout preconditioner and operator.
    void vcycle(const double *r, double *z, const int *done, cudaStream_t st);
    void apply(const double *u, double *r, double *dot_partial, const int *done, cudaStream_t st);
    cudaStream_t stream(void *s) const { return s ? (cudaStream_t)s : own_stream; }
    // Fine-operator sweep on a grid with K = sum CX_e Ke: the Hadamard-basis
    // kernel when it applies, else the dense element rows.
    template <typename T>
    bool use_hsweep(const Grid &gr) const { return opt.fine_op == 0 && hk.ok && hsweep_fits<T>(gr); }
    template <typename T>
    int fine_sweep(int l, int mode, const Lay &Lo, const ELay &E, const T *CXl, const T *u, const T *f,
                   const LevelBuf<T> &B, T *out, T omega, T pr, double *dot_partial, const int *done,
                   cudaStream_t st, const double *Rd = nullptr, const T *zo = nullptr, const T *uc = nullptr,
                   const Lay *Lc = nullptr) const
    {
        if (use_hsweep<T>(Lo.g) && B.rdiag)
            return launch_hsweep<T>(mode, Lo, E, hk, CXl, u, f, B.rdiag, mask[l], maskp[l], out, omega, pr,
                                    dot_partial, done, err, st, Rd, zo, uc, Lc, l == 0 ? opt.sweep_xchunk : 0,
                                    l == 0 && opt.sweep_pairs != 0);
        return launch_fine_sweep<T>(mode, Lo, E, CXl, u, f, B.diag, mask[l], out, omega, pr, dot_partial, done, err,
                                    st);
    }
    // Per-CTA partials written by the FP64 fine apply.
    int apply_blocks() const
    {
        return use_hsweep<double>(g[0]) && L[0].rdiag ? hsweep_blocks<double>(g[0], MODE_APPLY, opt.sweep_xchunk)
                                                      : fine_sweep_blocks(g[0]);
    }
    // Level 1 is applied matrix-free from the fine CX whenever it is not the
    // coarsest level (then it needs assembled matrices for the direct solve).
    bool quad_level1() const { return nl >= 3 && !redisc(); }
    // mgcg9's hierarchy: every level is K_l = sum_e CX_l Ke, CX_l = 2 mean(children)
    bool redisc() const { return opt.coarse == GPUTO_COARSE_REDISCRETIZED; }
    double *CXr[kMaxLevels]{};     // re-discretised element scales, natural order (l >= 1)
    double *CXrp[kMaxLevels]{};    // ... padded for the tile kernels (1 <= l < nl-1)
    float *CXrpf[kMaxLevels]{};    // ... and their FP32 copies (mixed precision)
    ELay elayr[kMaxLevels]{};
    int check_error_flags(cudaStream_t st);

  private:
    template <typename T>
    int alloc_levels(LevelBuf<T> *Lv, bool with_matrices);
    template <typename T>
    void vcycle_impl(LevelBuf<T> *Lv, const T *CXl, const T *r0, T *z0, const int *done,
                     cudaStream_t st, const double *dotR = nullptr, const T *dotZold = nullptr,
                     double *dotPartial = nullptr);
    // The mixed PCG's r'z and r'z_old come from its last fine smoothing sweep
    // (MODE_JACOBI_DOT) when that sweep is the Hadamard-basis kernel.
    bool fused_dot() const { return use_hsweep<float>(g[0]) && Lf[0].rdiag && opt.tc_parts == 0 && sweeps(0) > 0; }
    // Jacobi sweeps per smoothing step on level l
    int sweeps(int l) const
    {
        if (l == 0 && opt.nswp_fine > 0) return opt.nswp_fine;
        if (l >= (opt.coarse_from > 0 ? opt.coarse_from : 2) && opt.nswp_coarse > 0) return opt.nswp_coarse;
        return opt.nswp;
    }
    int run_graph(int batch, cudaStream_t st);
    void note(int s)
    {
        if (s && !launch_status) launch_status = s;
    }
};

}  // namespace gputo
