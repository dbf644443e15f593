// Batched solves and the option autotuner (host side; no reference
// counterpart: the reference solves one design per MEX call).
//
// Batch: several solvers, of any grid sizes, advance together.  One PCG
// iteration of every member is captured as a parallel branch of a single CUDA
// graph (each member on its own forked stream), so each CG step of the whole
// batch is one graph launch.  Members that have converged keep launching
// kernels that return at once (their device 'done' flag), so the graph stays
// fixed until the slowest member finishes; the host polls all members every
// check_every steps.
//
// Autotuner: the options that change neither the hierarchy nor its buffers
// (smoother back end and its x-chunk, Jacobi sweeps per smoothing step, host
// check interval) are chosen by timing complete solves of the caller's own
// problem with CUDA events and keeping the fastest that converges.
#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "gputo.h"
#include "gputo_internal.h"
#include "solver.h"

struct gputo_solver {
    gputo::Solver s;
};

struct gputo_batch {
    std::vector<gputo_solver *> members;
    cudaStream_t main = nullptr;
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> join;
    cudaEvent_t fork = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~gputo_batch()
    {
        if (main) cudaStreamSynchronize(main);
        if (exec) cudaGraphExecDestroy(exec);
        for (cudaEvent_t e : join) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        for (cudaStream_t s : side) cudaStreamDestroy(s);
        if (main) cudaStreamDestroy(main);
    }
};

using gputo::Solver;

extern "C" {

int gputo_batch_create(gputo_batch **out, gputo_solver **solvers, int n)
{
    if (!out || !solvers || n < 1) return GPUTO_ERR_ARG;
    *out = nullptr;
    int dev = 0;
    GPUTO_CUDA(cudaGetDevice(&dev));
    for (int i = 0; i < n; ++i) {
        if (!solvers[i] || solvers[i]->s.device != dev) {
            gputo::set_error("batch members must be solvers on the current device");
            return GPUTO_ERR_ARG;
        }
        for (int j = 0; j < i; ++j)
            if (solvers[j] == solvers[i]) {
                gputo::set_error("a solver appears twice in the batch");
                return GPUTO_ERR_ARG;
            }
    }
    auto *b = new (std::nothrow) gputo_batch();
    if (!b) return GPUTO_ERR_OOM;
    b->members.assign(solvers, solvers + n);
    auto fail = [&](cudaError_t e) {
        gputo::set_error(std::string("batch: ") + cudaGetErrorString(e));
        delete b;
        return GPUTO_ERR_CUDA;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(e);
    e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(e);
    b->side.resize(n, nullptr);
    b->join.resize(n, nullptr);
    for (int i = 0; i < n; ++i) {
        if ((e = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
        if ((e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    }
    *out = b;
    return GPUTO_OK;
}

void gputo_batch_destroy(gputo_batch *b) { delete b; }

int gputo_batch_solve_dev(gputo_batch *b, const double *const *F, double *const *U, double tol, int maxit,
                          int check_every, double *relres, int *nit)
{
    if (!b || !F || !U || !relres || !nit || check_every < 1 || maxit < 0) return GPUTO_ERR_ARG;
    const int n = (int)b->members.size();
    for (int i = 0; i < n; ++i)
        if (!F[i] || !U[i]) return GPUTO_ERR_ARG;
    // initial residuals and V-cycles, each member on its own stream
    GPUTO_CUDA(cudaEventRecord(b->fork, b->main));
    for (int i = 0; i < n; ++i) {
        Solver &s = b->members[i]->s;
        GPUTO_CUDA(cudaStreamWaitEvent(b->side[i], b->fork, 0));
        // the solver works in its row-padded layout (as gputo_solver_solve_dev)
        s.have_solution = false;
        gputo::launch_pack(s.lay[0], F[i], s.Fw, 0, b->side[i]);
        int st = s.solve_begin(s.Fw, tol, maxit, b->side[i]);
        if (st) return st;
        GPUTO_CUDA(cudaEventRecord(b->join[i], b->side[i]));
        GPUTO_CUDA(cudaStreamWaitEvent(b->main, b->join[i], 0));
    }
    // one iteration of every member as parallel branches of one graph; captured
    // per call because members may have changed options or attachments since
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    cudaGraph_t gr;
    GPUTO_CUDA(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal));
    GPUTO_CUDA(cudaEventRecord(b->fork, b->main));
    int cap_status = GPUTO_OK;
    for (int i = 0; i < n; ++i) {
        Solver &s = b->members[i]->s;
        cudaStreamWaitEvent(b->side[i], b->fork, 0);
        s.launch_status = GPUTO_OK;
        s.iteration(b->side[i]);
        if (s.launch_status && !cap_status) cap_status = s.launch_status;
        cudaEventRecord(b->join[i], b->side[i]);
        cudaStreamWaitEvent(b->main, b->join[i], 0);
    }
    cudaError_t ce = cudaStreamEndCapture(b->main, &gr);
    if (ce != cudaSuccess || cap_status) {
        if (ce == cudaSuccess) cudaGraphDestroy(gr);
        if (cap_status) return cap_status;
        GPUTO_CUDA(ce);
    }
    ce = cudaGraphInstantiate(&b->exec, gr, 0);
    cudaGraphDestroy(gr);
    GPUTO_CUDA(ce);

    int it = 0;
    for (;;) {
        bool all = true;
        for (int i = 0; i < n; ++i) {
            bool fin = false;
            int st = b->members[i]->s.solve_poll(b->main, &fin);
            if (st) return st;
            all = all && fin;
        }
        if (all || it >= maxit) break;
        const int steps = std::min(check_every, maxit - it);
        for (int k = 0; k < steps; ++k) GPUTO_CUDA(cudaGraphLaunch(b->exec, b->main));
        it += steps;
    }
    int first = GPUTO_OK;
    for (int i = 0; i < n; ++i) {
        Solver &s = b->members[i]->s;
        int st = s.solve_end(s.Uw, &relres[i], &nit[i], b->main);
        if (st && !first) first = st;
        if (!st || st == GPUTO_ERR_BREAKDOWN) gputo::launch_unpack(s.lay[0], s.Uw, U[i], 0, b->main);
    }
    GPUTO_CUDA(cudaStreamSynchronize(b->main));
    return first;
}

int gputo_solver_set_options(gputo_solver *h, const gputo_options *o)
{
    if (!h || !o) return GPUTO_ERR_ARG;
    return h->s.set_tunables(*o);
}

int gputo_autotune_dev(gputo_solver *h, const double *F, double *U, double tol, int maxit, gputo_options *best,
                       double *best_ms, double *table_ms, int *table_nit, int table_cap, int *ncand)
{
    if (!h || !F || !U || !best) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready) {
        gputo::set_error("autotune needs a solver after setup");
        return GPUTO_ERR_ARG;
    }
    const gputo_options base = s.opt;
    std::vector<gputo_options> cand;
    for (int nswp : {1, 2, 3, 4}) {
        gputo_options o = base;
        o.nswp = nswp;
        o.nswp_fine = 0;
        o.nswp_coarse = 0;
        o.coarse_from = 0;
        o.use_graph = 1;
        o.check_every = 8;
        o.tc_parts = 0;
        o.sweep_xchunk = 0;
        cand.push_back(o);
        for (int nf = 1; nf < nswp; ++nf) {   // fewer sweeps on the finest level, where they cost most
            o.nswp_fine = nf;
            cand.push_back(o);
        }
        if (nswp <= 3)   // the coarser levels apart, where a sweep costs least
            for (int from : {2, 3, 4})
                for (int nf : {1, 2})
                    for (int nc : {2, 3, 4, 6, 8, 12}) {
                        if (nc == nswp || nf > nswp || from > s.nl - 2) continue;
                        o.nswp_fine = nf;
                        o.nswp_coarse = nc;
                        o.coarse_from = from;
                        cand.push_back(o);
                    }
        o.nswp_coarse = 0;
        o.coarse_from = 0;
        if (nswp == 3)   // the fine sweeps' tile: node planes per CTA along x
            for (int nf : {0, 1})
                for (int xc : {16, 24}) {
                    o.nswp_fine = nf;
                    o.sweep_xchunk = xc;
                    cand.push_back(o);
                }
        o.nswp_fine = 0;
        o.sweep_xchunk = 0;
        if (s.opt.precision == GPUTO_PREC_MIXED)
            for (int xc : {8, 16}) {
                o.tc_parts = 2;
                o.tc_xchunk = xc;
                cand.push_back(o);
            }
    }
    cudaStream_t st = s.own_stream;
    s.have_solution = false;
    gputo::launch_pack(s.lay[0], F, s.Fw, 0, st);   // the solver's row-padded layout
    cudaEvent_t e0, e1;
    GPUTO_CUDA(cudaEventCreate(&e0));
    GPUTO_CUDA(cudaEventCreate(&e1));
    double bms = 1e300;
    int bi = -1;
    for (size_t c = 0; c < cand.size(); ++c) {
        int r = s.set_tunables(cand[c]);
        double rr = 0.0;
        int it = 0;
        float ms = 0.f;
        if (!r) r = s.solve(s.Fw, s.Uw, tol, maxit, &rr, &it, st, nullptr);   // warm-up (graph capture)
        if (!r) {
            cudaEventRecord(e0, st);
            r = s.solve(s.Fw, s.Uw, tol, maxit, &rr, &it, st, nullptr);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
        }
        const bool ok = !r && it < maxit && rr <= tol;
        if ((int)c < table_cap) {
            if (table_ms) table_ms[c] = ok ? (double)ms : -1.0;
            if (table_nit) table_nit[c] = ok ? it : -1;
        }
        if (ok && ms < bms) {
            bms = ms;
            bi = (int)c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ncand) *ncand = (int)cand.size();
    if (bi < 0) {
        s.set_tunables(base);
        gputo::set_error("autotune: no candidate converged");
        return GPUTO_ERR_BREAKDOWN;
    }
    *best = cand[bi];
    if (best_ms) *best_ms = bms;
    int r = s.set_tunables(cand[bi]);
    double rr = 0.0;
    int it = 0;
    if (!r) r = s.solve(s.Fw, s.Uw, tol, maxit, &rr, &it, st, nullptr);   // U: the solution with the choice
    if (!r) {
        gputo::launch_unpack(s.lay[0], s.Uw, U, 0, st);
        GPUTO_CUDA(cudaStreamSynchronize(st));
    }
    return r;
}

}  // extern "C"
