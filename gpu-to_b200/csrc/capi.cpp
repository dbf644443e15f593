// The C ABI of include/gputo.h.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "solver.h"

using gputo::Grid;
using gputo::Solver;

struct gputo_solver {
    Solver s;
};

struct gputo_net {
    gputo::Net n;
};

namespace gputo {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void set_error(const std::string &msg) { g_last_error = msg; }

int cuda_status(cudaError_t e, const char *what)
{
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? GPUTO_ERR_OOM : GPUTO_ERR_CUDA;
}

void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches_issued() { return g_launches.load(std::memory_order_relaxed); }

// The kernels are built for sm_100a only; refuse other devices up front
// instead of failing on the first launch.
static int check_device()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        set_error("no CUDA device is visible");
        return GPUTO_ERR_NO_DEVICE;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    int major = 0, minor = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    if (major != 10 || minor != 0) {
        set_error("gputo is built for sm_100a (B200); device " + std::to_string(dev) +
                  " is sm_" + std::to_string(major) + std::to_string(minor));
        return GPUTO_ERR_NO_DEVICE;
    }
    return GPUTO_OK;
}

}  // namespace gputo

extern "C" {

const char *gputo_status_string(int status)
{
    switch (status) {
    case GPUTO_OK: return "ok";
    case GPUTO_ERR_ARG: return "invalid argument";
    case GPUTO_ERR_CUDA: return "CUDA error";
    case GPUTO_ERR_OOM: return "out of device memory";
    case GPUTO_ERR_NOT_SPD: return "coarsest-grid matrix not positive definite";
    case GPUTO_ERR_BREAKDOWN: return "PCG breakdown";
    case GPUTO_ERR_NO_DEVICE: return "no usable CUDA device";
    case GPUTO_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
    }
}

const char *gputo_last_error(void) { return gputo::g_last_error.c_str(); }

const char *gputo_version(void) { return "gputo-b200 0.1 (sm_100a)"; }

int gputo_hex8_stiffness(double nu, double h, double *Ke)
{
    if (!Ke || !(h > 0) || !(nu > -1.0 && nu < 0.5)) return GPUTO_ERR_ARG;
    for (int m = 0; m < 576; ++m) Ke[m] = 0.0;
    for (int ix = 0; ix < 2; ++ix)
        for (int iy = 0; iy < 2; ++iy)
            for (int iz = 0; iz < 2; ++iz) {
                double K[24][24];
                gputo::gauss_part(nu, h, ix, iy, iz, K);
                for (int m = 0; m < 24; ++m)
                    for (int n = 0; n < 24; ++n) Ke[m * 24 + n] += K[m][n];
            }
    return GPUTO_OK;
}

void gputo_default_options(gputo_options *o)
{
    if (!o) return;
    o->precision = GPUTO_PREC_FP64;
    o->nswp = 3;
    o->omega = 0.48;
    o->prerelax = 0.7;
    o->nu = 0.3;
    o->check_every = 1;
    o->use_graph = 1;
    o->max_coarse_dofs = 12000;
    o->tc_parts = 0;
    o->tc_xchunk = 0;
    o->coarse = GPUTO_COARSE_GALERKIN;
    o->fine_op = 0;
    o->nswp_fine = 0;
    o->fuse_prolong = 0;
    o->sweep_xchunk = 0;
    o->sweep_pairs = 1;
    o->nswp_coarse = 0;
    o->coarse_from = 0;
}

int gputo_fine_op_constants(const double *Ke, double *c8)
{
    if (!Ke || !c8) return GPUTO_ERR_ARG;
    gputo::HadamardKe hk;
    if (!gputo::hadamard_ke(Ke, &hk)) {
        gputo::set_error("Ke does not have the Hadamard-basis pattern of an isotropic cube element");
        return GPUTO_ERR_ARG;
    }
    for (int q = 0; q < 8; ++q) c8[q] = hk.c[q];
    return GPUTO_OK;
}

int gputo_solver_create(gputo_solver **out, int nelx, int nely, int nelz, int nl,
                        const gputo_options *opt)
{
    if (!out) return GPUTO_ERR_ARG;
    *out = nullptr;
    int st = gputo::check_device();
    if (st) return st;
    auto *h = new gputo_solver();
    st = h->s.create(nelx, nely, nelz, nl, opt);
    if (st) {
        delete h;
        return st;
    }
    *out = h;
    return GPUTO_OK;
}

void gputo_solver_destroy(gputo_solver *s) { delete s; }

size_t gputo_solver_device_bytes(const gputo_solver *s) { return s ? s->s.bytes : 0; }

int gputo_solver_set_problem(gputo_solver *s, const double *Ke0, const double *fixed1b, int nfd)
{
    if (!s) return GPUTO_ERR_ARG;
    return s->s.set_problem(Ke0, fixed1b, nfd, s->s.own_stream);
}

int gputo_solver_setup_dev(gputo_solver *s, const double *CX, void *stream)
{
    if (!s || !CX) return GPUTO_ERR_ARG;
    return s->s.setup(CX, s->s.stream(stream));
}

int gputo_solver_solve_dev(gputo_solver *h, const double *F, double *U, double tol, int maxit,
                           double *relres, int *nit, void *stream)
{
    if (!h || !F || !U || !relres || !nit) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready) return GPUTO_ERR_ARG;
    cudaStream_t st = s.stream(stream);
    gputo::launch_pack(s.lay[0], F, s.Fw, 0, st);
    s.have_solution = false;
    int r = s.solve(s.Fw, s.Uw, tol, maxit, relres, nit, st, nullptr);
    if (r == GPUTO_OK || r == GPUTO_ERR_BREAKDOWN) {
        gputo::launch_unpack(s.lay[0], s.Uw, U, 0, st);
        GPUTO_CUDA(cudaStreamSynchronize(st));
        s.have_solution = r == GPUTO_OK;
    }
    return r;
}

int gputo_solver_energy_dev(gputo_solver *h, const double *dsK, double *ce, double *dc, double *compliance,
                            double *true_relres, void *stream)
{
    if (!h || !ce || (dc && !dsK)) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready || !s.have_solution) {
        gputo::set_error("gputo_solver_energy_dev needs a successful gputo_solver_solve_dev before it");
        return GPUTO_ERR_ARG;
    }
    cudaStream_t st = s.stream(stream);
    int r = s.energy(dsK, ce, dc, s.e2, st);
    if (r) return r;
    double hv[2] = {0.0, 0.0};
    GPUTO_CUDA(cudaMemcpyAsync(hv, s.e2, sizeof(hv), cudaMemcpyDeviceToHost, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    r = s.check_error_flags(st);
    if (r) return r;
    if (compliance) *compliance = hv[1];
    if (true_relres) *true_relres = hv[0] < 0.0 ? -1.0 : (s.last_res0 > 0.0 ? std::sqrt(hv[0]) / s.last_res0 : 0.0);
    return GPUTO_OK;
}

int gputo_solver_vcycle_dev(gputo_solver *h, const double *r, double *z, void *stream)
{
    if (!h || !r || !z) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready) return GPUTO_ERR_ARG;
    cudaStream_t st = s.stream(stream);
    s.launch_status = GPUTO_OK;
    s.have_solution = false;   // Fw is reused
    gputo::launch_pack(s.lay[0], r, s.Fw, 0, st);
    s.vcycle(s.Fw, s.Z, nullptr, st);
    gputo::launch_unpack(s.lay[0], s.Z, z, 0, st);
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    if (s.launch_status) return s.launch_status;
    return s.check_error_flags(st);
}

int gputo_solver_apply_dev(gputo_solver *h, const double *u, double *r, void *stream)
{
    if (!h || !u || !r) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready) return GPUTO_ERR_ARG;
    cudaStream_t st = s.stream(stream);
    s.launch_status = GPUTO_OK;
    gputo::launch_pack(s.lay[0], u, s.P, 0, st);
    s.apply(s.P, s.Q, nullptr, nullptr, st);
    gputo::launch_unpack(s.lay[0], s.Q, r, 0, st);
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    if (s.launch_status) return s.launch_status;
    return s.check_error_flags(st);
}

int gputo_solver_apply_fp32_dev(gputo_solver *h, const double *u, double *r, int tc_parts, void *stream)
{
    if (!h || !u || !r || tc_parts < 0 || tc_parts > 2) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready || s.opt.precision != GPUTO_PREC_MIXED) return GPUTO_ERR_ARG;
    cudaStream_t st = s.stream(stream);
    s.launch_status = GPUTO_OK;
    const long long nv = s.lay[0].size();
    gputo::launch_pack(s.lay[0], u, s.P, 0, st);
    gputo::launch_convert<double, float>(nv, s.P, s.Lf[0].u0, nullptr, st);
    int rs;
    if (tc_parts == 0)
        rs = s.fine_sweep<float>(0, gputo::MODE_APPLY, s.lay[0], s.elay, s.CXpf, s.Lf[0].u0, nullptr, s.Lf[0],
                                 s.Lf[0].u1, 1.f, 0.f, nullptr, nullptr, st);
    else
        rs = gputo::launch_tc_sweep(tc_parts, gputo::MODE_APPLY, s.lay[0], s.elay, s.CXpf, s.Lf[0].u0, nullptr,
                                    s.Lf[0].diag, s.mask[0], s.Lf[0].u1, 1.f, 0.f, s.opt.tc_xchunk, nullptr,
                                    s.err, st);
    if (rs) return rs;
    gputo::launch_convert<float, double>(nv, s.Lf[0].u1, s.Q, nullptr, st);
    gputo::launch_unpack(s.lay[0], s.Q, r, 0, st);
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    if (s.launch_status) return s.launch_status;
    return s.check_error_flags(st);
}

// ---------------------------------------------------------------------------
// learned coarse-grid correction
// ---------------------------------------------------------------------------

long long gputo_net_num_params(void) { return gputo::Net::num_params(); }

int gputo_net_create(gputo_net **out, unsigned long long seed)
{
    if (!out) return GPUTO_ERR_ARG;
    *out = nullptr;
    int st = gputo::check_device();
    if (st) return st;
    auto *h = new (std::nothrow) gputo_net();
    if (!h) return GPUTO_ERR_OOM;
    st = h->n.create(seed);
    if (st) {
        delete h;
        return st;
    }
    *out = h;
    return GPUTO_OK;
}

void gputo_net_destroy(gputo_net *h) { delete h; }

int gputo_net_get_params(const gputo_net *h, float *host)
{
    if (!h || !host) return GPUTO_ERR_ARG;
    GPUTO_CUDA(cudaMemcpy(host, h->n.params, sizeof(float) * gputo::Net::num_params(), cudaMemcpyDeviceToHost));
    return GPUTO_OK;
}

int gputo_net_set_params(gputo_net *h, const float *host)
{
    if (!h || !host) return GPUTO_ERR_ARG;
    const size_t b = sizeof(float) * gputo::Net::num_params();
    GPUTO_CUDA(cudaMemcpy(h->n.params, host, b, cudaMemcpyHostToDevice));
    GPUTO_CUDA(cudaMemset(h->n.grads, 0, b));
    GPUTO_CUDA(cudaMemset(h->n.m1, 0, b));
    GPUTO_CUDA(cudaMemset(h->n.m2, 0, b));
    h->n.step = 0;
    return GPUTO_OK;
}

int gputo_net_forward_dev(gputo_net *h, const float *x, int X, int Z, int Y, float *y, void *stream)
{
    if (!h || !x || !y || X < 1 || Z < 1 || Y < 1) return GPUTO_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    int s = gputo::init_net_kernels();
    if (!s) s = h->n.forward(x, gputo::NetDims{X, Z, Y}, y, st);
    if (s) return s;
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

int gputo_net_train_step_dev(gputo_net *h, const float *x, const float *t, const float *m, int nsamples, int X,
                             int Z, int Y, float lr, double *loss, float *grads_out, void *stream)
{
    if (!h || !x || !t || !m || nsamples < 1 || X < 1 || Z < 1 || Y < 1 || lr < 0.f) return GPUTO_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const gputo::NetDims d{X, Z, Y};
    const long long n = d.n();
    int s = gputo::init_net_kernels();
    if (s) return s;
    GPUTO_CUDA(cudaMemsetAsync(h->n.loss_acc, 0, sizeof(double), st));
    for (int q = 0; q < nsamples; ++q) {
        s = h->n.accumulate(x + (size_t)q * 4 * n, t + (size_t)q * 3 * n, m + (size_t)q * 3 * n, d, st);
        if (s) return s;
    }
    if (grads_out)
        GPUTO_CUDA(cudaMemcpyAsync(grads_out, h->n.grads, sizeof(float) * gputo::Net::num_params(),
                                   cudaMemcpyDeviceToHost, st));
    if (lr > 0.f) {
        s = h->n.adam(lr, nsamples, st);
        if (s) return s;
    } else {
        GPUTO_CUDA(cudaMemsetAsync(h->n.grads, 0, sizeof(float) * gputo::Net::num_params(), st));
    }
    double l = 0.0;
    GPUTO_CUDA(cudaMemcpyAsync(&l, h->n.loss_acc, sizeof(double), cudaMemcpyDeviceToHost, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    if (loss) *loss = l / nsamples;
    return GPUTO_OK;
}

int gputo_solver_set_net(gputo_solver *h, gputo_net *net, int mode)
{
    if (!h) return GPUTO_ERR_ARG;
    return h->s.attach_net(net ? &net->n : nullptr, net ? mode : 0);
}

int gputo_solver_net_state(const gputo_solver *h, int *on, int *plain_nit, int *net_nit)
{
    if (!h) return GPUTO_ERR_ARG;
    if (on) *on = h->s.net_on ? 1 : 0;
    if (plain_nit) *plain_nit = h->s.ref_plain_nit;
    if (net_nit) *net_nit = h->s.ref_net_nit;
    return GPUTO_OK;
}

int gputo_solver_net_dims(const gputo_solver *h, int *X, int *Z, int *Y)
{
    if (!h || !X || !Z || !Y) return GPUTO_ERR_ARG;
    const Solver &s = h->s;
    if (!s.net_x) return GPUTO_ERR_ARG;
    *X = s.nd.X;
    *Z = s.nd.Z;
    *Y = s.nd.Y;
    return GPUTO_OK;
}

int gputo_solver_net_features_dev(gputo_solver *h, const double *r, float *x, float *m, float *dsq, float *scale,
                                  void *stream)
{
    if (!h || !r || !x) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready || !s.net_x) return GPUTO_ERR_ARG;
    cudaStream_t st = s.stream(stream);
    gputo::launch_pack(s.lay[0], r, s.P, 0, st);
    gputo::launch_convert<double, float>(s.lay[0].size(), s.P, s.Lf[0].f, nullptr, st);
    gputo::launch_restrict<float>(s.lay[1], s.lay[0], s.Lf[0].f, s.mask[1], s.Lf[1].f, nullptr, st);
    gputo::launch_restrict<float>(s.lay[2], s.lay[1], s.Lf[1].f, s.mask[2], s.Lf[2].f, nullptr, st);
    gputo::launch_net_features(s.lay[2], s.Lf[2].f, s.Lf[2].diag, s.dens2, x, dsq, s.net_s, nullptr, st);
    if (m) gputo::launch_net_mask(s.g[2], s.mask[2], m, st);
    float sc = 0.f;
    GPUTO_CUDA(cudaMemcpyAsync(&sc, s.net_s, sizeof(float), cudaMemcpyDeviceToHost, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    if (scale) *scale = sc;
    return GPUTO_OK;
}

int gputo_solver_net_energy_rhs_dev(gputo_solver *h, const double *w, float scale, float *gt, void *stream)
{
    if (!h || !w || !gt || !(scale > 0.f)) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready || !s.net_x) return GPUTO_ERR_ARG;
    cudaStream_t st = s.stream(stream);
    gputo::launch_pack(s.lay[0], w, s.P, 0, st);
    gputo::launch_convert<double, float>(s.lay[0].size(), s.P, s.Lf[0].f, nullptr, st);
    gputo::launch_restrict<float>(s.lay[1], s.lay[0], s.Lf[0].f, s.mask[1], s.Lf[1].f, nullptr, st);
    gputo::launch_restrict<float>(s.lay[2], s.lay[1], s.Lf[1].f, s.mask[2], s.Lf[2].f, nullptr, st);
    gputo::launch_net_energy_rhs(s.lay[2], s.Lf[2].f, s.Lf[2].diag, s.mask[2], scale, gt, st);
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

int gputo_solver_net_train_step_dev(gputo_solver *h, gputo_net *net, const float *x, const float *gt, int nsamples,
                                    float lr, double *loss, float *grads_out, void *stream)
{
    if (!h || !net || !x || !gt || nsamples < 1 || lr < 0.f) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready || !s.net_x) return GPUTO_ERR_ARG;
    return s.net_train_energy(&net->n, x, gt, nsamples, lr, loss, grads_out, s.stream(stream));
}

int gputo_solver_level2_inject_dev(gputo_solver *h, const double *v, float *out, void *stream)
{
    if (!h || !v || !out) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (s.nl < 3) return GPUTO_ERR_ARG;
    cudaStream_t st = s.stream(stream);
    gputo::launch_level2_inject(s.g[2], s.g[0], v, out, st);
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

long long gputo_solver_launch_count(const gputo_solver *) { return gputo::launches_issued(); }

int gputo_debug_set_sweep_fault(int skip_stage, unsigned wait_us)
{
    return gputo::set_sweep_fault_hook(skip_stage, wait_us);
}

int gputo_solver_time_kernel(gputo_solver *h, int which, int reps, double *ms, void *stream)
{
    if (!h || !ms || reps < 1 || which < 0 || which > 6) return GPUTO_ERR_ARG;
    Solver &s = h->s;
    if (!s.ready) return GPUTO_ERR_ARG;
    if (which == 5 && !(s.use_hsweep<double>(s.g[0]) && gputo::hsweep_energy_fits(s.g[0]))) return GPUTO_ERR_ARG;
    if ((which == 1 || which == 2 || which == 4 || which == 6) && s.opt.precision != GPUTO_PREC_MIXED)
        return GPUTO_ERR_ARG;
    if (which == 6 && (s.nl < 4 || s.redisc())) return GPUTO_ERR_ARG;
    if ((which == 2 || which == 3) && s.nl < 2) return GPUTO_ERR_ARG;
    cudaStream_t st = s.stream(stream);
    cudaEvent_t e0, e1;
    GPUTO_CUDA(cudaEventCreate(&e0));
    GPUTO_CUDA(cudaEventCreate(&e1));
    int lst = GPUTO_OK;
    auto launch = [&]() {
        int r = GPUTO_OK;
        switch (which) {
        case 0:
            r = s.fine_sweep<double>(0, gputo::MODE_APPLY, s.lay[0], s.elay, s.CXp, s.P, nullptr, s.L[0], s.Q, 1.0,
                                     0.0, nullptr, nullptr, st);
            break;
        case 1:
            r = s.fine_sweep<float>(0, gputo::MODE_JACOBI, s.lay[0], s.elay, s.CXpf, s.Lf[0].u0, s.Lf[0].f, s.Lf[0],
                                    s.Lf[0].u1, 0.48f, 0.7f, nullptr, nullptr, st);
            break;
        case 5:   // the fused energy apply on the solver's U and F; ce into the staging buffer
            r = gputo::launch_hsweep_energy(s.lay[0], s.elay, s.hk, s.CXp, s.Uw, s.Fw, s.mask[0], s.maskp[0],
                                            nullptr, s.partial, s.Dn, nullptr, nullptr, s.err, st);
            break;
        case 4:
            r = gputo::launch_tc_sweep(s.opt.tc_parts > 0 ? s.opt.tc_parts : 1, gputo::MODE_JACOBI, s.lay[0],
                                       s.elay, s.CXpf, s.Lf[0].u0, s.Lf[0].f, s.Lf[0].diag, s.mask[0],
                                       s.Lf[0].u1, 0.48f, 0.7f, s.opt.tc_xchunk, nullptr, s.err, st);
            break;
        case 6:   // level 2, FP32 (stored Galerkin element matrices)
            if (s.Lf[2].yq)
                gputo::launch_packed_sweep_ec<float>(gputo::MODE_JACOBI, s.lay[2], s.Lf[2].Apk, s.Lf[2].u0,
                                                     s.Lf[2].f, s.Lf[2].rdiag, s.mask[2], s.Lf[2].u1, 0.48f, 0.7f,
                                                     s.Lf[2].yq, nullptr, st);
            else
                gputo::launch_packed_sweep<float>(gputo::MODE_JACOBI, s.lay[2], s.Lf[2].Apk, s.Lf[2].u0,
                                                  s.Lf[2].f, s.Lf[2].rdiag, s.mask[2], s.Lf[2].u1, 0.48f, 0.7f,
                                                  nullptr, st);
            break;
        case 2:
            if (s.quad_level1())
                r = gputo::launch_quad_sweep<float>(gputo::MODE_JACOBI, s.lay[1], s.elay, s.CXpf, s.Lf[1].u0,
                                                    s.Lf[1].f, s.Lf[1].rdiag, s.mask[1], s.Lf[1].u1, 0.48f,
                                                    0.7f, s.opt.nu, s.Lf[1].yq, nullptr, s.err, st);
            else
                gputo::launch_packed_sweep<float>(gputo::MODE_JACOBI, s.lay[1], s.Lf[1].Apk, s.Lf[1].u0,
                                                  s.Lf[1].f, s.Lf[1].rdiag, s.mask[1], s.Lf[1].u1, 0.48f,
                                                  0.7f, nullptr, st);
            break;
        default:
            if (s.quad_level1())
                r = gputo::launch_quad_sweep<double>(gputo::MODE_JACOBI, s.lay[1], s.elay, s.CXp, s.L[1].u0,
                                                     s.L[1].f, s.L[1].rdiag, s.mask[1], s.L[1].u1, 0.48,
                                                     0.7, s.opt.nu, s.L[1].yq, nullptr, s.err, st);
            else
                gputo::launch_packed_sweep<double>(gputo::MODE_JACOBI, s.lay[1], s.L[1].Apk, s.L[1].u0,
                                                   s.L[1].f, s.L[1].rdiag, s.mask[1], s.L[1].u1, 0.48,
                                                   0.7, nullptr, st);
        }
        if (r && !lst) lst = r;
    };
    launch();  // warm-up
    GPUTO_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < reps; ++r) launch();
    GPUTO_CUDA(cudaEventRecord(e1, st));
    GPUTO_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    GPUTO_CUDA(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    GPUTO_CUDA(cudaGetLastError());
    if (lst) return lst;
    *ms = (double)t / reps;
    return s.check_error_flags(st);
}

// ---------------------------------------------------------------------------
// drop-in MEX entry point with a per-shape solver cache
// ---------------------------------------------------------------------------

namespace {
// every option is part of the key: a call must never reuse a solver built
// with other options
using Key = std::tuple<int, int, int, int, int, int, int, double, double, double, int, int, int, int, int, int, int>;
std::mutex g_cache_mu;
std::map<Key, std::unique_ptr<gputo_solver>> g_cache;
std::vector<Key> g_cache_order;

gputo_solver *cached_solver(int nelx, int nely, int nelz, int nl, const gputo_options &o, int *st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    Key k{dev, nelx, nely, nelz, nl, o.precision, o.nswp, o.omega, o.prerelax, o.nu,
          o.check_every, o.use_graph, o.max_coarse_dofs, o.tc_parts, o.tc_xchunk, o.coarse, o.fine_op};
    auto it = g_cache.find(k);
    if (it != g_cache.end()) return it->second.get();
    // keep at most two shapes resident
    while (g_cache.size() >= 2) {
        g_cache.erase(g_cache_order.front());
        g_cache_order.erase(g_cache_order.begin());
    }
    gputo_solver *s = nullptr;
    *st = gputo_solver_create(&s, nelx, nely, nelz, nl, &o);
    if (*st == GPUTO_ERR_OOM) {
        // release everything cached and try once more
        g_cache.clear();
        g_cache_order.clear();
        cudaDeviceSynchronize();
        *st = gputo_solver_create(&s, nelx, nely, nelz, nl, &o);
    }
    if (*st) return nullptr;
    g_cache[k].reset(s);
    g_cache_order.push_back(k);
    return s;
}
}  // namespace

// One MEX-style solve on host buffers with the cached solver of these
// options; the log file (printLev >= 1) gets per-iteration lines from
// printLev >= cg_lines on.
static int mex_solve(const char *log_name, int cg_lines, const double *Ke0, const double *F, double *U,
                     const double *CX, const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl,
                     double tol, int maxit, int printLev, const gputo_options &o, double *relres, int *nit);

int gputo_mgcg1_ex(const double *Ke0, const double *F, double *U, const double *CX,
                   const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl,
                   double tol, int maxit, int printLev, const gputo_options *opt, double *relres,
                   int *nit)
{
    gputo_options o;
    if (opt) o = *opt;
    else gputo_default_options(&o);
    return mex_solve("mgcg1.log", 2, Ke0, F, U, CX, fixed1b, nfd, nelx, nely, nelz, nl, tol, maxit, printLev, o,
                     relres, nit);
}

int gputo_mgcg9(const double *Ae, const double *F, double *U, const double *CX, const double *fixed1b, int nfd,
                int nelx, int nely, int nelz, int nl, double tol, int maxit, int nswp, int printLev, double nu,
                double hx, double hy, double hz, double *relres, int *nit)
{
    (void)nu;   // read by the reference (mgcg9.cu:167-170) and not used on its solve path
    (void)hx;
    (void)hy;
    (void)hz;
    if (nswp < 0 || nl < 2) {
        if (relres) *relres = 0.0;
        if (nit) *nit = -1;
        gputo::set_error("mgcg9 needs nswp >= 0 and nl >= 2");
        return GPUTO_ERR_ARG;
    }
    gputo_options o;
    gputo_default_options(&o);
    o.coarse = GPUTO_COARSE_REDISCRETIZED;
    o.nswp = nswp;
    o.omega = 0.33;            // mgcg9.cu:929-935 Jacobc: U = 0.67 U + 0.33 (R + D U) / D
    o.prerelax = 0.7;          // mgcg9.cu:920-927 preRelc
    o.max_coarse_dofs = 19999; // mgcg9.cu:74,400 maxDofs0: direct coarsest solve below 20000 dofs
    return mex_solve("mgcg9.log", 3, Ae, F, U, CX, fixed1b, nfd, nelx, nely, nelz, nl, tol, maxit, printLev, o,
                     relres, nit);
}

static int mex_solve(const char *log_name, int cg_lines, const double *Ke0, const double *F, double *U,
                     const double *CX, const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl,
                     double tol, int maxit, int printLev, const gputo_options &o, double *relres, int *nit)
{
    if (relres) *relres = 0.0;
    if (nit) *nit = -1;
    if (!Ke0 || !F || !U || !CX || (nfd > 0 && !fixed1b) || !relres || !nit || nfd < 0) {
        gputo::set_error("null argument");
        return GPUTO_ERR_ARG;
    }
    auto t0 = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lock(g_cache_mu);
    int st = gputo::check_device();
    if (st) return st;
    gputo_solver *h = cached_solver(nelx, nely, nelz, nl, o, &st);
    if (!h) return st;
    Solver &s = h->s;
    cudaStream_t strm = s.own_stream;
    FILE *log = nullptr;
    if (printLev >= 1) log = std::fopen(log_name, "w");
    st = s.set_problem(Ke0, fixed1b, nfd, strm);
    if (st) {
        if (log) std::fclose(log);
        return st;
    }
    const long long nd = s.g[0].ndof(), ne = s.g[0].nel();
    std::unique_lock<std::mutex> io(gputo::host_io_mutex());
    GPUTO_CUDA(cudaStreamSynchronize(strm));   // set_problem's uploads have landed before Dn is reused
    // CX first: the hierarchy's setup kernels run on strm while F is staged
    // in (the setup reads neither Dn nor Fw)
    st = gputo::host_to_device(s.CX, CX, sizeof(double) * ne);
    if (!st) st = s.setup_enqueue(s.CX, strm);
    if (!st) st = gputo::host_to_device(s.Dn, F, sizeof(double) * nd);
    if (!st) gputo::launch_pack(s.lay[0], s.Dn, s.Fw, 0, strm);
    io.unlock();
    if (!st) st = s.setup_finish(strm);
    if (st) {
        if (log) std::fclose(log);
        return st;
    }
    if (!st) st = s.solve(s.Fw, s.Uw, tol, maxit, relres, nit, strm, printLev >= cg_lines ? log : nullptr);
    if (!st || st == GPUTO_ERR_BREAKDOWN) {
        // solver frame -> MATLAB frame: y components negated (mgcg1.cu:282-283)
        gputo::launch_unpack(s.lay[0], s.Uw, s.Dn, 1, strm);
        GPUTO_CUDA(cudaStreamSynchronize(strm));
        std::lock_guard<std::mutex> io2(gputo::host_io_mutex());
        const int cs = gputo::device_to_host(U, s.Dn, sizeof(double) * nd);
        if (cs && !st) st = cs;
    }
    if (log) {
        const double secs =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(log, "MGCG Initial residual=%12.6g\n", s.last_res0);
        std::fprintf(log, "MGCG Nit=%d  Time %8.3g  Final residual=%12.6g\n", *nit, secs, *relres);
        std::fclose(log);
    }
    return st;
}

int gputo_mgcg1(const double *Ke0, const double *F, double *U, const double *CX,
                const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl,
                double tol, int maxit, int printLev, double *relres, int *nit)
{
    return gputo_mgcg1_ex(Ke0, F, U, CX, fixed1b, nfd, nelx, nely, nelz, nl, tol, maxit, printLev,
                          nullptr, relres, nit);
}

// ---------------------------------------------------------------------------
// design-loop steps
// ---------------------------------------------------------------------------

int gputo_simp(const double *xPhys, long long n, double penal, double E0, double Emin, double *CX, double *dsK)
{
    if (!xPhys || !CX || n <= 0) return GPUTO_ERR_ARG;
    int st = gputo::check_device();
    if (st) return st;
    std::lock_guard<std::mutex> lock(gputo::host_io_mutex());
    double *dx = gputo::host_call_buffer(0, (size_t)n, &st);
    double *dcx = !st ? gputo::host_call_buffer(1, (size_t)n, &st) : nullptr;
    double *dds = (!st && dsK) ? gputo::host_call_buffer(2, (size_t)n, &st) : nullptr;
    if (st) return st;
    st = gputo::host_to_device(dx, xPhys, sizeof(double) * n);
    if (st) return st;
    gputo::launch_simp(n, dx, penal, E0, Emin, dcx, dds, nullptr);
    GPUTO_CUDA(cudaDeviceSynchronize());
    GPUTO_CUDA(cudaGetLastError());
    st = gputo::device_to_host(CX, dcx, sizeof(double) * n);
    if (!st && dsK) st = gputo::device_to_host(dsK, dds, sizeof(double) * n);
    return st;
}

namespace {
struct Scratch {
    double *partial = nullptr;
    unsigned *ticket = nullptr;
    double *scalar = nullptr;
    int *err = nullptr;
    double *big = nullptr;      // grown on demand (tensor-core partials)
    long long big_cap = 0;
    cudaStream_t st = nullptr;
    int reserve_big(long long n)
    {
        if (n <= big_cap) return GPUTO_OK;
        cudaFree(big);
        big = nullptr;
        big_cap = 0;
        GPUTO_CUDA(cudaMalloc(&big, sizeof(double) * (size_t)n));
        big_cap = n;
        return GPUTO_OK;
    }
    int init()
    {
        if (partial) return GPUTO_OK;
        GPUTO_CUDA(cudaMalloc(&partial, sizeof(double) * 2048));
        GPUTO_CUDA(cudaMalloc(&ticket, 16));
        GPUTO_CUDA(cudaMalloc(&scalar, sizeof(double)));
        GPUTO_CUDA(cudaMalloc(&err, sizeof(int)));
        GPUTO_CUDA(cudaMemset(err, 0, sizeof(int)));
        GPUTO_CUDA(cudaMemset(ticket, 0, 16));
        GPUTO_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        return GPUTO_OK;
    }
};
std::mutex g_scratch_mu;
Scratch g_scratch;

bool grid_ok(int nelx, int nely, int nelz)
{
    return nelx > 0 && nely > 0 && nelz > 0;
}
}  // namespace

int gputo_compliance_sens_dev(const double *Ke0, const double *U, const double *CX,
                              const double *dsK, int nelx, int nely, int nelz, double *ce,
                              double *dc, double *compliance, void *stream)
{
    if (!Ke0 || !U || !grid_ok(nelx, nely, nelz) || (dc && !dsK) || (compliance && !CX))
        return GPUTO_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    int st = gputo::check_device();
    if (st) return st;
    st = g_scratch.init();
    if (st) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : g_scratch.st;
    st = gputo::upload_fine_ke(Ke0, s);
    if (st) return st;
    Grid g{nelx, nely, nelz};
    gputo::launch_element_energy(g, U, CX, dsK, ce, dc, g_scratch.partial, g_scratch.ticket,
                                 compliance ? g_scratch.scalar : nullptr, s);
    if (compliance)
        GPUTO_CUDA(cudaMemcpyAsync(compliance, g_scratch.scalar, sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
    GPUTO_CUDA(cudaStreamSynchronize(s));
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

int gputo_compliance_sens_tc_dev(const double *Ke0, const double *U, const double *CX,
                                 const double *dsK, int nelx, int nely, int nelz, double *ce,
                                 double *dc, double *compliance, void *stream)
{
    if (!Ke0 || !U || !grid_ok(nelx, nely, nelz) || (dc && !dsK) || (compliance && !CX))
        return GPUTO_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    int st = gputo::check_device();
    if (st) return st;
    st = g_scratch.init();
    if (st) return st;
    Grid g{nelx, nely, nelz};
    if (!gputo::element_energy_tc_fits(g)) {
        gputo::set_error("grid too large for the tensor-core contraction (2^31 dofs)");
        return GPUTO_ERR_ARG;
    }
    st = g_scratch.reserve_big(gputo::element_energy_tc_partials(g));
    if (st) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : g_scratch.st;
    st = gputo::upload_fine_ke(Ke0, s);
    if (st) return st;
    gputo::launch_element_energy_tc(g, U, CX, dsK, ce, dc, g_scratch.big,
                                    compliance ? g_scratch.scalar : nullptr, g_scratch.err, s);
    if (compliance)
        GPUTO_CUDA(cudaMemcpyAsync(compliance, g_scratch.scalar, sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
    int h_err = 0;
    GPUTO_CUDA(cudaMemcpyAsync(&h_err, g_scratch.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    GPUTO_CUDA(cudaStreamSynchronize(s));
    GPUTO_CUDA(cudaGetLastError());
    if (h_err) {
        cudaMemset(g_scratch.err, 0, sizeof(int));
        gputo::set_error("tensor-core MMA completion wait gave up");
        return GPUTO_ERR_TIMEOUT;
    }
    return GPUTO_OK;
}

int gputo_compliance_sens(const double *Ke0, const double *U, const double *CX,
                          const double *dsK, int nelx, int nely, int nelz, double *ce,
                          double *dc, double *compliance)
{
    if (!Ke0 || !U || !grid_ok(nelx, nely, nelz) || (dc && !dsK) || (compliance && !CX))
        return GPUTO_ERR_ARG;
    int st = gputo::check_device();
    if (st) return st;
    Grid g{nelx, nely, nelz};
    const size_t nd = (size_t)g.ndof(), ne = (size_t)g.nel();
    std::lock_guard<std::mutex> lock(gputo::host_io_mutex());
    // device buffers kept between calls (slots 0-4 of the host-call workspace)
    double *dU = gputo::host_call_buffer(0, nd, &st);
    double *dCX = (!st && CX) ? gputo::host_call_buffer(1, ne, &st) : nullptr;
    double *dS = (!st && dsK) ? gputo::host_call_buffer(2, ne, &st) : nullptr;
    double *dce = (!st && ce) ? gputo::host_call_buffer(3, ne, &st) : nullptr;
    double *ddc = (!st && dc) ? gputo::host_call_buffer(4, ne, &st) : nullptr;
    if (st) return st;
    if (!st) st = gputo::host_to_device(dU, U, nd * 8);
    if (!st && CX) st = gputo::host_to_device(dCX, CX, ne * 8);
    if (!st && dsK) st = gputo::host_to_device(dS, dsK, ne * 8);
    if (st) return st;
    gputo::launch_flip_y(g.nnod(), dU, 0);  // MATLAB frame -> solver frame
    GPUTO_CUDA(cudaDeviceSynchronize());
    st = gputo_compliance_sens_dev(Ke0, dU, dCX, dS, nelx, nely, nelz, dce, ddc, compliance,
                                   nullptr);
    if (!st && ce) st = gputo::device_to_host(ce, dce, ne * 8);
    if (!st && dc) st = gputo::device_to_host(dc, ddc, ne * 8);
    return st;
}

int gputo_density_filter_dev(const double *in, const double *divisor, double *out, int nelx,
                             int nely, int nelz, double rmin, int normalize, void *stream)
{
    if (!in || !out || !grid_ok(nelx, nely, nelz) || !(rmin > 0)) return GPUTO_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    int st = gputo::check_device();
    if (st) return st;
    st = g_scratch.init();
    if (st) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : g_scratch.st;
    const int R = (int)std::ceil(rmin) - 1;
    if (nelx <= R || nely <= R || nelz <= R) {
        gputo::set_error("filter radius exceeds the grid");
        return GPUTO_ERR_ARG;
    }
    st = gputo::launch_filter(Grid{nelx, nely, nelz}, in, divisor, out, rmin, normalize, s);
    if (st) return st;
    GPUTO_CUDA(cudaStreamSynchronize(s));
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

int gputo_time_filter_dev(const double *const *in, double *const *out, int n, int nelx, int nely, int nelz,
                          double rmin, int reps, double *ms, void *stream)
{
    if (!in || !out || n < 1 || n > 64 || reps < 1 || !ms || !grid_ok(nelx, nely, nelz) || !(rmin > 0))
        return GPUTO_ERR_ARG;
    for (int q = 0; q < n; ++q)
        if (!in[q] || !out[q]) return GPUTO_ERR_ARG;
    int st = gputo::check_device();
    if (st) return st;
    const int R = (int)std::ceil(rmin) - 1;
    if (nelx <= R || nely <= R || nelz <= R) {
        gputo::set_error("filter radius exceeds the grid");
        return GPUTO_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const Grid g{nelx, nely, nelz};
    for (int q = 0; q < n; ++q)
        if ((st = gputo::launch_filter(g, in[q], nullptr, out[q], rmin, 1, s))) return st;
    cudaEvent_t e0, e1;
    GPUTO_CUDA(cudaEventCreate(&e0));
    GPUTO_CUDA(cudaEventCreate(&e1));
    GPUTO_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps && !st; ++r) st = gputo::launch_filter(g, in[r % n], nullptr, out[r % n], rmin, 1, s);
    GPUTO_CUDA(cudaEventRecord(e1, s));
    GPUTO_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    GPUTO_CUDA(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    GPUTO_CUDA(cudaGetLastError());
    *ms = (double)t / reps;
    return GPUTO_OK;
}

int gputo_density_filter(const double *in, const double *divisor, double *out, int nelx,
                         int nely, int nelz, double rmin, int normalize)
{
    if (!in || !out || !grid_ok(nelx, nely, nelz)) return GPUTO_ERR_ARG;
    int st = gputo::check_device();
    if (st) return st;
    const size_t ne = (size_t)nelx * nely * nelz;
    std::lock_guard<std::mutex> lock(gputo::host_io_mutex());
    double *din = gputo::host_call_buffer(0, ne, &st);
    double *ddiv = (!st && divisor) ? gputo::host_call_buffer(1, ne, &st) : nullptr;
    double *dout = !st ? gputo::host_call_buffer(2, ne, &st) : nullptr;
    if (st) return st;
    st = gputo::host_to_device(din, in, ne * 8);
    if (!st && divisor) st = gputo::host_to_device(ddiv, divisor, ne * 8);
    if (!st) st = gputo_density_filter_dev(din, ddiv, dout, nelx, nely, nelz, rmin, normalize, nullptr);
    if (!st) st = gputo::device_to_host(out, dout, ne * 8);
    return st;
}

int gputo_simp_dev(const double *xPhys, long long n, double penal, double E0, double Emin,
                   double *CX, double *dsK, void *stream)
{
    if (!xPhys || !CX || n <= 0) return GPUTO_ERR_ARG;
    int st = gputo::check_device();
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    gputo::launch_simp(n, xPhys, penal, E0, Emin, CX, dsK, s);
    GPUTO_CUDA(cudaStreamSynchronize(s));
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

namespace {
// Scratch of the OC update, grown on demand and kept for later calls.
struct OcScratch {
    double *ocp = nullptr, *partial = nullptr, *lmid_dev = nullptr;
    unsigned *ticket = nullptr;
    void *state = nullptr;
    long long cap = 0;
    int reserve(long long n)
    {
        if (!partial) {
            GPUTO_CUDA(cudaMalloc(&partial, sizeof(double) * 2048));
            GPUTO_CUDA(cudaMalloc(&ticket, 16));
            GPUTO_CUDA(cudaMemset(ticket, 0, 16));
            GPUTO_CUDA(cudaMalloc(&state, 64));
        }
        if (n > cap) {
            cudaFree(ocp);
            ocp = nullptr;
            cap = 0;
            GPUTO_CUDA(cudaMalloc(&ocp, sizeof(double) * (size_t)n));
            cap = n;
        }
        return GPUTO_OK;
    }
};
std::mutex g_oc_mu;
OcScratch g_oc;
constexpr int kHeavisideSteps = 60;   // Newton steps queued for the projection threshold
}  // namespace

int gputo_oc_update_dev(const double *x, const double *dc, const double *dV0, long long n,
                        double volfrac, double move, double *xnew, double *lmid, void *stream)
{
    if (!x || !dc || !dV0 || !xnew || n <= 0 || x == xnew || !(volfrac > 0) || !(move >= 0))
        return GPUTO_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_oc_mu);
    int st = gputo::check_device();
    if (st) return st;
    st = g_oc.reserve(n);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    gputo::launch_oc_update(n, x, dc, dV0, volfrac, move, g_oc.ocp, xnew, g_oc.partial,
                            g_oc.ticket, g_oc.state, 64, s);
    double hst[3] = {0, 0, 0};
    GPUTO_CUDA(cudaMemcpyAsync(hst, g_oc.state, sizeof(hst), cudaMemcpyDeviceToHost, s));
    GPUTO_CUDA(cudaStreamSynchronize(s));
    GPUTO_CUDA(cudaGetLastError());
    if (lmid) *lmid = hst[2];
    return GPUTO_OK;
}

int gputo_heaviside_dev(const double *xTilde, long long n, double volfrac, double beta, double *eta,
                        double *xPhys, double *dprj, void *stream)
{
    if (!xTilde || !xPhys || !eta || n <= 0 || xTilde == xPhys || !(volfrac > 0 && volfrac < 1) || !(beta > 0))
        return GPUTO_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_oc_mu);
    int st = gputo::check_device();
    if (st) return st;
    st = g_oc.reserve(n);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    gputo::launch_heaviside(n, xTilde, volfrac, beta, *eta, xPhys, dprj, g_oc.partial, g_oc.ticket, g_oc.state,
                            kHeavisideSteps, s);
    struct {
        double eta;
        int steps, done;
    } hst{};
    GPUTO_CUDA(cudaMemcpyAsync(&hst, g_oc.state, sizeof(hst), cudaMemcpyDeviceToHost, s));
    GPUTO_CUDA(cudaStreamSynchronize(s));
    GPUTO_CUDA(cudaGetLastError());
    *eta = hst.eta;
    if (!hst.done) {
        gputo::set_error("Heaviside threshold: the eta Newton iteration did not reach |f| <= 1e-6");
        return GPUTO_ERR_BREAKDOWN;
    }
    return GPUTO_OK;
}

int gputo_mul_dev(const double *a, const double *b, double *out, long long n, void *stream)
{
    if (!a || !b || !out || n <= 0) return GPUTO_ERR_ARG;
    int st = gputo::check_device();
    if (st) return st;
    gputo::launch_mul(n, a, b, out, (cudaStream_t)stream);
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

int gputo_oc_update(const double *x, const double *dc, const double *dV0, long long n,
                    double volfrac, double move, double *xnew, double *lmid)
{
    if (!x || !dc || !dV0 || !xnew || n <= 0) return GPUTO_ERR_ARG;
    int st = gputo::check_device();
    if (st) return st;
    std::lock_guard<std::mutex> lock(gputo::host_io_mutex());
    double *d = gputo::host_call_buffer(0, 4 * (size_t)n, &st);
    if (st) return st;
    st = gputo::host_to_device(d, x, sizeof(double) * n);
    if (!st) st = gputo::host_to_device(d + n, dc, sizeof(double) * n);
    if (!st) st = gputo::host_to_device(d + 2 * n, dV0, sizeof(double) * n);
    if (!st) st = gputo_oc_update_dev(d, d + n, d + 2 * n, n, volfrac, move, d + 3 * n, lmid, nullptr);
    if (!st) st = gputo::device_to_host(xnew, d + 3 * n, sizeof(double) * n);
    return st;
}

}  // extern "C"
