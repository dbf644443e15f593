// Host side of the MGCG solver: hierarchy allocation and setup, the V-cycle
// schedule and the PCG loop (Cantilever/TOP3D125MGCGCUDA/mgcg1.cu:184-651).
//
// Differences from the reference's host code, all behaviour-preserving:
//  * buffers are allocated once per solver (64-bit sizes) and reused across
//    calls instead of cudaDeviceReset + cudaMalloc on every call (:202-215);
//  * nodal vectors live in a row-padded layout (Lay) so the fine-level sweep
//    can load its tiles by TMA; the boundary packs / unpacks the reference's
//    dense layout;
//  * PCG scalars never leave the device inside an iteration; the host reads a
//    status block every opt.check_every iterations (the reference copies each
//    dot product back, :1033-1041);
//  * level 1 stores the quadrature operator, levels >= 2 the Galerkin
//    operator, both packed [300][nel] (structure of arrays, coalesced);
//  * the coarsest solve is two dense triangular products with the explicitly
//    inverted Cholesky factor instead of 2n single-block launches (:2175-2232);
//  * fixed dofs are a per-node bit mask on every level instead of index lists
//    built with atomics (:747-790).
#include "solver.h"

#include <type_traits>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace gputo {

static int checked_malloc(void **p, size_t bytes, size_t &total)
{
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        set_error(std::string("cudaMalloc of ") + std::to_string(bytes) + " bytes failed: " +
                  cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? GPUTO_ERR_OOM : GPUTO_ERR_CUDA;
    }
    total += bytes;
    return GPUTO_OK;
}

// Allocate, zero (padding must read as zero) and remember for release.
#define ALLOC(ptr, count)                                                                   \
    do {                                                                                    \
        const size_t _b = sizeof(*(ptr)) * (size_t)(count);                                 \
        int _st = checked_malloc((void **)&(ptr), _b, bytes);                               \
        if (_st) return _st;                                                                \
        owned.push_back((void *)(ptr));                                                     \
        GPUTO_CUDA(cudaMemsetAsync((void *)(ptr), 0, _b ? _b : 16, own_stream));             \
    } while (0)

Solver::~Solver()
{
    if (own_stream) cudaStreamSynchronize(own_stream);
    for (void *p : owned) cudaFree(p);
    drop_graphs();
    if (h_sc) cudaFreeHost(h_sc);
    if (own_stream) cudaStreamDestroy(own_stream);
}

template <typename T>
int Solver::alloc_levels(LevelBuf<T> *Lv, bool with_matrices)
{
    for (int l = 0; l < nl; ++l) {
        LevelBuf<T> &b = Lv[l];
        b.g = g[l];
        const long long nv = lay[l].size();
        ALLOC(b.u0, nv);
        ALLOC(b.r, nv);
        ALLOC(b.diag, nv);
        ALLOC(b.rdiag, nv);
        ALLOC(b.u1, nv);
        ALLOC(b.f, nv);
        // level 1 is applied matrix-free unless it is the coarsest level; the
        // re-discretised hierarchy stores element matrices for the coarsest only
        if (redisc()) {
            if (l > 0 && l == nl - 1 && with_matrices) ALLOC(b.Apk, 300 * g[l].nel());
            b.mask = mask[l];
            continue;
        }
        if (l > 0 && with_matrices && !(l == 1 && quad_level1())) ALLOC(b.Apk, 300 * g[l].nel());
        if (l >= 1 && (l == 1 ? quad_level1() : g[l].nel() >= kElementCentricMinElems))
            ALLOC(b.yq, 24 * g[l].nel());
        b.mask = mask[l];
    }
    return GPUTO_OK;
}

int Solver::create(int nelx, int nely, int nelz, int nl_, const gputo_options *o)
{
    if (o) opt = *o;
    else gputo_default_options(&opt);
    if (nl_ < 1 || nl_ > kMaxLevels || nelx < 1 || nely < 1 || nelz < 1) {
        set_error("grid sizes must be positive and 1 <= nl <= 12");
        return GPUTO_ERR_ARG;
    }
    if (nelx > 65534) {   // the transfer kernels take one row of CTAs per x node plane
        set_error("nelx must be at most 65534");
        return GPUTO_ERR_ARG;
    }
    const int m = 1 << (nl_ - 1);
    if (nelx % m || nely % m || nelz % m) {
        set_error("nelx, nely, nelz must be divisible by 2^(nl-1)");
        return GPUTO_ERR_ARG;
    }
    if (opt.nswp < 0 || opt.nswp_fine < 0 || opt.nswp_coarse < 0 || opt.coarse_from < 0 || opt.coarse_from == 1 ||
        opt.check_every < 1 || !(opt.omega > 0) ||
        opt.tc_parts < 0 ||
        (opt.sweep_xchunk != 0 && (opt.sweep_xchunk < 8 || opt.sweep_xchunk > 32)) ||
        opt.sweep_pairs < 0 || opt.sweep_pairs > 1 ||
        opt.tc_parts > 2 ||
        opt.tc_xchunk < 0 || (opt.coarse != GPUTO_COARSE_GALERKIN && opt.coarse != GPUTO_COARSE_REDISCRETIZED) ||
        (opt.precision != GPUTO_PREC_FP64 && opt.precision != GPUTO_PREC_MIXED)) {
        set_error("invalid solver options");
        return GPUTO_ERR_ARG;
    }
    nl = nl_;
    for (int l = 0; l < nl; ++l) {
        g[l] = Grid{nelx >> l, nely >> l, nelz >> l};
        lay[l] = Lay::of(g[l]);
    }
    elay = ELay::of(g[0]);
    nc = (int)g[nl - 1].ndof();
    if (nc > opt.max_coarse_dofs) {
        set_error("coarsest grid has " + std::to_string(nc) + " dofs, above max_coarse_dofs=" +
                  std::to_string(opt.max_coarse_dofs) + "; use more levels");
        return GPUTO_ERR_ARG;
    }
    GPUTO_CUDA(cudaGetDevice(&device));
    GPUTO_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    int ik = init_fine_kernels();
    if (!ik) ik = init_hsweep_kernels();
    if (!ik && opt.precision == GPUTO_PREC_MIXED) ik = init_tc_sweep_kernels();
    if (ik) return ik;

    const long long nv = lay[0].size(), ne = g[0].nel();
    for (int l = 0; l < nl; ++l) {
        ALLOC(mask[l], (g[l].nnod() + 3) & ~3LL);
        ALLOC(maskp[l], hsweep_mask_bytes(g[l]));
    }
    ALLOC(CX, ne);
    ALLOC(CXp, elay.size());
    ALLOC(R, nv);
    ALLOC(P, nv);
    ALLOC(Q, nv);
    ALLOC(Z, nv);
    ALLOC(Uw, nv);
    ALLOC(Fw, nv);
    ALLOC(Dn, g[0].ndof());
    if (opt.precision == GPUTO_PREC_MIXED) {
        ALLOC(Zold, nv);
        ALLOC(Zold32, nv);
    }
    if (redisc())
        for (int l = 1; l < nl; ++l) {
            elayr[l] = ELay::of(g[l]);
            ALLOC(CXr[l], g[l].nel());
            if (l < nl - 1) {
                ALLOC(CXrp[l], elayr[l].size());
                if (opt.precision == GPUTO_PREC_MIXED) ALLOC(CXrpf[l], elayr[l].size());
            }
        }
    int st = alloc_levels<double>(L, true);
    if (st) return st;
    if (opt.precision == GPUTO_PREC_MIXED) {
        st = alloc_levels<float>(Lf, true);
        if (st) return st;
        ALLOC(CXpf, elay.size());
        if (nl >= 3) {
            nd = NetDims{g[2].nx + 1, g[2].nz + 1, g[2].ny + 1};
            ALLOC(net_x, 4 * nd.n());
            ALLOC(net_y, 3 * nd.n());
            ALLOC(dens2, nd.n());
            ALLOC(net_s, 4);
        }
    }
    ALLOC(AQ, (long long)nc * nc);
    ALLOC(Linv, (long long)nc * nc);
    ALLOC(LinvT, (long long)nc * nc);
    ALLOC(ctmp, nc);
    if (nl == 1) ALLOC(Apk0, 300 * g[0].nel());
    // the smallest x chunk an option may ask for gives the most CTAs
    partial_cap = std::max({fine_sweep_blocks(g[0]), hsweep_blocks<double>(g[0], MODE_APPLY, 8),
                            2 * hsweep_blocks<float>(g[0], MODE_JACOBI_DOT, 8),
                            2 * hsweep_blocks<float>(g[0], MODE_JACOBI_DOT, 0),
                            2 * hsweep_blocks<float>(g[0], MODE_JACOBI_DOT, 8, true),
                            2 * hsweep_blocks<float>(g[0], MODE_JACOBI_DOT, 0, true),
                            2 * hsweep_blocks<double>(g[0], MODE_ENERGY), 1 << 12});
    ALLOC(partial, partial_cap);
    ALLOC(ticket, 4);
    ALLOC(sc, 1);
    ALLOC(e2, 2);
    ALLOC(info, 4);
    ALLOC(err, 4);
    ALLOC(fixed_dev, 1);
    GPUTO_CUDA(cudaMallocHost((void **)&h_sc, sizeof(PcgScalars)));
    GPUTO_CUDA(cudaStreamSynchronize(own_stream));
    return GPUTO_OK;
}

int Solver::set_problem(const double *Ke0, const double *fixed1b, int nfd, cudaStream_t st)
{
    if (!Ke0 || (nfd > 0 && !fixed1b) || nfd < 0) {
        set_error("Ke0 and fixed must be given");
        return GPUTO_ERR_ARG;
    }
    const long long nd = g[0].ndof();
    for (int n = 0; n < nfd; ++n) {
        const double v = fixed1b[n];
        if (!(v >= 1.0 && v <= (double)nd) || v != std::floor(v)) {
            set_error("fixed dof index " + std::to_string(v) + " outside 1.." + std::to_string(nd));
            return GPUTO_ERR_ARG;
        }
    }
    for (int m = 0; m < 576; ++m) {
        if (!std::isfinite(Ke0[m])) {
            set_error("Ke0 has a non-finite entry");
            return GPUTO_ERR_ARG;
        }
    }
    // Ke0 may arrive in either storage order; it is symmetric in every driver,
    // and the gateway reads it as mgcg1.cu:131-133 does (element [24*i+j]).
    std::memcpy(Ke, Ke0, sizeof(Ke));
    int s1 = upload_fine_ke(Ke, st);
    if (s1) return s1;
    HadamardKe nhk;
    hadamard_ke(Ke, &nhk);
    if (nhk.ok != hk.ok || std::memcmp(nhk.c, hk.c, sizeof(hk.c)) != 0)
        drop_graphs();   // the captured sweeps carry the constants
    hk = nhk;
    s1 = upload_quadrature_parts(opt.nu, st);
    if (s1) return s1;
    // the fixed list: unchanged lists are not re-uploaded
    std::vector<double> list(fixed1b, fixed1b + nfd);
    if (list != fixed_host || !have_problem) {
        if ((long long)list.size() > fixed_cap) {
            cudaStreamSynchronize(st);
            cudaFree(fixed_dev);
            owned.erase(std::find(owned.begin(), owned.end(), (void *)fixed_dev));
            fixed_dev = nullptr;
            ALLOC(fixed_dev, list.size());
            fixed_cap = (long long)list.size();
            GPUTO_CUDA(cudaStreamSynchronize(own_stream));
        }
        if (nfd > 0)
            GPUTO_CUDA(cudaMemcpyAsync(fixed_dev, list.data(), sizeof(double) * nfd,
                                       cudaMemcpyHostToDevice, st));
        launch_mask_from_list((g[0].nnod() + 3) & ~3LL, fixed_dev, nfd, mask[0], st);
        for (int l = 1; l < nl; ++l) launch_mask_restrict(g[l], mask[l - 1], mask[l], st);
        for (int l = 0; l < nl; ++l) launch_pad_mask(g[l], mask[l], maskp[l], st);
        GPUTO_CUDA(cudaStreamSynchronize(st));
        fixed_host.swap(list);
    }
    have_problem = true;
    return GPUTO_OK;
}

int Solver::check_error_flags(cudaStream_t st)
{
    int h_err = 0;
    GPUTO_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    if (h_err) {
        set_error(h_err == GPUTO_ERR_TIMEOUT ? "a bounded wait for a TMA tile load gave up"
                                             : "a fine sweep found its shared memory misaligned for TMA");
        cudaMemsetAsync(err, 0, sizeof(int), st);
        return h_err;
    }
    return GPUTO_OK;
}

int Solver::setup(const double *CX_in, cudaStream_t st)
{
    const int s = setup_enqueue(CX_in, st);
    return s ? s : setup_finish(st);
}

int Solver::setup_enqueue(const double *CX_in, cudaStream_t st)
{
    if (!have_problem) {
        set_error("gputo_solver_set_problem must come before setup");
        return GPUTO_ERR_ARG;
    }
    ready = false;
    have_solution = false;
    const long long ne = g[0].nel();
    if (CX_in != CX)
        GPUTO_CUDA(cudaMemcpyAsync(CX, CX_in, sizeof(double) * ne, cudaMemcpyDeviceToDevice, st));
    launch_pack_cx<double>(elay, CX, CXp, st);
    launch_diag_fine(lay[0], CX, L[0].diag, st);
    for (int l = 1; l < nl && redisc(); ++l) {
        launch_coarse_cx(g[l], l == 1 ? CX : CXr[l - 1], CXr[l], st);
        launch_diag_fine(lay[l], CXr[l], L[l].diag, st);
        if (l < nl - 1) launch_pack_cx<double>(elayr[l], CXr[l], CXrp[l], st);
        else launch_dense_fine(g[l], CXr[l], L[l].Apk, st);
    }
    for (int l = 1; l < nl && !redisc(); ++l) {
        if (l == 1 && quad_level1()) {
            launch_diag_quad(lay[1], CX, L[1].diag, st);
            continue;
        }
        if (l == 1) launch_build_level1(g[1], CX, L[1].Apk, st);
        else if (l == 2 && quad_level1()) launch_build_galerkin_from_quad(g[2], CX, L[2].Apk, st);
        else launch_build_galerkin(g[l], L[l - 1].Apk, L[l].Apk, st);
        if (l == nl - 1) launch_coarsest_penalty(g[l], mask[l], L[l].Apk, st);
        launch_diag_packed<double>(lay[l], L[l].Apk, L[l].diag, st);
    }
    const double *Acoarse = (nl > 1) ? L[nl - 1].Apk : Apk0;
    if (nl == 1) {
        launch_dense_fine(g[0], CX, Apk0, st);
        if (!redisc()) launch_coarsest_penalty(g[0], mask[0], Apk0, st);
    }
    launch_assemble_dense(g[nl - 1], Acoarse, AQ, st);
    if (redisc()) launch_dense_fix(g[nl - 1], mask[nl - 1], AQ, st);
    launch_cholesky(nc, AQ, info, st);
    launch_tri_inverse(nc, AQ, Linv, LinvT, st);
    if (opt.precision == GPUTO_PREC_MIXED) {
        if (dens2) launch_net_density(g[2], g[0], CX, dens2, st);
        launch_pack_cx<float>(elay, CX, CXpf, st);
        for (int l = 1; l < nl - 1 && redisc(); ++l) launch_pack_cx<float>(elayr[l], CXr[l], CXrpf[l], st);
        launch_cast_f32(lay[0].size(), L[0].diag, Lf[0].diag, st);
        for (int l = 1; l < nl; ++l) {
            if (L[l].Apk) launch_cast_f32(300 * g[l].nel(), L[l].Apk, Lf[l].Apk, st);
            launch_cast_f32(lay[l].size(), L[l].diag, Lf[l].diag, st);
        }
        for (int l = 0; l < nl; ++l)
            if (Lf[l].rdiag) launch_recip<float>(lay[l].size(), L[l].diag, Lf[l].rdiag, st);
    }
    for (int l = 0; l < nl; ++l)
        if (L[l].rdiag) launch_recip<double>(lay[l].size(), L[l].diag, L[l].rdiag, st);
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

int Solver::setup_finish(cudaStream_t st)
{
    int h_info = 0;
    GPUTO_CUDA(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    if (h_info) {
        set_error("coarsest-grid Cholesky met a non-positive pivot at row " + std::to_string(h_info));
        return GPUTO_ERR_NOT_SPD;
    }
    ready = true;
    return GPUTO_OK;
}

// V-cycle z = M r (mgcg1.cu:468-651): pre-smoothing with the initial guess
// prerelax*F/diag, nswp damped-Jacobi sweeps, defect, restriction; coarsest
// direct solve; prolongation, nswp sweeps.  The smoother ping-pongs between
// two buffers; the schedule is arranged so that every level's result lands
// in its second buffer (bufs[1]), which for level 0 is z itself.
template <typename T>
void Solver::vcycle_impl(LevelBuf<T> *Lv, const T *CXl, const T *r0, T *z0, const int *done,
                         cudaStream_t st, const double *dotR, const T *dotZold, double *dotPartial)
{
    const T om = (T)opt.omega, pr = (T)opt.prerelax;
    auto sweep = [&](int l, int mode, const T *u, const T *f, T *out, T w) {
        if (l == 0) {
            if constexpr (std::is_same<T, float>::value) {
                if (opt.tc_parts > 0) {
                    note(launch_tc_sweep(opt.tc_parts, mode, lay[0], elay, CXl, u, f, Lv[0].diag, mask[0], out, w,
                                         pr, opt.tc_xchunk, done, err, st));
                    return;
                }
            }
            note(fine_sweep<T>(0, mode, lay[0], elay, CXl, u, f, Lv[0], out, w, pr, nullptr, done, st));
        }
        else if (redisc()) {
            const T *cxl;
            if constexpr (std::is_same<T, float>::value) cxl = CXrpf[l];
            else cxl = CXrp[l];
            note(fine_sweep<T>(l, mode, lay[l], elayr[l], cxl, u, f, Lv[l], out, w, pr, nullptr, done, st));
        } else if (l == 1 && quad_level1())
            note(launch_quad_sweep<T>(mode, lay[1], elay, CXl, u, f, Lv[1].rdiag, mask[1], out, w, pr,
                                      opt.nu, Lv[1].yq, done, err, st));
        else if (Lv[l].yq)
            launch_packed_sweep_ec<T>(mode, lay[l], Lv[l].Apk, u, f, Lv[l].rdiag, mask[l], out, w, pr,
                                      Lv[l].yq, done, st);
        else
            launch_packed_sweep<T>(mode, lay[l], Lv[l].Apk, u, f, Lv[l].rdiag, mask[l], out, w, pr, done,
                                   st);
    };
    auto bufs = [&](int l, int which) -> T * {
        if (l == 0) return which ? z0 : Lv[0].u0;
        return which ? Lv[l].u1 : Lv[l].u0;
    };
    for (int l = 0; l < nl; ++l) {
        const int ns = sweeps(l);
        const T *f = (l == 0) ? r0 : Lv[l].f;
        if (l > 0) launch_restrict<T>(lay[l], lay[l - 1], Lv[l - 1].r, mask[l], Lv[l].f, done, st);
        if (l < nl - 1) {
            if (ns == 0) {
                sweep(l, MODE_JACOBI_PRE, nullptr, f, bufs(l, 1), T(0));  // U = prerelax F / diag
            } else {
                for (int s = 0; s < ns; ++s)
                    sweep(l, s == 0 ? MODE_JACOBI_PRE : MODE_JACOBI, s == 0 ? nullptr : bufs(l, (s - 1) & 1),
                          f, bufs(l, s & 1), om);
            }
            const T *upre = (ns == 0) ? bufs(l, 1) : bufs(l, (ns - 1) & 1);
            sweep(l, MODE_DEFECT, upre, f, Lv[l].r, om);
        } else {
            launch_coarse_solve<T>(lay[l], Linv, LinvT, f, bufs(l, 1), ctmp, done, st);
        }
    }
    for (int l = nl - 2; l >= 0; --l) {
        const int ns = sweeps(l);
        const T *f = (l == 0) ? r0 : Lv[l].f;
        int cur = (ns == 0) ? 1 : ((ns - 1) & 1);
        // the fine level's first post-smoothing sweep forms u + P e_c itself
        bool pro = opt.fuse_prolong && l == 0 && ns >= 1 && !(ns == 1 && dotR) && use_hsweep<T>(g[0]) &&
                   Lv[0].rdiag && hsweep_pro_fits<T>(g[0]);
        if constexpr (std::is_same<T, float>::value) pro = pro && opt.tc_parts == 0;
        if (!pro) launch_prolong_add<T>(lay[l], lay[l + 1], bufs(l + 1, 1), mask[l], bufs(l, cur), done, st);
        for (int s = 0; s < ns; ++s) {
            if (l == 0 && s == ns - 1 && dotR)   // the last sweep also sums r'z and r'z_old
                note(fine_sweep<T>(0, MODE_JACOBI_DOT, lay[0], elay, CXl, bufs(0, cur), f, Lv[0], bufs(0, cur ^ 1), om,
                                   pr, dotPartial, done, st, dotR, dotZold));
            else if (pro && s == 0)
                note(fine_sweep<T>(0, MODE_JACOBI_PRO, lay[0], elay, CXl, bufs(0, cur), f, Lv[0], bufs(0, cur ^ 1), om,
                                   pr, nullptr, done, st, nullptr, nullptr, bufs(1, 1), &lay[1]));
            else
                sweep(l, MODE_JACOBI, bufs(l, cur), f, bufs(l, cur ^ 1), om);
            cur ^= 1;
        }
    }
}

void Solver::vcycle(const double *r, double *z, const int *done, cudaStream_t st)
{
    if (opt.precision == GPUTO_PREC_MIXED) {
        // FP32 V-cycle between FP64 vectors
        launch_convert<double, float>(lay[0].size(), r, Lf[0].f, done, st);
        vcycle_impl<float>(Lf, CXpf, Lf[0].f, Lf[0].u1, done, st);
        launch_convert<float, double>(lay[0].size(), Lf[0].u1, z, done, st);
        if (net_on) learned_correction(z, done, st);
    } else {
        vcycle_impl<double>(L, CXp, r, z, done, st);
    }
}

// z += P0 P1 e2 with e2 = s D2^-1/2 net(density, D2^-1/2 R1 R0 r / s) on level 2
// (D2 the level-2 diagonal, s the RMS of the scaled residual), after the
// FP32 V-cycle (which leaves float(r) in Lf[0].f and no longer needs its level
// 1/2 buffers).  Additive, so the preconditioner stays a function of r alone;
// the flexible PCG absorbs that it is not exactly symmetric.
void Solver::learned_correction(double *z, const int *done, cudaStream_t st)
{
    launch_restrict<float>(lay[1], lay[0], Lf[0].f, mask[1], Lf[1].f, done, st);
    launch_restrict<float>(lay[2], lay[1], Lf[1].f, mask[2], Lf[2].f, done, st);
    launch_net_features(lay[2], Lf[2].f, Lf[2].diag, dens2, net_x, nullptr, net_s, done, st);
    note(net->forward(net_x, nd, net_y, st));
    launch_net_output(lay[2], net_y, Lf[2].diag, net_s, mask[2], Lf[2].u0, done, st);
    cudaMemsetAsync(Lf[1].u0, 0, sizeof(float) * lay[1].size(), st);
    launch_prolong_add<float>(lay[1], lay[2], Lf[2].u0, mask[1], Lf[1].u0, done, st);
    cudaMemsetAsync(Lf[0].u0, 0, sizeof(float) * lay[0].size(), st);
    launch_prolong_add<float>(lay[0], lay[1], Lf[1].u0, mask[0], Lf[0].u0, done, st);
    launch_add_f2d(lay[0].size(), Lf[0].u0, z, done, st);
}

void Solver::apply_level_f32(int l, const float *u, float *out, cudaStream_t st)
{
    if (Lf[l].yq)
        launch_packed_sweep_ec<float>(MODE_APPLY, lay[l], Lf[l].Apk, u, nullptr, Lf[l].rdiag, mask[l], out, 1.f, 0.f,
                                      Lf[l].yq, nullptr, st);
    else
        launch_packed_sweep<float>(MODE_APPLY, lay[l], Lf[l].Apk, u, nullptr, Lf[l].rdiag, mask[l], out, 1.f, 0.f,
                                   nullptr, st);
}

// Energy loss L = y'A~y - 2 y'g~ per sample (see launch_net_energy), summed
// over the samples; Adam with the mean gradient when lr > 0.  Uses Lf[2].u0/u1
// as scratch: not during a solve.
int Solver::net_train_energy(Net *n, const float *x, const float *gt, int ns, float lr, double *loss,
                             float *grads_out, cudaStream_t st)
{
    if (!n || !net_x || ns < 1 || redisc()) return GPUTO_ERR_ARG;
    int s = init_net_kernels();
    if (!s) s = n->reserve(nd.n());
    if (s) return s;
    const long long nn = nd.n();
    GPUTO_CUDA(cudaMemsetAsync(n->loss_acc, 0, sizeof(double), st));
    for (int q = 0; q < ns; ++q) {
        s = n->forward(x + (size_t)q * 4 * nn, nd, nullptr, st);
        if (s) return s;
        launch_net_to_padded(lay[2], n->act[4], Lf[2].diag, mask[2], Lf[2].u0, st);
        apply_level_f32(2, Lf[2].u0, Lf[2].u1, st);
        s = launch_net_energy(lay[2], n->act[4], Lf[2].u1, Lf[2].diag, gt + (size_t)q * 3 * nn, mask[2], n->gA,
                              n->part, 2048, n->loss_acc, st);
        if (!s) s = n->backward_from(nd, st);
        if (s) return s;
    }
    if (grads_out)
        GPUTO_CUDA(cudaMemcpyAsync(grads_out, n->grads, sizeof(float) * Net::num_params(), cudaMemcpyDeviceToHost, st));
    if (lr > 0.f) {
        s = n->adam(lr, ns, st);
        if (s) return s;
    } else {
        GPUTO_CUDA(cudaMemsetAsync(n->grads, 0, sizeof(float) * Net::num_params(), st));
    }
    double l = 0.0;
    GPUTO_CUDA(cudaMemcpyAsync(&l, n->loss_acc, sizeof(double), cudaMemcpyDeviceToHost, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    GPUTO_CUDA(cudaGetLastError());
    if (loss) *loss = l / ns;
    return GPUTO_OK;
}

int Solver::attach_net(Net *n, int mode)
{
    if (n && (opt.precision != GPUTO_PREC_MIXED || nl < 3 || !net_x || redisc())) {
        set_error("the learned correction needs precision GPUTO_PREC_MIXED, nl >= 3 and Galerkin coarse levels");
        return GPUTO_ERR_ARG;
    }
    if (mode < 0 || mode > 2) {
        set_error("net mode must be 0 (off), 1 (on) or 2 (auto)");
        return GPUTO_ERR_ARG;
    }
    if (n) {
        int d = 0;
        GPUTO_CUDA(cudaGetDevice(&d));
        if (d != n->device) {
            set_error("the network lives on another device");
            return GPUTO_ERR_ARG;
        }
        // everything the captured iteration needs exists before any capture
        int s = init_net_kernels();
        if (!s) s = n->reserve(nd.n());
        if (s) return s;
    }
    net = n;
    net_mode = n ? mode : 0;
    ref_plain_nit = ref_net_nit = -1;
    net_solves = 0;
    const bool want = net_mode == 1;
    if (want != net_on) drop_graphs();
    net_on = want;
    return GPUTO_OK;
}

void Solver::apply(const double *u, double *r, double *dot_partial, const int *done, cudaStream_t st)
{
    note(fine_sweep<double>(0, MODE_APPLY, lay[0], elay, CXp, u, nullptr, L[0], r, 1.0, 0.0, dot_partial, done, st));
}

// One PCG iteration (mgcg1.cu:254-275), every scalar on the device.
void Solver::iteration(cudaStream_t st)
{
    const long long nv = lay[0].size();
    const int *done = &sc->done;
    apply(P, Q, partial, done, st);
    launch_finish_apply_dot(apply_blocks(), partial, ticket, sc, st);
    if (opt.precision == GPUTO_PREC_MIXED && !net_on) {
        // float(r) comes from the residual update and z stays the FP32
        // V-cycle output: no precision-conversion passes
        launch_pcg_update(nv, R, Q, partial, ticket, sc, st, Lf[0].f);
        if (fused_dot()) {
            vcycle_impl<float>(Lf, CXpf, Lf[0].f, Lf[0].u1, done, st, R, Zold32, partial);
            launch_finish_dot2(hsweep_blocks<float>(g[0], MODE_JACOBI_DOT, opt.sweep_xchunk, opt.sweep_pairs != 0),
                               partial, sc, st);
        } else {
            vcycle_impl<float>(Lf, CXpf, Lf[0].f, Lf[0].u1, done, st);
            launch_dot2<float>(nv, R, Lf[0].u1, Zold32, partial, ticket, sc, done, st);
        }
        launch_p_update<float>(nv, Lf[0].u1, P, Zold32, Uw, sc, st);
        return;
    }
    launch_pcg_update(nv, R, Q, partial, ticket, sc, st);
    vcycle(R, Z, done, st);
    if (Zold) {
        launch_dot2<double>(nv, R, Z, Zold, partial, ticket, sc, done, st);
        launch_p_update<double>(nv, Z, P, Zold, Uw, sc, st);
    } else {
        launch_dot(nv, R, Z, partial, ticket, sc, 2 /*DOT_RZ*/, done, st);
        launch_p_update<double>(nv, Z, P, nullptr, Uw, sc, st);
    }
}

int Solver::solve_begin(const double *Fp, double tol, int maxit, cudaStream_t st)
{
    if (!ready) {
        set_error("solver setup has not succeeded");
        return GPUTO_ERR_ARG;
    }
    if (maxit < 0 || !(tol >= 0)) {
        set_error("maxit must be >= 0 and tol >= 0");
        return GPUTO_ERR_ARG;
    }
    launch_status = GPUTO_OK;
    // auto mode: measure a plain solve and a solve with the network, keep
    // whichever needed fewer iterations, re-measure the other every 8 solves
    if (net && net_mode == 2) {
        bool want;
        if (ref_plain_nit < 0) want = false;
        else if (ref_net_nit < 0) want = true;
        else {
            want = ref_net_nit < ref_plain_nit;
            if (net_solves % 8 == 7) want = !want;
        }
        if (want != net_on) drop_graphs();
        net_on = want;
    }
    const long long nv = lay[0].size();
    const int *done = &sc->done;
    launch_pcg_init(nv, Fp, Uw, R, partial, ticket, sc, tol, maxit, opt.precision == GPUTO_PREC_MIXED, st);
    vcycle(R, P, done, st);
    launch_dot(nv, R, P, partial, ticket, sc, 1 /*DOT_RHO0*/, done, st);
    if (Zold) launch_copy(nv, P, Zold, done, st);
    if (Zold32 && !net_on)   // the FP32 V-cycle output of the first step, for the fast iteration
        GPUTO_CUDA(cudaMemcpyAsync(Zold32, Lf[0].u1, sizeof(float) * nv, cudaMemcpyDeviceToDevice, st));
    return launch_status;
}

// Device scalars -> host (h_sc); true once the solve has converged or failed.
int Solver::solve_poll(cudaStream_t st, bool *finished)
{
    GPUTO_CUDA(cudaMemcpyAsync(h_sc, sc, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    *finished = h_sc->done != 0;
    return GPUTO_OK;
}

int Solver::solve_end(double *Up, double *relres, int *nit, cudaStream_t st)
{
    launch_flush_x(lay[0].size(), Uw, P, sc, st);   // the last iteration's U update, if still pending
    GPUTO_CUDA(cudaGetLastError());
    if (Up != Uw)
        GPUTO_CUDA(cudaMemcpyAsync(Up, Uw, sizeof(double) * lay[0].size(), cudaMemcpyDeviceToDevice, st));
    int fe = check_error_flags(st);
    if (fe) return fe;
    *relres = h_sc->relres;
    *nit = h_sc->nit;
    last_res0 = h_sc->res0;
    if (net && net_mode == 2) {
        (net_on ? ref_net_nit : ref_plain_nit) = h_sc->nit;
        ++net_solves;
    }
    if (h_sc->status) {
        if (!std::isfinite(h_sc->res0))
            set_error("PCG breakdown: the right-hand side F has a non-finite entry");
        else
            set_error("PCG breakdown: p'q <= 0 or a non-finite scalar at iteration " + std::to_string(h_sc->nit));
        return h_sc->status;
    }
    return GPUTO_OK;
}

int Solver::solve(const double *Fp, double *Up, double tol, int maxit, double *relres, int *nit,
                  cudaStream_t st, FILE *log)
{
    int s = solve_begin(Fp, tol, maxit, st);
    if (s) return s;
    const bool graph = opt.use_graph != 0;
    int it = 0;
    for (;;) {
        bool fin = false;
        s = solve_poll(st, &fin);
        if (s) return s;
        if (log && it > 0) std::fprintf(log, "CG It %d  %12.6g\n", h_sc->iter - 1, h_sc->relres);
        if (fin || it >= maxit) break;
        const int batch = std::min(opt.check_every, maxit - it);
        if (graph) {
            int gs = run_graph(batch, st);
            if (gs) return gs;
        } else {
            for (int b = 0; b < batch; ++b) iteration(st);
            if (launch_status) return launch_status;
        }
        it += batch;
    }
    return solve_end(Up, relres, nit, st);
}

// The last solve's U: element energies ce (dc = dsK ce), the compliance
// sum CX_e ce_e and |F - K U|^2 over the free dofs, from one FP64 operator
// apply with the energies in its epilogue (Hadamard-basis kernel).  out2
// (device, 2 doubles) receives (|F - K U|^2, compliance).  Without the
// Hadamard-basis kernel: the separate energy pass, and out2[0] = -1.
int Solver::energy(const double *dsK, double *ce, double *dc, double *out2, cudaStream_t st)
{
    if (!ready) {
        set_error("solver setup has not succeeded");
        return GPUTO_ERR_ARG;
    }
    if (!ce || (dc && !dsK) || !out2) {
        set_error("energy needs ce, out2, and dsK with dc");
        return GPUTO_ERR_ARG;
    }
    launch_status = GPUTO_OK;
    if (use_hsweep<double>(g[0]) && hsweep_energy_fits(g[0])) {
        const int nb = hsweep_blocks<double>(g[0], MODE_ENERGY);
        note(launch_hsweep_energy(lay[0], elay, hk, CXp, Uw, Fw, mask[0], maskp[0], nullptr, partial, ce, dc, dsK,
                                  err, st));
        if (launch_status) return launch_status;
        launch_sum_pairs(nb, partial, out2, st);
    } else {
        launch_unpack(lay[0], Uw, Dn, 0, st);
        launch_element_energy(g[0], Dn, CX, dsK, ce, dc, partial, ticket, out2 + 1, st);
        const double minus1 = -1.0;
        GPUTO_CUDA(cudaMemcpyAsync(out2, &minus1, sizeof(double), cudaMemcpyHostToDevice, st));
    }
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}

// Options that change neither the hierarchy nor its buffers.
int Solver::set_tunables(const gputo_options &o)
{
    if (o.nswp < 0 || o.nswp_fine < 0 || o.nswp_coarse < 0 || o.coarse_from < 0 || o.coarse_from == 1 ||
        o.check_every < 1 || !(o.omega > 0) || o.tc_parts < 0 ||
        o.tc_parts > 2 ||
        (o.sweep_xchunk != 0 && (o.sweep_xchunk < 8 || o.sweep_xchunk > 32)) ||
        o.sweep_pairs < 0 || o.sweep_pairs > 1 ||
        o.tc_xchunk < 0 ||
        o.fine_op < 0 || o.fine_op > 1 ||
        (o.tc_parts > 0 && opt.precision != GPUTO_PREC_MIXED)) {
        set_error("invalid solver options");
        return GPUTO_ERR_ARG;
    }
    opt.nswp = o.nswp;
    opt.nswp_fine = o.nswp_fine;
    opt.nswp_coarse = o.nswp_coarse;
    opt.coarse_from = o.coarse_from;
    opt.fuse_prolong = o.fuse_prolong;
    opt.sweep_xchunk = o.sweep_xchunk;
    opt.sweep_pairs = o.sweep_pairs;
    opt.omega = o.omega;
    opt.prerelax = o.prerelax;
    opt.check_every = o.check_every;
    opt.use_graph = o.use_graph;
    opt.tc_parts = o.tc_parts;
    opt.tc_xchunk = o.tc_xchunk;
    opt.fine_op = o.fine_op;
    drop_graphs();
    return GPUTO_OK;
}

void Solver::drop_graphs()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph_exec_n) cudaGraphExecDestroy(graph_exec_n);
    graph_exec = graph_exec_n = nullptr;
    graph_n = 0;
}

// 'iters' PCG iterations captured back to back into one executable graph
// (all pointers are solver-owned, all scalars device-resident; iteration()
// keeps no host state, so the capture equals 'iters' replays of one).
int Solver::capture_iterations(int iters, cudaStream_t st, cudaGraphExec_t *exec)
{
    cudaGraph_t gr;
    launch_status = GPUTO_OK;
    GPUTO_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    for (int b = 0; b < iters; ++b) iteration(st);
    GPUTO_CUDA(cudaStreamEndCapture(st, &gr));
    if (launch_status) {
        cudaGraphDestroy(gr);
        return launch_status;
    }
    cudaError_t e = cudaGraphInstantiate(exec, gr, 0);
    cudaGraphDestroy(gr);
    GPUTO_CUDA(e);
    return GPUTO_OK;
}

// 'batch' iterations between host checks: one launch of a graph that holds
// them all (no graph boundary between iterations); a shorter last batch
// replays the one-iteration graph.
int Solver::run_graph(int batch, cudaStream_t st)
{
    if (graph_stream != st) drop_graphs();
    graph_stream = st;
    if (batch > 1 && batch == opt.check_every) {
        if (!graph_exec_n || graph_n != batch) {
            if (graph_exec_n) cudaGraphExecDestroy(graph_exec_n);
            graph_exec_n = nullptr;
            graph_n = 0;
            const int s = capture_iterations(batch, st, &graph_exec_n);
            if (s) return s;
            graph_n = batch;
        }
        GPUTO_CUDA(cudaGraphLaunch(graph_exec_n, st));
        return GPUTO_OK;
    }
    if (!graph_exec) {
        const int s = capture_iterations(1, st, &graph_exec);
        if (s) return s;
    }
    for (int b = 0; b < batch; ++b) GPUTO_CUDA(cudaGraphLaunch(graph_exec, st));
    return GPUTO_OK;
}

template int Solver::alloc_levels<double>(LevelBuf<double> *, bool);
template int Solver::alloc_levels<float>(LevelBuf<float> *, bool);

}  // namespace gputo
