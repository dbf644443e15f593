// Multigrid kernels for the coarse levels: operator sweeps on packed element
// matrices, grid transfers, hierarchy setup and the coarsest direct solve.
//
// Every operator kernel is a node-centred gather over the (up to) 8 elements
// around a node, as the reference's defectc
// (Cantilever/TOP3D125MGCGCUDA/mgcg1.cu:1266-1324): one thread owns a node's
// three rows, so no atomics are needed, and the damped Jacobi update
// (:1199-1206) and Dirichlet zeroing (ZeroBCc, :1326-1331) are fused into the
// epilogue.  Vectors use the padded row layout (Lay); element arrays keep the
// reference's element order.
#include <algorithm>

#include "gputo_internal.h"

namespace gputo {

// Level-1 quadrature parts: Kg[g] packed (300), g = 4 ix + 2 iz + iy.
__constant__ double cKg[8 * 300];
// Prolongation weights of a coarse element onto its 8 children:
// cPc[c][b][a] = weight of coarse local node a at child c's local node b.
__constant__ double cPc[8 * 8 * 8];

// ---------------------------------------------------------------------------
// host-side element algebra for the constant tables
// ---------------------------------------------------------------------------

// B^T D B at one Gauss point of an h*h*h hex, E=1 (the integrand of
// mgcg1.c:1370-1418 Kem3 and mgcg1.cu:2000-2040 prepAelm).
void gauss_part(double nu, double h, int ix, int iy, int iz, double K[24][24])
{
    const double gp[2] = {-0.5773502691896257645, 0.5773502691896257645};
    const double s = gp[ix], e = gp[iy], t = gp[iz];
    double B[6][24] = {};
    for (int a = 0; a < 8; ++a) {
        const double xa = 2 * local_x(a) - 1, ya = 2 * local_y(a) - 1, za = 2 * local_z(a) - 1;
        const double fx = 1 + xa * s, fy = 1 + ya * e, fz = 1 + za * t;
        const double dx = 0.25 * xa * fy * fz / h, dy = 0.25 * ya * fx * fz / h,
                     dz = 0.25 * za * fx * fy / h;
        B[0][3 * a] = dx;
        B[1][3 * a + 1] = dy;
        B[2][3 * a + 2] = dz;
        B[3][3 * a] = dy;
        B[3][3 * a + 1] = dx;
        B[4][3 * a + 1] = dz;
        B[4][3 * a + 2] = dy;
        B[5][3 * a] = dz;
        B[5][3 * a + 2] = dx;
    }
    const double c = 1.0 / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double D[6][6] = {};
    for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) D[p][q] = c * (p == q ? 1.0 - nu : nu);
    for (int p = 3; p < 6; ++p) D[p][p] = c * (1.0 - 2.0 * nu) / 2.0;
    const double w = h * h * h / 8.0;
    for (int m = 0; m < 24; ++m)
        for (int n = 0; n <= m; ++n) {
            double acc = 0.0;
            for (int p = 0; p < 6; ++p) {
                double db = 0.0;
                for (int q = 0; q < 6; ++q) db += D[p][q] * B[q][n];
                acc += B[p][m] * db;
            }
            K[m][n] = K[n][m] = w * acc;
        }
}

// Level-2 Galerkin blocks of the quadrature level: the 2h-element matrix of
// level 1 is sum_g CX_g Kg[g], so the level-2 element matrix is
//   A_E = sum_{c,g} CX(fine element g of level-1 child c) * Pc^T Kg[g] Pc,
// a fixed combination of 64 constant matrices Mq[c*8+g] = Pc^T Kg[g] Pc
// (packed, 300 each), weighted by the 64 fine densities under E.
static double *g_mq_dev[64] = {};
static double g_mq_nu[64];

const double *quad_galerkin_blocks(int dev) { return dev >= 0 && dev < 64 ? g_mq_dev[dev] : nullptr; }

int upload_quadrature_parts(double nu, cudaStream_t st)
{
    int dev = 0;
    GPUTO_CUDA(cudaGetDevice(&dev));
    if (dev < 64 && g_mq_dev[dev] && g_mq_nu[dev] == nu) return GPUTO_OK;   // per device
    static double kg[8 * 300];
    for (int ix = 0; ix < 2; ++ix)
        for (int iz = 0; iz < 2; ++iz)
            for (int iy = 0; iy < 2; ++iy) {
                double K[24][24];
                gauss_part(nu, 2.0, ix, iy, iz, K);
                const int g = 4 * ix + 2 * iz + iy;
                for (int m = 0; m < 24; ++m)
                    for (int n = 0; n <= m; ++n) kg[g * 300 + packed_index(m, n)] = K[m][n];
            }
    static double pc[512];
    for (int c = 0; c < 8; ++c)
        for (int b = 0; b < 8; ++b)
            for (int a = 0; a < 8; ++a) {
                const int px = local_x(c) + local_x(b), py = local_y(c) + local_y(b),
                          pz = local_z(c) + local_z(b);
                const double wx = 1.0 - 0.5 * abs(px - 2 * local_x(a));
                const double wy = 1.0 - 0.5 * abs(py - 2 * local_y(a));
                const double wz = 1.0 - 0.5 * abs(pz - 2 * local_z(a));
                pc[(c * 8 + b) * 8 + a] = (wx > 0 && wy > 0 && wz > 0) ? wx * wy * wz : 0.0;
            }
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(cKg, kg, sizeof(kg), 0, cudaMemcpyHostToDevice, st));
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(cPc, pc, sizeof(pc), 0, cudaMemcpyHostToDevice, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    const int s2 = upload_quadrature_fine(kg, st);   // the sweep kernels' copy
    if (s2) return s2;
    // Mq[c][g] = Pc^T Kg[g] Pc
    static double mq[64 * 300];
    for (int c = 0; c < 8; ++c)
        for (int gq = 0; gq < 8; ++gq)
            for (int m = 0; m < 24; ++m)
                for (int n = 0; n <= m; ++n) {
                    const int am = m / 3, p = m % 3, an = n / 3, q = n % 3;
                    double acc = 0.0;
                    for (int b = 0; b < 8; ++b) {
                        const double wb = pc[(c * 8 + b) * 8 + am];
                        if (wb == 0.0) continue;
                        for (int b2 = 0; b2 < 8; ++b2) {
                            const double wb2 = pc[(c * 8 + b2) * 8 + an];
                            if (wb2 == 0.0) continue;
                            acc += wb * wb2 * kg[gq * 300 + packed_index(3 * b + p, 3 * b2 + q)];
                        }
                    }
                    mq[(c * 8 + gq) * 300 + packed_index(m, n)] = acc;
                }
    if (dev < 64) {
        if (!g_mq_dev[dev]) GPUTO_CUDA(cudaMalloc(&g_mq_dev[dev], sizeof(mq)));
        GPUTO_CUDA(cudaMemcpyAsync(g_mq_dev[dev], mq, sizeof(mq), cudaMemcpyHostToDevice, st));
        GPUTO_CUDA(cudaStreamSynchronize(st));
        g_mq_nu[dev] = nu;
    }
    return GPUTO_OK;
}

// ---------------------------------------------------------------------------
// coarse-level sweep: packed element matrices [300][nel]
// ---------------------------------------------------------------------------

__device__ __forceinline__ void node_ijk(const Grid &g, long long n, int &i, int &j, int &k)
{
    const long long t = n / (g.ny + 1);
    j = (int)(n - t * (g.ny + 1));
    i = (int)(t / (g.nz + 1));
    k = (int)(t - (long long)i * (g.nz + 1));
}

template <typename T, int MODE>
__global__ void __launch_bounds__(128)
packed_sweep_kernel(Lay L, const T *__restrict__ A, const T *__restrict__ u,
                    const T *__restrict__ f, const T *__restrict__ rdiag,
                    const uint8_t *__restrict__ mask, T *__restrict__ out, T omega, T prerelax,
                    const int *__restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    const Grid &g = L.g;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    int i, j, k;
    node_ijk(g, n, i, j, k);
    const long long nel = g.nel();
    T acc[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int ex = 0; ex < 2; ++ex) {
        const int ei = i - 1 + ex;
        if (ei < 0 || ei >= g.nx) continue;
#pragma unroll
        for (int ez = 0; ez < 2; ++ez) {
            const int ek = k - 1 + ez;
            if (ek < 0 || ek >= g.nz) continue;
#pragma unroll
            for (int ey = 0; ey < 2; ++ey) {
                const int ej = j - 1 + ey;
                if (ej < 0 || ej >= g.ny) continue;
                const long long e = g.elem(ei, ej, ek);
                const int a = local_index(1 - ex, 1 - ey, 1 - ez);
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    const long long nb = L.at(ei + local_x(b), ej + local_y(b), ek + local_z(b));
                    T ub[3];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        const long long dof = nb + q;
                        ub[q] = (MODE == MODE_JACOBI_PRE) ? prerelax * f[dof] * rdiag[dof] : u[dof];
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d)
#pragma unroll
                        for (int q = 0; q < 3; ++q)
                            acc[d] = fma(A[(long long)packed_index(3 * a + d, 3 * b + q) * nel + e], ub[q], acc[d]);
                }
            }
        }
    }
    const unsigned m = mask[n];
    const long long base = L.at(i, j, k);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const long long dof = base + d;
        const bool fixed = (m >> d) & 1u;
        if (MODE == MODE_APPLY) {
            out[dof] = fixed ? T(0) : acc[d];
        } else if (MODE == MODE_DEFECT) {
            out[dof] = fixed ? T(0) : f[dof] - acc[d];
        } else {
            const T r = fixed ? T(0) : f[dof] - acc[d];
            const T us = (MODE == MODE_JACOBI_PRE) ? prerelax * f[dof] * rdiag[dof] : u[dof];
            out[dof] = us + omega * r * rdiag[dof];
        }
    }
}

// Small coarse levels: a CTA finishes 32 consecutive nodes.  Warp w takes
// element slot w (the element at offset (ex, ey, ez) = bits of w from each
// node) and lane l node n0 + l, so every load of a matrix entry
// A[row, col] reads 32 neighbouring elements (the [300][nel] layout is
// element-fastest): four 32-byte sectors per warp instead of 32.  The eight
// slot partials are summed in a fixed order through shared memory.
// Warp w takes element slot (ex, ez, ey) = bits of w of the 8 around each
// node.  The element matrices do not change during a solve, so a thread
// loads its slot's 72 entries first, then lets the next kernel in the stream
// launch (griddepcontrol.launch_dependents: its entry loads overlap this
// kernel's tail), and only then waits for its predecessor before it reads u,
// f or 1/diag.  Kernels before a sweep that write the matrices (the setup)
// never release their successors early, so they have completed by then.
template <typename T, int MODE>
__global__ void __launch_bounds__(256)
packed_sweep_slot_kernel(Lay L, const T *__restrict__ A, const T *__restrict__ u, const T *__restrict__ f,
                         const T *__restrict__ rdiag, const uint8_t *__restrict__ mask, T *__restrict__ out,
                         T omega, T prerelax, const int *__restrict__ done)
{
    __shared__ T part[8][32][3];
    const Grid &g = L.g;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long n = (long long)blockIdx.x * 32 + lane;
    const bool have = n < g.nnod();
    int i = 0, j = 0, k = 0;
    if (have) node_ijk(g, n, i, j, k);
    const int ex = (w >> 2) & 1, ez = (w >> 1) & 1, ey = w & 1;
    const int ei = i - 1 + ex, ej = j - 1 + ey, ek = k - 1 + ez;
    const bool slot = have && ei >= 0 && ei < g.nx && ej >= 0 && ej < g.ny && ek >= 0 && ek < g.nz;
    const long long nel = g.nel();
    const long long e = slot ? g.elem(ei, ej, ek) : 0;
    const int a = local_index(1 - ex, 1 - ey, 1 - ez);
    // FP32: all 72 entries in registers before the wait; FP64 loads them after
    // it (144 registers of entries would halve the CTAs per SM)
    constexpr bool EARLY = sizeof(T) == 4;
    T am[3][24];   // rows 3 a + d of the slot's element matrix
    auto load_entries = [&]() {
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int col = 0; col < 24; ++col)
                am[d][col] = slot ? A[(long long)packed_index(3 * a + d, col) * nel + e] : T(0);
    };
    if (EARLY) load_entries();
    pdl_trigger();
    pdl_wait();
    if (done && *done) return;
    if (!EARLY) load_entries();
    // warp 0's epilogue operands, loaded together with the products' inputs
    // instead of after the slot sum
    T fe[3] = {T(0), T(0), T(0)}, re[3] = {T(0), T(0), T(0)}, ue[3] = {T(0), T(0), T(0)};
    unsigned me = 0;
    if (w == 0 && have) {
        const long long base = L.at(i, j, k);
        me = mask[n];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (MODE != MODE_APPLY) fe[d] = f[base + d];
            if (MODE == MODE_JACOBI || MODE == MODE_JACOBI_PRE) re[d] = rdiag[base + d];
            if (MODE == MODE_JACOBI) ue[d] = u[base + d];
        }
    }
    T acc[3] = {T(0), T(0), T(0)};
    if (slot) {
        T ub[24];
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const long long nb = L.at(ei + local_x(b), ej + local_y(b), ek + local_z(b));
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (MODE == MODE_JACOBI_PRE) {
                    ub[3 * b + q] = prerelax * f[nb + q] * rdiag[nb + q];
                } else {
                    ub[3 * b + q] = u[nb + q];
                }
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int col = 0; col < 24; ++col) acc[d] = fma(am[d][col], ub[col], acc[d]);
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) part[w][lane][d] = acc[d];
    __syncthreads();
    if (w == 0 && have) {
        T s[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            s[d] = part[0][lane][d];
#pragma unroll
            for (int q = 1; q < 8; ++q) s[d] += part[q][lane][d];
        }
        const long long base = L.at(i, j, k);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const long long dof = base + d;
            const bool fixed = (me >> d) & 1u;
            if (MODE == MODE_APPLY) {
                out[dof] = fixed ? T(0) : s[d];
            } else if (MODE == MODE_DEFECT) {
                out[dof] = fixed ? T(0) : fe[d] - s[d];
            } else {
                const T r = fixed ? T(0) : fe[d] - s[d];
                T us;
                if (MODE == MODE_JACOBI_PRE) {
                    us = prerelax * fe[d] * re[d];
                } else {
                    us = ue[d];
                }
                out[dof] = us + omega * r * re[d];
            }
        }
    }
}

template <typename T>
void launch_packed_sweep(int mode, const Lay &L, const T *Apk, const T *u, const T *f,
                         const T *rdiag, const uint8_t *mask, T *out, T omega, T prerelax,
                         const int *done, cudaStream_t st)
{
    const int bs = 128;
    if (L.g.nnod() < 65536) {
        const unsigned sb = (unsigned)((L.g.nnod() + 31) / 32);
        switch (mode) {
        case MODE_APPLY:
            launch_pdl(packed_sweep_slot_kernel<T, MODE_APPLY>, dim3(sb), dim3(256), 0, st, L, Apk, u, f, rdiag, mask, out, omega, prerelax, done);
            break;
        case MODE_DEFECT:
            launch_pdl(packed_sweep_slot_kernel<T, MODE_DEFECT>, dim3(sb), dim3(256), 0, st, L, Apk, u, f, rdiag, mask, out, omega, prerelax, done);
            break;
        case MODE_JACOBI:
            launch_pdl(packed_sweep_slot_kernel<T, MODE_JACOBI>, dim3(sb), dim3(256), 0, st, L, Apk, u, f, rdiag, mask, out, omega, prerelax, done);
            break;
        default:
            launch_pdl(packed_sweep_slot_kernel<T, MODE_JACOBI_PRE>, dim3(sb), dim3(256), 0, st, L, Apk, u, f, rdiag, mask, out, omega, prerelax, done);
        }
        count_launches(1);
        return;
    }
    const unsigned nb = (unsigned)((L.g.nnod() + bs - 1) / bs);
    switch (mode) {
    case MODE_APPLY:
        launch_pdl(packed_sweep_kernel<T, MODE_APPLY>, dim3(nb), dim3(bs), 0, st, L, Apk, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    case MODE_DEFECT:
        launch_pdl(packed_sweep_kernel<T, MODE_DEFECT>, dim3(nb), dim3(bs), 0, st, L, Apk, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    case MODE_JACOBI:
        launch_pdl(packed_sweep_kernel<T, MODE_JACOBI>, dim3(nb), dim3(bs), 0, st, L, Apk, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    default:
        launch_pdl(packed_sweep_kernel<T, MODE_JACOBI_PRE>, dim3(nb), dim3(bs), 0, st, L, Apk, u, f, rdiag, mask, out, omega, prerelax, done);
    }
    count_launches(1);
}

template void launch_packed_sweep<double>(int, const Lay &, const double *, const double *,
                                          const double *, const double *, const uint8_t *, double *,
                                          double, double, const int *, cudaStream_t);
template void launch_packed_sweep<float>(int, const Lay &, const float *, const float *,
                                         const float *, const float *, const uint8_t *, float *,
                                         float, float, const int *, cudaStream_t);

// ---------------------------------------------------------------------------
// grid transfers
// ---------------------------------------------------------------------------

// F_c = P^T R_f with the full-weighting weights 2^-(|di|+|dj|+|dk|) over the 27
// fine neighbours of each coarse node (mgcg1.cu:792-831 rstrFc), then the
// coarse Dirichlet rows are zeroed (ZeroBCc after rstrFc, mgcg1.cu:537).
template <typename T>
__device__ __forceinline__ void restrict_node(const Lay &Lc, const Lay &Lf, const T *__restrict__ rf,
                                              const uint8_t *__restrict__ maskc, T *__restrict__ fc, int i, int j,
                                              int k)
{
    const Grid &gc = Lc.g;
    const long long n = gc.node(i, j, k);
    const Grid &gf = Lf.g;
    T acc[3] = {T(0), T(0), T(0)};
    // all 27 taps unrolled with predicated loads (a tap outside the grid
    // adds an exact zero), so the loads of a plane issue together
#pragma unroll
    for (int di = -1; di <= 1; ++di) {
        const int fi = 2 * i + di;
        const bool oki = fi >= 0 && fi <= gf.nx;
#pragma unroll
        for (int dk = -1; dk <= 1; ++dk) {
            const int fk = 2 * k + dk;
            const bool okk = oki && fk >= 0 && fk <= gf.nz;
#pragma unroll
            for (int dj = -1; dj <= 1; ++dj) {
                const int fj = 2 * j + dj;
                const bool ok = okk && fj >= 0 && fj <= gf.ny;
                const T w = T(1.0 / (1 << ((di != 0) + (dj != 0) + (dk != 0))));
                const long long nf = ok ? Lf.at(fi, fj, fk) : 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) acc[d] = fma(w, ok ? rf[nf + d] : T(0), acc[d]);
            }
        }
    }
    const unsigned m = maskc[n];
    const long long base = Lc.at(i, j, k);
#pragma unroll
    for (int d = 0; d < 3; ++d) fc[base + d] = ((m >> d) & 1u) ? T(0) : acc[d];
}

template <typename T>
__global__ void restrict_kernel(Lay Lc, Lay Lf, const T *__restrict__ rf,
                                const uint8_t *__restrict__ maskc, T *__restrict__ fc,
                                const int *__restrict__ done)
{
    pdl_wait();
    pdl_trigger();   // the next kernel (a coarse sweep) may start loading its matrix
    if (done && *done) return;
    int i, j, k;
    if (!plane_ijk(Lc.g, i, j, k)) return;
    restrict_node<T>(Lc, Lf, rf, maskc, fc, i, j, k);
}

template <typename T>
void launch_restrict(const Lay &Lc, const Lay &Lf, const T *rf, const uint8_t *maskc, T *fc,
                     const int *done, cudaStream_t st)
{
    const int bs = 128;
    launch_pdl(restrict_kernel<T>, plane_grid(Lc.g, bs), dim3(bs), 0, st, Lc, Lf, rf, maskc, fc, done);
    count_launches(1);
}
template void launch_restrict<double>(const Lay &, const Lay &, const double *, const uint8_t *,
                                      double *, const int *, cudaStream_t);
template void launch_restrict<float>(const Lay &, const Lay &, const float *, const uint8_t *,
                                     float *, const int *, cudaStream_t);

// u_f += P u_c, trilinear (mgcg1.cu:1587-1641 interpc), then the fine
// Dirichlet dofs are zeroed (ZeroBCc after interpc, mgcg1.cu:631).  Fine
// node (i, j, k) takes the coarse nodes (i >> 1) + a, (j >> 1) + b,
// (k >> 1) + c for a < (i & 1) + 1 etc., summed in the order a, c, b, and
// scales the sum by 1 / (number of taps).  One thread per coarse cell: it
// reads the cell's (up to) 8 coarse nodes once and updates its 2 x 2 x 2 fine
// nodes (I, J, K the cell's lower coarse node; fine nodes past the grid's
// last plane, row or column are skipped), 3 coarse loads per fine node
// instead of 24 gathered ones (a thread per fine node took 45.9 us at the
// 256x128x128 level, bound by the gathers' L1 wavefronts).  The fine node
// pairs along y are 8-byte words.
template <typename T>
__global__ void prolong_cell_kernel(Lay Lf, Lay Lc, const T *__restrict__ uc, const uint8_t *__restrict__ maskf,
                                    T *__restrict__ uf, const int *__restrict__ done)
{
    pdl_wait();
    pdl_trigger();
    if (done && *done) return;
    int I, J, K;
    if (!plane_ijk(Lc.g, I, J, K)) return;
    const Grid &gf = Lf.g, &gc = Lc.g;
    const long long si = (long long)(gc.nz + 1) * Lc.pitch, sk = Lc.pitch;
    const T *c0 = uc + Lc.at(I, J, K);
    // coarse values C[a][c][b][d] of node (I + a, J + b, K + c), 0 where outside the grid
    const bool va = I < gc.nx, vb = J < gc.ny, vc = K < gc.nz;
    T C[2][2][2][3];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                const bool ok = (!a || va) && (!c || vc) && (!b || vb);
                const T *cr = c0 + (ok ? (a ? si : 0) + (c ? sk : 0) + 3 * b : 0);
#pragma unroll
                for (int d = 0; d < 3; ++d) C[a][c][b][d] = ok ? cr[d] : T(0);
            }
#pragma unroll
    for (int fi = 0; fi < 2; ++fi) {
        if (fi && !va) break;
#pragma unroll
        for (int fk = 0; fk < 2; ++fk) {
            if (fk && !vc) break;
            const int i = 2 * I + fi, k = 2 * K + fk, j = 2 * J;
            const long long base = Lf.at(i, j, k);
            const int ni = fi + 1, nk = fk + 1;
            T out[2][3];
            const bool pair = vb;   // fine node j + 1 exists
#pragma unroll
            for (int fj = 0; fj < 2; ++fj) {
                const int nj = fj + 1;
                T acc[3] = {T(0), T(0), T(0)};
                // tap order a (x), c (z), b (y); taps not taken add 0
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int c = 0; c < 2; ++c)
#pragma unroll
                        for (int b = 0; b < 2; ++b) {
                            const bool ok = a < ni && c < nk && b < nj;
#pragma unroll
                            for (int d = 0; d < 3; ++d) acc[d] += ok ? C[a][c][b][d] : T(0);
                        }
                const T w = T(1) / T(ni * nj * nk);
                const unsigned m = (fj && !pair) ? 0u : maskf[gf.node(i, j + fj, k)];
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const T v = (fj && !pair) ? T(0) : uf[base + 3 * fj + d];
                    out[fj][d] = ((m >> d) & 1u) ? T(0) : fma(w, acc[d], v);
                }
            }
            if (pair && sizeof(T) == 4) {
                float2 *o = reinterpret_cast<float2 *>(uf + base);
                o[0] = make_float2((float)out[0][0], (float)out[0][1]);
                o[1] = make_float2((float)out[0][2], (float)out[1][0]);
                o[2] = make_float2((float)out[1][1], (float)out[1][2]);
            } else {
#pragma unroll
                for (int d = 0; d < 3; ++d) uf[base + d] = out[0][d];
                if (pair)
#pragma unroll
                    for (int d = 0; d < 3; ++d) uf[base + 3 + d] = out[1][d];
            }
        }
    }
}

template <typename T>
void launch_prolong_add(const Lay &Lf, const Lay &Lc, const T *uc, const uint8_t *maskf, T *uf,
                        const int *done, cudaStream_t st)
{
    const int bs = 128;
    launch_pdl(prolong_cell_kernel<T>, plane_grid(Lc.g, bs), dim3(bs), 0, st, Lf, Lc, uc, maskf, uf, done);
    count_launches(1);
}
template void launch_prolong_add<double>(const Lay &, const Lay &, const double *, const uint8_t *,
                                         double *, const int *, cudaStream_t);
template void launch_prolong_add<float>(const Lay &, const Lay &, const float *, const uint8_t *,
                                        float *, const int *, cudaStream_t);

// ---------------------------------------------------------------------------
// hierarchy setup
// ---------------------------------------------------------------------------

// diag of a packed coarse level (mgcg1.cu:1404-1445 prepADc).
template <typename T>
__global__ void diag_packed_kernel(Lay L, const T *__restrict__ A, T *__restrict__ diag)
{
    const Grid &g = L.g;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    int i, j, k;
    node_ijk(g, n, i, j, k);
    const long long nel = g.nel();
    T acc[3] = {0, 0, 0};
    for (int ex = 0; ex < 2; ++ex)
        for (int ez = 0; ez < 2; ++ez)
            for (int ey = 0; ey < 2; ++ey) {
                const int ei = i - 1 + ex, ej = j - 1 + ey, ek = k - 1 + ez;
                if (ei < 0 || ei >= g.nx || ej < 0 || ej >= g.ny || ek < 0 || ek >= g.nz) continue;
                const long long e = g.elem(ei, ej, ek);
                const int a = local_index(1 - ex, 1 - ey, 1 - ez);
                for (int d = 0; d < 3; ++d) acc[d] += A[(long long)packed_index(3 * a + d, 3 * a + d) * nel + e];
            }
    const long long base = L.at(i, j, k);
    for (int d = 0; d < 3; ++d) diag[base + d] = acc[d];
}

template <typename T>
void launch_diag_packed(const Lay &L, const T *Apk, T *diag, cudaStream_t st)
{
    const int bs = 128;
    diag_packed_kernel<T><<<(unsigned)((L.g.nnod() + bs - 1) / bs), bs, 0, st>>>(L, Apk, diag);
    count_launches(1);
}
template void launch_diag_packed<double>(const Lay &, const double *, double *, cudaStream_t);
template void launch_diag_packed<float>(const Lay &, const float *, float *, cudaStream_t);

// dense reference layout <-> padded layout (y optionally negated)
__global__ void pack_kernel(Lay L, double *__restrict__ dense, double *__restrict__ padded,
                            int flip_y, int to_padded)
{
    const Grid &g = L.g;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= g.ndof()) return;
    const long long n = t / 3;
    const int d = (int)(t - 3 * n);
    const long long row = n / (g.ny + 1);
    const int j = (int)(n - row * (g.ny + 1));
    const long long p = row * L.pitch + 3LL * j + d;
    const double s = (flip_y && d == 1) ? -1.0 : 1.0;
    if (to_padded) padded[p] = s * dense[t];
    else dense[t] = s * padded[p];
}

void launch_pack(const Lay &L, const double *dense, double *padded, int flip_y, cudaStream_t st)
{
    const int bs = 256;
    pack_kernel<<<(unsigned)((L.g.ndof() + bs - 1) / bs), bs, 0, st>>>(L, const_cast<double *>(dense), padded,
                                                                        flip_y, 1);
    count_launches(1);
}

void launch_unpack(const Lay &L, const double *padded, double *dense, int flip_y, cudaStream_t st)
{
    const int bs = 256;
    pack_kernel<<<(unsigned)((L.g.ndof() + bs - 1) / bs), bs, 0, st>>>(L, dense, const_cast<double *>(padded),
                                                                        flip_y, 0);
    count_launches(1);
}

template <typename T>
__global__ void pack_cx_kernel(ELay E, const double *__restrict__ CX, T *__restrict__ out)
{
    const Grid &g = E.g;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= g.nel()) return;
    const long long row = e / g.ny;
    const int j = (int)(e - row * g.ny);
    out[row * E.pitch + j] = (T)CX[e];
}

template <typename T>
void launch_pack_cx(const ELay &E, const double *CX, T *padded, cudaStream_t st)
{
    const int bs = 256;
    pack_cx_kernel<T><<<(unsigned)((E.g.nel() + bs - 1) / bs), bs, 0, st>>>(E, CX, padded);
    count_launches(1);
}
template void launch_pack_cx<double>(const ELay &, const double *, double *, cudaStream_t);
template void launch_pack_cx<float>(const ELay &, const double *, float *, cudaStream_t);

// Level 1: A_E = sum_g CX(child containing Gauss point g) Kg[g]
// (mgcg1.cu:2042-2070 coarseAe2c).  One thread per (element, packed entry).
__global__ void build_level1_kernel(Grid gc, const double *__restrict__ CXf, double *__restrict__ A)
{
    const long long nel = gc.nel();
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nel) return;
    const long long t = e / gc.ny;
    const int j = (int)(e - t * gc.ny);
    const int i = (int)(t / gc.nz);
    const int k = (int)(t - (long long)i * gc.nz);
    const Grid gf{2 * gc.nx, 2 * gc.ny, 2 * gc.nz};
    double cx[8];
    for (int ix = 0; ix < 2; ++ix)
        for (int iz = 0; iz < 2; ++iz)
            for (int iy = 0; iy < 2; ++iy) cx[4 * ix + 2 * iz + iy] = CXf[gf.elem(2 * i + ix, 2 * j + iy, 2 * k + iz)];
    for (int p = 0; p < 300; ++p) {
        double acc = 0.0;
#pragma unroll
        for (int gq = 0; gq < 8; ++gq) acc = fma(cx[gq], cKg[gq * 300 + p], acc);
        A[(long long)p * nel + e] = acc;
    }
}

void launch_build_level1(const Grid &gc, const double *CXfine, double *Apk, cudaStream_t st)
{
    const int bs = 128;
    build_level1_kernel<<<(unsigned)((gc.nel() + bs - 1) / bs), bs, 0, st>>>(gc, CXfine, Apk);
    count_launches(1);
}

// Levels >= 2: Galerkin P^T A P over the 8 children of each coarse element
// (mgcg1.cu:1678-1743 coarseAe3c), computed child by child as
// A_E = sum_c Pc^T A_c Pc with the 8x8 node weights Pc.  One CTA of 576
// threads per coarse element; thread t owns entry (t/24, t%24).  The eight
// children's packed matrices (2,400 values) are staged in shared memory by
// one batch of independent loads (a plane's eight children side by side, so
// the two y-neighbours share a sector) before the products, and so are the
// 512 node weights (a warp reads up to 8 different weights at once, which
// constant memory would serialise).
__global__ void __launch_bounds__(576) build_galerkin_kernel(Grid gc, const double *__restrict__ Af,
                                                             double *__restrict__ A)
{
    const long long E = blockIdx.x;
    const long long nel = gc.nel();
    const long long t = E / gc.ny;
    const int j = (int)(E - t * gc.ny);
    const int i = (int)(t / gc.nz);
    const int k = (int)(t - (long long)i * gc.nz);
    const Grid gf{2 * gc.nx, 2 * gc.ny, 2 * gc.nz};
    const long long nelf = gf.nel();
    __shared__ double Sp[8][300];   // child c's packed matrix
    __shared__ double Tm[576];
    __shared__ double Pw[512];      // cPc
    const int tid = threadIdx.x;
    if (tid < 512) Pw[tid] = cPc[tid];
    for (int idx = tid; idx < 8 * 300; idx += 576) {
        const int c = idx & 7, pk = idx >> 3;
        Sp[c][pk] = Af[(long long)pk * nelf + gf.elem(2 * i + local_x(c), 2 * j + local_y(c), 2 * k + local_z(c))];
    }
    __syncthreads();
    const int m = tid / 24, n = tid - 24 * (tid / 24);
    const int am = m / 3, p = m - 3 * am;   // row: coarse local node, component
    const int an = n / 3, q = n - 3 * an;   // column
    double acc = 0.0;
    for (int c = 0; c < 8; ++c) {
        // Tm[(b,p)][(an,q)] = sum_b' S[(b,p)][(b',q)] Pc[b'][an]   (here m = (b,p))
        double tv = 0.0;
#pragma unroll
        for (int b2 = 0; b2 < 8; ++b2) tv = fma(Sp[c][packed_index(m, 3 * b2 + q)], Pw[(c * 8 + b2) * 8 + an], tv);
        Tm[tid] = tv;
        __syncthreads();
        // acc[(am,p)][n] += sum_b Pc[b][am] Tm[(b,p)][n]
#pragma unroll
        for (int b = 0; b < 8; ++b) acc = fma(Pw[(c * 8 + b) * 8 + am], Tm[(3 * b + p) * 24 + n], acc);
        __syncthreads();
    }
    if (n <= m) A[(long long)packed_index(m, n) * nel + E] = acc;
}

void launch_build_galerkin(const Grid &gc, const double *Afine, double *Apk, cudaStream_t st)
{
    build_galerkin_kernel<<<(unsigned)gc.nel(), 576, 0, st>>>(gc, Afine, Apk);
    count_launches(1);
}

// Level 2 from the fine CX: A_E[p] = sum_{f<64} CX_f Mq[f][p].  Persistent
// CTAs (one per SM) stage the whole 64 x 300 Mq (153.6 KB) in shared memory
// once, then take blocks of 32 consecutive level-2 elements: the block's 64
// fine CX values per element go to shared memory, warp w computes packed
// entries [30 w, 30 w + 30) three at a time with lane = element (each Mq
// value a broadcast read), and each store of an entry plane is 32
// consecutive elements.  The sum over f runs in order, as before.
constexpr int kL2qElems = 32;
constexpr int kL2qWarps = 10;
constexpr int kL2qPer = 30;   // packed entries per warp (10 x 30 = 300)
constexpr size_t kL2qSmem = sizeof(double) * (64 * 300 + kL2qElems * 65);

__global__ void __launch_bounds__(kL2qWarps * 32) build_level2_quad_kernel(Grid g2, const double *__restrict__ CXf,
                                                                          const double *__restrict__ Mq,
                                                                          double *__restrict__ A)
{
    extern __shared__ double l2q_smem[];
    double *Ms = l2q_smem;              // [64][300]
    double *cx = l2q_smem + 64 * 300;   // [32][65]
    const long long nel = g2.nel();
    const long long nblk = (nel + kL2qElems - 1) / kL2qElems;
    const Grid gff{4 * g2.nx, 4 * g2.ny, 4 * g2.nz};
    for (int idx = threadIdx.x; idx < 64 * 300; idx += kL2qWarps * 32) Ms[idx] = Mq[idx];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int p0 = w * kL2qPer;
    for (long long blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const long long E0 = blk * kL2qElems;
        __syncthreads();   // Ms staged (first block); the previous block's cx reads done
        for (int idx = threadIdx.x; idx < kL2qElems * 64; idx += kL2qWarps * 32) {
            const int el = idx >> 6, f = idx & 63;
            const long long E = E0 + el;
            double v = 0.0;
            if (E < nel) {
                const long long t = E / g2.ny;
                const int j = (int)(E - t * g2.ny);
                const int i = (int)(t / g2.nz);
                const int k = (int)(t - (long long)i * g2.nz);
                const int c = f >> 3, gq = f & 7;
                const int ix = gq >> 2, iz = (gq >> 1) & 1, iy = gq & 1;   // gq = 4 ix + 2 iz + iy
                v = CXf[gff.elem(2 * (2 * i + local_x(c)) + ix, 2 * (2 * j + local_y(c)) + iy,
                                 2 * (2 * k + local_z(c)) + iz)];
            }
            cx[el * 65 + f] = v;
        }
        __syncthreads();
        const long long E = E0 + lane;
        for (int pp = p0; pp < p0 + kL2qPer; pp += 3) {
            double a0 = 0.0, a1 = 0.0, a2 = 0.0;
#pragma unroll 8
            for (int f = 0; f < 64; ++f) {
                const double v = cx[lane * 65 + f];
                const double *mf = Ms + f * 300 + pp;
                a0 = fma(v, mf[0], a0);
                a1 = fma(v, mf[1], a1);
                a2 = fma(v, mf[2], a2);
            }
            if (E < nel) {
                A[(long long)pp * nel + E] = a0;
                A[(long long)(pp + 1) * nel + E] = a1;
                A[(long long)(pp + 2) * nel + E] = a2;
            }
        }
    }
}

void launch_build_galerkin_from_quad(const Grid &g2, const double *CXfine, double *Apk, cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    static bool attr_set[64] = {};
    static int sms[64] = {};
    if (dev < 64 && !attr_set[dev]) {   // setup runs outside stream capture
        cudaFuncSetAttribute(build_level2_quad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kL2qSmem);
        cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
        attr_set[dev] = true;
    }
    const long long nblk = (g2.nel() + kL2qElems - 1) / kL2qElems;
    const int sm = (dev < 64 && sms[dev] > 0) ? sms[dev] : 148;
    const unsigned grid = (unsigned)(nblk < sm ? nblk : sm);
    build_level2_quad_kernel<<<grid, kL2qWarps * 32, kL2qSmem, st>>>(g2, CXfine, quad_galerkin_blocks(dev), Apk);
    count_launches(1);
}

// Dirichlet penalty on the coarsest element matrices (mgcg1.cu:1368-1402
// CorrCsAc).  For a fixed dof of node (i,j,k) and each adjacent element
// (i+di, j+dj, k+dk), the reference writes 1e10 on the diagonal of the
// element-local node with offset (-di, 1+dj, -dk) -- its lookup table is the
// true local index mirrored in y -- and this kernel penalises the same
// entries.  Concurrent writers store the same value.
__global__ void penalty_kernel(Grid g, const uint8_t *__restrict__ mask, double *__restrict__ A)
{
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    const unsigned mk = mask[n];
    if (!mk) return;
    int i, j, k;
    node_ijk(g, n, i, j, k);
    const long long nel = g.nel();
    for (int d = 0; d < 3; ++d) {
        if (!((mk >> d) & 1u)) continue;
        for (int di = -1; di <= 0; ++di)
            for (int dk = -1; dk <= 0; ++dk)
                for (int dj = -1; dj <= 0; ++dj) {
                    const int ei = i + di, ej = j + dj, ek = k + dk;
                    if (ei < 0 || ei >= g.nx || ej < 0 || ej >= g.ny || ek < 0 || ek >= g.nz) continue;
                    const int a = local_index(-di, 1 + dj, -dk);
                    const int mm = 3 * a + d;
                    A[(long long)packed_index(mm, mm) * nel + g.elem(ei, ej, ek)] = 1e10;
                }
    }
}

void launch_coarsest_penalty(const Grid &g, const uint8_t *mask, double *Apk, cudaStream_t st)
{
    const int bs = 128;
    penalty_kernel<<<(unsigned)((g.nnod() + bs - 1) / bs), bs, 0, st>>>(g, mask, Apk);
    count_launches(1);
}

// Dense coarsest matrix, one thread per row (mgcg1.cu:1747-1806 assembAc).
__global__ void assemble_dense_kernel(Grid g, const double *__restrict__ A, double *__restrict__ AQ)
{
    const long long row = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long N = g.ndof();
    if (row >= N) return;
    const long long n = row / 3;
    const int d = (int)(row - 3 * n);
    int i, j, k;
    node_ijk(g, n, i, j, k);
    const long long nel = g.nel();
    double *out = AQ + row * N;
    for (long long c = 0; c < N; ++c) out[c] = 0.0;
    for (int ex = 0; ex < 2; ++ex)
        for (int ez = 0; ez < 2; ++ez)
            for (int ey = 0; ey < 2; ++ey) {
                const int ei = i - 1 + ex, ej = j - 1 + ey, ek = k - 1 + ez;
                if (ei < 0 || ei >= g.nx || ej < 0 || ej >= g.ny || ek < 0 || ek >= g.nz) continue;
                const long long e = g.elem(ei, ej, ek);
                const int a = local_index(1 - ex, 1 - ey, 1 - ez);
                for (int b = 0; b < 8; ++b) {
                    const long long nb = g.node(ei + local_x(b), ej + local_y(b), ek + local_z(b));
                    for (int q = 0; q < 3; ++q)
                        out[3 * nb + q] += A[(long long)packed_index(3 * a + d, 3 * b + q) * nel + e];
                }
            }
}

void launch_assemble_dense(const Grid &g, const double *Apk, double *AQ, cudaStream_t st)
{
    const int bs = 64;
    assemble_dense_kernel<<<(unsigned)((g.ndof() + bs - 1) / bs), bs, 0, st>>>(g, Apk, AQ);
    count_launches(1);
}

// Re-discretised coarse levels (Homogenization/QNC/mgcg9.cu:753-781 formCXc):
// a coarse element's scale is twice the mean of its eight children, the 2
// being Ke(2h) = 2 Ke(h) for the unit-modulus hex8 (the reference's choice
// among the mean forms it tried).
__global__ void coarse_cx_kernel(Grid gc, const double *__restrict__ CXf, double *__restrict__ CXc)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= gc.nel()) return;
    const int j = (int)(e % gc.ny);
    const long long r = e / gc.ny;
    const int k = (int)(r % gc.nz), i = (int)(r / gc.nz);
    const Grid gf{2 * gc.nx, 2 * gc.ny, 2 * gc.nz};
    double s = 0.0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) s += CXf[gf.elem(2 * i + a, 2 * j + c, 2 * k + b)];
    CXc[e] = 2.0 * (s / 8.0);
}

void launch_coarse_cx(const Grid &gc, const double *CXf, double *CXc, cudaStream_t st)
{
    const int bs = 256;
    coarse_cx_kernel<<<(unsigned)((gc.nel() + bs - 1) / bs), bs, 0, st>>>(gc, CXf, CXc);
    count_launches(1);
}

// Fixed dofs of a dense coarsest matrix, the mgcg9 way (mgcg9.cu:1005-1028
// CorrCsAQc): their rows and columns become zero and the diagonal 1e10.
__global__ void dense_fix_kernel(Grid g, const uint8_t *__restrict__ mask, double *__restrict__ AQ)
{
    const long long N = g.ndof();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= N * N) return;
    const long long r = idx / N, c = idx - r * N;
    const bool fr = (mask[r / 3] >> (r % 3)) & 1u, fc = (mask[c / 3] >> (c % 3)) & 1u;
    if (fr || fc) AQ[idx] = (r == c) ? 1e10 : 0.0;
}

void launch_dense_fix(const Grid &g, const uint8_t *mask, double *AQ, cudaStream_t st)
{
    const long long n2 = g.ndof() * g.ndof();
    const int bs = 256;
    dense_fix_kernel<<<(unsigned)((n2 + bs - 1) / bs), bs, 0, st>>>(g, mask, AQ);
    count_launches(1);
}

// Blocked right-looking Cholesky A = L L^T of the dense coarsest matrix, in
// place in the lower triangle, 32-column panels (textbook algorithm; the
// reference factors row by row, one kernel launch per row,
// mgcg1.cu:2099-2142).  For each panel [c0, c0 + w):
//   chol_diag_kernel   the w x w diagonal block, factored in shared memory
//                      (one CTA, a thread per entry);
//   chol_panel_kernel  each row r below it solves L[r][panel] D^T = A[r][panel]
//                      (a thread per row, many CTAs);
//   chol_trail_kernel  the trailing lower triangle loses the panel's rank-w
//                      product, A[r][c] -= sum_k L[r][c0 + k] L[c][c0 + k]
//                      (a CTA per 32 x 32 tile on or below the diagonal).
// Each step is a short latency-bound kernel (675 unknowns on the
// 256 x 128 x 128 grid), so all of them, and the inverse below, run back to
// back under programmatic dependent launch: a kernel lets the next one launch
// at its start and waits for its predecessor before it reads anything.
// info = 1-based index of the first non-positive (or NaN) pivot, 0 on
// success; once set, every later factor kernel returns at once.
constexpr int kCholB = 32;

// Column step j: every thread forms the pivot sqrt(D[j][j]) and the scaled
// entries it needs itself (the same operations on the same values, so the
// same bits as one thread forming them), the scaled column goes to Lc, and the
// trailing update writes only columns > j: one barrier per column.
__global__ void __launch_bounds__(1024) chol_diag_kernel(int n, int c0, int w, double *__restrict__ A,
                                                         int *__restrict__ info)
{
    pdl_wait();
    pdl_trigger();
    if (*info) return;
    __shared__ double D[kCholB][kCholB + 1];
    __shared__ double Lc[kCholB][kCholB + 1];
    const int tid = threadIdx.x, r = tid >> 5, c = tid & 31;
    D[r][c] = (r < w && c <= r) ? A[(long long)(c0 + r) * n + c0 + c] : 0.0;
    Lc[r][c] = 0.0;
    __syncthreads();
    for (int j = 0; j < w; ++j) {
        const double s = D[j][j];
        if (!(s > 0.0)) {   // the same value in every thread
            if (tid == 0) atomicCAS(info, 0, c0 + j + 1);
            return;
        }
        const double d = sqrt(s);
        if (r < w && r >= j) {
            const double lrj = r == j ? d : D[r][j] / d;
            if (c == j) Lc[r][j] = lrj;
            // trailing update inside the block: D[r][c] -= L[r][j] L[c][j], j < c <= r < w
            if (c > j && c <= r) D[r][c] = fma(-lrj, D[c][j] / d, D[r][c]);
        }
        __syncthreads();
    }
    if (r < w && c <= r) A[(long long)(c0 + r) * n + c0 + c] = Lc[r][c];
}

// A warp per row below the panel: x D^T = a by forward substitution, lane c
// holding entry c; step k finishes x_k on lane k and broadcasts it, and the
// later lanes subtract x_k D[c][k] (each lane's updates in order of k, as a
// thread-per-row substitution applies them).
constexpr int kCholPanelWarps = 8;

__global__ void __launch_bounds__(kCholPanelWarps * 32) chol_panel_kernel(int n, int c0, int w,
                                                                         double *__restrict__ A,
                                                                         const int *__restrict__ info)
{
    pdl_wait();
    pdl_trigger();
    if (*info) return;
    __shared__ double D[kCholB][kCholB + 1];
    for (int idx = threadIdx.x; idx < kCholB * kCholB; idx += kCholPanelWarps * 32) {
        const int r = idx / kCholB, c = idx - r * kCholB;
        D[r][c] = (r < w && c <= r) ? A[(long long)(c0 + r) * n + c0 + c] : 0.0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int r = c0 + w + blockIdx.x * kCholPanelWarps + (threadIdx.x >> 5);
    if (r >= n) return;   // the same for the whole warp
    double *row = A + (long long)r * n + c0;
    double s = lane < w ? row[lane] : 0.0;
    for (int k = 0; k < w; ++k) {
        double xk = lane == k ? s / D[k][k] : 0.0;
        xk = __shfl_sync(0xffffffffu, xk, k);
        if (lane == k) s = xk;
        else if (lane > k) s = fma(-xk, D[lane][k], s);
    }
    if (lane < w) row[lane] = s;
}

// grid (t, t) over the trailing 32 x 32 tiles; tiles above the diagonal return
__global__ void __launch_bounds__(256) chol_trail_kernel(int n, int c0, int w, double *__restrict__ A,
                                                         const int *__restrict__ info)
{
    pdl_wait();
    pdl_trigger();
    if (blockIdx.y > blockIdx.x || *info) return;
    __shared__ double Ar[kCholB][kCholB + 1];
    __shared__ double Ac[kCholB][kCholB + 1];
    const int t0 = c0 + w;
    const int r0 = t0 + blockIdx.x * kCholB, q0 = t0 + blockIdx.y * kCholB;
    for (int idx = threadIdx.x; idx < kCholB * kCholB; idx += 256) {
        const int rr = idx / kCholB, k = idx - rr * kCholB;
        Ar[rr][k] = (r0 + rr < n && k < w) ? A[(long long)(r0 + rr) * n + c0 + k] : 0.0;
        Ac[rr][k] = (q0 + rr < n && k < w) ? A[(long long)(q0 + rr) * n + c0 + k] : 0.0;
    }
    __syncthreads();
    const int ty = threadIdx.x >> 3, tx = threadIdx.x & 7;   // 32 rows x 8 threads, 4 columns each
    double acc[4] = {0, 0, 0, 0};
#pragma unroll 8
    for (int k = 0; k < kCholB; ++k) {
        const double a = Ar[ty][k];
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] = fma(a, Ac[tx * 4 + q][k], acc[q]);
    }
    const int r = r0 + ty;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int col = q0 + tx * 4 + q;
        if (r < n && col <= r) A[(long long)r * n + col] -= acc[q];
    }
}

void launch_cholesky(int n, double *A, int *info, cudaStream_t st)
{
    cudaMemsetAsync(info, 0, sizeof(int), st);
    for (int c0 = 0; c0 < n; c0 += kCholB) {
        const int w = (n - c0) < kCholB ? (n - c0) : kCholB;
        const int m = n - c0 - w;   // rows below the panel
        launch_pdl(chol_diag_kernel, dim3(1), dim3(kCholB * kCholB), 0, st, n, c0, w, A, info);
        count_launches(1);
        if (m > 0) {
            const int *cinfo = info;
            launch_pdl(chol_panel_kernel, dim3((unsigned)((m + kCholPanelWarps - 1) / kCholPanelWarps)),
                       dim3(kCholPanelWarps * 32), 0, st, n, c0, w, A, cinfo);
            const unsigned t = (unsigned)((m + kCholB - 1) / kCholB);
            launch_pdl(chol_trail_kernel, dim3(t, t), dim3(256), 0, st, n, c0, w, A, cinfo);
            count_launches(2);
        }
    }
}

// Explicit inverse of the lower Cholesky factor, so that each coarse solve is
// two dense triangular matrix-vector products instead of 2n dependent steps.
// Blocked by recursive doubling with the block formula
//   [A 0; B C]^-1 = [A^-1 0; -C^-1 B A^-1  C^-1]:
//   tri_diag_inverse_kernel  the inverse of every 32 x 32 diagonal block (a
//                            thread per column, forward substitution in
//                            shared memory; zeros above its diagonal);
//   for s = 32, 64, 128, ... < n, blocks [o, o + s) and [o + s, o + 2s)
//   (o = 2 s p, the second clipped at n) are paired:
//     tri_double_kernel<1>   T = B A^-1 into LinvT (scratch until the end);
//     tri_double_kernel<2>   the pair's lower-left block X = -C^-1 T;
//   tri_transpose_kernel     LinvT = Linv^T, zeros in Linv's strict upper
//                            triangle.
// Both products skip the 32 x 32 blocks that are zero by triangularity, so
// only blocks on or below the diagonal are read, and every one of them was
// written at an earlier level.  2 log2(n / 32) + 2 launches (12 for n = 675)
// instead of a serial chain of n steps per column.
__global__ void __launch_bounds__(kCholB) tri_diag_inverse_kernel(int n, const double *__restrict__ L,
                                                                  double *__restrict__ Linv)
{
    pdl_wait();
    pdl_trigger();
    __shared__ double Ls[kCholB][kCholB + 1];
    __shared__ double X[kCholB][kCholB + 1];   // X[i][j]: row i of column j of the block's inverse
    const int b0 = blockIdx.x * kCholB, w = min(kCholB, n - b0), j = threadIdx.x;
    for (int i = 0; i < w; ++i) Ls[i][j] = (j <= i) ? L[(long long)(b0 + i) * n + b0 + j] : 0.0;
    __syncwarp();
    if (j < w) {
        X[j][j] = 1.0 / Ls[j][j];
        for (int i = j + 1; i < w; ++i) {
            double s = 0.0;
            for (int k = j; k < i; ++k) s = fma(Ls[i][k], X[k][j], s);
            X[i][j] = -s / Ls[i][i];
        }
    }
    __syncwarp();
    if (j < w)
        for (int i = 0; i < w; ++i) Linv[(long long)(b0 + i) * n + b0 + j] = (j <= i) ? X[i][j] : 0.0;
}

// grid (s / 32 column tiles, s / 32 row tiles, pairs); 32 x 32 output tile per CTA
template <int STEP>
__global__ void __launch_bounds__(256) tri_double_kernel(int n, int s, const double *__restrict__ L,
                                                         double *__restrict__ Linv, double *__restrict__ Tb)
{
    pdl_wait();
    pdl_trigger();
    const int o = 2 * s * (int)blockIdx.z, rows0 = o + s;
    const int sc = min(s, n - rows0);   // rows of C (> 0 for every pair the grid holds)
    const int i0 = blockIdx.y * kCholB, j0 = blockIdx.x * kCholB;
    if (i0 >= sc) return;
    __shared__ double P[kCholB][kCholB + 1];
    __shared__ double Q[kCholB][kCholB + 1];
    const int ty = threadIdx.x >> 3, tx = threadIdx.x & 7;
    double acc[4] = {0, 0, 0, 0};
    // STEP 1: T[i][j] = sum_{k >= j} B[i][k] Ainv[k][j]  (k chunks from j0's on)
    // STEP 2: X[i][j] = -sum_{k <= i} Cinv[i][k] T[k][j] (k chunks up to i0's)
    const int kbeg = STEP == 1 ? j0 : 0;
    const int kend = STEP == 1 ? s : min(i0 + kCholB, sc);
    for (int k0 = kbeg; k0 < kend; k0 += kCholB) {
        for (int idx = threadIdx.x; idx < kCholB * kCholB; idx += 256) {
            const int a = idx / kCholB, b = idx - a * kCholB;
            const bool pin = i0 + a < sc && k0 + b < kend;   // P[a][b]: row i0 + a, column k0 + b
            const bool qin = k0 + a < kend;                   // Q[a][b]: row k0 + a, column j0 + b
            if (STEP == 1) {
                P[a][b] = pin ? L[(long long)(rows0 + i0 + a) * n + o + k0 + b] : 0.0;
                Q[a][b] = qin ? Linv[(long long)(o + k0 + a) * n + o + j0 + b] : 0.0;
            } else {
                P[a][b] = pin ? Linv[(long long)(rows0 + i0 + a) * n + rows0 + k0 + b] : 0.0;
                Q[a][b] = qin ? Tb[(long long)(rows0 + k0 + a) * n + o + j0 + b] : 0.0;
            }
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < kCholB; ++k) {
            const double a = P[ty][k];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] = fma(a, Q[k][tx * 4 + q], acc[q]);
        }
        __syncthreads();
    }
    const int i = i0 + ty;
    if (i >= sc) return;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const long long at = (long long)(rows0 + i) * n + o + j0 + tx * 4 + q;
        if (STEP == 1) Tb[at] = acc[q];
        else Linv[at] = -acc[q];
    }
}

// The last kernel of the setup's factor chain: it does not release its
// successor early, because the coarse-solve GEMVs read the inverse before
// they wait on their predecessor.
__global__ void __launch_bounds__(256) tri_transpose_kernel(int n, double *__restrict__ Linv,
                                                            double *__restrict__ LinvT)
{
    pdl_wait();
    __shared__ double t[kCholB][kCholB + 1];
    const int bx = blockIdx.x * kCholB, by = blockIdx.y * kCholB;   // Linv tile: rows by.., columns bx..
    for (int a = threadIdx.y; a < kCholB; a += 8) {
        const int r = by + a, c = bx + threadIdx.x;
        double v = 0.0;
        if (r < n && c < n) {
            if (c <= r) v = Linv[(long long)r * n + c];
            else Linv[(long long)r * n + c] = 0.0;
        }
        t[a][threadIdx.x] = v;
    }
    __syncthreads();
    for (int a = threadIdx.y; a < kCholB; a += 8) {
        const int r = bx + a, c = by + threadIdx.x;   // LinvT[r][c] = Linv[c][r]
        if (r < n && c < n) LinvT[(long long)r * n + c] = t[threadIdx.x][a];
    }
}

void launch_tri_inverse(int n, const double *L, double *Linv, double *LinvT, cudaStream_t st)
{
    const unsigned nb = (unsigned)((n + kCholB - 1) / kCholB);
    launch_pdl(tri_diag_inverse_kernel, dim3(nb), dim3(kCholB), 0, st, n, L, Linv);
    count_launches(1);
    for (int s = kCholB; s < n; s *= 2) {
        const unsigned pairs = (unsigned)((n - s + 2 * s - 1) / (2 * s));
        const dim3 grid((unsigned)(s / kCholB), (unsigned)(s / kCholB), pairs);
        launch_pdl(tri_double_kernel<1>, grid, dim3(256), 0, st, n, s, L, Linv, LinvT);
        launch_pdl(tri_double_kernel<2>, grid, dim3(256), 0, st, n, s, L, Linv, LinvT);
        count_launches(2);
    }
    launch_pdl(tri_transpose_kernel, dim3(nb, nb), dim3(kCholB, 8), 0, st, n, Linv, LinvT);
    count_launches(1);
}

// Position of dense (reference-order) dof r in the padded layout.
__device__ __forceinline__ long long padded_pos(const Lay &L, long long r)
{
    const long long n = r / 3;
    const long long row = n / (L.g.ny + 1);
    const long long j = n - row * (L.g.ny + 1);
    return row * L.pitch + 3 * j + (r - 3 * n);
}

// y = M x for a dense row-major n x n triangular matrix, one warp per row,
// FP64 accumulation.  in_padded / out_padded: x / y live in the level's padded
// layout (otherwise dense vectors of n).
// The inverse factor does not change during a solve: a lane loads its first
// kGemvPre entries of the row before waiting on the previous kernel (the
// rest, for n > 32 kGemvPre, after it), and lets the next kernel launch.  A
// warp per row: lane l sums columns l, l + 32, ... in order, then the lanes
// are summed by shuffles.
constexpr int kGemvPre = 24;

template <typename Tin, typename Tout>
__global__ void gemv_warp_kernel(Lay L, const double *__restrict__ M, const Tin *__restrict__ x,
                                 Tout *__restrict__ y, int lower, int in_padded, int out_padded,
                                 const int *__restrict__ done)
{
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int n = (int)L.g.ndof();
    const bool live = row < n;
    const int lo = lower ? 0 : row, hi = !live ? 0 : (lower ? row + 1 : n);
    const double *mr = M + (long long)(live ? row : 0) * n;
    double pre[kGemvPre];
#pragma unroll
    for (int q = 0; q < kGemvPre; ++q) {
        const int c = lo + lane + 32 * q;
        pre[q] = c < hi ? mr[c] : 0.0;
    }
    pdl_trigger();
    pdl_wait();
    if (done && *done) return;
    if (!live) return;
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < kGemvPre; ++q) {
        const int c = lo + lane + 32 * q;
        if (c < hi) s = fma(pre[q], (double)x[in_padded ? padded_pos(L, c) : c], s);
    }
    for (int c = lo + lane + 32 * kGemvPre; c < hi; c += 32)
        s = fma(mr[c], (double)x[in_padded ? padded_pos(L, c) : c], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[out_padded ? padded_pos(L, row) : row] = (Tout)s;
}

// Coarsest solve x = A^-1 b = Linv^T (Linv b) with the explicit inverse of the
// Cholesky factor (replaces cholsl1's 2n single-block launches, mgcg1.cu:2175-2232).
template <typename T>
void launch_coarse_solve(const Lay &L, const double *Linv, const double *LinvT, const T *b, T *x,
                         double *tmp, const int *done, cudaStream_t st)
{
    const int n = (int)L.g.ndof();
    const int bs = 256;
    const unsigned nb = (unsigned)((n * 32 + bs - 1) / bs);
    launch_pdl(gemv_warp_kernel<T, double>, dim3(nb), dim3(bs), 0, st, L, Linv, b, tmp, 1, 1, 0, done);
    launch_pdl(gemv_warp_kernel<double, T>, dim3(nb), dim3(bs), 0, st, L, LinvT, tmp, x, 0, 0, 1, done);
    count_launches(2);
}
template void launch_coarse_solve<double>(const Lay &, const double *, const double *, const double *,
                                          double *, double *, const int *, cudaStream_t);
template void launch_coarse_solve<float>(const Lay &, const double *, const double *, const float *,
                                         float *, double *, const int *, cudaStream_t);

// Fixed-dof mask from the 1-based list (indices validated on the host).
__global__ void mask_from_list_kernel(const double *__restrict__ fixed1b, int nfd, uint8_t *mask)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nfd) return;
    const long long dof = (long long)fixed1b[t] - 1;
    const long long n = dof / 3;
    const unsigned bit = 1u << (unsigned)(dof - 3 * n);
    // byte-wise OR through the enclosing aligned 32-bit word
    unsigned *word = reinterpret_cast<unsigned *>(reinterpret_cast<uintptr_t>(mask + n) & ~uintptr_t(3));
    const unsigned shift = 8u * (unsigned)(reinterpret_cast<uintptr_t>(mask + n) & 3u);
    atomicOr(word, bit << shift);
}

void launch_mask_from_list(long long nnod_bytes, const double *fixed1b, int nfd, uint8_t *mask,
                           cudaStream_t st)
{
    cudaMemsetAsync(mask, 0, (size_t)nnod_bytes, st);
    if (nfd > 0) {
        const int bs = 256;
        mask_from_list_kernel<<<(nfd + bs - 1) / bs, bs, 0, st>>>(fixed1b, nfd, mask);
        count_launches(1);
    }
}

// Coarse fixed dofs: those of the fine nodes with even (i,j,k)
// (mgcg1.cu:747-790 rstrFDc; a mask instead of an atomically ordered list).
__global__ void mask_restrict_kernel(Grid gc, const uint8_t *__restrict__ mf, uint8_t *__restrict__ mc)
{
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= gc.nnod()) return;
    int i, j, k;
    node_ijk(gc, n, i, j, k);
    const Grid gf{2 * gc.nx, 2 * gc.ny, 2 * gc.nz};
    mc[n] = mf[gf.node(2 * i, 2 * j, 2 * k)];
}

void launch_mask_restrict(const Grid &gc, const uint8_t *maskf, uint8_t *maskc, cudaStream_t st)
{
    const int bs = 256;
    mask_restrict_kernel<<<(unsigned)((gc.nnod() + bs - 1) / bs), bs, 0, st>>>(gc, maskf, maskc);
    count_launches(1);
}


}  // namespace gputo
