// Periodic homogenization of a voxel unit cell: the six unit-strain load
// cases solved together as six right-hand sides, and the effective 6x6
// elasticity tensor.  No counterpart in the reference (its Homogenization
// directory solves a self-weight problem, Homogenization/QNC/QNC_V1_mod1m.m:
// 180-199); the method is the reference's MGCG (mgcg1.cu:184-651) carried to
// a periodic grid:
//
//  * grid: n_x x n_y x n_z elements = nodes, node / element (i, j, k) at
//    (n_z n_y) i + n_y k + j (y fastest, the reference's order); element
//    (i, j, k) has the corners (i + x_a, j + y_a, k + z_a) mod n in the
//    reference's local order.  Node 0 is held (its three dofs) to remove the
//    rigid translations, the periodic operator's only null space;
//  * vectors: [dof][6] with dof = 3 node + d, the six load cases of a dof
//    next to each other, so one thread applies the operator to all six;
//  * load case r (Voigt xx, yy, zz, yz, xz, xy; engineering shears): the
//    fluctuation chi_r solves K chi_r = -sum_e CX_e Ke u0_r, u0_r the affine
//    field of unit strain r at an element's local corners;
//  * operator: a node-centred gather over the 27 neighbours; the 3x3 block
//    of each neighbour, sum over the shared elements of CX_e Ke(a, b), is
//    formed once per node and applied to all six load cases;
//  * preconditioner: an FP32 V-cycle (damped Jacobi, the reference's
//    nswp / omega / pre-relaxation; trilinear periodic transfers) on
//    re-discretised coarse levels (CX_l = 2 mean of the eight children, as
//    the reference's mgcg9 builds them, Homogenization/QNC/mgcg9.cu:753-781),
//    and a dense Cholesky solve on the coarsest grid;
//  * outer iteration: flexible PCG (Polak-Ribiere beta) in FP64, one
//    recurrence per load case, a load case frozen (alpha = 0) once it meets
//    the tolerance; one CUDA graph launch per iteration of all six;
//  * C_rs = (1 / n_el) sum_e CX_e (u0_r + chi_r)_e' Ke (u0_s + chi_s)_e.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gputo_internal.h"

namespace gputo {

namespace {

constexpr int NR = 6;                  // load cases
constexpr int kHBlocks = 1184;         // CTAs of the reduction kernels (8 per SM)

__constant__ double cPKe64[576];
__constant__ float cPKe32[576];
__constant__ double cPG[24 * NR];      // Ke u0_r, [24][6]
__constant__ double cPU0[NR * 24];     // u0_r at the local corners, [6][24]

struct PGrid {
    int nx, ny, nz;
    __host__ __device__ long long nnod() const { return (long long)nx * ny * nz; }
    __host__ __device__ long long ndof() const { return 3 * nnod(); }
    __host__ __device__ long long node(int i, int j, int k) const
    {
        return ((long long)nz * ny) * i + (long long)ny * k + j;
    }
};

__host__ __device__ constexpr int corner_of(int x, int y, int z) { return 4 * z + (y ? (x ? 2 : 3) : (x ? 1 : 0)); }

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

template <typename T> __device__ __forceinline__ T pke(int idx);
template <> __device__ __forceinline__ double pke<double>(int idx) { return cPKe64[idx]; }
template <> __device__ __forceinline__ float pke<float>(int idx) { return cPKe32[idx]; }

enum PMode { P_APPLY = 0, P_DEFECT = 1, P_JACOBI = 2, P_PRE = 3 };

// One operator sweep over all six load cases, thread per node.  Modes as the
// fine sweeps: K u (with the per-case p'q partials), f - K u, damped Jacobi
// z = u + omega (f - K u) / diag, and the pre-relaxation that starts from
// u = prerelax f / diag.  Node 0's dofs are held at zero residual.
template <typename T, int MODE>
__global__ void __launch_bounds__(256)
psweep_kernel(PGrid g, const T *__restrict__ CX, const T *__restrict__ u, const T *__restrict__ f,
              const T *__restrict__ rdiag, T *__restrict__ out, T omega, T prerelax, double *__restrict__ partial,
              const int *__restrict__ done)
{
    if (done && *done) return;
    const long long nn = g.nnod();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dsum[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) dsum[r] = 0.0;
    if (n < nn) {
        const int j = (int)(n % g.ny);
        const long long t = n / g.ny;
        const int k = (int)(t % g.nz), i = (int)(t / g.nz);
        const int xi[3] = {wrap(i - 1, g.nx), i, wrap(i + 1, g.nx)};
        const int yj[3] = {wrap(j - 1, g.ny), j, wrap(j + 1, g.ny)};
        const int zk[3] = {wrap(k - 1, g.nz), k, wrap(k + 1, g.nz)};
        // the eight elements around the node: element (i - 1 + ex, j - 1 + ey, k - 1 + ez)
        T cxe[8];
#pragma unroll
        for (int ex = 0; ex < 2; ++ex)
#pragma unroll
            for (int ey = 0; ey < 2; ++ey)
#pragma unroll
                for (int ez = 0; ez < 2; ++ez) cxe[(ex * 2 + ey) * 2 + ez] = CX[g.node(xi[ex], yj[ey], zk[ez])];
        T acc[3][NR], uc[3][NR];
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[d][r] = T(0);
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dz = -1; dz <= 1; ++dz) {
                    // 3x3 block between the node and neighbour (dx, dy, dz)
                    T B[3][3];
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b) B[a][b] = T(0);
#pragma unroll
                    for (int ex = 0; ex < 2; ++ex)
#pragma unroll
                        for (int ey = 0; ey < 2; ++ey)
#pragma unroll
                            for (int ez = 0; ez < 2; ++ez) {
                                const int bx = dx + 1 - ex, by = dy + 1 - ey, bz = dz + 1 - ez;
                                if (bx < 0 || bx > 1 || by < 0 || by > 1 || bz < 0 || bz > 1) continue;
                                const int ca = corner_of(1 - ex, 1 - ey, 1 - ez), cb = corner_of(bx, by, bz);
                                const T c = cxe[(ex * 2 + ey) * 2 + ez];
#pragma unroll
                                for (int a = 0; a < 3; ++a)
#pragma unroll
                                    for (int b = 0; b < 3; ++b)
                                        B[a][b] = fma(c, pke<T>((3 * ca + a) * 24 + 3 * cb + b), B[a][b]);
                            }
                    const long long nb = g.node(xi[dx + 1], yj[dy + 1], zk[dz + 1]);
                    T v[3][NR];
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        const long long base = (3 * nb + b) * NR;
                        if (MODE == P_PRE) {
                            const T s = prerelax * rdiag[3 * nb + b];
#pragma unroll
                            for (int r = 0; r < NR; ++r) v[b][r] = s * f[base + r];
                        } else {
#pragma unroll
                            for (int r = 0; r < NR; ++r) v[b][r] = u[base + r];
                        }
                    }
                    if (dx == 0 && dy == 0 && dz == 0) {
#pragma unroll
                        for (int b = 0; b < 3; ++b)
#pragma unroll
                            for (int r = 0; r < NR; ++r) uc[b][r] = v[b][r];
                    }
#pragma unroll
                    for (int a = 0; a < 3; ++a)
#pragma unroll
                        for (int b = 0; b < 3; ++b)
#pragma unroll
                            for (int r = 0; r < NR; ++r) acc[a][r] = fma(B[a][b], v[b][r], acc[a][r]);
                }
        const bool held = n == 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const long long base = (3 * n + d) * NR;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                if (MODE == P_APPLY) {
                    const T q = held ? T(0) : acc[d][r];
                    out[base + r] = q;
                    dsum[r] = fma((double)uc[d][r], (double)q, dsum[r]);
                } else if (MODE == P_DEFECT) {
                    out[base + r] = held ? T(0) : f[base + r] - acc[d][r];
                } else {
                    const T res = held ? T(0) : f[base + r] - acc[d][r];
                    out[base + r] = uc[d][r] + omega * res * rdiag[3 * n + d];
                }
            }
        }
    }
    if (MODE == P_APPLY && partial) {
        __shared__ double red[8][NR];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            for (int o = 16; o > 0; o >>= 1) dsum[r] += __shfl_xor_sync(0xffffffffu, dsum[r], o);
        if ((threadIdx.x & 31) == 0)
#pragma unroll
            for (int r = 0; r < NR; ++r) red[threadIdx.x >> 5][r] = dsum[r];
        __syncthreads();
        if (threadIdx.x < NR) {
            double s = 0.0;
            for (int w = 0; w < 8; ++w) s += red[w][threadIdx.x];
            partial[blockIdx.x * NR + threadIdx.x] = s;
        }
    }
}

// 1/diag of K per dof (the same for all six cases); 0 on node 0.
__global__ void pdiag_kernel(PGrid g, const double *__restrict__ CX, double *__restrict__ rdiag)
{
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    const int j = (int)(n % g.ny);
    const long long t = n / g.ny;
    const int k = (int)(t % g.nz), i = (int)(t / g.nz);
    double dg[3] = {0.0, 0.0, 0.0};
    for (int ex = 0; ex < 2; ++ex)
        for (int ey = 0; ey < 2; ++ey)
            for (int ez = 0; ez < 2; ++ez) {
                const double c = CX[g.node(wrap(i - 1 + ex, g.nx), wrap(j - 1 + ey, g.ny), wrap(k - 1 + ez, g.nz))];
                const int ca = corner_of(1 - ex, 1 - ey, 1 - ez);
                for (int d = 0; d < 3; ++d) dg[d] += c * cPKe64[(3 * ca + d) * 24 + 3 * ca + d];
            }
    for (int d = 0; d < 3; ++d) rdiag[3 * n + d] = n == 0 ? 0.0 : 1.0 / dg[d];
}

// Coarse element scales: CX_c = 2 mean of the eight children (mgcg9.cu:753-781).
__global__ void pcoarse_cx_kernel(PGrid gc, const double *__restrict__ CXf, double *__restrict__ CXc)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= gc.nnod()) return;
    const PGrid gf{2 * gc.nx, 2 * gc.ny, 2 * gc.nz};
    const int j = (int)(e % gc.ny);
    const long long t = e / gc.ny;
    const int k = (int)(t % gc.nz), i = (int)(t / gc.nz);
    double s = 0.0;
    for (int a = 0; a < 2; ++a)
        for (int c = 0; c < 2; ++c)
            for (int b = 0; b < 2; ++b) s += CXf[gf.node(2 * i + a, 2 * j + b, 2 * k + c)];
    CXc[e] = 0.25 * s;
}

// Full-weighting restriction (the transpose of the trilinear prolongation):
// coarse node (I, J, K) gathers fine nodes (2I + dx, ...) with weights
// 1, 1/2 per direction; node 0 gets zero.
__global__ void prestrict_kernel(PGrid gc, const float *__restrict__ rf, float *__restrict__ fc, const int *done)
{
    if (done && *done) return;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= gc.nnod()) return;
    const PGrid gf{2 * gc.nx, 2 * gc.ny, 2 * gc.nz};
    const int J = (int)(n % gc.ny);
    const long long t = n / gc.ny;
    const int K = (int)(t % gc.nz), I = (int)(t / gc.nz);
    float acc[3 * NR];
#pragma unroll
    for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.f;
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                const float w = (dx ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dz ? 0.5f : 1.f);
                const long long fn = gf.node(wrap(2 * I + dx, gf.nx), wrap(2 * J + dy, gf.ny), wrap(2 * K + dz, gf.nz));
                const float *src = rf + fn * 3 * NR;
#pragma unroll
                for (int q = 0; q < 3 * NR; ++q) acc[q] = fmaf(w, src[q], acc[q]);
            }
    float *dst = fc + n * 3 * NR;
#pragma unroll
    for (int q = 0; q < 3 * NR; ++q) dst[q] = n == 0 ? 0.f : acc[q];
}

// u_f += P u_c (trilinear, periodic); node 0 stays zero.
__global__ void pprolong_kernel(PGrid gf, const float *__restrict__ uc, float *__restrict__ uf, const int *done)
{
    if (done && *done) return;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= gf.nnod()) return;
    const PGrid gc{gf.nx / 2, gf.ny / 2, gf.nz / 2};
    const int j = (int)(n % gf.ny);
    const long long t = n / gf.ny;
    const int k = (int)(t % gf.nz), i = (int)(t / gf.nz);
    const int ix[2] = {i >> 1, (i & 1) ? wrap((i >> 1) + 1, gc.nx) : (i >> 1)};
    const int iy[2] = {j >> 1, (j & 1) ? wrap((j >> 1) + 1, gc.ny) : (j >> 1)};
    const int iz[2] = {k >> 1, (k & 1) ? wrap((k >> 1) + 1, gc.nz) : (k >> 1)};
    const int mx = (i & 1) ? 2 : 1, my = (j & 1) ? 2 : 1, mz = (k & 1) ? 2 : 1;
    const float w = 1.f / (float)(mx * my * mz);
    float acc[3 * NR];
#pragma unroll
    for (int q = 0; q < 3 * NR; ++q) acc[q] = 0.f;
    for (int a = 0; a < mx; ++a)
        for (int c = 0; c < mz; ++c)
            for (int b = 0; b < my; ++b) {
                const float *src = uc + gc.node(ix[a], iy[b], iz[c]) * 3 * NR;
#pragma unroll
                for (int q = 0; q < 3 * NR; ++q) acc[q] += src[q];
            }
    float *dst = uf + n * 3 * NR;
#pragma unroll
    for (int q = 0; q < 3 * NR; ++q) dst[q] = n == 0 ? 0.f : fmaf(w, acc[q], dst[q]);
}

// Dense coarsest matrix (row per thread, no atomics); node 0's rows and
// columns become the identity.
__global__ void pdense_kernel(PGrid g, const double *__restrict__ CX, double *__restrict__ A)
{
    const int nd = (int)g.ndof();
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nd) return;
    double *Ar = A + (long long)row * nd;
    for (int c = 0; c < nd; ++c) Ar[c] = 0.0;
    const int n = row / 3, d = row - 3 * n;
    if (n == 0) {
        Ar[row] = 1.0;
        return;
    }
    const int j = n % g.ny, t = n / g.ny, k = t % g.nz, i = t / g.nz;
    for (int ex = 0; ex < 2; ++ex)
        for (int ey = 0; ey < 2; ++ey)
            for (int ez = 0; ez < 2; ++ez) {
                const int ei = wrap(i - 1 + ex, g.nx), ej = wrap(j - 1 + ey, g.ny), ek = wrap(k - 1 + ez, g.nz);
                const double c = CX[g.node(ei, ej, ek)];
                const int ca = corner_of(1 - ex, 1 - ey, 1 - ez);
                for (int cb = 0; cb < 8; ++cb) {
                    const int bx = local_x(cb), by = local_y(cb), bz = local_z(cb);
                    const long long nb = g.node(wrap(ei + bx, g.nx), wrap(ej + by, g.ny), wrap(ek + bz, g.nz));
                    if (nb == 0) continue;
                    for (int b = 0; b < 3; ++b) Ar[3 * nb + b] += c * cPKe64[(3 * ca + d) * 24 + 3 * cb + b];
                }
            }
}

// y = M x on the coarsest grid for the six cases (warp per row; lower: the
// lower triangle of M, else the upper).
template <typename Tin, typename Tout>
__global__ void pgemv6_kernel(int n, const double *__restrict__ M, const Tin *__restrict__ x, Tout *__restrict__ y,
                              int lower, const int *done)
{
    if (done && *done) return;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= n) return;
    const int lo = lower ? 0 : row, hi = lower ? row + 1 : n;
    const double *mr = M + (long long)row * n;
    double s[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) s[r] = 0.0;
    for (int c = lo + lane; c < hi; c += 32) {
        const double m = mr[c];
#pragma unroll
        for (int r = 0; r < NR; ++r) s[r] = fma(m, (double)x[(long long)c * NR + r], s[r]);
    }
#pragma unroll
    for (int r = 0; r < NR; ++r)
        for (int o = 16; o > 0; o >>= 1) s[r] += __shfl_xor_sync(0xffffffffu, s[r], o);
    if (lane < NR) {
        double v = s[0];
#pragma unroll
        for (int r = 1; r < NR; ++r)
            if (lane == r) v = s[r];
        y[(long long)row * NR + lane] = (Tout)v;
    }
}

// The right-hand sides f[dof][r] = -sum_e CX_e (Ke u0_r)[local dof].
__global__ void pload_kernel(PGrid g, const double *__restrict__ CX, double *__restrict__ F)
{
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    const int j = (int)(n % g.ny);
    const long long t = n / g.ny;
    const int k = (int)(t % g.nz), i = (int)(t / g.nz);
    double f[3][NR] = {};
    for (int ex = 0; ex < 2; ++ex)
        for (int ey = 0; ey < 2; ++ey)
            for (int ez = 0; ez < 2; ++ez) {
                const double c = CX[g.node(wrap(i - 1 + ex, g.nx), wrap(j - 1 + ey, g.ny), wrap(k - 1 + ez, g.nz))];
                const int ca = corner_of(1 - ex, 1 - ey, 1 - ez);
                for (int d = 0; d < 3; ++d)
                    for (int r = 0; r < NR; ++r) f[d][r] -= c * cPG[(3 * ca + d) * NR + r];
            }
    for (int d = 0; d < 3; ++d)
        for (int r = 0; r < NR; ++r) F[(3 * n + d) * NR + r] = n == 0 ? 0.0 : f[d][r];
}

// ---- PCG over the six cases (FP64) ----------------------------------------

struct HScal {
    double res0[NR], rho[NR], alpha[NR], beta[NR], relres[NR], rr[NR];
    int done_r[NR], nit[NR];
    double tol;
    int iter, maxit, done, status;
};

// Per-block partial sums of K values per dof group -> partial[block][K].
template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double *partial)
{
    __shared__ double red[8][K];
#pragma unroll
    for (int q = 0; q < K; ++q)
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) red[threadIdx.x >> 5][q] = v[q];
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += red[w][threadIdx.x];
        partial[blockIdx.x * K + threadIdx.x] = s;
    }
}

// U = 0, R = F, float(R), |F_r|^2 partials.
__global__ void __launch_bounds__(256) pinit_kernel(long long nd, const double *__restrict__ F, double *__restrict__ U,
                                                    double *__restrict__ R, float *__restrict__ Rf,
                                                    double *__restrict__ partial)
{
    double s[NR] = {};
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < nd; d += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const double f = F[d * NR + r];
            U[d * NR + r] = 0.0;
            R[d * NR + r] = f;
            Rf[d * NR + r] = (float)f;
            s[r] = fma(f, f, s[r]);
        }
    block_partials<NR>(s, partial);
}

// U += alpha P, R -= alpha Q, float(R), |R_r|^2 partials.
__global__ void __launch_bounds__(256) pupdate_kernel(long long nd, double *__restrict__ U, double *__restrict__ R,
                                                      const double *__restrict__ P, const double *__restrict__ Q,
                                                      float *__restrict__ Rf, const HScal *__restrict__ sc,
                                                      double *__restrict__ partial)
{
    if (sc->done) return;
    double al[NR], s[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        al[r] = sc->alpha[r];
        s[r] = 0.0;
    }
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < nd; d += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const long long q = d * NR + r;
            U[q] = fma(al[r], P[q], U[q]);
            const double rv = fma(-al[r], Q[q], R[q]);
            R[q] = rv;
            Rf[q] = (float)rv;
            s[r] = fma(rv, rv, s[r]);
        }
    block_partials<NR>(s, partial);
}

// r'z and r'z_old per case.
__global__ void __launch_bounds__(256) pdot2_kernel(long long nd, const double *__restrict__ R,
                                                    const float *__restrict__ Z, const float *__restrict__ Zo,
                                                    double *__restrict__ partial, const HScal *__restrict__ sc)
{
    if (sc && sc->done) return;
    double s[2 * NR] = {};
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < nd; d += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const long long q = d * NR + r;
            const double rv = R[q];
            s[r] = fma(rv, (double)Z[q], s[r]);
            if (Zo) s[NR + r] = fma(rv, (double)Zo[q], s[NR + r]);
        }
    block_partials<2 * NR>(s, partial);
}

// P = z + beta P (beta = 0: P = z), z_old = z.
__global__ void __launch_bounds__(256) ppupdate_kernel(long long nd, const float *__restrict__ Z, double *__restrict__ P,
                                                       float *__restrict__ Zo, const HScal *__restrict__ sc, int first)
{
    if (sc->done && !first) return;
    double be[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) be[r] = first ? 0.0 : sc->beta[r];
    for (long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x; d < nd; d += (long long)gridDim.x * blockDim.x)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const long long q = d * NR + r;
            const float z = Z[q];
            P[q] = first ? (double)z : fma(be[r], P[q], (double)z);
            Zo[q] = z;
        }
}

enum PFinish { PF_INIT = 0, PF_RHO0 = 1, PF_ALPHA = 2, PF_END = 3 };

// Sums the per-block partials in fixed order and moves the scalars (one
// block).  INIT: res0; RHO0: rho; ALPHA: alpha = rho / p'q (0 for finished
// cases); END (partials: r'z, r'z_old; rr from the update): beta, relres,
// convergence per case, iteration count.
__global__ void __launch_bounds__(256) pfinish_kernel(int nb, const double *__restrict__ partial,
                                                      const double *__restrict__ partial_rr, HScal *sc, int which)
{
    if (which >= PF_ALPHA && sc->done) return;
    // pdot2 writes 2 NR partials per block (INIT: pinit, ALPHA: the apply, NR each)
    const int K = (which == PF_END || which == PF_RHO0) ? 2 * NR : NR;
    __shared__ double tot[2 * NR], tot_rr[NR];
    // thread q sums column q (fixed order: deterministic)
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += partial[(long long)b * K + threadIdx.x];
        tot[threadIdx.x] = s;
    }
    if (which == PF_END && threadIdx.x >= 32 && threadIdx.x < 32 + NR) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += partial_rr[(long long)b * NR + threadIdx.x - 32];
        tot_rr[threadIdx.x - 32] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    if (which == PF_INIT) {
        for (int r = 0; r < NR; ++r) {
            sc->res0[r] = sqrt(tot[r]);
            sc->relres[r] = 1.0;
            sc->nit[r] = sc->maxit;
            sc->done_r[r] = 0;
            if (!isfinite(sc->res0[r])) {
                sc->status = GPUTO_ERR_BREAKDOWN;
                sc->done_r[r] = 1;
            } else if (!(sc->res0[r] > 0.0)) {   // F_r = 0: chi_r = 0
                sc->done_r[r] = 1;
                sc->relres[r] = 0.0;
                sc->nit[r] = 0;
            }
        }
        int all = 1;
        for (int r = 0; r < NR; ++r) all &= sc->done_r[r];
        sc->done = all || sc->status || sc->maxit <= 0;
        sc->iter = 0;
    } else if (which == PF_RHO0) {
        for (int r = 0; r < NR; ++r) sc->rho[r] = tot[r];
    } else if (which == PF_ALPHA) {
        for (int r = 0; r < NR; ++r) {
            const double a = sc->rho[r] / tot[r];
            if (sc->done_r[r]) {
                sc->alpha[r] = 0.0;
            } else if (!(tot[r] > 0.0) || !isfinite(a)) {
                sc->alpha[r] = 0.0;
                sc->status = GPUTO_ERR_BREAKDOWN;
                sc->done = 1;
            } else {
                sc->alpha[r] = a;
            }
        }
    } else {
        const int it = sc->iter;
        int all = 1;
        for (int r = 0; r < NR; ++r) {
            if (!sc->done_r[r]) {
                const double rz = tot[r], rzo = tot[NR + r];
                sc->beta[r] = (rz - rzo) / sc->rho[r];
                sc->rho[r] = rz;
                sc->rr[r] = tot_rr[r];
                sc->relres[r] = sqrt(tot_rr[r]) / sc->res0[r];
                if (!isfinite(sc->relres[r]) || !isfinite(sc->beta[r])) {
                    sc->status = GPUTO_ERR_BREAKDOWN;
                    sc->done_r[r] = 1;
                    sc->nit[r] = it;
                } else if (sc->relres[r] < sc->tol) {
                    sc->done_r[r] = 1;
                    sc->nit[r] = it;
                }
            } else {
                sc->beta[r] = 0.0;
            }
            all &= sc->done_r[r];
        }
        sc->iter = it + 1;
        if (all || sc->status || it + 1 >= sc->maxit) sc->done = 1;
    }
}

// C_rs partials: per element W_r = u0_r + chi_r (24 values), C_rs += CX_e
// W_r' Ke W_s; the 21 upper-triangle entries per block.
__global__ void __launch_bounds__(256) pceff_kernel(PGrid g, const double *__restrict__ CX,
                                                    const double *__restrict__ U, double *__restrict__ partial)
{
    double c[21] = {};
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < g.nnod();
         e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e % g.ny);
        const long long t = e / g.ny;
        const int k = (int)(t % g.nz), i = (int)(t / g.nz);
        long long nodes[8];
#pragma unroll
        for (int a = 0; a < 8; ++a)
            nodes[a] = g.node(wrap(i + local_x(a), g.nx), wrap(j + local_y(a), g.ny), wrap(k + local_z(a), g.nz));
        const double cx = CX[e];
        int q = 0;
#pragma unroll 1
        for (int r = 0; r < NR; ++r) {
            double w[24], kw[24];
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    w[3 * a + d] = cPU0[r * 24 + 3 * a + d] + U[(3 * nodes[a] + d) * NR + r];
#pragma unroll
            for (int m = 0; m < 24; ++m) {
                double s = 0.0;
#pragma unroll
                for (int p = 0; p < 24; ++p) s = fma(cPKe64[m * 24 + p], w[p], s);
                kw[m] = s;
            }
#pragma unroll 1
            for (int s2 = r; s2 < NR; ++s2, ++q) {
                double dot = 0.0;
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        dot = fma(cPU0[s2 * 24 + 3 * a + d] + U[(3 * nodes[a] + d) * NR + s2], kw[3 * a + d], dot);
                // q indexes the upper triangle in row order
#pragma unroll
                for (int z = 0; z < 21; ++z)
                    if (z == q) c[z] = fma(cx, dot, c[z]);
            }
        }
    }
    block_partials<21>(c, partial);
}

inline unsigned nblk(long long n, int bs = 256) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

// ---------------------------------------------------------------------------

struct Homog {
    int nl = 0, device = 0, nc = 0;
    PGrid g[kMaxLevels]{};
    gputo_options opt{};
    cudaStream_t own_stream = nullptr;
    std::vector<void *> owned;
    size_t bytes = 0;
    // FP64 outer vectors [ndof][6]
    double *F = nullptr, *U = nullptr, *R = nullptr, *P = nullptr, *Q = nullptr;
    float *Rf = nullptr, *Zold = nullptr;
    // per level: element scales (FP64 natural, FP32), 1/diag (FP64, FP32), FP32 buffers [ndof_l][6]
    double *CXd[kMaxLevels]{}, *rdd[kMaxLevels]{};
    float *CXf[kMaxLevels]{}, *rdf[kMaxLevels]{};
    float *u0[kMaxLevels]{}, *u1[kMaxLevels]{}, *fl[kMaxLevels]{}, *rl[kMaxLevels]{};
    // coarsest
    double *A = nullptr, *Linv = nullptr, *LinvT = nullptr, *ctmp = nullptr;
    int *info = nullptr;
    HScal *sc = nullptr, *h_sc = nullptr;
    double *part = nullptr, *part_rr = nullptr, *part_c = nullptr;
    int nb_red = 0;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;

    ~Homog()
    {
        if (own_stream) cudaStreamSynchronize(own_stream);
        if (graph) cudaGraphExecDestroy(graph);
        for (void *p : owned) cudaFree(p);
        if (h_sc) cudaFreeHost(h_sc);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    template <typename T>
    int alloc(T **p, long long count)
    {
        const size_t b = sizeof(T) * (size_t)std::max(count, 1LL);
        cudaError_t e = cudaMalloc((void **)p, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            *p = nullptr;
            set_error("cudaMalloc of " + std::to_string(b) + " bytes failed: " + cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? GPUTO_ERR_OOM : GPUTO_ERR_CUDA;
        }
        owned.push_back(*p);
        bytes += b;
        GPUTO_CUDA(cudaMemsetAsync(*p, 0, b, own_stream));
        return GPUTO_OK;
    }

    int create(int nx, int ny, int nz, int nl_, const gputo_options *o)
    {
        if (o) opt = *o;
        else gputo_default_options(&opt);
        if (nl_ < 1 || nl_ > kMaxLevels || nx < 2 || ny < 2 || nz < 2) {
            set_error("periodic cell sizes must be >= 2 and 1 <= nl <= 12");
            return GPUTO_ERR_ARG;
        }
        const int m = 1 << (nl_ - 1);
        if (nx % m || ny % m || nz % m || nx / m < 2 || ny / m < 2 || nz / m < 2) {
            set_error("nx, ny, nz must be divisible by 2^(nl-1), with at least 2 coarsest elements per direction");
            return GPUTO_ERR_ARG;
        }
        if (opt.nswp < 1 || !(opt.omega > 0) || opt.check_every < 1) {
            set_error("homogenization needs nswp >= 1, omega > 0 and check_every >= 1");
            return GPUTO_ERR_ARG;
        }
        nl = nl_;
        for (int l = 0; l < nl; ++l) g[l] = PGrid{nx >> l, ny >> l, nz >> l};
        nc = (int)g[nl - 1].ndof();
        if (nc > opt.max_coarse_dofs) {
            set_error("coarsest grid has " + std::to_string(nc) + " dofs, above max_coarse_dofs=" +
                      std::to_string(opt.max_coarse_dofs) + "; use more levels");
            return GPUTO_ERR_ARG;
        }
        GPUTO_CUDA(cudaGetDevice(&device));
        GPUTO_CUDA(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
        const long long nv = g[0].ndof() * NR;
        int s = GPUTO_OK;
        if (!s) s = alloc(&F, nv);
        if (!s) s = alloc(&U, nv);
        if (!s) s = alloc(&R, nv);
        if (!s) s = alloc(&P, nv);
        if (!s) s = alloc(&Q, nv);
        if (!s) s = alloc(&Rf, nv);
        if (!s) s = alloc(&Zold, nv);
        for (int l = 0; l < nl && !s; ++l) {
            const long long nvl = g[l].ndof() * NR;
            s = alloc(&CXd[l], g[l].nnod());
            if (!s) s = alloc(&CXf[l], g[l].nnod());
            if (!s) s = alloc(&rdd[l], g[l].ndof());
            if (!s) s = alloc(&rdf[l], g[l].ndof());
            if (!s) s = alloc(&u0[l], nvl);
            if (!s) s = alloc(&u1[l], nvl);
            if (!s && l > 0) s = alloc(&fl[l], nvl);
            if (!s) s = alloc(&rl[l], nvl);
        }
        if (!s) s = alloc(&A, (long long)nc * nc);
        if (!s) s = alloc(&Linv, (long long)nc * nc);
        if (!s) s = alloc(&LinvT, (long long)nc * nc);
        if (!s) s = alloc(&ctmp, (long long)nc * NR);
        if (!s) s = alloc(&info, 4);
        if (!s) s = alloc(&sc, 1);
        nb_red = (int)std::min<long long>(kHBlocks, std::max(1LL, (g[0].ndof() + 255) / 256));
        const int nb_apply = (int)nblk(g[0].nnod());
        if (!s) s = alloc(&part, (long long)std::max(nb_apply, nb_red) * 2 * NR);
        if (!s) s = alloc(&part_rr, (long long)nb_red * NR);
        if (!s) s = alloc(&part_c, (long long)nb_red * 21);
        if (s) return s;
        GPUTO_CUDA(cudaMallocHost((void **)&h_sc, sizeof(HScal)));
        GPUTO_CUDA(cudaStreamSynchronize(own_stream));
        return GPUTO_OK;
    }

    int upload_ke(const double *Ke, cudaStream_t st)
    {
        for (int m = 0; m < 576; ++m)
            if (!std::isfinite(Ke[m])) {
                set_error("Ke0 has a non-finite entry");
                return GPUTO_ERR_ARG;
            }
        float kf[576];
        for (int m = 0; m < 576; ++m) kf[m] = (float)Ke[m];
        // u0_r at the local corners and G = Ke u0
        double u0h[NR * 24] = {}, gh[24 * NR] = {};
        for (int a = 0; a < 8; ++a) {
            const double x = local_x(a), y = local_y(a), z = local_z(a);
            const double f[NR][3] = {{x, 0, 0}, {0, y, 0}, {0, 0, z}, {0, z / 2, y / 2}, {z / 2, 0, x / 2},
                                     {y / 2, x / 2, 0}};
            for (int r = 0; r < NR; ++r)
                for (int d = 0; d < 3; ++d) u0h[r * 24 + 3 * a + d] = f[r][d];
        }
        for (int m = 0; m < 24; ++m)
            for (int r = 0; r < NR; ++r) {
                double sum = 0.0;
                for (int p = 0; p < 24; ++p) sum += Ke[m * 24 + p] * u0h[r * 24 + p];
                gh[m * NR + r] = sum;
            }
        GPUTO_CUDA(cudaMemcpyToSymbolAsync(cPKe64, Ke, sizeof(double) * 576, 0, cudaMemcpyHostToDevice, st));
        GPUTO_CUDA(cudaMemcpyToSymbolAsync(cPKe32, kf, sizeof(kf), 0, cudaMemcpyHostToDevice, st));
        GPUTO_CUDA(cudaMemcpyToSymbolAsync(cPU0, u0h, sizeof(u0h), 0, cudaMemcpyHostToDevice, st));
        GPUTO_CUDA(cudaMemcpyToSymbolAsync(cPG, gh, sizeof(gh), 0, cudaMemcpyHostToDevice, st));
        GPUTO_CUDA(cudaStreamSynchronize(st));   // the host arrays are on the stack
        return GPUTO_OK;
    }

    // Hierarchy for CX (device, natural order, FP64).
    int setup(const double *CX, cudaStream_t st)
    {
        GPUTO_CUDA(cudaMemcpyAsync(CXd[0], CX, sizeof(double) * g[0].nnod(), cudaMemcpyDeviceToDevice, st));
        for (int l = 1; l < nl; ++l)
            pcoarse_cx_kernel<<<nblk(g[l].nnod()), 256, 0, st>>>(g[l], CXd[l - 1], CXd[l]);
        for (int l = 0; l < nl; ++l) {
            pdiag_kernel<<<nblk(g[l].nnod()), 256, 0, st>>>(g[l], CXd[l], rdd[l]);
            launch_cast_f32(g[l].nnod(), CXd[l], CXf[l], st);
            launch_cast_f32(g[l].ndof(), rdd[l], rdf[l], st);
        }
        pdense_kernel<<<nblk(nc), 256, 0, st>>>(g[nl - 1], CXd[nl - 1], A);
        launch_cholesky(nc, A, info, st);
        launch_tri_inverse(nc, A, Linv, LinvT, st);
        pload_kernel<<<nblk(g[0].nnod()), 256, 0, st>>>(g[0], CXd[0], F);
        count_launches(4 * nl + 4);
        int h_info = 0;
        GPUTO_CUDA(cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, st));
        GPUTO_CUDA(cudaStreamSynchronize(st));
        GPUTO_CUDA(cudaGetLastError());
        if (h_info) {
            set_error("coarsest periodic matrix is not positive definite (pivot " + std::to_string(h_info) + ")");
            return GPUTO_ERR_NOT_SPD;
        }
        return GPUTO_OK;
    }

    template <int MODE>
    void sweep(int l, const float *u, const float *f, float *out, const int *done, cudaStream_t st)
    {
        psweep_kernel<float, MODE><<<nblk(g[l].nnod()), 256, 0, st>>>(
            g[l], CXf[l], u, f, rdf[l], out, (float)opt.omega, (float)opt.prerelax, nullptr, done);
        count_launches(1);
    }

    // z = M r on all six cases (FP32), the solver's V-cycle schedule.
    void vcycle(const float *r0, float *z0, const int *done, cudaStream_t st)
    {
        const int ns = opt.nswp;
        auto buf = [&](int l, int which) -> float * {
            if (l == 0) return which ? z0 : u0[0];
            return which ? u1[l] : u0[l];
        };
        for (int l = 0; l < nl; ++l) {
            const float *f = l == 0 ? r0 : fl[l];
            if (l > 0) {
                prestrict_kernel<<<nblk(g[l].nnod()), 256, 0, st>>>(g[l], rl[l - 1], fl[l], done);
                count_launches(1);
            }
            if (l < nl - 1) {
                for (int s = 0; s < ns; ++s) {
                    if (s == 0) sweep<P_PRE>(l, nullptr, f, buf(l, 0), done, st);
                    else sweep<P_JACOBI>(l, buf(l, (s - 1) & 1), f, buf(l, s & 1), done, st);
                }
                sweep<P_DEFECT>(l, buf(l, (ns - 1) & 1), f, rl[l], done, st);
            } else {
                const unsigned nbw = (unsigned)((nc * 32 + 255) / 256);
                pgemv6_kernel<float, double><<<nbw, 256, 0, st>>>(nc, Linv, f, ctmp, 1, done);
                pgemv6_kernel<double, float><<<nbw, 256, 0, st>>>(nc, LinvT, ctmp, buf(l, 1), 0, done);
                count_launches(2);
            }
        }
        for (int l = nl - 2; l >= 0; --l) {
            const float *f = l == 0 ? r0 : fl[l];
            int cur = (ns - 1) & 1;
            pprolong_kernel<<<nblk(g[l].nnod()), 256, 0, st>>>(g[l], buf(l + 1, 1), buf(l, cur), done);
            count_launches(1);
            // starting from buffer (ns - 1) & 1, ns sweeps end in buffer 1
            for (int s = 0; s < ns; ++s) {
                sweep<P_JACOBI>(l, buf(l, cur), f, buf(l, cur ^ 1), done, st);
                cur ^= 1;
            }
        }
    }

    // One flexible PCG iteration of all six cases.
    void iteration(cudaStream_t st)
    {
        const long long nd = g[0].ndof();
        const int *done = &sc->done;
        const int nb = (int)nblk(g[0].nnod());
        psweep_kernel<double, P_APPLY><<<nb, 256, 0, st>>>(g[0], CXd[0], P, nullptr, nullptr, Q, 1.0, 0.0, part, done);
        pfinish_kernel<<<1, 256, 0, st>>>(nb, part, nullptr, sc, PF_ALPHA);
        pupdate_kernel<<<nb_red, 256, 0, st>>>(nd, U, R, P, Q, Rf, sc, part_rr);
        vcycle(Rf, u1[0], done, st);
        pdot2_kernel<<<nb_red, 256, 0, st>>>(nd, R, u1[0], Zold, part, sc);
        pfinish_kernel<<<1, 256, 0, st>>>(nb_red, part, part_rr, sc, PF_END);
        ppupdate_kernel<<<nb_red, 256, 0, st>>>(nd, u1[0], P, Zold, sc, 0);
        count_launches(7);
    }

    int run_graph(int batch, cudaStream_t st)
    {
        if (!graph || graph_stream != st) {
            if (graph) cudaGraphExecDestroy(graph);
            graph = nullptr;
            cudaGraph_t gr;
            GPUTO_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            iteration(st);
            GPUTO_CUDA(cudaStreamEndCapture(st, &gr));
            cudaError_t e = cudaGraphInstantiate(&graph, gr, 0);
            cudaGraphDestroy(gr);
            GPUTO_CUDA(e);
            graph_stream = st;
        }
        for (int b = 0; b < batch; ++b) GPUTO_CUDA(cudaGraphLaunch(graph, st));
        return GPUTO_OK;
    }

    int solve(double tol, int maxit, double *Ceff, double *relres, int *nit, cudaStream_t st)
    {
        if (maxit < 0 || !(tol >= 0)) {
            set_error("maxit must be >= 0 and tol >= 0");
            return GPUTO_ERR_ARG;
        }
        const long long nd = g[0].ndof();
        HScal z{};
        z.tol = tol;
        z.maxit = maxit;
        GPUTO_CUDA(cudaMemcpyAsync(sc, &z, sizeof(HScal), cudaMemcpyHostToDevice, st));
        pinit_kernel<<<nb_red, 256, 0, st>>>(nd, F, U, R, Rf, part);
        pfinish_kernel<<<1, 256, 0, st>>>(nb_red, part, nullptr, sc, PF_INIT);
        vcycle(Rf, u1[0], &sc->done, st);
        pdot2_kernel<<<nb_red, 256, 0, st>>>(nd, R, u1[0], nullptr, part, nullptr);
        pfinish_kernel<<<1, 256, 0, st>>>(nb_red, part, nullptr, sc, PF_RHO0);
        ppupdate_kernel<<<nb_red, 256, 0, st>>>(nd, u1[0], P, Zold, sc, 1);
        count_launches(5);
        GPUTO_CUDA(cudaStreamSynchronize(st));   // the host struct z is on the stack
        int it = 0;
        for (;;) {
            GPUTO_CUDA(cudaMemcpyAsync(h_sc, sc, sizeof(HScal), cudaMemcpyDeviceToHost, st));
            GPUTO_CUDA(cudaStreamSynchronize(st));
            if (h_sc->done || it >= maxit) break;
            const int batch = std::min(opt.check_every, maxit - it);
            if (opt.use_graph) {
                int s = run_graph(batch, st);
                if (s) return s;
            } else {
                for (int b = 0; b < batch; ++b) iteration(st);
            }
            it += batch;
        }
        GPUTO_CUDA(cudaGetLastError());
        for (int r = 0; r < NR; ++r) {
            if (relres) relres[r] = h_sc->relres[r];
            if (nit) nit[r] = h_sc->done_r[r] ? h_sc->nit[r] : h_sc->iter;
        }
        if (h_sc->status) {
            set_error("homogenization PCG breakdown (non-finite loads or p'q <= 0)");
            return h_sc->status;
        }
        if (Ceff) {
            const unsigned nbc = (unsigned)std::min<long long>(kHBlocks, (long long)nblk(g[0].nnod()));
            pceff_kernel<<<nbc, 256, 0, st>>>(g[0], CXd[0], U, part_c);
            count_launches(1);
            std::vector<double> hp((size_t)nbc * 21);
            GPUTO_CUDA(cudaMemcpyAsync(hp.data(), part_c, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, st));
            GPUTO_CUDA(cudaStreamSynchronize(st));
            double c[21] = {};
            for (unsigned b = 0; b < nbc; ++b)
                for (int q = 0; q < 21; ++q) c[q] += hp[(size_t)b * 21 + q];
            const double inv = 1.0 / (double)g[0].nnod();
            int q = 0;
            for (int r = 0; r < NR; ++r)
                for (int s2 = r; s2 < NR; ++s2, ++q) Ceff[r * NR + s2] = Ceff[s2 * NR + r] = c[q] * inv;
        }
        return GPUTO_OK;
    }
};

}  // namespace gputo

struct gputo_homog {
    gputo::Homog h;
};

extern "C" {

int gputo_homog_create(gputo_homog **out, int nx, int ny, int nz, int nl, const gputo_options *opt)
{
    if (!out) return GPUTO_ERR_ARG;
    *out = nullptr;
    int dev = 0, major = 0, n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        gputo::set_error("no CUDA device is visible");
        return GPUTO_ERR_NO_DEVICE;
    }
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) {
        gputo::set_error("gputo is built for sm_100a (B200)");
        return GPUTO_ERR_NO_DEVICE;
    }
    auto *h = new gputo_homog();
    const int st = h->h.create(nx, ny, nz, nl, opt);
    if (st) {
        delete h;
        return st;
    }
    *out = h;
    return GPUTO_OK;
}

void gputo_homog_destroy(gputo_homog *h) { delete h; }

size_t gputo_homog_device_bytes(const gputo_homog *h) { return h ? h->h.bytes : 0; }

int gputo_homog_solve_dev(gputo_homog *hh, const double *Ke0, const double *CX, double tol, int maxit,
                          double *Ceff, double *relres, int *nit, double *chi, void *stream)
{
    if (!hh || !Ke0 || !CX) return GPUTO_ERR_ARG;
    gputo::Homog &h = hh->h;
    cudaStream_t st = stream ? (cudaStream_t)stream : h.own_stream;
    int s = h.upload_ke(Ke0, st);
    if (!s) s = h.setup(CX, st);
    if (!s) s = h.solve(tol, maxit, Ceff, relres, nit, st);
    if (!s && chi) {
        GPUTO_CUDA(cudaMemcpyAsync(chi, h.U, sizeof(double) * h.g[0].ndof() * gputo::NR, cudaMemcpyDeviceToDevice, st));
        GPUTO_CUDA(cudaStreamSynchronize(st));
    }
    return s;
}

}  // extern "C"
