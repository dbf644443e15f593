// Level-1 multigrid operator without stored element matrices.
//
// The reference's first coarse level (mgcg1.cu:2042-2070 coarseAe2c) is the
// stiffness of each 2h element integrated with its 2x2x2 Gauss rule, every
// Gauss point weighted by the density of the fine element it lies in:
//     A_E = sum_g CX_g Kg[g],   Kg[g] = w B_g^T D B_g   (w = (h/2)^3 = 1 at h = 2).
// The reference stores 300 doubles per coarse element for it.  Here it is
// applied on the fly in two deterministic passes:
//   1. one thread per coarse element: strain at each Gauss point, stress
//      CX_g D eps_g, and y_E = sum_g B_g^T sigma_g into a scratch of 24 values
//      per element (structure of arrays, coalesced);
//   2. one thread per node: the sum of its rows of y over the (up to) 8
//      elements around it, followed by the same epilogues as the other sweeps
//      (K u, f - K u, damped Jacobi, Dirichlet rows zeroed).
// The strain-displacement values at the Gauss points are compile-time
// constants, so pass 1 costs about 1250 FMAs per element with no table reads.
#include "gputo_internal.h"

namespace gputo {

// dN_a/dx_p at Gauss point (ix, iy, iz) of a cube of edge h = 2:
// 0.25 * sgn_p(a) * (product of (1 + sgn_q(a) gp_q) over the other axes) / h.
__host__ __device__ constexpr double gauss_coord(int i) { return i ? 0.57735026918962576451 : -0.57735026918962576451; }
__host__ __device__ constexpr double sgn(int v) { return v ? 1.0 : -1.0; }
__host__ __device__ constexpr double dN(int a, int p, int ix, int iy, int iz)
{
    const double fx = 1.0 + sgn(local_x(a)) * gauss_coord(ix);
    const double fy = 1.0 + sgn(local_y(a)) * gauss_coord(iy);
    const double fz = 1.0 + sgn(local_z(a)) * gauss_coord(iz);
    return p == 0 ? 0.125 * sgn(local_x(a)) * fy * fz
         : p == 1 ? 0.125 * sgn(local_y(a)) * fx * fz
                  : 0.125 * sgn(local_z(a)) * fx * fy;
}

template <typename T, bool PRE>
__global__ void __launch_bounds__(128)
quad_element_kernel(Lay L, const T *__restrict__ CXp, ELay Ef,
                    const T *__restrict__ u, const T *__restrict__ f, const T *__restrict__ diag,
                    T prerelax, T lam, T mu, T *__restrict__ y, const int *__restrict__ done)
{
    if (done && *done) return;
    const Grid &g = L.g;
    const long long nel = g.nel();
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nel) return;
    const long long t = e / g.ny;
    const int j = (int)(e - t * g.ny);
    const int i = (int)(t / g.nz);
    const int k = (int)(t - (long long)i * g.nz);
    T ue[24];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const long long nb = L.at(i + local_x(a), j + local_y(a), k + local_z(a));
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            if (PRE) {
                const T dv = diag[nb + q];
                ue[3 * a + q] = dv != T(0) ? prerelax * f[nb + q] / dv : T(0);
            } else {
                ue[3 * a + q] = u[nb + q];
            }
        }
    }
    T ye[24];
#pragma unroll
    for (int m = 0; m < 24; ++m) ye[m] = T(0);
#pragma unroll
    for (int ix = 0; ix < 2; ++ix)
#pragma unroll
        for (int iz = 0; iz < 2; ++iz)
#pragma unroll
            for (int iy = 0; iy < 2; ++iy) {
                const T c = CXp[Ef.at(2 * i + ix, 2 * j + iy, 2 * k + iz)];
                // displacement gradient G[d][p] = sum_a dN_a/dx_p u_{a,d}
                T G[3][3];
#pragma unroll
                for (int d = 0; d < 3; ++d)
#pragma unroll
                    for (int p = 0; p < 3; ++p) {
                        T s = T(0);
#pragma unroll
                        for (int a = 0; a < 8; ++a) s = fma(T(dN(a, p, ix, iy, iz)), ue[3 * a + d], s);
                        G[d][p] = s;
                    }
                // sigma = CX (lam tr(eps) I + 2 mu eps), eps = sym(G)
                const T tr = G[0][0] + G[1][1] + G[2][2];
                const T cl = c * lam, cm = c * mu;
                T S[3][3];
                S[0][0] = fma(cl, tr, T(2) * cm * G[0][0]);
                S[1][1] = fma(cl, tr, T(2) * cm * G[1][1]);
                S[2][2] = fma(cl, tr, T(2) * cm * G[2][2]);
                S[0][1] = S[1][0] = cm * (G[0][1] + G[1][0]);
                S[1][2] = S[2][1] = cm * (G[1][2] + G[2][1]);
                S[0][2] = S[2][0] = cm * (G[0][2] + G[2][0]);
                // y_{a,d} += sum_p dN_a/dx_p sigma[d][p]
#pragma unroll
                for (int a = 0; a < 8; ++a)
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        T s = ye[3 * a + d];
#pragma unroll
                        for (int p = 0; p < 3; ++p) s = fma(T(dN(a, p, ix, iy, iz)), S[d][p], s);
                        ye[3 * a + d] = s;
                    }
            }
#pragma unroll
    for (int m = 0; m < 24; ++m) y[(long long)m * nel + e] = ye[m];
}

template <typename T, int MODE>
__global__ void __launch_bounds__(128)
quad_node_kernel(Lay L, const T *__restrict__ y, const T *__restrict__ u, const T *__restrict__ f,
                 const T *__restrict__ diag, const uint8_t *__restrict__ mask, T *__restrict__ out,
                 T omega, T prerelax, const int *__restrict__ done)
{
    if (done && *done) return;
    const Grid &g = L.g;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    const long long t = n / (g.ny + 1);
    const int j = (int)(n - t * (g.ny + 1));
    const int i = (int)(t / (g.nz + 1));
    const int k = (int)(t - (long long)i * (g.nz + 1));
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
                for (int d = 0; d < 3; ++d) acc[d] += y[(long long)(3 * a + d) * nel + e];
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
            T us;
            if (MODE == MODE_JACOBI_PRE) {
                const T dv = diag[dof];
                us = dv != T(0) ? prerelax * f[dof] / dv : T(0);
            } else {
                us = u[dof];
            }
            out[dof] = us + omega * r / diag[dof];
        }
    }
}

template <typename T>
int launch_quad_sweep(int mode, const Lay &L, const ELay &Ef, const T *CX, const T *u, const T *f,
                      const T *diag, const uint8_t *mask, T *out, T omega, T prerelax, double nu,
                      T *yscratch, const int *done, int *, cudaStream_t st)
{
    const T lam = (T)(nu / ((1.0 + nu) * (1.0 - 2.0 * nu)));
    const T mu = (T)(1.0 / (2.0 * (1.0 + nu)));
    const int bs = 128;
    const unsigned eb = (unsigned)((L.g.nel() + bs - 1) / bs);
    const unsigned nb = (unsigned)((L.g.nnod() + bs - 1) / bs);
    if (mode == MODE_JACOBI_PRE)
        quad_element_kernel<T, true><<<eb, bs, 0, st>>>(L, CX, Ef, u, f, diag, prerelax, lam, mu,
                                                        yscratch, done);
    else
        quad_element_kernel<T, false><<<eb, bs, 0, st>>>(L, CX, Ef, u, f, diag, prerelax, lam, mu,
                                                         yscratch, done);
    switch (mode) {
    case MODE_APPLY:
        quad_node_kernel<T, MODE_APPLY><<<nb, bs, 0, st>>>(L, yscratch, u, f, diag, mask, out, omega, prerelax, done);
        break;
    case MODE_DEFECT:
        quad_node_kernel<T, MODE_DEFECT><<<nb, bs, 0, st>>>(L, yscratch, u, f, diag, mask, out, omega, prerelax, done);
        break;
    case MODE_JACOBI:
        quad_node_kernel<T, MODE_JACOBI><<<nb, bs, 0, st>>>(L, yscratch, u, f, diag, mask, out, omega, prerelax, done);
        break;
    default:
        quad_node_kernel<T, MODE_JACOBI_PRE><<<nb, bs, 0, st>>>(L, yscratch, u, f, diag, mask, out, omega, prerelax, done);
    }
    count_launches(2);
    return GPUTO_OK;
}

template int launch_quad_sweep<double>(int, const Lay &, const ELay &, const double *, const double *,
                                       const double *, const double *, const uint8_t *, double *, double,
                                       double, double, double *, const int *, int *, cudaStream_t);
template int launch_quad_sweep<float>(int, const Lay &, const ELay &, const float *, const float *,
                                      const float *, const float *, const uint8_t *, float *, float, float,
                                      double, float *, const int *, int *, cudaStream_t);

}  // namespace gputo

namespace gputo {

// Element-centric sweep for a level with stored (packed) element matrices:
// one thread per element reads its 300 matrix entries once (coalesced,
// structure of arrays) and writes y_E = A_E u_E; the node pass is the same
// deterministic gather as for level 1.  Used for the large coarse levels,
// where the node-centred form re-reads every entry from the 8 nodes around it.
template <typename T, bool PRE>
__global__ void __launch_bounds__(128)
packed_element_kernel(Lay L, const T *__restrict__ A, const T *__restrict__ u, const T *__restrict__ f,
                      const T *__restrict__ diag, T prerelax, T *__restrict__ y, const int *__restrict__ done)
{
    if (done && *done) return;
    const Grid &g = L.g;
    const long long nel = g.nel();
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nel) return;
    const long long t = e / g.ny;
    const int j = (int)(e - t * g.ny);
    const int i = (int)(t / g.nz);
    const int k = (int)(t - (long long)i * g.nz);
    T ue[24];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const long long nb = L.at(i + local_x(a), j + local_y(a), k + local_z(a));
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            if (PRE) {
                const T dv = diag[nb + q];
                ue[3 * a + q] = dv != T(0) ? prerelax * f[nb + q] / dv : T(0);
            } else {
                ue[3 * a + q] = u[nb + q];
            }
        }
    }
    T ye[24];
#pragma unroll
    for (int m = 0; m < 24; ++m) ye[m] = T(0);
#pragma unroll
    for (int m = 0; m < 24; ++m) {
#pragma unroll
        for (int n = 0; n <= m; ++n) {
            const T amn = A[(long long)packed_index(m, n) * nel + e];
            ye[m] = fma(amn, ue[n], ye[m]);
            if (n != m) ye[n] = fma(amn, ue[m], ye[n]);
        }
    }
#pragma unroll
    for (int m = 0; m < 24; ++m) y[(long long)m * nel + e] = ye[m];
}

template <typename T>
void launch_packed_sweep_ec(int mode, const Lay &L, const T *Apk, const T *u, const T *f, const T *diag,
                            const uint8_t *mask, T *out, T omega, T prerelax, T *yscratch,
                            const int *done, cudaStream_t st)
{
    const int bs = 128;
    const unsigned eb = (unsigned)((L.g.nel() + bs - 1) / bs);
    const unsigned nb = (unsigned)((L.g.nnod() + bs - 1) / bs);
    if (mode == MODE_JACOBI_PRE)
        packed_element_kernel<T, true><<<eb, bs, 0, st>>>(L, Apk, u, f, diag, prerelax, yscratch, done);
    else
        packed_element_kernel<T, false><<<eb, bs, 0, st>>>(L, Apk, u, f, diag, prerelax, yscratch, done);
    switch (mode) {
    case MODE_APPLY:
        quad_node_kernel<T, MODE_APPLY><<<nb, bs, 0, st>>>(L, yscratch, u, f, diag, mask, out, omega, prerelax, done);
        break;
    case MODE_DEFECT:
        quad_node_kernel<T, MODE_DEFECT><<<nb, bs, 0, st>>>(L, yscratch, u, f, diag, mask, out, omega, prerelax, done);
        break;
    case MODE_JACOBI:
        quad_node_kernel<T, MODE_JACOBI><<<nb, bs, 0, st>>>(L, yscratch, u, f, diag, mask, out, omega, prerelax, done);
        break;
    default:
        quad_node_kernel<T, MODE_JACOBI_PRE><<<nb, bs, 0, st>>>(L, yscratch, u, f, diag, mask, out, omega, prerelax, done);
    }
    count_launches(2);
}

template void launch_packed_sweep_ec<double>(int, const Lay &, const double *, const double *,
                                             const double *, const double *, const uint8_t *, double *,
                                             double, double, double *, const int *, cudaStream_t);
template void launch_packed_sweep_ec<float>(int, const Lay &, const float *, const float *, const float *,
                                            const float *, const uint8_t *, float *, float, float, float *,
                                            const int *, cudaStream_t);

}  // namespace gputo
