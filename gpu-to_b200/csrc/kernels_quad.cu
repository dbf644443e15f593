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
// Pass 1 works in the Hadamard basis of the element's corners: with
// V = T u, T[p][c] = (-1)^(p.c), the trilinear displacement is
// u(xi) = (1/8) sum_p (-1)^|p| xi^p V_p.  A derivative along one axis needs
// only the four modes with that axis' bit set and does not vary along that
// axis, so the gradients at all 8 Gauss points cost 72 operations; the
// adjoint sum_g B_g^T sigma_g comes back as y = (1/8) T W, W built from sums
// of the stress over the Gauss points.  About 530 operations per element
// instead of 1250 FMAs for the strain-displacement products.  In FP32 a
// thread takes two elements adjacent along y on float2 pairs.
#include "gputo_internal.h"
#include "hadamard.h"

namespace gputo {

// Hadamard transform of 8 values indexed by c = 4 x + 2 y + z:
// x_p <- sum_c (-1)^(p.c) x_c.
template <typename T>
__device__ __forceinline__ void fwht8(T (&x)[8])
{
#pragma unroll
    for (int b = 1; b < 8; b <<= 1)
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if (!(i & b)) {
                const T u = x[i], v = x[i | b];
                x[i] = u + v;
                x[i | b] = u - v;
            }
}

// Signed sums of P[i][j] (sign of the i-th and j-th Gauss coordinate):
// H = [sum P, sum s_i P, sum s_j P, sum s_i s_j P].
template <typename T>
__device__ __forceinline__ void h22(const T (&P)[2][2], T (&H)[4])
{
    const T r0 = P[0][0] + P[0][1], r1 = P[1][0] + P[1][1];
    const T q0 = P[0][1] - P[0][0], q1 = P[1][1] - P[1][0];
    H[0] = r0 + r1;
    H[1] = r1 - r0;
    H[2] = q0 + q1;
    H[3] = q1 - q0;
}

// Pass 1 of one element from its 24 corner values ue (corner a, component
// d at 3 a + d) and its 8 Gauss-point densities cg[ix][iz][iy] to its 24
// outputs.  V is the arithmetic type: float or double for one element, float2
// for two elements in one instruction stream (paired FP32 instructions).
template <typename V>
__device__ __forceinline__ void quad_body(const V (&ue)[24], const V (&cg)[2][2][2], V lam, V mu, V (&ye)[24])
{
    // corner a -> index c = 4 x + 2 y + z; modes p use the same bits
    V Vm[3][8];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int d = 0; d < 3; ++d) Vm[d][4 * local_x(a) + 2 * local_y(a) + local_z(a)] = ue[3 * a + d];
#pragma unroll
    for (int d = 0; d < 3; ++d) fwht8(Vm[d]);
    const V s = hconst<V>(0.57735026918962576451);   // Gauss coordinate 1/sqrt(3)
    // 8 x displacement gradient: Gx[d][iy][iz] = 8 du_d/dx at Gauss points
    // (., iy, iz), Gy[d][ix][iz], Gz[d][ix][iy] likewise
    V Gx[3][2][2], Gy[3][2][2], Gz[3][2][2];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const V si = i ? s : -s;
            const V ax = hfma(si, Vm[d][6], -Vm[d][4]), bx = hfma(-si, Vm[d][7], Vm[d][5]);
            const V ay = hfma(si, Vm[d][6], -Vm[d][2]), by = hfma(-si, Vm[d][7], Vm[d][3]);
            const V az = hfma(si, Vm[d][5], -Vm[d][1]), bz = hfma(-si, Vm[d][7], Vm[d][3]);
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const V sj = j ? s : -s;
                Gx[d][i][j] = hfma(sj, bx, ax);
                Gy[d][i][j] = hfma(sj, by, ay);
                Gz[d][i][j] = hfma(sj, bz, az);
            }
        }
    // stress at each Gauss point, summed over the axis its column does not
    // depend on: Px[d][iy][iz] = sum_ix sigma[d][x], Py[d][ix][iz], Pz[d][ix][iy]
    V Px[3][2][2], Py[3][2][2], Pz[3][2][2];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) Px[d][i][j] = Py[d][i][j] = Pz[d][i][j] = hzero<V>();
#pragma unroll
    for (int ix = 0; ix < 2; ++ix)
#pragma unroll
        for (int iz = 0; iz < 2; ++iz)
#pragma unroll
            for (int iy = 0; iy < 2; ++iy) {
                const V c = cg[ix][iz][iy];
                const V cl = c * lam, cm = c * mu, cm2 = cm + cm;   // lam, mu carry 1/64
                const V g00 = Gx[0][iy][iz], g01 = Gy[0][ix][iz], g02 = Gz[0][ix][iy];
                const V g10 = Gx[1][iy][iz], g11 = Gy[1][ix][iz], g12 = Gz[1][ix][iy];
                const V g20 = Gx[2][iy][iz], g21 = Gy[2][ix][iz], g22 = Gz[2][ix][iy];
                const V tr = g00 + g11 + g22;
                const V s00 = hfma(cl, tr, cm2 * g00), s11 = hfma(cl, tr, cm2 * g11), s22 = hfma(cl, tr, cm2 * g22);
                const V s01 = cm * (g01 + g10), s02 = cm * (g02 + g20), s12 = cm * (g12 + g21);
                Px[0][iy][iz] = Px[0][iy][iz] + s00;
                Px[1][iy][iz] = Px[1][iy][iz] + s01;
                Px[2][iy][iz] = Px[2][iy][iz] + s02;
                Py[0][ix][iz] = Py[0][ix][iz] + s01;
                Py[1][ix][iz] = Py[1][ix][iz] + s11;
                Py[2][ix][iz] = Py[2][ix][iz] + s12;
                Pz[0][ix][iy] = Pz[0][ix][iy] + s02;
                Pz[1][ix][iy] = Pz[1][ix][iy] + s12;
                Pz[2][ix][iy] = Pz[2][ix][iy] + s22;
            }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        V X[4], Y[4], Z[4];   // [00, 10, 01, 11]: sums weighted by the signs of the two Gauss coordinates
        h22(Px[d], X);
        h22(Py[d], Y);
        h22(Pz[d], Z);
        V W[8];
        W[0] = hzero<V>();
        W[1] = -Z[0];
        W[2] = -Y[0];
        W[3] = s * (Y[2] + Z[2]);
        W[4] = -X[0];
        W[5] = s * (X[2] + Z[1]);
        W[6] = s * (X[1] + Y[1]);
        W[7] = -(s * s) * (X[3] + Y[3] + Z[3]);
        fwht8(W);
#pragma unroll
        for (int a = 0; a < 8; ++a) ye[3 * a + d] = W[4 * local_x(a) + 2 * local_y(a) + local_z(a)];
    }
}

template <typename T, bool PRE>
__global__ void __launch_bounds__(128)
quad_element_kernel(Lay L, const T *__restrict__ CXp, ELay Ef,
                    const T *__restrict__ u, const T *__restrict__ f, const T *__restrict__ rdiag,
                    T prerelax, T lam, T mu, T *__restrict__ y, const int *__restrict__ done)
{
    pdl_wait();
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
                ue[3 * a + q] = prerelax * f[nb + q] * rdiag[nb + q];
            } else {
                ue[3 * a + q] = u[nb + q];
            }
        }
    }
    T cg[2][2][2];
#pragma unroll
    for (int ix = 0; ix < 2; ++ix)
#pragma unroll
        for (int iz = 0; iz < 2; ++iz)
#pragma unroll
            for (int iy = 0; iy < 2; ++iy) cg[ix][iz][iy] = CXp[Ef.at(2 * i + ix, 2 * j + iy, 2 * k + iz)];
    T ye[24];
    quad_body<T>(ue, cg, lam, mu, ye);
#pragma unroll
    for (int m = 0; m < 24; ++m) y[(long long)m * nel + e] = ye[m];
}

// FP32 pass 1 on element pairs (j, j + 1), j even (the level-1 ny is even):
// the shared node column j + 1 is loaded once, the arithmetic runs on float2
// (about half the instructions), and each output pair is one 8-byte store.
template <bool PRE>
__global__ void __launch_bounds__(128)
quad_element2_kernel(Lay L, const float *__restrict__ CXp, ELay Ef, const float *__restrict__ u,
                     const float *__restrict__ f, const float *__restrict__ rdiag, float prerelax, float lam,
                     float mu, float *__restrict__ y, const int *__restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    const Grid &g = L.g;
    const long long nel = g.nel();
    const long long e = 2 * ((long long)blockIdx.x * blockDim.x + threadIdx.x);
    if (e >= nel) return;
    const long long t = e / g.ny;
    const int j = (int)(e - t * g.ny);
    const int i = (int)(t / g.nz);
    const int k = (int)(t - (long long)i * g.nz);
    float2 ue[24];
#pragma unroll
    for (int x = 0; x < 2; ++x)
#pragma unroll
        for (int z = 0; z < 2; ++z) {
            const long long nb = L.at(i + x, j, k + z);   // node columns j, j + 1, j + 2
            float v[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) v[q] = PRE ? hmul(hmul(prerelax, f[nb + q]), rdiag[nb + q]) : u[nb + q];
#pragma unroll
            for (int yy = 0; yy < 2; ++yy) {
                const int a = local_index(x, yy, z);
#pragma unroll
                for (int d = 0; d < 3; ++d) ue[3 * a + d] = make_float2(v[3 * yy + d], v[3 * yy + 3 + d]);
            }
        }
    float2 cg[2][2][2];
#pragma unroll
    for (int ix = 0; ix < 2; ++ix)
#pragma unroll
        for (int iz = 0; iz < 2; ++iz)
#pragma unroll
            for (int iy = 0; iy < 2; ++iy) {
                const long long c0 = Ef.at(2 * i + ix, 2 * j + iy, 2 * k + iz);
                cg[ix][iz][iy] = make_float2(CXp[c0], CXp[c0 + 2]);
            }
    float2 ye[24];
    quad_body<float2>(ue, cg, make_float2(lam, lam), make_float2(mu, mu), ye);
#pragma unroll
    for (int m = 0; m < 24; ++m) *reinterpret_cast<float2 *>(y + (long long)m * nel + e) = ye[m];
}

template <typename T, int MODE>
__global__ void __launch_bounds__(128)
quad_node_kernel(Lay L, const T *__restrict__ y, const T *__restrict__ u, const T *__restrict__ f,
                 const T *__restrict__ rdiag, const uint8_t *__restrict__ mask, T *__restrict__ out,
                 T omega, T prerelax, const int *__restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    const Grid &g = L.g;
    int i, j, k;
    if (!plane_ijk(g, i, j, k)) return;
    const long long n = g.node(i, j, k);
    const long long nel = g.nel();
    // all 24 loads issue before any is used (predicated, no branches), so the
    // gather waits for memory once instead of once per element
    const bool vx[2] = {i >= 1, i < g.nx}, vz[2] = {k >= 1, k < g.nz}, vy[2] = {j >= 1, j < g.ny};
    T v[2][2][2][3];
#pragma unroll
    for (int ex = 0; ex < 2; ++ex)
#pragma unroll
        for (int ez = 0; ez < 2; ++ez)
#pragma unroll
            for (int ey = 0; ey < 2; ++ey) {
                const bool ok = vx[ex] && vz[ez] && vy[ey];
                const long long e = ok ? g.elem(i - 1 + ex, j - 1 + ey, k - 1 + ez) : 0;
                const int a = local_index(1 - ex, 1 - ey, 1 - ez);
#pragma unroll
                for (int d = 0; d < 3; ++d) v[ex][ez][ey][d] = ok ? __ldg(y + (long long)(3 * a + d) * nel + e) : T(0);
            }
    T acc[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int ex = 0; ex < 2; ++ex)
#pragma unroll
        for (int ez = 0; ez < 2; ++ez)
#pragma unroll
            for (int ey = 0; ey < 2; ++ey)
#pragma unroll
                for (int d = 0; d < 3; ++d) acc[d] += v[ex][ez][ey][d];
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
                us = prerelax * f[dof] * rdiag[dof];
            } else {
                us = u[dof];
            }
            out[dof] = us + omega * r * rdiag[dof];
        }
    }
}

template <typename T>
int launch_quad_sweep(int mode, const Lay &L, const ELay &Ef, const T *CX, const T *u, const T *f,
                      const T *rdiag, const uint8_t *mask, T *out, T omega, T prerelax, double nu,
                      T *yscratch, const int *done, int *, cudaStream_t st)
{
    // Lame constants of the unit-modulus material, with the 1/64 of the two
    // Hadamard transforms folded in
    const T lam = (T)(nu / ((1.0 + nu) * (1.0 - 2.0 * nu)) / 64.0);
    const T mu = (T)(1.0 / (2.0 * (1.0 + nu)) / 64.0);
    const int bs = 128;
    const unsigned eb = (unsigned)((L.g.nel() + bs - 1) / bs);
    const dim3 nb = plane_grid(L.g, bs);   // quad_node_kernel: one row of CTAs per node plane
    bool paired = false;
    if constexpr (sizeof(T) == 4) {
        if (L.g.ny % 2 == 0) {   // element pairs
            paired = true;
            const unsigned eb2 = (unsigned)((L.g.nel() / 2 + bs - 1) / bs);
            if (mode == MODE_JACOBI_PRE)
                launch_pdl(quad_element2_kernel<true>, dim3(eb2), dim3(bs), 0, st, L, CX, Ef, u, f, rdiag, prerelax,
                           lam, mu, yscratch, done);
            else
                launch_pdl(quad_element2_kernel<false>, dim3(eb2), dim3(bs), 0, st, L, CX, Ef, u, f, rdiag, prerelax,
                           lam, mu, yscratch, done);
        }
    }
    if (!paired) {
        if (mode == MODE_JACOBI_PRE)
            launch_pdl(quad_element_kernel<T, true>, dim3(eb), dim3(bs), 0, st, L, CX, Ef, u, f, rdiag, prerelax, lam,
                       mu, yscratch, done);
        else
            launch_pdl(quad_element_kernel<T, false>, dim3(eb), dim3(bs), 0, st, L, CX, Ef, u, f, rdiag, prerelax, lam,
                       mu, yscratch, done);
    }
    switch (mode) {
    case MODE_APPLY:
        launch_pdl(quad_node_kernel<T, MODE_APPLY>, dim3(nb), dim3(bs), 0, st, L, yscratch, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    case MODE_DEFECT:
        launch_pdl(quad_node_kernel<T, MODE_DEFECT>, dim3(nb), dim3(bs), 0, st, L, yscratch, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    case MODE_JACOBI:
        launch_pdl(quad_node_kernel<T, MODE_JACOBI>, dim3(nb), dim3(bs), 0, st, L, yscratch, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    default:
        launch_pdl(quad_node_kernel<T, MODE_JACOBI_PRE>, dim3(nb), dim3(bs), 0, st, L, yscratch, u, f, rdiag, mask, out, omega, prerelax, done);
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
// y_E = A_E u_E into the 24-per-element scratch, then the node pass (the same
// deterministic gather as for level 1).  Used for the large coarse levels,
// where the node-centred form re-reads every entry from the 8 nodes around it.
// A CTA of 4 warps takes 32 elements (lane = element, so every entry load is
// coalesced over the [300][nel] layout); warp g multiplies the packed rows
// [M0, M1) of its share (78, 75, 78 and 69 of the 300 entries), using each
// off-diagonal entry for both of its products, into a partial 24-vector; the
// four partials are summed in a fixed order through shared memory.
template <typename T, int M0, int M1>
__device__ __forceinline__ void packed_rows(const T *__restrict__ A, long long nel, long long e, const T (&ue)[24],
                                            T (&ye)[24])
{
#pragma unroll
    for (int m = M0; m < M1; ++m)
#pragma unroll
        for (int n = 0; n <= m; ++n) {
            const T amn = A[(long long)packed_index(m, n) * nel + e];
            ye[m] = fma(amn, ue[n], ye[m]);
            if (n != m) ye[n] = fma(amn, ue[m], ye[n]);
        }
}

template <typename T, bool PRE>
__global__ void __launch_bounds__(128)
packed_element_kernel(Lay L, const T *__restrict__ A, const T *__restrict__ u, const T *__restrict__ f,
                      const T *__restrict__ rdiag, T prerelax, T *__restrict__ y, const int *__restrict__ done)
{
    pdl_wait();
    if (done && *done) return;
    __shared__ T part[4][24][32];
    const Grid &g = L.g;
    const long long nel = g.nel();
    const int lane = threadIdx.x & 31, wg = threadIdx.x >> 5;
    const long long e = (long long)blockIdx.x * 32 + lane;
    const bool have = e < nel;
    T ye[24];
#pragma unroll
    for (int m = 0; m < 24; ++m) ye[m] = T(0);
    if (have) {
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
                    ue[3 * a + q] = prerelax * f[nb + q] * rdiag[nb + q];
                } else {
                    ue[3 * a + q] = u[nb + q];
                }
            }
        }
        switch (wg) {
        case 0: packed_rows<T, 0, 12>(A, nel, e, ue, ye); break;
        case 1: packed_rows<T, 12, 17>(A, nel, e, ue, ye); break;
        case 2: packed_rows<T, 17, 21>(A, nel, e, ue, ye); break;
        default: packed_rows<T, 21, 24>(A, nel, e, ue, ye);
        }
    }
#pragma unroll
    for (int m = 0; m < 24; ++m) part[wg][m][lane] = ye[m];
    __syncthreads();
    if (!have) return;
    // warp wg writes rows 6 wg .. 6 wg + 5
#pragma unroll
    for (int r = 0; r < 6; ++r) {
        const int m = 6 * wg + r;
        const T s = ((part[0][m][lane] + part[1][m][lane]) + part[2][m][lane]) + part[3][m][lane];
        y[(long long)m * nel + e] = s;
    }
}

template <typename T>
void launch_packed_sweep_ec(int mode, const Lay &L, const T *Apk, const T *u, const T *f, const T *rdiag,
                            const uint8_t *mask, T *out, T omega, T prerelax, T *yscratch,
                            const int *done, cudaStream_t st)
{
    const int bs = 128;
    const unsigned eb = (unsigned)((L.g.nel() + 31) / 32);   // 32 elements per CTA of 4 warps
    const dim3 nb = plane_grid(L.g, bs);   // quad_node_kernel: one row of CTAs per node plane
    if (mode == MODE_JACOBI_PRE)
        launch_pdl(packed_element_kernel<T, true>, dim3(eb), dim3(bs), 0, st, L, Apk, u, f, rdiag, prerelax, yscratch, done);
    else
        launch_pdl(packed_element_kernel<T, false>, dim3(eb), dim3(bs), 0, st, L, Apk, u, f, rdiag, prerelax, yscratch, done);
    switch (mode) {
    case MODE_APPLY:
        launch_pdl(quad_node_kernel<T, MODE_APPLY>, dim3(nb), dim3(bs), 0, st, L, yscratch, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    case MODE_DEFECT:
        launch_pdl(quad_node_kernel<T, MODE_DEFECT>, dim3(nb), dim3(bs), 0, st, L, yscratch, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    case MODE_JACOBI:
        launch_pdl(quad_node_kernel<T, MODE_JACOBI>, dim3(nb), dim3(bs), 0, st, L, yscratch, u, f, rdiag, mask, out, omega, prerelax, done);
        break;
    default:
        launch_pdl(quad_node_kernel<T, MODE_JACOBI_PRE>, dim3(nb), dim3(bs), 0, st, L, yscratch, u, f, rdiag, mask, out, omega, prerelax, done);
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
