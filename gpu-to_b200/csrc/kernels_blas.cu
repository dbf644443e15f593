// PCG vector kernels with device-resident scalars.
//
// The reference computes every dot product with a single 1024-thread block,
// a cudaMalloc per call and a blocking copy to the host (mgcg1.cu:1033-1067),
// and every axpy with one block (:1016-1023).  Here each reduction is a
// grid-wide two-level reduction in FP64: per-CTA partials, then the last CTA
// to finish (ticket counter) adds the partials in a fixed order -- so results
// are deterministic -- and applies the PCG scalar recurrence in place on the
// device.  The host reads the scalars only to test convergence.
#include "gputo_internal.h"

#include <cmath>

namespace gputo {

constexpr int kRedThreads = 256;
constexpr int kMaxRedBlocks = 1184;   // 148 SMs x 8

int reduce_partials_capacity() { return 1 << 16; }

static int red_blocks(long long n)
{
    long long b = (n + kRedThreads * 4 - 1) / (kRedThreads * 4);
    if (b < 1) b = 1;
    if (b > kMaxRedBlocks) b = kMaxRedBlocks;
    return (int)b;
}

__device__ __forceinline__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (w == 0) {
        s = l < (int)(blockDim.x >> 5) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;  // valid in thread 0
}

// Sum of partial[0..nb) in a fixed order by one CTA.
__device__ double sum_partials(const double *partial, int nb, double *red)
{
    double v = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) v += partial[i];
    __syncthreads();
    return block_sum(v, red);
}

// Returns true in thread 0 of the last CTA to arrive; that CTA then sums.
__device__ bool last_block(unsigned *ticket)
{
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return is_last;
}

enum DotWhich { DOT_RES0 = 0, DOT_RHO0 = 1, DOT_RZ = 2 };

__device__ void finalize_dot(PcgScalars *sc, int which, double s, double s_old = 0.0)
{
    if (which == DOT_RES0) {
        sc->res0 = sqrt(s);
    } else if (which == DOT_RHO0) {
        sc->rho_p = s;
        sc->rz = s;
    } else {
        // end of a PCG iteration (mgcg1.cu:263-275)
        // flexible PCG (Polak-Ribiere): beta = r'(z - z_old) / rho_p, which
        // equals the classical r'z / rho_p for a fixed SPD preconditioner
        const double rho = s;
        const double beta = (sc->flexible ? (rho - s_old) : rho) / sc->rho_p;
        sc->rz_old = s_old;
        sc->beta = beta;
        sc->rz = rho;
        sc->rho_p = rho;
        const double rel = sqrt(sc->rr) / sc->res0;
        sc->relres = rel;
        const int it = sc->iter;
        sc->iter = it + 1;
        if (!isfinite(rel) || !isfinite(beta)) {
            sc->status = GPUTO_ERR_BREAKDOWN;
            sc->done = 1;
            sc->nit = it;
        } else if (rel < sc->tol) {
            sc->done = 1;
            sc->nit = it;
        } else if (it + 1 >= sc->maxit) {
            sc->done = 1;
            sc->nit = sc->maxit;
        }
    }
}

__global__ void __launch_bounds__(kRedThreads)
dot_kernel(long long n, const double *__restrict__ a, const double *__restrict__ b,
           double *__restrict__ partial, unsigned *ticket, PcgScalars *sc, int which,
           const int *done)
{
    if (done && *done) return;
    __shared__ double red[kRedThreads / 32];
    double v = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        v = fma(a[i], b[i], v);
    v = block_sum(v, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
    if (last_block(ticket)) {
        const double s = sum_partials(partial, gridDim.x, red);
        if (threadIdx.x == 0) {
            finalize_dot(sc, which, s);
            *ticket = 0;
        }
    }
}

void launch_dot(long long n, const double *a, const double *b, double *partial, unsigned *ticket,
                PcgScalars *sc, int which, const int *done, cudaStream_t st)
{
    dot_kernel<<<red_blocks(n), kRedThreads, 0, st>>>(n, a, b, partial, ticket, sc, which, done);
    count_launches(1);
}

// r'z and r'z_old in one pass, for the flexible recurrence.  Z is FP64, or
// the FP32 V-cycle output itself (the FP64 z would be its exact widening).
template <typename Z>
__global__ void __launch_bounds__(kRedThreads)
dot2_kernel(long long n, const double *__restrict__ r, const Z *__restrict__ z,
            const Z *__restrict__ zold, double *__restrict__ partial, unsigned *ticket,
            PcgScalars *sc, const int *done)
{
    if (done && *done) return;
    __shared__ double red[kRedThreads / 32];
    double v = 0.0, w = 0.0;
    // two neighbouring entries per trip (16-byte loads); n odd leaves a tail
    const long long n2 = n >> 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2;
         i += (long long)gridDim.x * blockDim.x) {
        const double2 ri = reinterpret_cast<const double2 *>(r)[i];
        const double z0 = (double)z[2 * i], z1 = (double)z[2 * i + 1];
        const double o0 = (double)zold[2 * i], o1 = (double)zold[2 * i + 1];
        v = fma(ri.x, z0, v);
        w = fma(ri.x, o0, w);
        v = fma(ri.y, z1, v);
        w = fma(ri.y, o1, w);
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        v = fma(r[n - 1], (double)z[n - 1], v);
        w = fma(r[n - 1], (double)zold[n - 1], w);
    }
    v = block_sum(v, red);
    __syncthreads();
    w = block_sum(w, red);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = v;
        partial[2 * blockIdx.x + 1] = w;
    }
    if (last_block(ticket)) {
        double a = 0.0, b = 0.0;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
            a += partial[2 * i];
            b += partial[2 * i + 1];
        }
        __syncthreads();
        a = block_sum(a, red);
        __syncthreads();
        b = block_sum(b, red);
        if (threadIdx.x == 0) {
            finalize_dot(sc, DOT_RZ, a, b);
            *ticket = 0;
        }
    }
}

template <typename Z>
void launch_dot2(long long n, const double *r, const Z *z, const Z *zold, double *partial, unsigned *ticket,
                 PcgScalars *sc, const int *done, cudaStream_t st)
{
    dot2_kernel<Z><<<red_blocks(n), kRedThreads, 0, st>>>(n, r, z, zold, partial, ticket, sc, done);
    count_launches(1);
}
template void launch_dot2<double>(long long, const double *, const double *, const double *, double *, unsigned *,
                                  PcgScalars *, const int *, cudaStream_t);
template void launch_dot2<float>(long long, const double *, const float *, const float *, double *, unsigned *,
                                 PcgScalars *, const int *, cudaStream_t);

// R -= alpha Q and r'r (mgcg1.cu:259,269); R32, when given, receives
// float(R) for the mixed-precision V-cycle.  The solution's update U += alpha
// P (mgcg1.cu:258) is left pending: p_update_kernel applies it, as it reads P
// anyway, and a solve that stops before the direction update applies it in
// launch_flush_x.  Same values as updating U here (P does not change in
// between), 16 bytes per dof less traffic.
__global__ void __launch_bounds__(kRedThreads)
pcg_update_kernel(long long n, double *__restrict__ R, const double *__restrict__ Q,
                  double *__restrict__ partial, unsigned *ticket, PcgScalars *sc, float *__restrict__ R32)
{
    pdl_wait();
    if (sc->done) return;
    __shared__ double red[kRedThreads / 32];
    const double alpha = sc->alpha;
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->x_pending = 1;
    double v = 0.0;
    // two neighbouring entries per trip (16-byte loads and stores)
    const long long n2 = n >> 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2;
         i += (long long)gridDim.x * blockDim.x) {
        const double2 q = reinterpret_cast<const double2 *>(Q)[i];
        double2 r = reinterpret_cast<double2 *>(R)[i];
        r.x = fma(-alpha, q.x, r.x);
        r.y = fma(-alpha, q.y, r.y);
        reinterpret_cast<double2 *>(R)[i] = r;
        if (R32) reinterpret_cast<float2 *>(R32)[i] = make_float2((float)r.x, (float)r.y);
        v = fma(r.x, r.x, v);
        v = fma(r.y, r.y, v);
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const long long i = n - 1;
        const double r = fma(-alpha, Q[i], R[i]);
        R[i] = r;
        if (R32) R32[i] = (float)r;
        v = fma(r, r, v);
    }
    v = block_sum(v, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
    if (last_block(ticket)) {
        const double s = sum_partials(partial, gridDim.x, red);
        if (threadIdx.x == 0) {
            sc->rr = s;
            *ticket = 0;
        }
    }
}

void launch_pcg_update(long long n, double *R, const double *Q, double *partial, unsigned *ticket, PcgScalars *sc,
                       cudaStream_t st, float *R32)
{
    launch_pdl(pcg_update_kernel, dim3(red_blocks(n)), dim3(kRedThreads), 0, st, n, R, Q, partial, ticket, sc, R32);
    count_launches(1);
}

// U += alpha P (the update pcg_update_kernel left pending, with the old P),
// then P = Z + beta P (mgcg1.cu:258,265); the flexible variant also keeps Z as
// Z_old.
template <typename Z>
__global__ void p_update_kernel(long long n, const Z *__restrict__ z_in, double *__restrict__ P,
                                Z *__restrict__ Zold, double *__restrict__ U, PcgScalars *sc)
{
    pdl_wait();
    if (sc->done) return;
    const double beta = sc->beta, alpha = sc->alpha;
    // read only by launch_flush_x, after this kernel in stream order
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->x_pending = 0;
    const long long n2 = n >> 1;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n2;
         i += (long long)gridDim.x * blockDim.x) {
        const Z z0 = z_in[2 * i], z1 = z_in[2 * i + 1];
        double2 p = reinterpret_cast<double2 *>(P)[i], u = reinterpret_cast<double2 *>(U)[i];
        u.x = fma(alpha, p.x, u.x);
        u.y = fma(alpha, p.y, u.y);
        reinterpret_cast<double2 *>(U)[i] = u;
        p.x = fma(beta, p.x, (double)z0);
        p.y = fma(beta, p.y, (double)z1);
        reinterpret_cast<double2 *>(P)[i] = p;
        if (Zold) {
            Zold[2 * i] = z0;
            Zold[2 * i + 1] = z1;
        }
    }
    if ((n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        const Z z = z_in[n - 1];
        U[n - 1] = fma(alpha, P[n - 1], U[n - 1]);
        P[n - 1] = fma(beta, P[n - 1], (double)z);
        if (Zold) Zold[n - 1] = z;
    }
}

template <typename Z>
void launch_p_update(long long n, const Z *z, double *P, Z *Zold, double *U, PcgScalars *sc, cudaStream_t st)
{
    launch_pdl(p_update_kernel<Z>, dim3(red_blocks(n)), dim3(kRedThreads), 0, st, n, z, P, Zold, U, sc);
    count_launches(1);
}
template void launch_p_update<double>(long long, const double *, double *, double *, double *, PcgScalars *,
                                      cudaStream_t);
template void launch_p_update<float>(long long, const float *, double *, float *, double *, PcgScalars *,
                                     cudaStream_t);

// The solution update still pending when a solve stopped after its residual
// update (converged, maxit, or a breakdown found by the dot at the end of the
// iteration): U += alpha P.
__global__ void flush_x_kernel(long long n, double *__restrict__ U, const double *__restrict__ P,
                               const PcgScalars *sc)
{
    if (!sc->x_pending) return;
    const double alpha = sc->alpha;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        U[i] = fma(alpha, P[i], U[i]);
}

void launch_flush_x(long long n, double *U, const double *P, const PcgScalars *sc, cudaStream_t st)
{
    flush_x_kernel<<<red_blocks(n), kRedThreads, 0, st>>>(n, U, P, sc);
    count_launches(1);
}

// U = 0, R = F, res0 = ||F|| and the scalar state (mgcg1.cu:235-238).
__global__ void __launch_bounds__(kRedThreads)
pcg_init_kernel(long long n, const double *__restrict__ F, double *__restrict__ U,
                double *__restrict__ R, double *__restrict__ partial, unsigned *ticket,
                PcgScalars *sc, double tol, int maxit, int flexible)
{
    __shared__ double red[kRedThreads / 32];
    double v = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double f = F[i];
        U[i] = 0.0;
        R[i] = f;
        v = fma(f, f, v);
    }
    v = block_sum(v, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = v;
    if (last_block(ticket)) {
        const double s = sum_partials(partial, gridDim.x, red);
        if (threadIdx.x == 0) {
            PcgScalars z{};
            z.res0 = sqrt(s);
            z.tol = tol;
            z.maxit = maxit;
            z.relres = 1.0;
            z.flexible = flexible;
            z.nit = maxit;
            z.done = (maxit <= 0) ? 1 : 0;
            if (!isfinite(z.res0)) {
                // a non-finite F: nothing to iterate on (the reference would
                // run its loop on NaNs to maxit)
                z.status = GPUTO_ERR_BREAKDOWN;
                z.done = 1;
                z.nit = 0;
            } else if (!(z.res0 > 0.0)) {
                // F = 0: U = 0 is the solution; the reference would divide 0/0.
                z.done = 1;
                z.nit = 0;
                z.relres = 0.0;
            }
            *sc = z;
            *ticket = 0;
        }
    }
}

void launch_pcg_init(long long n, const double *F, double *U, double *R, double *partial,
                     unsigned *ticket, PcgScalars *sc, double tol, int maxit, int flexible,
                     cudaStream_t st)
{
    pcg_init_kernel<<<red_blocks(n), kRedThreads, 0, st>>>(n, F, U, R, partial, ticket, sc, tol,
                                                             maxit, flexible);
    count_launches(1);
}

// alpha = rho_p / p'q from the per-CTA partials of the fused apply.
__global__ void __launch_bounds__(kRedThreads)
finish_apply_dot_kernel(int nb, const double *__restrict__ partial, PcgScalars *sc)
{
    pdl_wait();
    if (sc->done) return;
    __shared__ double red[kRedThreads / 32];
    const double s = sum_partials(partial, nb, red);
    if (threadIdx.x == 0) {
        sc->pq = s;
        const double alpha = sc->rho_p / s;
        sc->alpha = alpha;
        if (!(s > 0.0) || !isfinite(alpha)) {
            sc->status = GPUTO_ERR_BREAKDOWN;
            sc->done = 1;
            sc->nit = sc->iter;
        }
    }
}

void launch_finish_apply_dot(int nblocks, double *partial, unsigned *, PcgScalars *sc,
                             cudaStream_t st)
{
    launch_pdl(finish_apply_dot_kernel, dim3(1), dim3(kRedThreads), 0, st, nblocks, (const double *)partial, sc);
    count_launches(1);
}

__global__ void __launch_bounds__(kRedThreads)
finish_dot2_kernel(int nb, const double *__restrict__ partial, PcgScalars *sc)
{
    pdl_wait();
    if (sc->done) return;
    __shared__ double red[kRedThreads / 32];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        a += partial[2 * i];
        b += partial[2 * i + 1];
    }
    a = block_sum(a, red);
    __syncthreads();
    b = block_sum(b, red);
    if (threadIdx.x == 0) finalize_dot(sc, DOT_RZ, a, b);
}

void launch_finish_dot2(int nblocks, const double *partial, PcgScalars *sc, cudaStream_t st)
{
    launch_pdl(finish_dot2_kernel, dim3(1), dim3(kRedThreads), 0, st, nblocks, partial, sc);
    count_launches(1);
}

__global__ void copy_kernel(long long n, const double *__restrict__ a, double *__restrict__ b,
                            const int *done)
{
    if (done && *done) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        b[i] = a[i];
}

void launch_copy(long long n, const double *a, double *b, const int *done, cudaStream_t st)
{
    copy_kernel<<<red_blocks(n), kRedThreads, 0, st>>>(n, a, b, done);
    count_launches(1);
}

// y components negated on output (mgcg1.cu:282-283).
__global__ void flip_y_kernel(long long nnod, double *U)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnod;
         i += (long long)gridDim.x * blockDim.x)
        U[3 * i + 1] = -U[3 * i + 1];
}

void launch_flip_y(long long nnod, double *U, cudaStream_t st)
{
    flip_y_kernel<<<red_blocks(nnod), kRedThreads, 0, st>>>(nnod, U);
    count_launches(1);
}

template <typename Tin, typename Tout>
__global__ void convert_kernel(long long n, const Tin *__restrict__ in, Tout *__restrict__ out,
                               const int *done)
{
    if (done && *done) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = (Tout)in[i];
}

template <typename Tin, typename Tout>
void launch_convert(long long n, const Tin *in, Tout *out, const int *done, cudaStream_t st)
{
    convert_kernel<Tin, Tout><<<red_blocks(n), kRedThreads, 0, st>>>(n, in, out, done);
    count_launches(1);
}
template void launch_convert<double, float>(long long, const double *, float *, const int *, cudaStream_t);
template void launch_convert<float, double>(long long, const float *, double *, const int *, cudaStream_t);

template <typename T>
__global__ void recip_kernel(long long n, const double *__restrict__ in, T *__restrict__ out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = in[i] != 0.0 ? (T)(1.0 / in[i]) : T(0);
}

template <typename T>
void launch_recip(long long n, const double *in, T *out, cudaStream_t st)
{
    recip_kernel<T><<<red_blocks(n), kRedThreads, 0, st>>>(n, in, out);
    count_launches(1);
}
template void launch_recip<double>(long long, const double *, double *, cudaStream_t);
template void launch_recip<float>(long long, const double *, float *, cudaStream_t);

void launch_cast_f32(long long n, const double *in, float *out, cudaStream_t st)
{
    launch_convert<double, float>(n, in, out, nullptr, st);
}

}  // namespace gputo
