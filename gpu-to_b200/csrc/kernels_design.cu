// Design-loop steps that the MATLAB driver runs around the solve
// (Cantilever/TOP3D125MGCGCUDA/top3D125modCuda.m:95-96,109,139-141,163).
#include "gputo_internal.h"
#include "hadamard.h"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

namespace gputo {

// Element matrix for the energy kernel.  Constant memory is per translation
// unit without relocatable device code, so this file keeps its own copy,
// written by upload_fine_ke() together with the solver's.  When Ke has the
// cube element's Hadamard pattern, its eight constants (per device) select
// the Hadamard-basis energy pass.
__constant__ double cKeD[576];
static HadamardKe g_design_hk[64];
static std::mutex g_design_hk_mu;   // writers (upload) and readers (launch) on other threads

int upload_design_ke(const double *Ke_host, cudaStream_t st)
{
    int dev = 0;
    GPUTO_CUDA(cudaGetDevice(&dev));
    HadamardKe hk;
    (void)hadamard_ke(Ke_host, &hk);   // sets ok = false without the pattern
    {
        std::lock_guard<std::mutex> lock(g_design_hk_mu);
        g_design_hk[dev < 64 ? dev : 63] = hk;
    }
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(cKeD, Ke_host, sizeof(double) * 576, 0,
                                       cudaMemcpyHostToDevice, st));
    return GPUTO_OK;
}

constexpr int kMaxFilterRadius = 6;           // stencil up to 13^3
constexpr int kFilterW = 2 * kMaxFilterRadius + 1;
__constant__ double cFilterH[kFilterW * kFilterW * kFilterW];

// ce_e = u_e^T Ke u_e, dc_e = dsK_e ce_e, and sum_e CX_e ce_e.  Thread per
// element.  U is in the solver frame: the driver's U(cMat) gather
// (top3D125modCuda.m:39-41,139) lists element nodes in an order mirrored in y,
// which matches the y-negated U the MEX hands back, so both give the same ce.
// HAD: u_e' Ke u_e as (T u_e)' (S / 64) (T u_e) in the element's Hadamard
// basis (about 140 FP64 operations, so the pass is bound by memory); else
// the dense 24x24 product with Ke from constant memory (1152 FLOP).
template <bool HAD>
__global__ void __launch_bounds__(256)
element_energy_kernel(Grid g, HC<double> hc, const double *__restrict__ U, const double *__restrict__ CX,
                      const double *__restrict__ dsK, double *__restrict__ ce,
                      double *__restrict__ dc, double *__restrict__ partial, unsigned *ticket,
                      double *compliance)
{
    __shared__ double red[8];
    __shared__ bool is_last;
    const long long nel = g.nel();
    double csum = 0.0;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
         e += (long long)gridDim.x * blockDim.x) {
        const long long t = e / g.ny;
        const int j = (int)(e - t * g.ny);
        const int i = (int)(t / g.nz);
        const int k = (int)(t - (long long)i * g.nz);
        double s = 0.0;
        if constexpr (HAD) {
            // corners (cx, cy, cz) into the two x faces, [(2 cy + cz) 4 + d]
            double Fp[HF], Fn[HF];
#pragma unroll
            for (int cy = 0; cy < 2; ++cy)
#pragma unroll
                for (int cz = 0; cz < 2; ++cz) {
                    const long long n0 = g.node(i, j + cy, k + cz), n1 = g.node(i + 1, j + cy, k + cz);
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        Fp[(2 * cy + cz) * 4 + d] = U[3 * n0 + d];
                        Fn[(2 * cy + cz) * 4 + d] = U[3 * n1 + d];
                    }
                }
            face_h(Fp);
            face_h(Fn);
            s = element_energy_h(Fp, Fn, hc);
        } else {
            double ue[24];
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const long long n = g.node(i + local_x(a), j + local_y(a), k + local_z(a));
#pragma unroll
                for (int d = 0; d < 3; ++d) ue[3 * a + d] = U[3 * n + d];
            }
#pragma unroll 4
            for (int m = 0; m < 24; ++m) {
                double tm = 0.0;
#pragma unroll
                for (int q = 0; q < 24; ++q) tm = fma(cKeD[m * 24 + q], ue[q], tm);
                s = fma(ue[m], tm, s);
            }
        }
        if (ce) ce[e] = s;
        if (dc) dc[e] = dsK[e] * s;
        if (CX) csum = fma(CX[e], s, csum);
    }
    if (!compliance) return;
    for (int o = 16; o > 0; o >>= 1) csum += __shfl_xor_sync(0xffffffffu, csum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = csum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w];
        partial[blockIdx.x] = v;
        __threadfence();
        is_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        __threadfence();
        double v = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) v += partial[b];
        *compliance = v;
        *ticket = 0;
    }
}

// Same kernel with an explicit number of CTAs (one partial slot per CTA).
void launch_element_energy_blocks(const Grid &g, const double *U, const double *CX,
                                  const double *dsK, double *ce, double *dc, double *partial,
                                  unsigned *ticket, double *compliance, int nblocks,
                                  cudaStream_t st)
{
    int dev = 0;
    cudaGetDevice(&dev);
    HadamardKe hk;
    {
        std::lock_guard<std::mutex> lock(g_design_hk_mu);
        hk = g_design_hk[dev < 64 ? dev : 63];
    }
    if (hk.ok)
        element_energy_kernel<true><<<(unsigned)nblocks, 256, 0, st>>>(g, make_hc<double>(hk), U, CX, dsK, ce, dc,
                                                                       partial, ticket, compliance);
    else
        element_energy_kernel<false><<<(unsigned)nblocks, 256, 0, st>>>(g, HC<double>{}, U, CX, dsK, ce, dc,
                                                                        partial, ticket, compliance);
    count_launches(1);
}

void launch_element_energy(const Grid &g, const double *U, const double *CX, const double *dsK,
                           double *ce, double *dc, double *partial, unsigned *ticket,
                           double *compliance, cudaStream_t st)
{
    long long nb = (g.nel() + 255) / 256;
    if (nb > 1184) nb = 1184;
    if (nb < 1) nb = 1;
    launch_element_energy_blocks(g, U, CX, dsK, ce, dc, partial, ticket, compliance, (int)nb, st);
}

// MATLAB 'symmetric' padding: mirror including the edge sample.
__device__ __forceinline__ int mirror_index(int i, int n)
{
    while (i < 0 || i >= n) {
        if (i < 0) i = -1 - i;
        if (i >= n) i = 2 * n - 1 - i;
    }
    return i;
}

// out = correlate(in ./ div, h) [/ sum h], elements in (y fastest) order
// (imfilter(..., 'symmetric'), top3D125modCuda.m:109,140-141).
//
// Shared-memory tiled: a CTA owns an output tile of 32 (y, one per lane) x 8
// (z, one per warp) element columns and marches along x through a chunk of
// planes.  Each input plane of the tile plus its R-wide halo, mirrored at the
// grid faces, is loaded from global memory once (the quotient in ./ div is
// taken at load time) into a ring of 2R + 2 plane slots; the loads of the
// plane FPF steps ahead are in flight while the current output plane is
// computed from shared memory, with one barrier per plane (the slot being
// filled is never one being read).  The weights are in constant memory and
// the same for every lane (broadcast).  The sum runs in the order x offset,
// z offset, y offset, as a direct 3-D correlation would.
constexpr int kFTY = 32, kFTZ = 8, kFPF = 2;

template <int R> struct FiltTile {
    static constexpr int W = 2 * R + 1;
    static constexpr int TYH = kFTY + 2 * R, TZH = kFTZ + 2 * R;
    static constexpr int PLANE = TYH * TZH;
    static constexpr int NPOS = (PLANE + 255) / 256;   // halo-tile positions per thread
    static constexpr int SLOTS = 2 * R + 2;
    static constexpr size_t bytes = sizeof(double) * SLOTS * PLANE;
};

template <int R>
__global__ void __launch_bounds__(256)
filter_kernel(Grid g, const double *__restrict__ in, const double *__restrict__ div,
              double *__restrict__ out, double scale, int xc)
{
    using FT = FiltTile<R>;
    constexpr int W = FT::W;
    extern __shared__ double fs[];   // [SLOTS][PLANE]
    const int tid = threadIdx.x, ly = tid & 31, lz = tid >> 5;
    const int j0 = blockIdx.x * kFTY, k0 = blockIdx.y * kFTZ;
    const int x0 = blockIdx.z * xc, x1 = min(x0 + xc, g.nx);
    const long long ps = (long long)g.ny * g.nz;   // elements per x plane
    // this thread's positions in a halo tile: offset inside an x plane (-1: none)
    long long off[FT::NPOS];
#pragma unroll
    for (int q = 0; q < FT::NPOS; ++q) {
        const int p = tid + 256 * q;
        off[q] = -1;
        if (p < FT::PLANE) {
            const int zz = p / FT::TYH, yy = p - zz * FT::TYH;
            off[q] = (long long)mirror_index(k0 + zz - R, g.nz) * g.ny + mirror_index(j0 + yy - R, g.ny);
        }
    }
    auto fetch = [&](int px, double (&v)[FT::NPOS]) {
        const long long base = (long long)mirror_index(px, g.nx) * ps;
#pragma unroll
        for (int q = 0; q < FT::NPOS; ++q)
            if (off[q] >= 0) {
                const long long s = base + off[q];
                v[q] = div ? in[s] / div[s] : in[s];
            }
    };
    auto put = [&](int px, const double (&v)[FT::NPOS]) {
        double *P = fs + ((px - x0 + R) % FT::SLOTS) * FT::PLANE;
#pragma unroll
        for (int q = 0; q < FT::NPOS; ++q)
            if (off[q] >= 0) P[tid + 256 * q] = v[q];
    };
    // planes x0 - R .. x0 + R - 1 before the first output plane
    for (int px = x0 - R; px < x0 + R; ++px) {
        double v[FT::NPOS];
        fetch(px, v);
        put(px, v);
    }
    double pre[kFPF][FT::NPOS];
#pragma unroll
    for (int d = 0; d < kFPF; ++d)
        if (x0 + d < x1) fetch(x0 + R + d, pre[d]);
    const int j = j0 + ly, k = k0 + lz;
    const bool mine = j < g.ny && k < g.nz;
    for (int i0 = x0; i0 < x1; i0 += kFPF)
#pragma unroll
    for (int pf = 0; pf < kFPF; ++pf) {   // register sets by constant index
        const int i = i0 + pf;
        if (i >= x1) break;               // the same for the whole CTA
        put(i + R, pre[pf]);
        __syncthreads();
        if (i + kFPF < x1) fetch(i + R + kFPF, pre[pf]);   // in flight while plane i is computed
        if (mine) {
            double acc = 0.0;
#pragma unroll
            for (int a = -R; a <= R; ++a) {
                const double *P = fs + ((i + a - x0 + R) % FT::SLOTS) * FT::PLANE;
#pragma unroll
                for (int c = -R; c <= R; ++c) {
                    const double *row = P + (lz + R + c) * FT::TYH + ly + R;
#pragma unroll
                    for (int b = -R; b <= R; ++b)
                        acc = fma(cFilterH[((a + R) * W + (b + R)) * W + (c + R)], row[b], acc);
                }
            }
            out[(long long)i * ps + (long long)k * g.ny + j] = acc * scale;
        }
    }
}

// The same correlation for 1 <= R <= 3, decomposed by x plane: h[a][b][c] =
// h[-a][b][c], so plane q contributes P_|a|(q) = sum_{c,b} h[a][b][c] in(q, j+b,
// k+c) (R + 1 two-dimensional sums over the same (2R + 1)^2 shared-memory
// values) to the output at plane q - a, for every a in -R..R.  A thread keeps
// the 2R + 1 outputs still open in registers (a ring indexed at compile time:
// the march is unrolled by 2 (2R + 1)), so each input plane sits in shared
// memory once (two slots, one barrier per plane) and costs (2R + 1)^2 shared
// loads per output instead of (2R + 1)^3.  Output i sums P_R(i - R), ...,
// P_0(i), ..., P_R(i + R) in plane order.
// Planes arrive by cp.async into a ring of kFPS shared-memory slots (input,
// and the divisor when given), kFPS - 1 planes ahead of the one in use, one
// barrier per plane (two planes ahead in registers reached 0.40 of HBM).
constexpr int kFPS = 4;

__device__ __forceinline__ void cp_async8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int R>
__global__ void __launch_bounds__(256)
filter_plane_kernel(Grid g, const double *__restrict__ in, const double *__restrict__ div,
                    double *__restrict__ out, double scale, int xc)
{
    using FT = FiltTile<R>;
    constexpr int W = FT::W;
    extern __shared__ double fs[];   // [kFPS][PLANE] input planes, then (with a divisor) [kFPS][PLANE] divisor planes
    double *fd = fs + kFPS * FT::PLANE;
    const int tid = threadIdx.x, ly = tid & 31, lz = tid >> 5;
    const int j0 = blockIdx.x * kFTY, k0 = blockIdx.y * kFTZ;
    const int x0 = blockIdx.z * xc, x1 = min(x0 + xc, g.nx);
    const long long ps = (long long)g.ny * g.nz;
    long long off[FT::NPOS];
#pragma unroll
    for (int q = 0; q < FT::NPOS; ++q) {
        const int p = tid + 256 * q;
        off[q] = -1;
        if (p < FT::PLANE) {
            const int zz = p / FT::TYH, yy = p - zz * FT::TYH;
            off[q] = (long long)mirror_index(k0 + zz - R, g.nz) * g.ny + mirror_index(j0 + yy - R, g.ny);
        }
    }
    const int T = x1 - x0 + 2 * R;   // planes x0 - R .. x1 + R - 1
    // plane t (t < T) into slot t mod kFPS; one commit group per plane, empty past the end
    auto fetch = [&](int t) {
        if (t < T) {
            const long long base = (long long)mirror_index(x0 - R + t, g.nx) * ps;
            const int sl = (t % kFPS) * FT::PLANE;
#pragma unroll
            for (int q = 0; q < FT::NPOS; ++q)
                if (off[q] >= 0) {
                    cp_async8(fs + sl + tid + 256 * q, in + base + off[q]);
                    if (div) cp_async8(fd + sl + tid + 256 * q, div + base + off[q]);
                }
        }
        cp_async_commit();
    };
    const int j = j0 + ly, k = k0 + lz;
    const bool mine = j < g.ny && k < g.nz;
    const long long obase = (long long)k * g.ny + j;
    double acc[W];
#pragma unroll
    for (int s = 0; s < W; ++s) acc[s] = 0.0;
#pragma unroll
    for (int t = 0; t < kFPS - 1; ++t) fetch(t);
    for (int t0 = 0; t0 < T; t0 += 2 * W)
#pragma unroll
    for (int u = 0; u < 2 * W; ++u) {
        const int t = t0 + u;
        if (t >= T) break;                 // the same for the whole CTA
        const int q = x0 - R + t;          // this plane
        cp_async_wait<kFPS - 2>();         // this thread's copies of plane t have landed
        __syncthreads();                   // everyone's have; slot (t - 1) mod kFPS is free
        fetch(t + kFPS - 1);
        double *P = fs + (t % kFPS) * FT::PLANE;
        if (div) {   // in / divisor, in place, once per plane
            const double *D = fd + (t % kFPS) * FT::PLANE;
#pragma unroll
            for (int v = 0; v < FT::NPOS; ++v)
                if (off[v] >= 0) P[tid + 256 * v] = P[tid + 256 * v] / D[tid + 256 * v];
            __syncthreads();
        }
        auto val = [&](int zz, int yy) { return P[zz * FT::TYH + yy]; };
        double pa[R + 1];
        if constexpr (R == 1) {
            // radius 1: the weight of a tap depends only on how many of its
            // offsets are non-zero (centre, face, edge, corner), so each plane
            // needs the centre, the sum of its 4 edge neighbours and the sum
            // of its 4 corners
            const int zc = lz + 1, yc = ly + 1;
            const double s0 = val(zc, yc);
            const double s1 = (val(zc, yc - 1) + val(zc, yc + 1)) + (val(zc - 1, yc) + val(zc + 1, yc));
            const double s2 = (val(zc - 1, yc - 1) + val(zc - 1, yc + 1)) + (val(zc + 1, yc - 1) + val(zc + 1, yc + 1));
            const double w0 = cFilterH[13], w1 = cFilterH[12], w2 = cFilterH[9], w3 = cFilterH[0];
            pa[0] = fma(w2, s2, fma(w1, s1, w0 * s0));
            pa[1] = fma(w3, s2, fma(w2, s1, w1 * s0));
        } else {
#pragma unroll
            for (int a = 0; a <= R; ++a) pa[a] = 0.0;
#pragma unroll
            for (int c = -R; c <= R; ++c)
#pragma unroll
                for (int b = -R; b <= R; ++b) {
                    const double x = val(lz + R + c, ly + R + b);
#pragma unroll
                    for (int a = 0; a <= R; ++a)
                        pa[a] = fma(cFilterH[((a + R) * W + (b + R)) * W + (c + R)], x, pa[a]);
                }
        }
        // output q + a (a = -R..R) sits in slot (t + a + R) mod W
#pragma unroll
        for (int a = -R; a <= R; ++a) {
            const int sl = (u + a + R) % W;
            acc[sl] += pa[a < 0 ? -a : a];
        }
        // output q - R is complete
        const int i = q - R, sl = u % W;
        if (i >= x0 && mine) out[(long long)i * ps + obase] = acc[sl] * scale;
        acc[sl] = 0.0;
    }
    cp_async_wait<0>();   // the empty trailing groups
}

// Radius 1 with four output rows along z per thread, tiles of 32 (y) x 32 (z)
// outputs: a thread reads its 6 x 3 window of each plane once for its four
// outputs, 4.5 shared loads per output instead of 9 (the 32 x 8 tiles above
// are bound by shared-memory bandwidth in FP64).  The same ring and the same
// arithmetic per output as filter_plane_kernel<1>.
constexpr int kF1Y = 32, kF1Z = 32;

template <bool DIV>
__global__ void __launch_bounds__(256)
filter_r1_kernel(Grid g, const double *__restrict__ in, const double *__restrict__ div,
                 double *__restrict__ out, double scale, int xc)
{
    constexpr int TYH = kF1Y + 2, TZH = kF1Z + 2, PLANE = TYH * TZH, NPOS = (PLANE + 255) / 256;
    extern __shared__ double fs[];   // [kFPS][PLANE] input planes, then (DIV) [kFPS][PLANE] divisor planes
    double *fd = fs + kFPS * PLANE;
    const int tid = threadIdx.x, ly = tid & 31, lg = tid >> 5;
    const int j0 = blockIdx.x * kF1Y, k0 = blockIdx.y * kF1Z;
    const int x0 = blockIdx.z * xc, x1 = min(x0 + xc, g.nx);
    const long long ps = (long long)g.ny * g.nz;
    long long off[NPOS];
#pragma unroll
    for (int q = 0; q < NPOS; ++q) {
        const int p = tid + 256 * q;
        off[q] = -1;
        if (p < PLANE) {
            const int zz = p / TYH, yy = p - zz * TYH;
            off[q] = (long long)mirror_index(k0 + zz - 1, g.nz) * g.ny + mirror_index(j0 + yy - 1, g.ny);
        }
    }
    const int T = x1 - x0 + 2;   // planes x0 - 1 .. x1
    auto fetch = [&](int t) {
        if (t < T) {
            const long long base = (long long)mirror_index(x0 - 1 + t, g.nx) * ps;
            const int sl = (t % kFPS) * PLANE;
#pragma unroll
            for (int q = 0; q < NPOS; ++q)
                if (off[q] >= 0) {
                    cp_async8(fs + sl + tid + 256 * q, in + base + off[q]);
                    if (DIV) cp_async8(fd + sl + tid + 256 * q, div + base + off[q]);
                }
        }
        cp_async_commit();
    };
    const int j = j0 + ly, kr = k0 + 4 * lg;   // output column; first of the thread's four rows
    const bool jok = j < g.ny;
    const double w0 = cFilterH[13], w1 = cFilterH[12], w2 = cFilterH[9], w3 = cFilterH[0];
    double acc[3][4];
#pragma unroll
    for (int s = 0; s < 3; ++s)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[s][r] = 0.0;
#pragma unroll
    for (int t = 0; t < kFPS - 1; ++t) fetch(t);
    for (int t0 = 0; t0 < T; t0 += 6)
#pragma unroll
    for (int u = 0; u < 6; ++u) {
        const int t = t0 + u;
        if (t >= T) break;   // the same for the whole CTA
        const int q = x0 - 1 + t;
        cp_async_wait<kFPS - 2>();
        __syncthreads();
        fetch(t + kFPS - 1);
        double *P = fs + (t % kFPS) * PLANE;
        if (DIV) {   // in / divisor, in place, once per plane
            const double *D = fd + (t % kFPS) * PLANE;
#pragma unroll
            for (int v = 0; v < NPOS; ++v)
                if (off[v] >= 0) P[tid + 256 * v] = P[tid + 256 * v] / D[tid + 256 * v];
            __syncthreads();
        }
        double v[6][3];
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) v[r][c] = P[(4 * lg + r) * TYH + ly + c];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const double s0 = v[r + 1][1];
            const double s1 = (v[r + 1][0] + v[r + 1][2]) + (v[r][1] + v[r + 2][1]);
            const double s2 = (v[r][0] + v[r][2]) + (v[r + 2][0] + v[r + 2][2]);
            const double p0 = fma(w2, s2, fma(w1, s1, w0 * s0));
            const double p1 = fma(w3, s2, fma(w2, s1, w1 * s0));
            // output q + a (a = -1, 0, 1) sits in slot (u + a + 1) mod 3
            acc[u % 3][r] += p1;
            acc[(u + 1) % 3][r] += p0;
            acc[(u + 2) % 3][r] += p1;
        }
        // output q - 1 is complete
        const int i = q - 1, sl = u % 3;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            if (i >= x0 && jok && kr + r < g.nz) out[(long long)i * ps + (long long)(kr + r) * g.ny + j] = acc[sl][r] * scale;
            acc[sl][r] = 0.0;
        }
    }
    cp_async_wait<0>();   // the empty trailing groups
}

template <int R>
int filter_launch(const Grid &g, const double *in, const double *div, double *out, double scale,
                  cudaStream_t st)
{
    using FT = FiltTile<R>;
    if (FT::bytes > 48 * 1024) {
        static std::once_flag once[64];
        int dev = 0;
        GPUTO_CUDA(cudaGetDevice(&dev));
        cudaError_t e = cudaSuccess;
        std::call_once(once[dev < 64 ? dev : 63], [&]() {
            e = cudaFuncSetAttribute(filter_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)FT::bytes);
        });
        GPUTO_CUDA(e);
    }
    if constexpr (R == 1) {
        // tiles of 32 x 32 outputs; x chunks for about 592 CTAs (4 per SM, one wave), at least 6 planes each
        constexpr size_t plane = sizeof(double) * (kF1Y + 2) * (kF1Z + 2);
        const size_t smem = (div ? 2 : 1) * kFPS * plane;
        if (div) {
            static std::once_flag once[64];
            int dev = 0;
            GPUTO_CUDA(cudaGetDevice(&dev));
            cudaError_t e = cudaSuccess;
            std::call_once(once[dev < 64 ? dev : 63], [&]() {
                e = cudaFuncSetAttribute(filter_r1_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(2 * kFPS * plane));
            });
            GPUTO_CUDA(e);
        }
        const unsigned ty = (unsigned)((g.ny + kF1Y - 1) / kF1Y), tz = (unsigned)((g.nz + kF1Z - 1) / kF1Z);
        const long long tiles = (long long)ty * tz;
        const long long want = std::max(1LL, (592 + tiles - 1) / tiles);
        int xc = (int)std::max(6LL, ((long long)g.nx + want - 1) / want);
        if (xc > g.nx) xc = g.nx;
        const unsigned tx = (unsigned)((g.nx + xc - 1) / xc);
        if (div)
            filter_r1_kernel<true><<<dim3(ty, tz, tx), 256, smem, st>>>(g, in, div, out, scale, xc);
        else
            filter_r1_kernel<false><<<dim3(ty, tz, tx), 256, smem, st>>>(g, in, div, out, scale, xc);
        count_launches(1);
        return GPUTO_OK;
    }
    const unsigned ty = (unsigned)((g.ny + kFTY - 1) / kFTY), tz = (unsigned)((g.nz + kFTZ - 1) / kFTZ);
    // x chunks: about 1184 CTAs (8 per SM) in all, at least 16 planes each
    const long long tiles = (long long)ty * tz;
    const long long want = std::max(1LL, (1184 + tiles - 1) / tiles);
    int xc = (int)std::max(16LL, ((long long)g.nx + want - 1) / want);
    if (xc > g.nx) xc = g.nx;
    const unsigned tx = (unsigned)((g.nx + xc - 1) / xc);
    if constexpr (R >= 1 && R <= 3)
        filter_plane_kernel<R><<<dim3(ty, tz, tx), 256, sizeof(double) * (div ? 2 : 1) * kFPS * FT::PLANE, st>>>(
            g, in, div, out, scale, xc);
    else
        filter_kernel<R><<<dim3(ty, tz, tx), 256, FT::bytes, st>>>(g, in, div, out, scale, xc);
    count_launches(1);
    return GPUTO_OK;
}

int launch_filter(const Grid &g, const double *in, const double *div, double *out, double rmin,
                  int normalize, cudaStream_t st)
{
    const int R = (int)std::ceil(rmin) - 1;
    if (R < 0 || R > kMaxFilterRadius) return GPUTO_ERR_ARG;
    const int W = 2 * R + 1;
    std::vector<double> h((size_t)W * W * W);
    double hs = 0.0;
    for (int a = -R; a <= R; ++a)
        for (int b = -R; b <= R; ++b)
            for (int c = -R; c <= R; ++c) {
                const double v = rmin - std::sqrt((double)(a * a + b * b + c * c));
                const double w = v > 0 ? v : 0.0;
                h[((a + R) * W + (b + R)) * W + (c + R)] = w;
                hs += w;
            }
    static double last_rmin[64];
    static bool have[64] = {};
    int dev = 0;
    GPUTO_CUDA(cudaGetDevice(&dev));
    const int slot = dev < 64 ? dev : 63;
    if (!have[slot] || rmin != last_rmin[slot] || dev >= 64) {   // constant memory is per device
        GPUTO_CUDA(cudaMemcpyToSymbolAsync(cFilterH, h.data(), sizeof(double) * h.size(), 0,
                                           cudaMemcpyHostToDevice, st));
        GPUTO_CUDA(cudaStreamSynchronize(st));
        last_rmin[slot] = rmin;
        have[slot] = true;
    }
    const double scale = normalize ? 1.0 / hs : 1.0;
    switch (R) {
    case 0: return filter_launch<0>(g, in, div, out, scale, st);
    case 1: return filter_launch<1>(g, in, div, out, scale, st);
    case 2: return filter_launch<2>(g, in, div, out, scale, st);
    case 3: return filter_launch<3>(g, in, div, out, scale, st);
    case 4: return filter_launch<4>(g, in, div, out, scale, st);
    case 5: return filter_launch<5>(g, in, div, out, scale, st);
    default: return filter_launch<6>(g, in, div, out, scale, st);
    }
}

}  // namespace gputo

namespace gputo {

// SIMP stiffness and its derivative (top3D125modCuda.m:124,130):
//   CX = Emin + x^p (E0 - Emin),   dsK = -p (E0 - Emin) x^(p-1)
__global__ void simp_kernel(long long n, const double *__restrict__ x, double penal, double E0,
                            double Emin, double *__restrict__ CX, double *__restrict__ dsK)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double xi = x[i];
        const double xp1 = pow(xi, penal - 1.0);
        CX[i] = Emin + xp1 * xi * (E0 - Emin);
        if (dsK) dsK[i] = -penal * (E0 - Emin) * xp1;
    }
}

void launch_simp(long long n, const double *x, double penal, double E0, double Emin, double *CX,
                 double *dsK, cudaStream_t st)
{
    long long nb = (n + 255) / 256;
    if (nb > 4736) nb = 4736;
    simp_kernel<<<(unsigned)nb, 256, 0, st>>>(n, x, penal, E0, Emin, CX, dsK);
    count_launches(1);
}

// OC update with bisection on the Lagrange multiplier
// (top3D125modCuda.m:143-151).  The multiplier bracket lives on the device;
// each bisection step is one pass that evaluates the candidate design at
// lmid, sums it in a fixed order and moves the bracket, so the whole loop
// needs no host round trip.  A step whose bracket is already tight returns
// at once, leaving the design of the last evaluated lmid, as the MATLAB loop
// does.
struct OcState {
    double l1, l2, lmid;
    int steps, done;
};

constexpr int kOcThreads = 256;
constexpr int kOcBlocks = 1184;

__device__ __forceinline__ double oc_candidate(double x, double ocp, double lmid, double move)
{
    // max(max(min(min(ocP/lmid, xU), 1), xL), 0)
    const double xU = x + move, xL = x - move;
    double v = ocp / lmid;
    v = fmin(v, xU);
    v = fmin(v, 1.0);
    v = fmax(v, xL);
    return fmax(v, 0.0);
}

__global__ void __launch_bounds__(kOcThreads)
oc_prepare_kernel(long long n, const double *__restrict__ x, const double *__restrict__ dc,
                  const double *__restrict__ dv0, double *__restrict__ ocp, double volfrac,
                  double *__restrict__ partial, unsigned *ticket, OcState *state)
{
    __shared__ double red[kOcThreads / 32];
    __shared__ bool is_last;
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = x[i] * sqrt(-dc[i] / dv0[i]);
        ocp[i] = v;
        s += v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < kOcThreads / 32; ++w) b += red[w];
        partial[blockIdx.x] = b;
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        __threadfence();
        double t = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) t += partial[b];
        OcState z;
        z.l1 = 0.0;
        z.l2 = (t / (double)n) / volfrac;
        z.lmid = 0.5 * (z.l1 + z.l2);
        z.steps = 0;
        z.done = !((z.l2 - z.l1) / (z.l2 + z.l1) > 1e-4);
        *state = z;
        *ticket = 0;
    }
}

__global__ void __launch_bounds__(kOcThreads)
oc_bisect_kernel(long long n, const double *__restrict__ x, const double *__restrict__ ocp,
                 double move, double volfrac, double *__restrict__ xnew,
                 double *__restrict__ partial, unsigned *ticket, OcState *state)
{
    if (state->done) return;
    __shared__ double red[kOcThreads / 32];
    __shared__ bool is_last;
    const double lmid = 0.5 * (state->l1 + state->l2);
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const double v = oc_candidate(x[i], ocp[i], lmid, move);
        xnew[i] = v;
        s += v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < kOcThreads / 32; ++w) b += red[w];
        partial[blockIdx.x] = b;
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        __threadfence();
        double t = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) t += partial[b];
        OcState z = *state;
        z.lmid = lmid;
        if (t / (double)n > volfrac) z.l1 = lmid;
        else z.l2 = lmid;
        z.steps += 1;
        z.done = !((z.l2 - z.l1) / (z.l2 + z.l1) > 1e-4);
        *state = z;
        *ticket = 0;
    }
}

// x_new = x when the loop body never runs (bracket already tight).
__global__ void copy_if_untouched_kernel(long long n, const double *__restrict__ x,
                                         double *__restrict__ xnew, const OcState *state)
{
    if (state->steps > 0) return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        xnew[i] = x[i];
}

int oc_state_bytes() { return (int)sizeof(OcState); }

// ---------------------------------------------------------------------------
// Heaviside projection with the volume-preserving threshold
// (top3D125modCuda.m:60-64 prj/deta/dprj, :111-119 the eta Newton loop):
//   while |mean(prj(xTilde, eta, beta)) - volfrac| > 1e-6:
//       eta -= f / mean(deta(xTilde, eta, beta))
//   xPhys = prj(xTilde, eta, beta),  dprj(xTilde, eta, beta) for the chain rule
// Each Newton step is one pass with a fixed-order sum; the threshold lives
// on the device, so the loop needs no host round trip.
// ---------------------------------------------------------------------------
struct ProjState {
    double eta;
    int steps, done;
};

__device__ __forceinline__ double prj_v(double v, double eta, double beta)
{
    return (tanh(beta * eta) + tanh(beta * (v - eta))) / (tanh(beta * eta) + tanh(beta * (1.0 - eta)));
}

__device__ __forceinline__ double deta_v(double v, double eta, double beta)
{
    const double c = cosh(beta * (v - eta));
    return -beta / sinh(beta) / (c * c) * sinh(v * beta) * sinh((1.0 - v) * beta);
}

__device__ __forceinline__ double dprj_v(double v, double eta, double beta)
{
    const double t = tanh(beta * (v - eta));
    return beta * (1.0 - t * t) / (tanh(beta * eta) + tanh(beta * (1.0 - eta)));
}

__global__ void proj_init_kernel(ProjState *state, double eta0)
{
    state->eta = eta0;
    state->steps = 0;
    state->done = 0;
}

__global__ void __launch_bounds__(kOcThreads)
proj_newton_kernel(long long n, const double *__restrict__ xt, double beta, double volfrac,
                   double *__restrict__ partial, unsigned *ticket, ProjState *state)
{
    if (state->done) return;
    __shared__ double rp[kOcThreads / 32], rd[kOcThreads / 32];
    __shared__ bool is_last;
    const double eta = state->eta;
    double sp = 0.0, sd = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        sp += prj_v(xt[i], eta, beta);
        sd += deta_v(xt[i], eta, beta);
    }
    for (int o = 16; o > 0; o >>= 1) {
        sp += __shfl_xor_sync(0xffffffffu, sp, o);
        sd += __shfl_xor_sync(0xffffffffu, sd, o);
    }
    if ((threadIdx.x & 31) == 0) rp[threadIdx.x >> 5] = sp, rd[threadIdx.x >> 5] = sd;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < kOcThreads / 32; ++w) a += rp[w], b += rd[w];
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
        __threadfence();
        is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (is_last && threadIdx.x == 0) {
        __threadfence();
        double a = 0.0, b = 0.0;
        for (unsigned q = 0; q < gridDim.x; ++q) a += partial[2 * q], b += partial[2 * q + 1];
        const double f = a / (double)n - volfrac;
        ProjState z = *state;
        if (fabs(f) > 1e-6) {
            z.eta = eta - f / (b / (double)n);
            z.steps += 1;
        } else {
            z.done = 1;
        }
        *state = z;
        *ticket = 0;
    }
}

__global__ void proj_apply_kernel(long long n, const double *__restrict__ xt, double beta,
                                  const ProjState *__restrict__ state, double *__restrict__ xphys,
                                  double *__restrict__ dprj)
{
    const double eta = state->eta;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        xphys[i] = prj_v(xt[i], eta, beta);
        if (dprj) dprj[i] = dprj_v(xt[i], eta, beta);
    }
}

int proj_state_bytes() { return (int)sizeof(ProjState); }

void launch_heaviside(long long n, const double *xt, double volfrac, double beta, double eta0, double *xphys,
                      double *dprj, double *partial, unsigned *ticket, void *state, int max_steps, cudaStream_t st)
{
    long long nb = (n + kOcThreads - 1) / kOcThreads;
    if (nb > kOcBlocks / 2) nb = kOcBlocks / 2;   // partial holds 2 sums per CTA
    ProjState *s = (ProjState *)state;
    proj_init_kernel<<<1, 1, 0, st>>>(s, eta0);
    for (int k = 0; k < max_steps; ++k)
        proj_newton_kernel<<<(unsigned)nb, kOcThreads, 0, st>>>(n, xt, beta, volfrac, partial, ticket, s);
    proj_apply_kernel<<<(unsigned)nb, kOcThreads, 0, st>>>(n, xt, beta, s, xphys, dprj);
    count_launches(2 + max_steps);
}

__global__ void mul_kernel(long long n, const double *__restrict__ a, const double *__restrict__ b,
                           double *__restrict__ out)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = a[i] * b[i];
}

void launch_mul(long long n, const double *a, const double *b, double *out, cudaStream_t st)
{
    long long nb = (n + 255) / 256;
    if (nb > 4096) nb = 4096;
    mul_kernel<<<(unsigned)nb, 256, 0, st>>>(n, a, b, out);
    count_launches(1);
}

void launch_oc_update(long long n, const double *x, const double *dc, const double *dv0,
                      double volfrac, double move, double *ocp, double *xnew, double *partial,
                      unsigned *ticket, void *state, int max_steps, cudaStream_t st)
{
    long long nb = (n + kOcThreads - 1) / kOcThreads;
    if (nb > kOcBlocks) nb = kOcBlocks;
    OcState *s = (OcState *)state;
    oc_prepare_kernel<<<(unsigned)nb, kOcThreads, 0, st>>>(n, x, dc, dv0, ocp, volfrac, partial,
                                                           ticket, s);
    for (int k = 0; k < max_steps; ++k)
        oc_bisect_kernel<<<(unsigned)nb, kOcThreads, 0, st>>>(n, x, ocp, move, volfrac, xnew,
                                                              partial, ticket, s);
    copy_if_untouched_kernel<<<(unsigned)nb, kOcThreads, 0, st>>>(n, x, xnew, s);
    count_launches(2 + max_steps);
}

}  // namespace gputo
