// Element-batched stiffness contraction on the 5th-generation tensor cores.
//
// ce_e = u_e^T Ke u_e for every element (the compliance sensitivity of
// top3D125modCuda.m:139) is the product Y = U Ke of the [n_elem x 24]
// element-displacement matrix with the 24 x 24 element matrix, followed by a
// row-wise dot with U.  One CTA takes 128 elements (M = 128):
//   * U and Ke are each split into three BF16 parts (hi + mid + lo carry the
//     24 bits of an FP32 value); Ke's parts sit side by side in B = [K1|K2|K3]
//     (N = 72, padded to 80), K = 24 padded to 32;
//   * one thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) for the
//     three U parts and both K halves into one TMEM accumulator, so TMEM holds
//     U K1, U K2 and U K3;
//   * tcgen05.ld brings each element's row back (one TMEM lane per thread);
//     Y = U K1 + U K2 + U K3 and ce = u . Y with the FP64 displacements.
// Each element's rigid-body motion is projected out of u_e in FP64 first
// (remove_rigid_motion), so each ce carries FP32 accuracy relative to itself
// (about 1e-7), well inside the 1e-6 compliance tolerance; the FP64 CUDA-core
// kernel remains the default.
#include <cuda_bf16.h>

#include "gputo_internal.h"
#include "tma.h"

namespace gputo {

// This translation unit's copy of the element matrix (constant memory is per
// translation unit without relocatable device code).
__constant__ double cKeTC[576];

int upload_tc_ke(const double *Ke_host, cudaStream_t st)
{
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(cKeTC, Ke_host, sizeof(double) * 576, 0, cudaMemcpyHostToDevice, st));
    return GPUTO_OK;
}

namespace {

constexpr int TC_M = 128;        // elements per CTA (TMEM lanes)
constexpr int TC_K = 32;         // 24 padded to a multiple of 16
constexpr int TC_N = 80;         // 3 x 24 padded to a multiple of 16
constexpr int TC_COLS = 128;     // TMEM columns allocated (power of 2 >= TC_N)
constexpr uint32_t kTcWaitPolls = 1u << 22;

// Byte offset of (row, col) in a K-major BF16 operand stored as 8x8 core
// matrices (16-byte rows), four core matrices along K per 8-row block:
// leading (K) byte offset 128, stride (M/N) byte offset 512, no swizzle.
__device__ __forceinline__ uint32_t core_offset(int row, int col)
{
    return (uint32_t)(((row >> 3) * 4 + (col >> 3)) * 128 + (row & 7) * 16 + (col & 7) * 2);
}

// Shared-memory matrix descriptor (sm_100): start address, leading and stride
// byte offsets (all >> 4), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t make_desc(const void *smem_ptr)
{
    const uint64_t addr = smem_u32(smem_ptr);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;             // bits  0-13 start address
    d |= (uint64_t)(128 >> 4) << 16;          // bits 16-29 leading byte offset (K)
    d |= (uint64_t)(512 >> 4) << 32;          // bits 32-45 stride byte offset (M/N)
    d |= (uint64_t)1 << 46;                   // bits 46-47 version
    return d;                                 // base offset 0, SWIZZLE_NONE (bits 61-63 = 0)
}

// Instruction descriptor, kind::f16: FP32 accumulate, BF16 A and B, both
// K-major, N = 80, M = 128.
constexpr uint32_t kInstrDesc = (1u << 4)               // D format F32
                              | (1u << 7)               // A format BF16
                              | (1u << 10)              // B format BF16
                              | ((uint32_t)(TC_N >> 3) << 17)
                              | ((uint32_t)(TC_M >> 4) << 24);

__device__ __forceinline__ void split3(float v, __nv_bfloat16 &a, __nv_bfloat16 &b, __nv_bfloat16 &c)
{
    a = __float2bfloat16_rn(v);
    const float r1 = v - __bfloat162float(a);
    b = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(b);
    c = __float2bfloat16_rn(r2);
}

__device__ __forceinline__ void store_bf16(unsigned char *base, uint32_t off, __nv_bfloat16 v)
{
    *reinterpret_cast<__nv_bfloat16 *>(base + off) = v;
}

// Removes the element's rigid-body motion from u_e in FP64.  Ke u_rigid = 0,
// so u^T Ke u is unchanged, but an element that mostly translates or rotates
// (far from the supports) keeps a large |u| with a small energy, and FP32
// accumulation of Ke u would lose that energy to cancellation.  With node
// coordinates centred on the element (+-1/2) the three translations and three
// rotations are mutually orthogonal over the 8 corners (norms 8 and 4), so the
// projection is six independent coefficients.
__device__ __forceinline__ void remove_rigid_motion(double (&u)[24])
{
    double tx = 0.0, ty = 0.0, tz = 0.0, wx = 0.0, wy = 0.0, wz = 0.0;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const double x = local_x(a) - 0.5, y = local_y(a) - 0.5, z = local_z(a) - 0.5;
        const double ux = u[3 * a], uy = u[3 * a + 1], uz = u[3 * a + 2];
        tx += ux;
        ty += uy;
        tz += uz;
        wx += y * uz - z * uy;   // rotation about x: (0, -z, y)
        wy += z * ux - x * uz;   // rotation about y: (z, 0, -x)
        wz += x * uy - y * ux;   // rotation about z: (-y, x, 0)
    }
    tx *= 0.125, ty *= 0.125, tz *= 0.125;
    wx *= 0.25, wy *= 0.25, wz *= 0.25;
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const double x = local_x(a) - 0.5, y = local_y(a) - 0.5, z = local_z(a) - 0.5;
        u[3 * a] -= tx + wy * z - wz * y;
        u[3 * a + 1] -= ty - wx * z + wz * x;
        u[3 * a + 2] -= tz + wx * y - wy * x;
    }
}

}  // namespace

// v = hi + mid + lo exactly, each part a BF16 value held in the upper half
// of a 32-bit word (truncating splits: hi keeps the top 8 significand bits,
// the exact remainder keeps at most 16, mid the top 8 of those, and lo the
// at most 8 bits left, which BF16 holds exactly).
__device__ __forceinline__ void split3_bits(float v, uint32_t (&w)[3])
{
    const uint32_t b0 = __float_as_uint(v);
    const float r1 = v - __uint_as_float(b0 & 0xFFFF0000u);
    const uint32_t b1 = __float_as_uint(r1);
    const float r2 = r1 - __uint_as_float(b1 & 0xFFFF0000u);
    w[0] = b0;
    w[1] = b1;
    w[2] = __float_as_uint(r2);
}

// Persistent: each CTA allocates its TMEM and builds B once, then walks
// 128-element tiles blockIdx.x, blockIdx.x + gridDim.x, ...
__global__ void __launch_bounds__(TC_M, 4)
element_energy_tc_kernel(Grid g, const double *__restrict__ U,
                         const double *__restrict__ CX, const double *__restrict__ dsK,
                         double *__restrict__ ce, double *__restrict__ dc, double *__restrict__ partial,
                         int *__restrict__ err)
{
    __shared__ __align__(128) unsigned char sA[3][TC_M * TC_K * 2];
    __shared__ __align__(128) unsigned char sB[TC_N * TC_K * 2];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ double red[TC_M / 32];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long nel = g.nel();
    const long long ntiles = (nel + TC_M - 1) / TC_M;

    // TMEM accumulator: 128 lanes x 128 columns, allocated by warp 0
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(TC_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }

    // B = [K1 | K2 | K3 | 0]: row n = 24 q + m of B is row m of Ke part q
    for (int idx = tid; idx < TC_N * TC_K; idx += TC_M) {
        const int n = idx / TC_K, k = idx - n * TC_K;
        __nv_bfloat16 v = __float2bfloat16_rn(0.f);
        if (n < 72 && k < 24) {
            const int q = n / 24, m = n - 24 * q;
            __nv_bfloat16 p0, p1, p2;
            split3((float)cKeTC[m * 24 + k], p0, p1, p2);
            v = q == 0 ? p0 : (q == 1 ? p1 : p2);
        }
        store_bf16(sB, core_offset(n, k), v);
    }
    // A's K padding (columns 24..31) stays zero for every tile
#pragma unroll
    for (int part = 0; part < 3; ++part)
        *reinterpret_cast<uint4 *>(sA[part] + core_offset(tid, 24)) = make_uint4(0u, 0u, 0u, 0u);

    const uint32_t row_addr_off = (uint32_t)(warp * 32) << 16;
    double cs = 0.0;
    uint32_t phase = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, phase ^= 1u) {
        const long long e = tile * TC_M + tid;
        // this thread's element row; the FP64 row stays in registers.  Index
        // arithmetic is 32-bit: the launcher admits only grids whose dof
        // count fits.
        double ue[24];
        if (e < nel) {
            const uint32_t e32 = (uint32_t)e, t32 = e32 / (uint32_t)g.ny;
            const uint32_t j = e32 - t32 * (uint32_t)g.ny;
            const uint32_t i = t32 / (uint32_t)g.nz, k = t32 - i * (uint32_t)g.nz;
            const uint32_t sk = (uint32_t)g.ny + 1u, si = sk * ((uint32_t)g.nz + 1u);
            const uint32_t nb = si * i + sk * k + j;
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                const uint32_t n = nb + si * (uint32_t)local_x(a) + sk * (uint32_t)local_z(a) + (uint32_t)local_y(a);
#pragma unroll
                for (int d = 0; d < 3; ++d) ue[3 * a + d] = U[3u * n + (uint32_t)d];
            }
        } else {
#pragma unroll
            for (int m = 0; m < 24; ++m) ue[m] = 0.0;
        }
        remove_rigid_motion(ue);
        // three BF16 parts, eight columns (one 16-byte core-matrix row) per store
#pragma unroll
        for (int c0 = 0; c0 < 24; c0 += 8) {
            uint32_t w[3][4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint32_t a[3], b[3];
                split3_bits((float)ue[c0 + 2 * q], a);
                split3_bits((float)ue[c0 + 2 * q + 1], b);
#pragma unroll
                for (int part = 0; part < 3; ++part) w[part][q] = __byte_perm(a[part], b[part], 0x7632);
            }
            const uint32_t off = core_offset(tid, c0);
#pragma unroll
            for (int part = 0; part < 3; ++part)
                *reinterpret_cast<uint4 *>(sA[part] + off) = make_uint4(w[part][0], w[part][1], w[part][2], w[part][3]);
        }
        // generic-proxy smem writes -> visible to the tensor core (async proxy);
        // the barrier also orders the previous tile's TMEM reads before the MMAs
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

        const uint32_t tmem = tmem_base;
        if (tid == 0) {
#pragma unroll
            for (int part = 0; part < 3; ++part) {
#pragma unroll
                for (int kk = 0; kk < TC_K / 16; ++kk) {
                    // K half kk starts two core matrices (256 bytes) further along K
                    const uint64_t da = make_desc(sA[part] + kk * 256);
                    const uint64_t db = make_desc(sB + kk * 256);
                    const uint32_t acc = (part | kk) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                        ::"r"(tmem), "l"(da), "l"(db), "r"(kInstrDesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                        : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bar))
                         : "memory");
        }
        const bool timed_out = !mbar_wait_bounded(&bar, phase, kTcWaitPolls);
        if (timed_out) {
            if (err) atomicExch(err, GPUTO_ERR_TIMEOUT);
            // let the MMAs drain before TMEM or shared memory is touched again
            mbar_wait_bounded(&bar, phase, kTcWaitPolls);
        }
        if (__syncthreads_or(timed_out)) break;   // block-uniform: every thread leaves
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

        // this warp's 32 TMEM lanes (its 32 elements): column c holds
        // (U Kq)[c mod 24] for part q = c / 24; y = U K1 + U K2 + U K3 is
        // summed in FP32 (largest part first), ce = u . y in FP64
        float y[24];
#pragma unroll
        for (int c0 = 0; c0 < 72; c0 += 16) {
            uint32_t r[16];
            // the wait is in the same statement: no use of r can move above it
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
                "tcgen05.wait::ld.sync.aligned;"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(tmem + row_addr_off + (uint32_t)c0)
                : "memory");
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int c = c0 + q;
                if (c < 24) y[c] = __uint_as_float(r[q]);
                else if (c < 72) y[c % 24] += __uint_as_float(r[q]);
            }
        }
        double s = 0.0;
#pragma unroll
        for (int m = 0; m < 24; ++m) s = fma(ue[m], (double)y[m], s);
        if (e < nel) {
            if (ce) ce[e] = s;
            if (dc) dc[e] = dsK[e] * s;
            if (CX) cs = fma(CX[e], s, cs);
        }
    }
    for (int o = 16; o > 0; o >>= 1) cs += __shfl_xor_sync(0xffffffffu, cs, o);
    if (lane == 0) red[warp] = cs;

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TC_COLS)
                     : "memory");
    }
    if (tid == 0 && partial) partial[blockIdx.x] = red[0] + red[1] + red[2] + red[3];
}

// Second pass: sum of the per-CTA compliance partials in a fixed order.
__global__ void sum_partials_kernel(const double *__restrict__ partial, long long n, double *__restrict__ out)
{
    __shared__ double red[32];
    double v = 0.0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) v += partial[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        *out = t;
    }
}

bool element_energy_tc_fits(const Grid &g) { return g.ndof() < (1LL << 31); }

// Persistent grid: four CTAs per SM (the TMEM and register budget), never
// more CTAs than tiles.
long long element_energy_tc_partials(const Grid &g)
{
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (g.nel() + TC_M - 1) / TC_M;
    const long long cap = 4LL * sms;
    return tiles < cap ? tiles : cap;
}

// Ke comes from constant memory (upload_fine_ke); partial: one slot per CTA
// (element_energy_tc_partials); compliance: device scalar or NULL.
void launch_element_energy_tc(const Grid &g, const double *U, const double *CX, const double *dsK,
                              double *ce, double *dc, double *partial, double *compliance, int *err,
                              cudaStream_t st)
{
    const long long nb = element_energy_tc_partials(g);
    element_energy_tc_kernel<<<(unsigned)nb, TC_M, 0, st>>>(g, U, CX, dsK, ce, dc,
                                                            compliance ? partial : nullptr, err);
    count_launches(1);
    if (compliance) {
        sum_partials_kernel<<<1, 1024, 0, st>>>(partial, nb, compliance);
        count_launches(1);
    }
}

}  // namespace gputo
