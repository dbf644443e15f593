// Fine-level operator sweeps, K = sum_e CX_e Ke on the voxel grid.
//
// One kernel does K u (MODE_APPLY, optionally with the CTA partials of u'Ku),
// f - K u (MODE_DEFECT), or a damped Jacobi sweep u + w (f - K u)/diag
// (MODE_JACOBI; MODE_JACOBI_PRE starts from u = prerelax f / diag), with the
// Dirichlet rows zeroed in the epilogue.  It is the node-centred gather of the
// reference's multAV0c / defect0c + Jacobc + ZeroBCc
// (Cantilever/TOP3D125MGCGCUDA/mgcg1.cu:941-997,1199-1264,1326-1331) reorganised
// for sm_100a:
//  * a CTA owns a 32 (y) x 8 (z) x 4 (x) block of nodes; its halo tiles of u
//    (and of f and diag for MODE_JACOBI_PRE) and of CX arrive in shared memory
//    by TMA (cp.async.bulk.tensor, zero fill outside the grid) on one mbarrier;
//  * each thread owns a column of 4 nodes along x and visits the 20 elements
//    around it once, using each element's 24 displacements for both column
//    nodes the element touches;
//  * the element-local row block of Ke is the same for the whole warp at every
//    step, so Ke is an operand from constant memory.
// Nodes on the three far faces (j = ny, k = nz or i = nx) are handled by a
// small gather kernel so that the tile grid divides the element grid exactly.
#include "gputo_internal.h"
#include "tma.h"

#include <mutex>

namespace gputo {

__constant__ double cKe64[576];
__constant__ float cKe32[576];
__constant__ float2 cKe32p[288];   // the same FP32 rows as (q, q+1) pairs for packed FMAs

template <typename T> __device__ __forceinline__ T ke(int idx);
template <> __device__ __forceinline__ double ke<double>(int idx) { return cKe64[idx]; }
template <> __device__ __forceinline__ float ke<float>(int idx) { return cKe32[idx]; }

int upload_fine_ke(const double *Ke_host, cudaStream_t st)
{
    // constant memory is per device: remember what each device holds
    static std::mutex mu;
    static double last[64][576];
    static bool have[64] = {};
    static unsigned long long ctx_of[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    int dev = 0;
    GPUTO_CUDA(cudaGetDevice(&dev));
    const int slot = dev < 64 ? dev : 63;
    // Ke0 is an argument of every MEX call; skip the copy when it repeats
    // (in the same context: a device reset clears constant memory).
    const unsigned long long ctx = current_context_id();
    bool same = have[slot] && dev < 64 && ctx != 0 && ctx_of[slot] == ctx;
    for (int m = 0; same && m < 576; ++m) same = (last[slot][m] == Ke_host[m]);
    if (same) return GPUTO_OK;
    float kf[576];
    for (int m = 0; m < 576; ++m) {
        last[slot][m] = Ke_host[m];
        kf[m] = (float)Ke_host[m];
    }
    have[slot] = true;
    ctx_of[slot] = ctx;
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(cKe64, last[slot], sizeof(double) * 576, 0, cudaMemcpyHostToDevice, st));
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(cKe32, kf, sizeof(kf), 0, cudaMemcpyHostToDevice, st));
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(cKe32p, kf, sizeof(kf), 0, cudaMemcpyHostToDevice, st));
    int s2 = upload_design_ke(last[slot], st);
    if (!s2) s2 = upload_tc_ke(last[slot], st);
    if (!s2) s2 = upload_tcsweep_ke(last[slot], st);
    if (s2) return s2;
    GPUTO_CUDA(cudaStreamSynchronize(st));
    return GPUTO_OK;
}

// ---------------------------------------------------------------------------
// level-1 quadrature parts (constant memory, this translation unit's copy)
// ---------------------------------------------------------------------------

// Kg[g] packed lower triangle (300), g = 4 ix + 2 iz + iy: the 2h element's
// stiffness evaluated at one Gauss point (mgcg1.cu:2000-2040 prepAelm); used
// here for the diagonal of the level-1 operator.
__constant__ double cKq64[8 * 300];

int upload_quadrature_fine(const double *kg_packed, cudaStream_t st)
{
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(cKq64, kg_packed, sizeof(double) * 8 * 300, 0,
                                       cudaMemcpyHostToDevice, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    return GPUTO_OK;
}

// ---------------------------------------------------------------------------
// tile geometry
// ---------------------------------------------------------------------------
//
// OP_FINE: K = sum_e CX_e Ke (the fine level).  The operator is a template
// parameter so that other element operators can share the tile machinery.

constexpr int OP_FINE = 0;
constexpr int TY = 32, TZ = 8;                    // nodes per tile in y, z
constexpr int NT = TY * TZ;                       // threads per CTA (one x-column each)
constexpr int UW = 104;                           // u box width: 3*(TY+2) = 102 values from
                                                  // 3(j0-1)-1 (16-byte aligned start)
constexpr int UOFF = 1;                           // value offset of halo node 0 in a u row
constexpr int TX_FINE = 4;                        // nodes per thread column along x

// CX box width / offset (16-byte aligned start per element type)
template <typename T, int OP> struct CxBox;
template <> struct CxBox<double, OP_FINE> { static constexpr int W = 34, OFF = 1; };
template <> struct CxBox<float, OP_FINE> { static constexpr int W = 36, OFF = 3; };

template <typename T, int OP, int TXN>
struct TileSmem {
    static constexpr int CZ = TZ + 1;                                   // CX box rows in z
    static constexpr int CX_ = TXN + 1;                                 // CX box planes in x
    static constexpr int U = (TXN + 2) * (TZ + 2) * UW;                // values
    static constexpr int C = CX_ * CZ * CxBox<T, OP>::W;
    static constexpr size_t u_bytes = sizeof(T) * U;
    static constexpr size_t c_bytes = sizeof(T) * C;
    static constexpr size_t u_off = 0;
    static constexpr size_t d_off = (u_bytes + 127) & ~size_t(127);   // diag tile (PRE only)
    __host__ __device__ static constexpr size_t c_off(bool pre) { return pre ? 2 * d_off : d_off; }
    __host__ __device__ static constexpr size_t bar_off(bool pre) { return (c_off(pre) + c_bytes + 127) & ~size_t(127); }
    __host__ __device__ static constexpr size_t bytes(bool pre) { return bar_off(pre) + 16; }
};

constexpr uint32_t kWaitPolls = 1u << 22;   // bounded mbarrier wait (seconds, not forever)

// rows (3a..3a+2) of one element operator times its 24 displacements
template <typename T, int OP>
__device__ __forceinline__ void element_rows(int a, const T (&ue)[24], const T *cg, T &t0, T &t1, T &t2)
{
#pragma unroll
    for (int q = 0; q < 24; ++q) {
        t0 = fma(ke<T>((3 * a) * 24 + q), ue[q], t0);
        t1 = fma(ke<T>((3 * a + 1) * 24 + q), ue[q], t1);
        t2 = fma(ke<T>((3 * a + 2) * 24 + q), ue[q], t2);
    }
    t0 *= cg[0];
    t1 *= cg[0];
    t2 *= cg[0];
}

// FP32: packed two-wide FMAs (sm_100 FFMA2), each row summed as two interleaved
// partial sums over (q, q+1) pairs, so one instruction issues two FMAs; the
// FP32 sweep is issue-bound, not FMA-bound.
template <>
__device__ __forceinline__ void element_rows<float, OP_FINE>(int a, const float (&ue)[24], const float *cg, float &t0,
                                                             float &t1, float &t2)
{
    float2 s0 = make_float2(0.f, 0.f), s1 = s0, s2 = s0;
#pragma unroll
    for (int q = 0; q < 24; q += 2) {
        const float2 u2 = make_float2(ue[q], ue[q + 1]);
        s0 = __ffma2_rn(cKe32p[((3 * a) * 24 + q) >> 1], u2, s0);
        s1 = __ffma2_rn(cKe32p[((3 * a + 1) * 24 + q) >> 1], u2, s1);
        s2 = __ffma2_rn(cKe32p[((3 * a + 2) * 24 + q) >> 1], u2, s2);
    }
    t0 = fmaf(s0.x + s0.y, cg[0], t0);
    t1 = fmaf(s1.x + s1.y, cg[0], t1);
    t2 = fmaf(s2.x + s2.y, cg[0], t2);
}

// FP32 instances are held to 3 CTAs per SM (85 registers): with packed FMAs
// the sweep is latency-bound, and the third CTA hides more than the spare
// registers would.
template <typename T, int MODE, int OP, int TXN>
__global__ void __launch_bounds__(NT, sizeof(T) == 4 ? 3 : 2)
tile_kernel(const __grid_constant__ CUtensorMap tm_u, const __grid_constant__ CUtensorMap tm_d,
            const __grid_constant__ CUtensorMap tm_c, Lay L, const T *__restrict__ f,
            const T *__restrict__ diag, const uint8_t *__restrict__ mask, T *__restrict__ out,
            T omega, T prerelax, double *__restrict__ dot_partial, const int *__restrict__ done,
            int *__restrict__ err)
{
    if (done && *done) return;
    constexpr bool PRE = (MODE == MODE_JACOBI_PRE);
    using S = TileSmem<T, OP, TXN>;
    constexpr int CW = CxBox<T, OP>::W, COFF = CxBox<T, OP>::OFF;
    extern __shared__ __align__(128) unsigned char smem[];
    T *su = reinterpret_cast<T *>(smem + S::u_off);
    T *sd = reinterpret_cast<T *>(smem + S::d_off);
    T *sc = reinterpret_cast<T *>(smem + S::c_off(PRE));
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + S::bar_off(PRE));

    const Grid &g = L.g;
    const int j0 = blockIdx.x * TY, k0 = blockIdx.y * TZ, i0 = blockIdx.z * TXN;
    const int tid = threadIdx.x;

    if (tid == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        const uint32_t bytes = (uint32_t)(S::u_bytes * (PRE ? 2 : 1) + S::c_bytes);
        mbar_arrive_expect_tx(bar, bytes);
        const int cu = 3 * (j0 - 1) - UOFF;
        tma_load_3d(su, &tm_u, cu, k0 - 1, i0 - 1, bar);
        if (PRE) tma_load_3d(sd, &tm_d, cu, k0 - 1, i0 - 1, bar);
        tma_load_3d(sc, &tm_c, j0 - 1 - COFF, k0 - 1, i0 - 1, bar);
    }
    const bool ok = mbar_wait_bounded(bar, 0, kWaitPolls);
    if (__syncthreads_or(!ok)) {
        if (tid == 0 && err) atomicExch(err, GPUTO_ERR_TIMEOUT);
        return;
    }
    if (PRE) {
        // halo of the initial smoother guess u = prerelax f / diag (0 outside)
        for (int idx = tid; idx < S::U; idx += NT) {
            const T dv = sd[idx];
            su[idx] = dv != T(0) ? prerelax * su[idx] / dv : T(0);
        }
        __syncthreads();
    }

    const int ty = tid & 31, tz = tid >> 5;
    T acc[TXN][3];
#pragma unroll
    for (int n = 0; n < TXN; ++n) acc[n][0] = acc[n][1] = acc[n][2] = T(0);

#pragma unroll
    for (int l = 0; l <= TXN; ++l) {          // element x-layer i0-1+l
#pragma unroll
        for (int ez = 0; ez < 2; ++ez) {
#pragma unroll
            for (int ey = 0; ey < 2; ++ey) {
                T cg[1];
                cg[0] = sc[(l * S::CZ + tz + ez) * CW + COFF + ty + ey];
                T ue[24];
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    const T *p = su + ((l + local_x(b)) * (TZ + 2) + tz + ez + local_z(b)) * UW + UOFF +
                                 3 * (ty + ey + local_y(b));
                    ue[3 * b] = p[0];
                    ue[3 * b + 1] = p[1];
                    ue[3 * b + 2] = p[2];
                }
#pragma unroll
                for (int side = 0; side < 2; ++side) {
                    // side 0: the element's x = 0 face node (column node l-1);
                    // side 1: its x = 1 face node (column node l)
                    const int n = side ? l : l - 1;
                    if (n < 0 || n >= TXN) continue;
                    const int a = local_index(side, 1 - ey, 1 - ez);
                    T t0 = T(0), t1 = T(0), t2 = T(0);
                    element_rows<T, OP>(a, ue, cg, t0, t1, t2);
                    acc[n][0] += t0;
                    acc[n][1] += t1;
                    acc[n][2] += t2;
                }
            }
        }
    }

    double dsum = 0.0;
    const int j = j0 + ty, k = k0 + tz;
#pragma unroll
    for (int n = 0; n < TXN; ++n) {
        const int i = i0 + n;
        if (j >= g.ny || k >= g.nz || i >= g.nx) continue;   // far faces: face kernel
        const unsigned m = mask[g.node(i, j, k)];
        const long long base = L.at(i, j, k);
        const T *us = su + ((n + 1) * (TZ + 2) + tz + 1) * UW + UOFF + 3 * (ty + 1);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const bool fixed = (m >> d) & 1u;
            if (MODE == MODE_APPLY) {
                const T q = fixed ? T(0) : acc[n][d];
                out[base + d] = q;
                if (dot_partial) dsum += (double)us[d] * (double)q;
            } else if (MODE == MODE_DEFECT) {
                out[base + d] = fixed ? T(0) : f[base + d] - acc[n][d];
            } else {
                const T r = fixed ? T(0) : f[base + d] - acc[n][d];
                out[base + d] = us[d] + omega * r / diag[base + d];
            }
        }
    }
    if (MODE == MODE_APPLY && dot_partial) {
        __shared__ double red[NT / 32];
        for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
        if ((tid & 31) == 0) red[tid >> 5] = dsum;
        __syncthreads();
        if (tid < 32) {
            double v = tid < NT / 32 ? red[tid] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (tid == 0)
                dot_partial[blockIdx.x + gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z)] = v;
        }
    }
}


// Nodes on the far faces j = ny, k = nz, i = nx: a direct gather, one thread
// per node.  Face A: j = ny; face B: k = nz, j < ny; face C: i = nx, j < ny, k < nz.
// E is the layout of the CX array.
template <typename T, int MODE, int OP>
__global__ void __launch_bounds__(128)
face_kernel(Lay L, ELay E, const T *__restrict__ CX, const T *__restrict__ u,
            const T *__restrict__ f, const T *__restrict__ diag,
            const uint8_t *__restrict__ mask, T *__restrict__ out, T omega, T prerelax,
            double *__restrict__ dot_partial, const int *__restrict__ done)
{
    if (done && *done) return;
    const Grid &g = L.g;
    const long long nA = (long long)(g.nx + 1) * (g.nz + 1);
    const long long nB = (long long)(g.nx + 1) * g.ny;
    const long long nC = (long long)g.ny * g.nz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dsum = 0.0;
    if (t < nA + nB + nC) {
        int i, j, k;
        if (t < nA) {
            j = g.ny;
            i = (int)(t / (g.nz + 1));
            k = (int)(t - (long long)i * (g.nz + 1));
        } else if (t < nA + nB) {
            const long long s = t - nA;
            k = g.nz;
            i = (int)(s / g.ny);
            j = (int)(s - (long long)i * g.ny);
        } else {
            const long long s = t - nA - nB;
            i = g.nx;
            k = (int)(s / g.ny);
            j = (int)(s - (long long)k * g.ny);
        }
        T acc[3] = {T(0), T(0), T(0)};
        for (int ex = 0; ex < 2; ++ex) {
            const int ei = i - 1 + ex;
            if (ei < 0 || ei >= g.nx) continue;
            for (int ez = 0; ez < 2; ++ez) {
                const int ek = k - 1 + ez;
                if (ek < 0 || ek >= g.nz) continue;
                for (int ey = 0; ey < 2; ++ey) {
                    const int ej = j - 1 + ey;
                    if (ej < 0 || ej >= g.ny) continue;
                    T cg[1] = {CX[E.at(ei, ej, ek)]};
                    const int a = local_index(1 - ex, 1 - ey, 1 - ez);
                    T ue[24];
#pragma unroll
                    for (int b = 0; b < 8; ++b) {
                        const long long nb = L.at(ei + local_x(b), ej + local_y(b), ek + local_z(b));
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            if (MODE == MODE_JACOBI_PRE) {
                                const T dv = diag[nb + q];
                                ue[3 * b + q] = dv != T(0) ? prerelax * f[nb + q] / dv : T(0);
                            } else {
                                ue[3 * b + q] = u[nb + q];
                            }
                        }
                    }
                    T t0 = T(0), t1 = T(0), t2 = T(0);
                    element_rows<T, OP>(a, ue, cg, t0, t1, t2);
                    acc[0] += t0;
                    acc[1] += t1;
                    acc[2] += t2;
                }
            }
        }
        const unsigned m = mask[g.node(i, j, k)];
        const long long base = L.at(i, j, k);
        for (int d = 0; d < 3; ++d) {
            const bool fixed = (m >> d) & 1u;
            if (MODE == MODE_APPLY) {
                const T q = fixed ? T(0) : acc[d];
                out[base + d] = q;
                if (dot_partial) dsum += (double)u[base + d] * (double)q;
            } else if (MODE == MODE_DEFECT) {
                out[base + d] = fixed ? T(0) : f[base + d] - acc[d];
            } else {
                const T r = fixed ? T(0) : f[base + d] - acc[d];
                T us;
                if (MODE == MODE_JACOBI_PRE) {
                    const T dv = diag[base + d];
                    us = dv != T(0) ? prerelax * f[base + d] / dv : T(0);
                } else {
                    us = u[base + d];
                }
                out[base + d] = us + omega * r / diag[base + d];
            }
        }
    }
    if (MODE == MODE_APPLY && dot_partial) {
        __shared__ double red[4];
        for (int o = 16; o > 0; o >>= 1) dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dsum;
        __syncthreads();
        if (threadIdx.x == 0) dot_partial[blockIdx.x] = red[0] + red[1] + red[2] + red[3];
    }
}

template <int TXN>
static dim3 tile_grid(const Grid &g)
{
    return dim3((g.ny + TY - 1) / TY, (g.nz + TZ - 1) / TZ, (g.nx + TXN - 1) / TXN);
}

static long long face_nodes(const Grid &g)
{
    return (long long)(g.nx + 1) * (g.nz + 1) + (long long)(g.nx + 1) * g.ny + (long long)g.ny * g.nz;
}

int fine_sweep_blocks(const Grid &g)
{
    const dim3 tg = tile_grid<TX_FINE>(g);
    return (int)(tg.x * tg.y * tg.z + (face_nodes(g) + 127) / 128);
}

// Tensor maps for one sweep: u (or f), diag (PRE only) and CX (layout E).
template <typename T, int OP, int TXN>
static int make_maps(const Lay &L, const ELay &E, const T *u, const T *d, const T *CX, CUtensorMap *mu,
                     CUtensorMap *md, CUtensorMap *mc)
{
    using S = TileSmem<T, OP, TXN>;
    const Grid &g = L.g;
    const uint64_t es = sizeof(T);
    int st = make_tmap_3d(mu, u, (int)es, (uint64_t)L.pitch, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1,
                          L.pitch * es, L.pitch * es * (g.nz + 1), UW, TZ + 2, TXN + 2);
    if (!st && d)
        st = make_tmap_3d(md, d, (int)es, (uint64_t)L.pitch, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1,
                          L.pitch * es, L.pitch * es * (g.nz + 1), UW, TZ + 2, TXN + 2);
    if (!st)
        st = make_tmap_3d(mc, CX, (int)es, (uint64_t)E.pitch, (uint64_t)E.g.nz, (uint64_t)E.g.nx,
                          E.pitch * es, E.pitch * es * E.g.nz, CxBox<T, OP>::W, S::CZ, S::CX_);
    return st;
}

template <typename T, int MODE, int OP, int TXN>
static int launch_mode(const Lay &L, const ELay &E, const T *CX, const T *u, const T *f, const T *diag,
                       const uint8_t *mask, T *out, T omega, T prerelax, double *dot_partial,
                       const int *done, int *err, cudaStream_t st)
{
    constexpr bool PRE = (MODE == MODE_JACOBI_PRE);
    CUtensorMap mu, md, mc;
    int s = make_maps<T, OP, TXN>(L, E, PRE ? f : u, PRE ? diag : nullptr, CX, &mu, &md, &mc);
    if (s) return s;
    if (!PRE) md = mu;
    const size_t smem = TileSmem<T, OP, TXN>::bytes(PRE);
    const dim3 tg = tile_grid<TXN>(L.g);
    tile_kernel<T, MODE, OP, TXN><<<tg, NT, smem, st>>>(mu, md, mc, L, f, diag, mask, out, omega, prerelax,
                                                        dot_partial, done, err);
    const long long nf = face_nodes(L.g);
    const unsigned fb = (unsigned)((nf + 127) / 128);
    double *fp = dot_partial ? dot_partial + (long long)tg.x * tg.y * tg.z : nullptr;
    face_kernel<T, MODE, OP><<<fb, 128, 0, st>>>(L, E, CX, u, f, diag, mask, out, omega, prerelax, fp, done);
    count_launches(2);
    return GPUTO_OK;
}

template <typename T, int MODE, int OP, int TXN>
static cudaError_t set_smem_attr()
{
    return cudaFuncSetAttribute(tile_kernel<T, MODE, OP, TXN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)TileSmem<T, OP, TXN>::bytes(MODE == MODE_JACOBI_PRE));
}

template <typename T, int OP, int TXN>
static cudaError_t set_attrs_all_modes()
{
    cudaError_t e;
    if ((e = set_smem_attr<T, MODE_APPLY, OP, TXN>()) != cudaSuccess) return e;
    if ((e = set_smem_attr<T, MODE_DEFECT, OP, TXN>()) != cudaSuccess) return e;
    if ((e = set_smem_attr<T, MODE_JACOBI, OP, TXN>()) != cudaSuccess) return e;
    return set_smem_attr<T, MODE_JACOBI_PRE, OP, TXN>();
}

// Dynamic shared-memory opt-in for every tile-kernel instance, once per
// process and device, outside any stream capture.
int init_fine_kernels()
{
    static std::mutex mu;
    static bool done_dev[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && done_dev[dev]) return GPUTO_OK;
    GPUTO_CUDA((set_attrs_all_modes<double, OP_FINE, TX_FINE>()));
    GPUTO_CUDA((set_attrs_all_modes<float, OP_FINE, TX_FINE>()));
    if (dev < 64) done_dev[dev] = true;
    return GPUTO_OK;
}

template <typename T, int OP, int TXN>
static int launch_any(int mode, const Lay &L, const ELay &E, const T *CX, const T *u, const T *f,
                      const T *diag, const uint8_t *mask, T *out, T omega, T prerelax,
                      double *dot_partial, const int *done, int *err, cudaStream_t st)
{
    switch (mode) {
    case MODE_APPLY:
        return launch_mode<T, MODE_APPLY, OP, TXN>(L, E, CX, u, f, diag, mask, out, omega, prerelax,
                                                   dot_partial, done, err, st);
    case MODE_DEFECT:
        return launch_mode<T, MODE_DEFECT, OP, TXN>(L, E, CX, u, f, diag, mask, out, omega, prerelax,
                                                    nullptr, done, err, st);
    case MODE_JACOBI:
        return launch_mode<T, MODE_JACOBI, OP, TXN>(L, E, CX, u, f, diag, mask, out, omega, prerelax,
                                                    nullptr, done, err, st);
    default:
        return launch_mode<T, MODE_JACOBI_PRE, OP, TXN>(L, E, CX, u, f, diag, mask, out, omega, prerelax,
                                                        nullptr, done, err, st);
    }
}

template <typename T>
int launch_fine_sweep(int mode, const Lay &L, const ELay &E, const T *CX, const T *u, const T *f,
                      const T *diag, const uint8_t *mask, T *out, T omega, T prerelax,
                      double *dot_partial, const int *done, int *err, cudaStream_t st)
{
    return launch_any<T, OP_FINE, TX_FINE>(mode, L, E, CX, u, f, diag, mask, out, omega, prerelax,
                                           dot_partial, done, err, st);
}

// The far-face gather alone (nodes j = ny, k = nz, i = nx), for sweeps whose
// interior comes from another kernel.
template <typename T>
int launch_fine_faces(int mode, const Lay &L, const ELay &E, const T *CX, const T *u, const T *f, const T *diag,
                      const uint8_t *mask, T *out, T omega, T prerelax, const int *done, cudaStream_t st)
{
    const unsigned fb = (unsigned)((face_nodes(L.g) + 127) / 128);
    switch (mode) {
    case MODE_APPLY:
        face_kernel<T, MODE_APPLY, OP_FINE><<<fb, 128, 0, st>>>(L, E, CX, u, f, diag, mask, out, omega, prerelax,
                                                                nullptr, done);
        break;
    case MODE_DEFECT:
        face_kernel<T, MODE_DEFECT, OP_FINE><<<fb, 128, 0, st>>>(L, E, CX, u, f, diag, mask, out, omega, prerelax,
                                                                 nullptr, done);
        break;
    case MODE_JACOBI:
        face_kernel<T, MODE_JACOBI, OP_FINE><<<fb, 128, 0, st>>>(L, E, CX, u, f, diag, mask, out, omega, prerelax,
                                                                 nullptr, done);
        break;
    default:
        face_kernel<T, MODE_JACOBI_PRE, OP_FINE><<<fb, 128, 0, st>>>(L, E, CX, u, f, diag, mask, out, omega,
                                                                     prerelax, nullptr, done);
    }
    count_launches(1);
    return GPUTO_OK;
}
template int launch_fine_faces<float>(int, const Lay &, const ELay &, const float *, const float *, const float *,
                                      const float *, const uint8_t *, float *, float, float, const int *,
                                      cudaStream_t);

template int launch_fine_sweep<double>(int, const Lay &, const ELay &, const double *, const double *,
                                       const double *, const double *, const uint8_t *, double *,
                                       double, double, double *, const int *, int *, cudaStream_t);
template int launch_fine_sweep<float>(int, const Lay &, const ELay &, const float *, const float *,
                                      const float *, const float *, const uint8_t *, float *, float,
                                      float, double *, const int *, int *, cudaStream_t);

// diag of the level-1 quadrature operator from the fine CX (natural order):
// sum over adjacent coarse elements and Gauss points of CX_g Kg[g][m][m].
__global__ void diag_quad_kernel(Lay L, const double *__restrict__ CXf, double *__restrict__ diag)
{
    const Grid &g = L.g;
    const Grid gf{2 * g.nx, 2 * g.ny, 2 * g.nz};
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    const long long t = n / (g.ny + 1);
    const int j = (int)(n - t * (g.ny + 1));
    const int i = (int)(t / (g.nz + 1));
    const int k = (int)(t - (long long)i * (g.nz + 1));
    double acc[3] = {0, 0, 0};
    for (int ex = 0; ex < 2; ++ex)
        for (int ez = 0; ez < 2; ++ez)
            for (int ey = 0; ey < 2; ++ey) {
                const int ei = i - 1 + ex, ej = j - 1 + ey, ek = k - 1 + ez;
                if (ei < 0 || ei >= g.nx || ej < 0 || ej >= g.ny || ek < 0 || ek >= g.nz) continue;
                const int a = local_index(1 - ex, 1 - ey, 1 - ez);
                for (int ix = 0; ix < 2; ++ix)
                    for (int iz = 0; iz < 2; ++iz)
                        for (int iy = 0; iy < 2; ++iy) {
                            const double c = CXf[gf.elem(2 * ei + ix, 2 * ej + iy, 2 * ek + iz)];
                            const int gq = 4 * ix + 2 * iz + iy;
                            for (int d = 0; d < 3; ++d)
                                acc[d] += c * cKq64[gq * 300 + packed_index(3 * a + d, 3 * a + d)];
                        }
            }
    const long long base = L.at(i, j, k);
    for (int d = 0; d < 3; ++d) diag[base + d] = acc[d];
}

void launch_diag_quad(const Lay &L, const double *CXf, double *diag, cudaStream_t st)
{
    const int bs = 128;
    diag_quad_kernel<<<(unsigned)((L.g.nnod() + bs - 1) / bs), bs, 0, st>>>(L, CXf, diag);
    count_launches(1);
}

// ---------------------------------------------------------------------------
// fine-level setup kernels that need Ke
// ---------------------------------------------------------------------------

// diag(K) on the fine level: sum over adjacent elements of CX_e Ke[m][m]
// (mgcg1.cu:1447-1487 prepAD0c).  CX in natural element order.
__global__ void diag_fine_kernel(Lay L, const double *__restrict__ CX, double *__restrict__ diag)
{
    const Grid &g = L.g;
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    const long long t = n / (g.ny + 1);
    const int j = (int)(n - t * (g.ny + 1));
    const int i = (int)(t / (g.nz + 1));
    const int k = (int)(t - (long long)i * (g.nz + 1));
    double acc[3] = {0, 0, 0};
    for (int ex = 0; ex < 2; ++ex)
        for (int ez = 0; ez < 2; ++ez)
            for (int ey = 0; ey < 2; ++ey) {
                const int ei = i - 1 + ex, ej = j - 1 + ey, ek = k - 1 + ez;
                if (ei < 0 || ei >= g.nx || ej < 0 || ej >= g.ny || ek < 0 || ek >= g.nz) continue;
                const double c = CX[g.elem(ei, ej, ek)];
                const int a = local_index(1 - ex, 1 - ey, 1 - ez);
                for (int d = 0; d < 3; ++d) acc[d] += c * cKe64[(3 * a + d) * 25];
            }
    const long long base = L.at(i, j, k);
    for (int d = 0; d < 3; ++d) diag[base + d] = acc[d];
}

void launch_diag_fine(const Lay &L, const double *CX, double *diag, cudaStream_t st)
{
    const int bs = 128;
    diag_fine_kernel<<<(unsigned)((L.g.nnod() + bs - 1) / bs), bs, 0, st>>>(L, CX, diag);
    count_launches(1);
}

// Fine level as packed element matrices (only for a single-level hierarchy).
__global__ void dense_fine_kernel(Grid g, const double *__restrict__ CX, double *__restrict__ A)
{
    const long long nel = g.nel();
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nel) return;
    const double c = CX[e];
    for (int m = 0; m < 24; ++m)
        for (int n = 0; n <= m; ++n) A[(long long)packed_index(m, n) * nel + e] = c * cKe64[m * 24 + n];
}

void launch_dense_fine(const Grid &g, const double *CX, double *Apk, cudaStream_t st)
{
    const int bs = 128;
    dense_fine_kernel<<<(unsigned)((g.nel() + bs - 1) / bs), bs, 0, st>>>(g, CX, Apk);
    count_launches(1);
}

// ---------------------------------------------------------------------------
// tensor-map encoding through the driver entry point (no libcuda link)
// ---------------------------------------------------------------------------

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault,
                                             &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);

unsigned long long current_context_id()
{
    static CtxGetIdFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, []() {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetIdFn>(p);
    });
    if (!fn) return 0;
    // 0 as well before the runtime has made its primary context current on
    // this thread: callers then treat their cache as stale
    unsigned long long id = 0;
    return fn(nullptr, &id) == CUDA_SUCCESS ? id : 0;
}

int make_tmap_3d(CUtensorMap *m, const void *base, int elem_bytes, uint64_t d0, uint64_t d1,
                 uint64_t d2, uint64_t stride1_bytes, uint64_t stride2_bytes, uint32_t b0,
                 uint32_t b1, uint32_t b2)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled is not available from the driver");
        return GPUTO_ERR_CUDA;
    }
    const cuuint64_t dims[3] = {d0, d1, d2};
    const cuuint64_t strides[2] = {stride1_bytes, stride2_bytes};
    const cuuint32_t box[3] = {b0, b1, b2};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt = elem_bytes == 8   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                   : elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                                     : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    CUresult r = fn(m, dt, 3, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
        return GPUTO_ERR_CUDA;
    }
    return GPUTO_OK;
}

}  // namespace gputo
