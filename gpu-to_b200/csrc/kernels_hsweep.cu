// Fine-level operator sweeps with the element matrix in its Hadamard basis.
//
// Same modes and results as tile_kernel (K u, f - K u, damped Jacobi with the
// Dirichlet rows zeroed: mgcg1.cu:941-997,1199-1264,1326-1331), with far
// fewer operations per element; MODE_JACOBI_DOT is the FP32 Jacobi sweep that
// also sums the mixed PCG's r'z and r'z_old (mgcg1.cu:263-265).
//
// The algebra (its helpers are in hadamard.h).  Let H be the 2x2 Hadamard matrix and T = H (x) H (x) H act on
// the eight corners of an element (corner (cx, cy, cz), mode (px, py, pz),
// sign (-1)^(px cx + py cy + pz cz)).  For the trilinear hex8 of an isotropic
// material on a cube, Ke is a sum of Kronecker products of the 1-D mass,
// stiffness and gradient matrices [a b; b a] / [a a; -a -a], which H turns
// into diagonal / single-entry matrices.  So S = T Ke T' (per displacement
// component, 24x24) has only 45 non-zeros in a fixed pattern:
//   three 2x2 blocks a [1 1; 1 1], two 3x3 blocks (b - c) I + c 11', three 2x2
//   blocks [f g; g f], the diagonal h on mode (1,1,1), and zero on mode
//   (0,0,0) (rigid translation).
// Ke u = T' S T u / 64.  T factors into butterflies: two per face (y, z),
// shared by the two elements that meet at the face, and one across the
// element (x).  Per element: 24 + 24 operations forward, 41 in S (with the
// element's CX folded into eight scaled constants), 36 + 24 back, against
// 576 FMAs for the dense 24x24 product.  The host derives the eight
// constants from the caller's Ke and checks the pattern to 1e-12; any other
// Ke runs on the dense kernel.
//
// The tiling.  A thread owns one element column along x (lane = y, warp = z)
// and marches through an x chunk of HTX node planes, one element per step:
//  * node planes arrive by TMA into a ring of HRING shared-memory slots (u,
//    or f and diag for MODE_JACOBI_PRE, plus the CX plane), each slot on its
//    own mbarrier, with bounded waits;
//  * the back face of element i is the front face of element i + 1, so each
//    face is loaded and transformed once and its accumulator carries over;
//  * when a node plane is complete, the four corner partials of each column
//    are summed across columns: over y by a warp shuffle, over z through
//    shared memory (one barrier per plane, which also frees the ring slot);
//  * a cluster of CTAs spans all of y (ny <= 256): the partial of the node
//    column on the seam between two CTAs goes to the right neighbour's
//    shared memory (DSMEM), which finishes those nodes after one cluster
//    barrier at the end of the chunk; in z, tiles overlap by one element
//    column; in x, chunks overlap by one element.
// No atomics: results are deterministic.  Nodes on the far faces need no
// separate kernel.
#include <cooperative_groups.h>

#include <cmath>
#include <mutex>

#include "gputo_internal.h"
#include "hadamard.h"
#include "tma.h"

namespace cg = cooperative_groups;

namespace gputo {

namespace {

constexpr int HY = 32;           // element columns per CTA along y (one per lane)
constexpr int HUW = 100;         // u box width in values: 3 (HY + 1) = 99, rounded to 16 bytes
constexpr int HRING = 4;         // ring slots; loads run HRING - 2 node planes ahead (4 measured
                                 // faster than 5 and than 3 CTAs per SM)
constexpr int HM = 48;           // mask box width in bytes: HY + 1 = 33 nodes, rounded to 16
constexpr int HTX = 32;          // node planes per x chunk
constexpr int HMAXP = HTX + 1;   // planes one chunk may finish (the last chunk also takes plane nx)
constexpr int HMAXCY = 8;        // CTAs per cluster (portable limit): ny <= 256
constexpr int HCZ = 6;           // MODE_JACOBI_PRO: coarse rows of a tile (fine rows kc0 .. kc0 + 8)
constexpr int HCW = 52;          // ... and coarse values per row: 3 (HY / 2 + 1) = 51, rounded to 16 bytes
constexpr uint32_t kHDrainNs = 1000000000u;   // wait for copies in flight before leaving after a failure

__host__ __device__ constexpr size_t al128(size_t x) { return (x + 127) & ~size_t(127); }

// What each mode reads besides u: f (defect, Jacobi, pre-relaxation) and
// 1/diag (Jacobi, pre-relaxation) at the node plane being finished.
template <int MODE> struct HNeeds {
    static constexpr bool PRE = MODE == MODE_JACOBI_PRE;
    static constexpr bool PRO = MODE == MODE_JACOBI_PRO;   // u = u_pre + P e_c formed in the face tiles
    static constexpr bool F = MODE != MODE_APPLY;   // MODE_ENERGY: the residual f - K u
    static constexpr bool D = MODE == MODE_JACOBI || MODE == MODE_JACOBI_PRE || MODE == MODE_JACOBI_DOT || PRO;
    static constexpr bool DOT = MODE == MODE_JACOBI_DOT;   // also the FP64 residual and z_old tiles
};

// Shared memory of one CTA.  Ring slot s holds: the face tile of node plane
// E0 + s (u; f and diag for pre-relaxation), the CX tile of element plane
// E0 + s - 1, and the epilogue tiles of node plane E0 + s - 1 (f, diag, the
// Dirichlet mask; with MODE_JACOBI_DOT also the FP64 residual and z_old),
// which that stage finishes.
template <typename T, int WZ, int MODE>
struct HSmem {
    using N = HNeeds<MODE>;
    // every TMA destination starts on a 128-byte boundary
    static constexpr size_t u_bytes = sizeof(T) * (WZ + 1) * HUW;   // one node plane tile
    static constexpr size_t ua = al128(u_bytes);
    static constexpr size_t c_bytes = sizeof(T) * WZ * HY;          // one CX plane tile
    static constexpr size_t m_bytes = (size_t)WZ * HM;              // one mask plane tile
    static constexpr size_t d_off = ua;                               // face 1/diag (pre-relaxation)
    static constexpr size_t ef_off = d_off + (N::PRE ? ua : 0);       // epilogue f
    static constexpr size_t ed_off = ef_off + (N::F ? ua : 0);        // epilogue 1/diag
    static constexpr size_t r_bytes = sizeof(double) * (WZ + 1) * HUW;   // FP64 residual tile
    static constexpr size_t er_off = ed_off + (N::D ? ua : 0);        // epilogue residual (MODE_JACOBI_DOT)
    static constexpr size_t ez_off = er_off + (N::DOT ? al128(r_bytes) : 0);   // epilogue z_old
    static constexpr size_t c_off = ez_off + (N::DOT ? ua : 0);
    static constexpr size_t m_off = c_off + al128(c_bytes);
    // MODE_JACOBI_PRO: the coarse correction's node plane (E0 + s + 1) / 2 and
    // the Dirichlet bits of face plane E0 + s (WZ + 1 rows)
    static constexpr size_t co_bytes = sizeof(T) * HCZ * HCW;
    static constexpr size_t mf_bytes = (size_t)(WZ + 1) * HM;
    static constexpr size_t co_off = al128(m_off + m_bytes);
    static constexpr size_t mf_off = co_off + (N::PRO ? al128(co_bytes) : 0);
    static constexpr size_t slot = al128(mf_off + (N::PRO ? mf_bytes : 0));
    static constexpr int ZROW = HY + 1;                               // lanes + the seam column
    static constexpr size_t x0_off = HRING * slot;                    // PRO: coarse plane E0 / 2 (odd E0)
    static constexpr size_t z_off = x0_off + (N::PRO ? al128(co_bytes) : 0);
    static constexpr size_t z_bytes = sizeof(T) * 2 * WZ * ZROW * 3;
    static constexpr int SEAM = HMAXP * WZ * 3;
    static constexpr size_t s_off = al128(z_off + z_bytes);
    // seam node partials: own (row sums, z partners), received (the same from
    // the left neighbour), and with MODE_JACOBI_PRO the tile's corrected u
    static constexpr size_t s_bytes = sizeof(T) * (N::PRO ? 5 : 4) * SEAM;
    static constexpr size_t bar_off = al128(s_off + s_bytes);
    static constexpr size_t red_off = bar_off + 8 * HRING;            // per-warp dot partials (two per warp)
    static constexpr size_t bytes = red_off + 16 * WZ;
    static_assert(ua % 128 == 0 && c_off % 128 == 0 && m_off % 128 == 0 && slot % 128 == 0 && er_off % 128 == 0 &&
                      ez_off % 128 == 0 && co_off % 128 == 0 && mf_off % 128 == 0 && x0_off % 128 == 0,
                  "TMA shared-memory destinations must be 128-byte aligned");
};
// Two CTAs of the FP32 Jacobi sweep with the PCG dots share an SM (228 KB,
// 1 KB of it reserved per CTA).
static_assert(2 * (HSmem<float, 8, MODE_JACOBI_DOT>::bytes + 1024) <= 228 * 1024,
              "the FP32 sweep with dots must fit two CTAs per SM");

// One element in the Hadamard basis.  Fp, Fn: transformed front (x = 0) and
// back (x = 1) faces.  Adds the element's front-face output (still in face
// modes) to A and sets An to its back-face output.
template <typename T>
__device__ __forceinline__ void element_h(const T (&Fp)[HF], const T (&Fn)[HF], T cx, const HC<T> &k, T (&A)[HF],
                                          T (&An)[HF])
{
    T v0[HF], v1[HF], w0[HF], w1[HF];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v0[4 * c + d] = Fp[4 * c + d] + Fn[4 * c + d];
            v1[4 * c + d] = Fp[4 * c + d] - Fn[4 * c + d];
        }
    element_s(v0, v1, cx, k, w0, w1);
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            A[4 * c + d] += w0[4 * c + d] + w1[4 * c + d];
            An[4 * c + d] = w0[4 * c + d] - w1[4 * c + d];
        }
}

// element_h that also returns v . w with w = S v / 64 (CX applied after the
// S step), the element's energy u_e' Ke u_e: the FP64 apply with the element
// energies.
__device__ __forceinline__ double element_h_energy(const double (&Fp)[HF], const double (&Fn)[HF], double cx,
                                                   const HC<double> &k, double (&A)[HF], double (&An)[HF])
{
    double v0[HF], v1[HF], w0[HF], w1[HF];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v0[4 * c + d] = Fp[4 * c + d] + Fn[4 * c + d];
            v1[4 * c + d] = Fp[4 * c + d] - Fn[4 * c + d];
        }
    element_s(v0, v1, 1.0, k, w0, w1);
    double en = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int q = 4 * c + d;
            en = fma(v0[q], w0[q], en);
            en = fma(v1[q], w1[q], en);
            A[q] = fma(cx, w0[q] + w1[q], A[q]);
            An[q] = cx * (w0[q] - w1[q]);
        }
    return en;
}

// FP32: the sums and differences of faces and outputs on (x, y) pairs.  All
// FP32 steps are rounding intrinsics (never contracted into an FMA), so the
// one- and two-column kernels give the same results bit for bit.
template <>
__device__ __forceinline__ void element_h<float>(const float (&Fp)[HF], const float (&Fn)[HF], float cx,
                                                 const HC<float> &k, float (&A)[HF], float (&An)[HF])
{
    float v0[HF], v1[HF], w0[HF], w1[HF];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float2 p = f2(Fp, 4 * c), n = f2(Fn, 4 * c);
        f2set(v0, 4 * c, __fadd2_rn(p, n));
        f2set(v1, 4 * c, sub2(p, n));
        v0[4 * c + 2] = __fadd_rn(Fp[4 * c + 2], Fn[4 * c + 2]);
        v1[4 * c + 2] = __fsub_rn(Fp[4 * c + 2], Fn[4 * c + 2]);
    }
    element_s(v0, v1, cx, k, w0, w1);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float2 a = f2(w0, 4 * c), b = f2(w1, 4 * c);
        f2set(A, 4 * c, __fadd2_rn(f2(A, 4 * c), __fadd2_rn(a, b)));
        f2set(An, 4 * c, sub2(a, b));
        A[4 * c + 2] = __fadd_rn(A[4 * c + 2], __fadd_rn(w0[4 * c + 2], w1[4 * c + 2]));
        An[4 * c + 2] = __fsub_rn(w0[4 * c + 2], w1[4 * c + 2]);
    }
}

template <typename T, int MODE>
__device__ __forceinline__ void h_store(long long base, unsigned m, const T (&ku)[3], const T (&u)[3], const T *fv,
                                        const T *rv, T *__restrict__ out, T omega, double &dsum, const double *rdv,
                                        const T *zov, double &dsum2)
{
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const bool fixed = (m >> d) & 1u;
        if (MODE == MODE_APPLY) {
            const T q = fixed ? T(0) : ku[d];
            out[base + d] = q;
            dsum += (double)u[d] * (double)q;
        } else if (MODE == MODE_DEFECT) {
            out[base + d] = fixed ? T(0) : fv[d] - ku[d];
        } else if (MODE == MODE_ENERGY) {
            const T r = fixed ? T(0) : fv[d] - ku[d];
            if (out) out[base + d] = r;
            dsum = fma((double)r, (double)r, dsum);
        } else {
            const T r = fixed ? T(0) : fv[d] - ku[d];
            const T z = hfma(hmul(omega, r), rv[d], u[d]);
            out[base + d] = z;
            if (MODE == MODE_JACOBI_DOT) {   // r'z and r'z_old with the FP64 residual
                const double rd = rdv[d];
                dsum = fma(rd, (double)z, dsum);
                dsum2 = fma(rd, (double)zov[d], dsum2);
            }
        }
    }
}

// Grid: x = rank along y inside the cluster (the cluster spans all of y),
// y = z tile (element columns kc0 .. kc0 + WZ - 1, kc0 = (WZ - 1) tile),
// z = x chunk (node planes [c htx, (c + 1) htx), the last one up to nx;
// htx <= HTX).  The Dirichlet bits come by TMA from a copy with rows padded
// to 16 bytes (tm_m); rdiag = 1/diag.
// CTAs per SM the compiler budgets registers for: 2, and 3 for the FP64
// energy apply (128 registers: 135.6 us against 153.7 us at 2; the FP64 apply
// measured no faster at 3 or 4).
template <typename T, int MODE> struct HMinBlocks {
    static constexpr int value = (sizeof(T) == 8 && MODE == MODE_ENERGY) ? 3 : 2;
};

template <typename T, int MODE, int WZ>
__global__ void __launch_bounds__(32 * WZ, HMinBlocks<T, MODE>::value)
hsweep_kernel(const __grid_constant__ CUtensorMap tm_u, const __grid_constant__ CUtensorMap tm_d,
              const __grid_constant__ CUtensorMap tm_f, const __grid_constant__ CUtensorMap tm_c,
              const __grid_constant__ CUtensorMap tm_m, const __grid_constant__ CUtensorMap tm_r,
              const __grid_constant__ CUtensorMap tm_z, Lay L, HC<T> hc, int htx, const T *__restrict__ f,
              const T *__restrict__ rdiag, const uint8_t *__restrict__ mask, T *__restrict__ out, T omega,
              T prerelax, double *__restrict__ dot_partial, const int *__restrict__ done, int *__restrict__ err,
              const double *__restrict__ Rd, const T *__restrict__ zo, uint32_t wait_ns, int skip_stage,
              double *__restrict__ ce, double *__restrict__ dcv, const double *__restrict__ dsK,
              const T *__restrict__ ucoarse, Lay Lc, const T *__restrict__ ug)
{
    if (done && *done) return;   // the same value for every CTA of the cluster
    using N = HNeeds<MODE>;
    constexpr int NT = 32 * WZ;
    using S = HSmem<T, WZ, MODE>;
    extern __shared__ __align__(128) unsigned char smem[];
    if (smem_u32(smem) & 127u) {   // TMA destinations need 128-byte alignment (same for every CTA)
        if (threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && err)
            atomicExch(err, GPUTO_ERR_CUDA);
        return;
    }
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + S::bar_off);
    T *zb = reinterpret_cast<T *>(smem + S::z_off);
    T *s_own = reinterpret_cast<T *>(smem + S::s_off);
    T *s_ownz = s_own + S::SEAM;
    T *s_recv = s_own + 2 * S::SEAM;
    T *s_recvz = s_own + 3 * S::SEAM;
    T *s_ownu = s_own + 4 * S::SEAM;   // MODE_JACOBI_PRO only

    cg::cluster_group cluster = cg::this_cluster();
    const Grid &g = L.g;
    const int tid = threadIdx.x, l = tid & 31, w = tid >> 5;
    const int r = blockIdx.x, CY = gridDim.x;
    const int jc0 = HY * r;
    const int zt = blockIdx.y, kc0 = (WZ - 1) * zt;
    const int P0 = blockIdx.z * htx;
    const int P1 = (blockIdx.z == gridDim.z - 1) ? g.nx + 1 : P0 + htx;
    const int E0 = P0 > 0 ? P0 - 1 : 0, E1 = P1 < g.nx ? P1 : g.nx;
    const int nE = E1 - E0;                          // elements of the chunk (>= 1)
    const bool last_plane = E1 == g.nx && E1 < P1;   // plane nx: only element nx - 1 touches it
    const int nst = nE + 1 + (last_plane ? 1 : 0);   // ring stages
    const bool tail_owner = (r == CY - 1) && (jc0 + HY == g.ny);
    const bool zok = (w >= 1 || zt == 0) && kc0 + w <= g.nz;   // this warp's node row is output here

    if (tid == 0) {
        for (int s = 0; s < HRING; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int issued = 0;   // meaningful on thread 0
    auto issue = [&](int s) {
        unsigned char *sb = smem + (s % HRING) * S::slot;
        uint64_t *b = &bar[s % HRING];
        const bool face = s <= nE, cxp = s >= 1 && s <= nE, epi = s >= 1 && E0 + s - 1 >= P0;
        uint32_t bytes = 0;
        if (face) bytes += (uint32_t)(S::u_bytes * (N::PRE ? 2 : 1));
        if (face && N::PRO)
            bytes += (uint32_t)(S::co_bytes * ((s == 0 && (E0 & 1)) ? 2 : 1) + S::mf_bytes);
        if (cxp) bytes += (uint32_t)S::c_bytes;
        if (epi) bytes += (uint32_t)(S::u_bytes * ((N::F ? 1 : 0) + (N::D ? 1 : 0) + (N::DOT ? 1 : 0)) + S::m_bytes +
                                     (N::DOT ? S::r_bytes : 0));
        mbar_arrive_expect_tx(b, bytes);
        if (s == skip_stage) {   // test hook: the stage stays armed with no copy in flight
            issued = s + 1;
            return;
        }
        if (face) {
            tma_load_3d(sb, &tm_u, 3 * jc0, kc0, E0 + s, b);
            if (N::PRE) tma_load_3d(sb + S::d_off, &tm_d, 3 * jc0, kc0, E0 + s, b);
            if (N::PRO) {   // tm_r: the coarse correction, tm_z: the Dirichlet bits, WZ + 1 rows
                tma_load_3d(sb + S::co_off, &tm_r, 3 * (jc0 >> 1), kc0 >> 1, (E0 + s + 1) >> 1, b);
                tma_load_3d(sb + S::mf_off, &tm_z, jc0, kc0, E0 + s, b);
                if (s == 0 && (E0 & 1)) tma_load_3d(smem + S::x0_off, &tm_r, 3 * (jc0 >> 1), kc0 >> 1, E0 >> 1, b);
            }
        }
        if (cxp) tma_load_3d(sb + S::c_off, &tm_c, jc0, kc0, E0 + s - 1, b);
        if (epi) {
            if (N::F) tma_load_3d(sb + S::ef_off, &tm_f, 3 * jc0, kc0, E0 + s - 1, b);
            if (N::D) tma_load_3d(sb + S::ed_off, &tm_d, 3 * jc0, kc0, E0 + s - 1, b);
            if (N::DOT) {
                tma_load_3d(sb + S::er_off, &tm_r, 3 * jc0, kc0, E0 + s - 1, b);
                tma_load_3d(sb + S::ez_off, &tm_z, 3 * jc0, kc0, E0 + s - 1, b);
            }
            tma_load_3d(sb + S::m_off, &tm_m, jc0, kc0, E0 + s - 1, b);
        }
        issued = s + 1;
    };
    if (tid == 0)
        for (int s = 0; s < HRING && s < nst; ++s) issue(s);
    cluster.sync();   // every CTA of the cluster is running before any remote store

    bool bad = false;
    auto wait_stage = [&](int s) {
        if (!bad && !mbar_wait_for(&bar[s % HRING], (uint32_t)((s / HRING) & 1), wait_ns)) bad = true;
    };
    auto load_face = [&](int s, T (&U)[HF]) {
        const unsigned char *sb = smem + (s % HRING) * S::slot;
        const T *su = reinterpret_cast<const T *>(sb);
        const T *sd = reinterpret_cast<const T *>(sb + S::d_off);
#pragma unroll
        for (int cy = 0; cy < 2; ++cy)
#pragma unroll
            for (int cz = 0; cz < 2; ++cz)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const int idx = (w + cz) * HUW + 3 * (l + cy) + d;
                    T v = su[idx];
                    if (N::PRE) v = hmul(hmul(prerelax, v), sd[idx]);   // 1/diag is 0 outside the grid
                    U[(cy * 2 + cz) * 4 + d] = v;
                }
    };
    // MODE_JACOBI_PRO: add the prolonged coarse correction to the u tile of
    // ring stage s (node plane p = E0 + s) in place, from the coarse tiles
    // that came by TMA with the stage (plane p / 2 in slot s, for odd p plane
    // (p - 1) / 2 in slot s - 1 or, at s = 0, the extra tile), with the same
    // taps in the same order as prolong_cell_kernel, the fixed dofs zeroed from the
    // stage's own Dirichlet tile.  Tile t + 1 is corrected during step t,
    // before the barrier that ends it, so no barrier of its own is needed
    // (tile 0 before the first one).
    auto prolong_tile = [&](int s) {
        unsigned char *sb = smem + (s % HRING) * S::slot;
        T *su = reinterpret_cast<T *>(sb);
        const int p = E0 + s, ni = (p & 1) + 1;
        const T *tb = reinterpret_cast<const T *>(sb + S::co_off);   // plane (p + 1) / 2
        const T *ta = (p & 1) ? reinterpret_cast<const T *>(s == 0 ? smem + S::x0_off
                                                                   : smem + ((s - 1) % HRING) * S::slot + S::co_off)
                              : tb;                                     // plane p / 2
        const uint8_t *mf = sb + S::mf_off;
        const int K0 = kc0 >> 1, J0 = jc0 >> 1;
        for (int idx = tid; idx < (WZ + 1) * (HY + 1); idx += NT) {
            const int zz = idx / (HY + 1), jj = idx - zz * (HY + 1);
            const int j = jc0 + jj, k = kc0 + zz;
            if (j > g.ny || k > g.nz) continue;
            const int nj = (j & 1) + 1, nk = (k & 1) + 1;
            T acc[3] = {T(0), T(0), T(0)};
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const T *cr = (a && a < ni ? tb : ta) + ((k >> 1) - K0 + ((c && c < nk) ? 1 : 0)) * HCW +
                                  3 * ((j >> 1) - J0);
#pragma unroll
                    for (int b = 0; b < 2; ++b) {
                        const bool ok = a < ni && c < nk && b < nj;
                        const int off = (b < nj) ? 3 * b : 0;
#pragma unroll
                        for (int d = 0; d < 3; ++d) acc[d] += ok ? cr[off + d] : T(0);
                    }
                }
            const T wgt = T(1) / T(ni * nj * nk);
            const unsigned m = mf[zz * HM + jj];
            T *v = su + zz * HUW + 3 * jj;
#pragma unroll
            for (int d = 0; d < 3; ++d) v[d] = ((m >> d) & 1u) ? T(0) : fma(wgt, acc[d], v[d]);
        }
    };
    double dsum = 0.0, dsum2 = 0.0;
    // Corner partials P of node plane p -> y sums through the warp, z partner
    // values into the exchange buffer (read after the next barrier).
    auto reduce_y = [&](int p, T (&P)[HF], T (&q0)[3]) {
        T *z = zb + (p & 1) * (WZ * S::ZROW * 3);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T a0 = __shfl_up_sync(0xffffffffu, P[8 + d], 1);
            const T a1 = __shfl_up_sync(0xffffffffu, P[12 + d], 1);
            q0[d] = P[d] + (l > 0 ? a0 : T(0));
            z[(w * S::ZROW + l) * 3 + d] = P[4 + d] + (l > 0 ? a1 : T(0));
            if (l == HY - 1) z[(w * S::ZROW + HY) * 3 + d] = P[12 + d];
        }
    };
    // Finish node plane p with the epilogue tiles of ring stage s.
    auto emit = [&](int p, int s, const T (&P)[HF], const T (&q0)[3], const T (&Uu)[HF]) {
        if (!zok) return;
        const unsigned char *sb = smem + (s % HRING) * S::slot;
        const T *ef = reinterpret_cast<const T *>(sb + S::ef_off) + w * HUW;
        const T *ed = reinterpret_cast<const T *>(sb + S::ed_off) + w * HUW;
        const double *er = reinterpret_cast<const double *>(sb + S::er_off) + w * HUW;   // MODE_JACOBI_DOT only
        const T *ez = reinterpret_cast<const T *>(sb + S::ez_off) + w * HUW;
        const uint8_t *em = sb + S::m_off + w * HM;
        const T *z = zb + (p & 1) * (WZ * S::ZROW * 3);
        const int k = kc0 + w, j = jc0 + l, at = ((p - P0) * WZ + w) * 3;
        T R[3], Z[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            Z[d] = w > 0 ? z[((w - 1) * S::ZROW + l) * 3 + d] : T(0);
            R[d] = q0[d] + Z[d];
        }
        if (l == 0 && r > 0) {   // seam node: finished after the cluster barrier
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                s_own[at + d] = q0[d];
                s_ownz[at + d] = Z[d];
                if (N::PRO) s_ownu[at + d] = Uu[d];
            }
        } else if (j <= g.ny) {
            const T uu[3] = {Uu[0], Uu[1], Uu[2]};
            h_store<T, MODE>(L.at(p, j, k), em[l], R, uu, ef + 3 * l, ed + 3 * l, out, omega, dsum, er + 3 * l,
                             ez + 3 * l, dsum2);
        }
        if (l == HY - 1) {   // this CTA's part of node column jc0 + HY
            T Sq[3], Sz[3], Sd[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                Sq[d] = P[8 + d];
                Sz[d] = w > 0 ? z[((w - 1) * S::ZROW + HY) * 3 + d] : T(0);
                Sd[d] = Sq[d] + Sz[d];
            }
            if (r + 1 < CY) {
                T *rem = cluster.map_shared_rank(s_recv, r + 1);
                T *remz = cluster.map_shared_rank(s_recvz, r + 1);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    rem[at + d] = Sq[d];
                    remz[at + d] = Sz[d];
                }
            } else if (tail_owner) {
                const T uu[3] = {Uu[8], Uu[9], Uu[10]};
                h_store<T, MODE>(L.at(p, g.ny, k), em[HY], Sd, uu, ef + 3 * HY, ed + 3 * HY, out, omega, dsum,
                                 er + 3 * HY, ez + 3 * HY, dsum2);
            }
        }
    };

    // One march step: element E0 + t - 1 between faces (Uc, Fc) and the next
    // face (Un, Fn); Ac collects node plane E0 + t - 1, An starts plane E0 + t.
    // The loop runs two steps per trip with the roles swapped, so no arrays
    // are copied.
    int cur = 0;   // the stage being consumed
    bool fail = false;
    auto step = [&](int t, T (&Uc)[HF], T (&Fc)[HF], T (&Ac)[HF], T (&Un)[HF], T (&Fn)[HF], T (&An)[HF]) {
        cur = t;
        wait_stage(t);
        load_face(t, Un);   // MODE_JACOBI_PRO: tile t got its correction in step t - 1
#pragma unroll
        for (int q = 0; q < HF; ++q)
            if ((q & 3) != 3) Fn[q] = Un[q];
        face_h(Fn);
        const T cx = reinterpret_cast<const T *>(smem + (t % HRING) * S::slot + S::c_off)[w * HY + l];
        if constexpr (MODE == MODE_ENERGY) {
            const double en = element_h_energy(Fc, Fn, cx, hc, Ac, An);
            // element (E0 + t - 1, jc0 + l, kc0 + w): written by the one CTA that
            // owns it (x chunks overlap by one element, z tiles by one row)
            const int ei = E0 + t - 1, ej = jc0 + l, ek = kc0 + w;
            if (ei >= P0 && (w < WZ - 1 || zt == (int)gridDim.y - 1) && ek < g.nz && ej < g.ny) {
                const long long e = g.elem(ei, ej, ek);
                ce[e] = en;
                if (dcv) dcv[e] = dsK[e] * en;
                dsum2 = fma((double)cx, en, dsum2);
            }
        } else {
            element_h(Fc, Fn, cx, hc, Ac, An);
        }
        const int p = E0 + t - 1;   // node plane finished by this element
        const bool out_plane = p >= P0;
        T q0[3];
        if (out_plane) {
            face_h(Ac);   // node partials of plane p
            reduce_y(p, Ac, q0);
        }
        if constexpr (N::PRO) {   // the next face tile, before the barrier that publishes it
            if (t + 1 <= nE) {
                wait_stage(t + 1);
                if (!bad) prolong_tile(t + 1);
            }
        }
        fail = __syncthreads_or(bad);   // z partners visible; ring slot t - 1 free
        if (!fail && tid == 0 && t - 1 + HRING < nst) issue(t - 1 + HRING);
        if (!fail && out_plane) emit(p, t, Ac, q0, Uc);
    };
    auto finish_last = [&](T (&Uc)[HF], T (&Ac)[HF]) {   // plane nx: only element nx - 1 touches it
        cur = nE + 1;
        wait_stage(nE + 1);
        T q0[3];
        face_h(Ac);
        reduce_y(E1, Ac, q0);
        fail = __syncthreads_or(bad);
        if (!fail) emit(E1, nE + 1, Ac, q0, Uc);
    };

    T U0[HF], F0[HF], A0[HF], U1[HF], F1[HF], A1[HF];
    wait_stage(0);
    if constexpr (N::PRO) {
        if (!bad) prolong_tile(0);
        __syncthreads();
    }
    load_face(0, U0);
#pragma unroll
    for (int q = 0; q < HF; ++q) {
        F0[q] = (q & 3) != 3 ? U0[q] : T(0);
        A0[q] = T(0);
    }
    face_h(F0);
    if constexpr (N::PRO) {
        if (1 <= nE) {
            wait_stage(1);
            if (!bad) prolong_tile(1);
        }
    }
    fail = __syncthreads_or(bad);
    if constexpr (sizeof(T) == 8) {   // FP64: one step per trip, the state copied back
        for (int t = 1; !fail && t <= nE; ++t) {
            step(t, U0, F0, A0, U1, F1, A1);
#pragma unroll
            for (int q = 0; q < HF; ++q)
                if ((q & 3) != 3) {
                    U0[q] = U1[q];
                    F0[q] = F1[q];
                    A0[q] = A1[q];
                }
        }
        if (!fail && last_plane) finish_last(U0, A0);
    } else {
        int t = 1;
        for (; !fail && t + 1 <= nE; t += 2) {
            step(t, U0, F0, A0, U1, F1, A1);
            if (!fail) step(t + 1, U1, F1, A1, U0, F0, A0);
        }
        if (!fail && t <= nE) {   // odd count: one more step, the state ends in set 1
            step(t, U0, F0, A0, U1, F1, A1);
            if (!fail && last_plane) finish_last(U1, A1);
        } else if (!fail && last_plane) {
            finish_last(U0, A0);
        }
    }
    if (fail && tid == 0) {
        // let the loads still in flight (stages cur .. issued - 1, each the
        // latest phase of its slot) land before the CTA ends (bounded); a
        // stage the test hook left unissued has nothing in flight
        for (int s = cur; s < issued; ++s)
            if (s != skip_stage) (void)mbar_wait_for(&bar[s % HRING], (uint32_t)((s / HRING) & 1), kHDrainNs);
        if (err) atomicExch(err, GPUTO_ERR_TIMEOUT);
    }
    cluster.sync();   // seam partials from the left neighbour have arrived
    if (!fail && r > 0) {   // node column jc0, from both sides of the seam
        const int np = P1 - P0;
        for (int idx = tid; idx < np * WZ; idx += NT) {
            const int pp = idx / WZ, ww = idx - pp * WZ;
            const int k = kc0 + ww, p = P0 + pp, at = idx * 3;
            if (!((ww >= 1 || zt == 0) && k <= g.nz)) continue;
            // the interior nodes' order: (row sums) + (z partners), each own + left
            const long long base = L.at(p, jc0, k);
            T v[3], uu[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                v[d] = (s_own[at + d] + s_recv[at + d]) + (s_ownz[at + d] + s_recvz[at + d]);
                if (N::PRO)
                    uu[d] = s_ownu[at + d];
                else if (N::PRE)
                    uu[d] = hmul(hmul(prerelax, f[base + d]), rdiag[base + d]);
                else
                    uu[d] = (MODE == MODE_APPLY || N::D) ? ug[base + d] : T(0);
            }
            h_store<T, MODE>(base, mask[g.node(p, jc0, k)], v, uu, f + base, rdiag + base, out, omega, dsum,
                             Rd + base, zo + base, dsum2);
        }
    }
    if ((MODE == MODE_APPLY || MODE == MODE_JACOBI_DOT || MODE == MODE_ENERGY) && dot_partial) {
        constexpr bool PAIR = MODE == MODE_JACOBI_DOT || MODE == MODE_ENERGY;
        double *red = reinterpret_cast<double *>(smem + S::red_off);
        for (int o = 16; o > 0; o >>= 1) {
            dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
            if (PAIR) dsum2 += __shfl_xor_sync(0xffffffffu, dsum2, o);
        }
        if (l == 0) {
            red[w] = dsum;
            red[WZ + w] = dsum2;
        }
        __syncthreads();
        if (tid == 0) {
            double v = 0.0, v2 = 0.0;
            for (int q = 0; q < WZ; ++q) {
                v += red[q];
                v2 += red[WZ + q];
            }
            const long long cta = blockIdx.x + gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
            if (MODE == MODE_APPLY) {
                dot_partial[cta] = v;
            } else {
                dot_partial[2 * cta] = v;
                dot_partial[2 * cta + 1] = v2;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// FP32 sweeps with two element columns per lane (hsweep2_kernel).
//
// The same sweeps as hsweep_kernel with the same results bit for bit (the
// dot partials aside, which group their FP64 sums differently), but each lane
// owns elements j = jc0 + 2l and 2l + 1, so a CTA covers 64 element columns
// along y.  The two elements run one instruction stream: every arithmetic
// step of the Hadamard form is a paired FP32 instruction on a float2 (element
// 2l in .x, 2l + 1 in .y), the node column between the two is summed inside
// the lane, and the per-step costs (the ring wait, the barrier, the shuffles,
// the index arithmetic, the seam branches) are shared by two elements.  The
// node pairs of the epilogue move as 8-byte words (f, 1/diag, the z
// partners, the output).  About 40 % fewer instructions per element than
// hsweep_kernel.  Twice the state per thread (165-200 registers): CTAs of
// four warps, two or three per SM.  The per-step CTA barrier holds all of a
// CTA's warps in the same phase (element arithmetic, then shuffles and shared
// memory, then stores); the other CTAs on the SM issue during one CTA's
// barrier, latency and ring-filling phases.  (Eight warps per CTA, with the
// barrier or with the warps synchronised point to point by mbarriers, and
// loading the next face before the barrier, all measured slower.)
constexpr int HY2 = 64;     // element columns per CTA along y (two per lane)
constexpr int HUW2 = 196;   // u box width: 3 (HY2 + 1) = 195 values, rounded to 16 bytes
constexpr int HM2 = 80;     // mask box width in bytes: HY2 + 1 = 65 nodes, rounded to 16
constexpr int ZROW2 = 66;   // z exchange row: 65 node columns, even so node pairs are 8-byte aligned
constexpr int HWZ2 = 4;     // warps (element rows along z) per CTA (measured 79 us against 84 us for one
                            // CTA of eight warps per SM, despite the extra overlapping row in four)

template <int MODE>
struct HSmem2 {
    using N = HNeeds<MODE>;
    static constexpr int WZ = HWZ2;
    static constexpr size_t u_bytes = sizeof(float) * (WZ + 1) * HUW2;   // one node plane tile
    static constexpr size_t ua = al128(u_bytes);
    static constexpr size_t c_bytes = sizeof(float) * WZ * HY2;          // one CX plane tile
    static constexpr size_t m_bytes = (size_t)WZ * HM2;                  // one mask plane tile
    static constexpr size_t r_bytes = sizeof(double) * (WZ + 1) * HUW2;   // FP64 residual tile
    static constexpr size_t d_off = ua;
    static constexpr size_t ef_off = d_off + (N::PRE ? ua : 0);
    static constexpr size_t ed_off = ef_off + (N::F ? ua : 0);
    static constexpr size_t er_off = ed_off + (N::D ? ua : 0);
    static constexpr size_t ez_off = er_off + (N::DOT ? al128(r_bytes) : 0);
    static constexpr size_t c_off = ez_off + (N::DOT ? ua : 0);
    static constexpr size_t m_off = c_off + al128(c_bytes);
    static constexpr size_t slot = al128(m_off + m_bytes);
    static constexpr size_t z_off = HRING * slot;
    static constexpr size_t z_bytes = sizeof(float) * 2 * WZ * ZROW2 * 3;
    static constexpr int SEAM = HMAXP * WZ * 3;
    static constexpr size_t s_off = al128(z_off + z_bytes);
    static constexpr size_t s_bytes = sizeof(float) * 4 * SEAM;   // own and received row sums and z partners
    static constexpr size_t bar_off = al128(s_off + s_bytes);
    static constexpr size_t red_off = bar_off + 8 * HRING;
    static constexpr size_t bytes = red_off + 16 * WZ;
    static_assert(ua % 128 == 0 && c_off % 128 == 0 && m_off % 128 == 0 && slot % 128 == 0 && er_off % 128 == 0 &&
                      ez_off % 128 == 0 && z_off % 128 == 0,
                  "TMA shared-memory destinations must be 128-byte aligned");
};
static_assert(2 * (HSmem2<MODE_JACOBI_DOT>::bytes + 1024) <= 228 * 1024,
              "two CTAs of the paired FP32 sweep with dots must share an SM");

// Node columns 2l, 2l + 1, 2l + 2 of rows w, w + 1 (raw[cz][n][d]) -> the
// face modes of elements 2l and 2l + 1, F[4 c + d] with mode c = 2 py + pz:
// the y butterflies in scalar form (each node column 2l + 1 serves both
// elements), the z butterflies paired.
__device__ __forceinline__ void face_h2(const float (&raw)[2][3][3], float2 (&F)[HF])
{
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float2 s[2], df[2];
#pragma unroll
        for (int cz = 0; cz < 2; ++cz) {
            const float a = raw[cz][0][d], b = raw[cz][1][d], c = raw[cz][2][d];
            s[cz] = make_float2(__fadd_rn(a, b), __fadd_rn(b, c));
            df[cz] = make_float2(__fsub_rn(a, b), __fsub_rn(b, c));
        }
        F[d] = s[0] + s[1];
        F[4 + d] = s[0] - s[1];
        F[8 + d] = df[0] + df[1];
        F[12 + d] = df[0] - df[1];
    }
}

// element_h on a pair of elements.
__device__ __forceinline__ void element_h2(const float2 (&Fp)[HF], const float2 (&Fn)[HF], float2 cx,
                                           const HC<float2> &k, float2 (&A)[HF], float2 (&An)[HF])
{
    float2 v0[HF], v1[HF], w0[HF], w1[HF];
#pragma unroll
    for (int q = 0; q < HF; ++q)
        if ((q & 3) != 3) {
            v0[q] = Fp[q] + Fn[q];
            v1[q] = Fp[q] - Fn[q];
        }
    element_s(v0, v1, cx, k, w0, w1);
#pragma unroll
    for (int q = 0; q < HF; ++q)
        if ((q & 3) != 3) {
            A[q] = A[q] + (w0[q] + w1[q]);
            An[q] = w0[q] - w1[q];
        }
}

__device__ __forceinline__ void lds6(const float *p, float (&v)[6])
{
    const float2 *q = reinterpret_cast<const float2 *>(p);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float2 x = q[i];
        v[2 * i] = x.x;
        v[2 * i + 1] = x.y;
    }
}

// The epilogue operands of a lane's node pair (f, 1/diag, the Dirichlet
// bits; with the dots also the FP64 residual and z_old), read from the ring
// slot before the step's barrier so that their latency overlaps it.
struct Epi2 {
    float fv[6], rv[6], zv[6];
    double rd[6];
    unsigned mm;
};

template <int MODE>
__device__ __forceinline__ void load_epi2(const unsigned char *sb, int w, int l, Epi2 &e)
{
    using N = HNeeds<MODE>;
    using S = HSmem2<MODE>;
    const int o = w * HUW2 + 6 * l;
    if (N::F) lds6(reinterpret_cast<const float *>(sb + S::ef_off) + o, e.fv);
    if (N::D) lds6(reinterpret_cast<const float *>(sb + S::ed_off) + o, e.rv);
    if (N::DOT) {
        lds6(reinterpret_cast<const float *>(sb + S::ez_off) + o, e.zv);
        const double2 *q = reinterpret_cast<const double2 *>(reinterpret_cast<const double *>(sb + S::er_off) + o);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double2 x = q[i];
            e.rd[2 * i] = x.x;
            e.rd[2 * i + 1] = x.y;
        }
    }
    e.mm = *reinterpret_cast<const uint16_t *>(sb + S::m_off + w * HM2 + 2 * l);
}

// Finish node columns j0 = jc0 + 2l and j0 + 1 of one row (h_store on a node
// pair): 'base' is the dof of node j0, in1 whether node j0 + 1 is in the grid
// (node j0 is), count0 whether node j0 enters the dot sums (not on a CTA
// seam, where it is written here with this CTA's partial and rewritten after
// the cluster barrier).  u comes from the face registers.
template <int MODE>
__device__ __forceinline__ void h_store2(long long base, bool in1, bool count0, const Epi2 &e, const float (&R)[6],
                                         const float (&u)[9], float *__restrict__ out, float omega, double &dsum,
                                         double &dsum2)
{
    float o[6];
    const unsigned mm = e.mm;
    const float(&fv)[6] = e.fv;
    const float(&rv)[6] = e.rv;
    const float(&zv)[6] = e.zv;
    const double(&rd)[6] = e.rd;
#pragma unroll
    for (int n = 0; n < 2; ++n) {
        const bool counted = n ? in1 : count0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int i = 3 * n + d;
            const bool fixed = (mm >> (8 * n + d)) & 1u;
            if (MODE == MODE_APPLY) {
                const float q = fixed ? 0.f : R[i];
                o[i] = q;
                if (counted) dsum += (double)u[i] * (double)q;
            } else if (MODE == MODE_DEFECT) {
                o[i] = fixed ? 0.f : fv[i] - R[i];
            } else {
                const float r = fixed ? 0.f : fv[i] - R[i];
                const float z = hfma(hmul(omega, r), rv[i], u[i]);
                o[i] = z;
                if (MODE == MODE_JACOBI_DOT && counted) {
                    dsum = fma(rd[i], (double)z, dsum);
                    dsum2 = fma(rd[i], (double)zv[i], dsum2);
                }
            }
        }
    }
    if (in1) {
        float2 *o2 = reinterpret_cast<float2 *>(out + base);
#pragma unroll
        for (int i = 0; i < 3; ++i) o2[i] = make_float2(o[2 * i], o[2 * i + 1]);
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) out[base + d] = o[d];
    }
}

// CTAs per SM the compiler budgets registers for: three where three fit in
// shared memory (168 registers, no spills; the Jacobi sweep measured 73.7
// against 78.2 us at two), else two.
template <int MODE> struct HMinBlocks2 {
    static constexpr int value = (MODE == MODE_APPLY || MODE == MODE_DEFECT || MODE == MODE_JACOBI) ? 3 : 2;
};
static_assert(3 * (HSmem2<MODE_JACOBI>::bytes + 1024) <= 228 * 1024, "three Jacobi CTAs must share an SM");

template <int MODE>
__global__ void __launch_bounds__(32 * HWZ2, HMinBlocks2<MODE>::value)
hsweep2_kernel(const __grid_constant__ CUtensorMap tm_u, const __grid_constant__ CUtensorMap tm_d,
               const __grid_constant__ CUtensorMap tm_f, const __grid_constant__ CUtensorMap tm_c,
               const __grid_constant__ CUtensorMap tm_m, const __grid_constant__ CUtensorMap tm_r,
               const __grid_constant__ CUtensorMap tm_z, Lay L, HC<float2> hc, int htx, const float *__restrict__ f,
               const float *__restrict__ rdiag, const uint8_t *__restrict__ mask, float *__restrict__ out,
               float omega, float prerelax, double *__restrict__ dot_partial, const int *__restrict__ done,
               int *__restrict__ err, const double *__restrict__ Rd, const float *__restrict__ zo, uint32_t wait_ns,
               int skip_stage, const float *__restrict__ ug)
{
    static_assert(MODE != MODE_ENERGY && MODE != MODE_JACOBI_PRO, "FP64 energy and the fused prolongation use hsweep_kernel");
    if (done && *done) return;   // the same value for every CTA of the cluster
    using N = HNeeds<MODE>;
    constexpr int WZ = HWZ2, NT = 32 * WZ;
    using S = HSmem2<MODE>;
    extern __shared__ __align__(128) unsigned char smem[];
    if (smem_u32(smem) & 127u) {
        if (threadIdx.x == 0 && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && err)
            atomicExch(err, GPUTO_ERR_CUDA);
        return;
    }
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + S::bar_off);
    float *zb = reinterpret_cast<float *>(smem + S::z_off);
    float *s_own = reinterpret_cast<float *>(smem + S::s_off);
    float *s_ownz = s_own + S::SEAM;
    float *s_recv = s_own + 2 * S::SEAM;
    float *s_recvz = s_own + 3 * S::SEAM;

    cg::cluster_group cluster = cg::this_cluster();
    const Grid &g = L.g;
    const int tid = threadIdx.x, l = tid & 31, w = tid >> 5;
    const int r = blockIdx.x, CY = gridDim.x;
    const int jc0 = HY2 * r;
    const int zt = blockIdx.y, kc0 = (WZ - 1) * zt;
    const int P0 = blockIdx.z * htx;
    const int P1 = (blockIdx.z == gridDim.z - 1) ? g.nx + 1 : P0 + htx;
    const int E0 = P0 > 0 ? P0 - 1 : 0, E1 = P1 < g.nx ? P1 : g.nx;
    const int nE = E1 - E0;
    const bool last_plane = E1 == g.nx && E1 < P1;
    const int nst = nE + 1 + (last_plane ? 1 : 0);
    const bool tail_owner = (r == CY - 1) && (jc0 + HY2 == g.ny);
    const bool zok = (w >= 1 || zt == 0) && kc0 + w <= g.nz;
    const int j0 = jc0 + 2 * l;
    const bool in0 = j0 <= g.ny, in1 = j0 + 1 <= g.ny, seam = l == 0 && r > 0;

    if (tid == 0) {
        for (int s = 0; s < HRING; ++s) mbar_init(&bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    int issued = 0;
    auto issue = [&](int s) {
        unsigned char *sb = smem + (s % HRING) * S::slot;
        uint64_t *b = &bar[s % HRING];
        const bool face = s <= nE, cxp = s >= 1 && s <= nE, epi = s >= 1 && E0 + s - 1 >= P0;
        uint32_t bytes = 0;
        if (face) bytes += (uint32_t)(S::u_bytes * (N::PRE ? 2 : 1));
        if (cxp) bytes += (uint32_t)S::c_bytes;
        if (epi) bytes += (uint32_t)(S::u_bytes * ((N::F ? 1 : 0) + (N::D ? 1 : 0) + (N::DOT ? 1 : 0)) + S::m_bytes +
                                     (N::DOT ? S::r_bytes : 0));
        mbar_arrive_expect_tx(b, bytes);
        if (s == skip_stage) {   // test hook: the stage stays armed with no copy in flight
            issued = s + 1;
            return;
        }
        if (face) {
            tma_load_3d(sb, &tm_u, 3 * jc0, kc0, E0 + s, b);
            if (N::PRE) tma_load_3d(sb + S::d_off, &tm_d, 3 * jc0, kc0, E0 + s, b);
        }
        if (cxp) tma_load_3d(sb + S::c_off, &tm_c, jc0, kc0, E0 + s - 1, b);
        if (epi) {
            if (N::F) tma_load_3d(sb + S::ef_off, &tm_f, 3 * jc0, kc0, E0 + s - 1, b);
            if (N::D) tma_load_3d(sb + S::ed_off, &tm_d, 3 * jc0, kc0, E0 + s - 1, b);
            if (N::DOT) {
                tma_load_3d(sb + S::er_off, &tm_r, 3 * jc0, kc0, E0 + s - 1, b);
                tma_load_3d(sb + S::ez_off, &tm_z, 3 * jc0, kc0, E0 + s - 1, b);
            }
            tma_load_3d(sb + S::m_off, &tm_m, jc0, kc0, E0 + s - 1, b);
        }
        issued = s + 1;
    };
    if (tid == 0)
        for (int s = 0; s < HRING && s < nst; ++s) issue(s);
    cluster.sync();   // every CTA of the cluster is running before any remote store

    bool bad = false;
    auto wait_stage = [&](int s) {
        if (!bad && !mbar_wait_for(&bar[s % HRING], (uint32_t)((s / HRING) & 1), wait_ns)) bad = true;
    };
    // Face of ring stage s: raw node values (u, or the pre-relaxed f / diag)
    // and the element pair's CX, read a step ahead (before the barrier of the
    // step that precedes their use).
    auto load_face = [&](int s, float (&raw)[2][3][3], float2 &cx) {
        const unsigned char *sb = smem + (s % HRING) * S::slot;
        const float *su = reinterpret_cast<const float *>(sb) + w * HUW2 + 6 * l;
        const float *sd = reinterpret_cast<const float *>(sb + S::d_off) + w * HUW2 + 6 * l;
#pragma unroll
        for (int cz = 0; cz < 2; ++cz)
#pragma unroll
            for (int n = 0; n < 3; ++n)
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const int idx = cz * HUW2 + 3 * n + d;
                    float v = su[idx];
                    if (N::PRE) v = hmul(hmul(prerelax, v), sd[idx]);   // 1/diag is 0 outside the grid
                    raw[cz][n][d] = v;
                }
        if (s >= 1)
            cx = *reinterpret_cast<const float2 *>(reinterpret_cast<const float *>(sb + S::c_off) + w * HY2 + 2 * l);
    };
    // Row cz = 0 kept for the epilogue, and the face modes.
    auto take_face = [&](const float (&raw)[2][3][3], float (&Uk)[9], float2 (&F)[HF]) {
#pragma unroll
        for (int n = 0; n < 3; ++n)
#pragma unroll
            for (int d = 0; d < 3; ++d) Uk[3 * n + d] = raw[0][n][d];
        face_h2(raw, F);
    };
    double dsum = 0.0, dsum2 = 0.0;
    // Corner partial pairs P of node plane p -> the row-w sums of node
    // columns 2l, 2l + 1 (q), and the row-(w + 1) partials into the z
    // exchange buffer (read by warp w + 1 after the next barrier).
    auto reduce_y = [&](int p, const float2 (&P)[HF], float (&q)[6]) {
        float *z = zb + (p & 1) * (WZ * ZROW2 * 3);
        float zp[6];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float a0 = __shfl_up_sync(0xffffffffu, P[8 + d].y, 1);
            const float a1 = __shfl_up_sync(0xffffffffu, P[12 + d].y, 1);
            q[d] = P[d].x + (l > 0 ? a0 : 0.f);
            q[3 + d] = P[d].y + P[8 + d].x;
            zp[d] = P[4 + d].x + (l > 0 ? a1 : 0.f);
            zp[3 + d] = P[4 + d].y + P[12 + d].x;
        }
        float2 *zr = reinterpret_cast<float2 *>(z + (w * ZROW2 + 2 * l) * 3);
#pragma unroll
        for (int i = 0; i < 3; ++i) zr[i] = make_float2(zp[2 * i], zp[2 * i + 1]);
        if (l == 31)
#pragma unroll
            for (int d = 0; d < 3; ++d) z[(w * ZROW2 + HY2) * 3 + d] = P[12 + d].y;
    };
    // Finish node plane p with the epilogue tiles of ring stage s.
    auto emit = [&](int p, int s, const float2 (&P)[HF], const float (&q)[6], const float (&Uu)[9], const Epi2 &e) {
        if (!zok) return;
        const unsigned char *sb = smem + (s % HRING) * S::slot;
        const float *ef = reinterpret_cast<const float *>(sb + S::ef_off) + w * HUW2;
        const float *ed = reinterpret_cast<const float *>(sb + S::ed_off) + w * HUW2;
        const double *er = reinterpret_cast<const double *>(sb + S::er_off) + w * HUW2;
        const float *ez = reinterpret_cast<const float *>(sb + S::ez_off) + w * HUW2;
        const uint8_t *em = sb + S::m_off + w * HM2;
        const float *z = zb + (p & 1) * (WZ * ZROW2 * 3);
        const int k = kc0 + w, at = ((p - P0) * WZ + w) * 3;
        float zv[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (w > 0) lds6(z + ((w - 1) * ZROW2 + 2 * l) * 3, zv);
        float R[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) R[i] = q[i] + zv[i];
        if (seam) {   // node column jc0: finished after the cluster barrier
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                s_own[at + d] = q[d];
                s_ownz[at + d] = zv[d];
            }
        }
        if (in0) h_store2<MODE>(L.at(p, j0, k), in1, !seam, e, R, Uu, out, omega, dsum, dsum2);
        if (l == 31) {   // this CTA's part of node column jc0 + HY2
            float Sq[3], Sz[3], Sd[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                Sq[d] = P[8 + d].y;
                Sz[d] = w > 0 ? z[((w - 1) * ZROW2 + HY2) * 3 + d] : 0.f;
                Sd[d] = Sq[d] + Sz[d];
            }
            if (r + 1 < CY) {
                float *rem = cluster.map_shared_rank(s_recv, r + 1);
                float *remz = cluster.map_shared_rank(s_recvz, r + 1);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    rem[at + d] = Sq[d];
                    remz[at + d] = Sz[d];
                }
            } else if (tail_owner) {
                const float uu[3] = {Uu[6], Uu[7], Uu[8]};
                h_store<float, MODE>(L.at(p, g.ny, k), em[HY2], Sd, uu, ef + 3 * HY2, ed + 3 * HY2, out, omega,
                                     dsum, er + 3 * HY2, ez + 3 * HY2, dsum2);
            }
        }
    };

    int cur = 0;
    bool fail = false;
    // Step t: the element pair between faces t - 1 (Fc) and t (from raw,
    // waited for and read in step t - 1); then, before the barrier, the face
    // of stage t + 1 and the epilogue operands of node plane p = E0 + t - 1
    // (both in ring slots already waited for), so that their shared-memory
    // latency overlaps the barrier.
    float raw[2][3][3];
    float2 cxn = make_float2(0.f, 0.f);
    auto step = [&](int t, float (&Uc)[9], float2 (&Fc)[HF], float2 (&Ac)[HF], float (&Un)[9], float2 (&Fn)[HF],
                    float2 (&An)[HF]) {
        cur = t;
        wait_stage(t);
        load_face(t, raw, cxn);
        take_face(raw, Un, Fn);
        element_h2(Fc, Fn, cxn, hc, Ac, An);
        const int p = E0 + t - 1;   // node plane finished by this element pair
        const bool out_plane = p >= P0;
        float q[6];
        Epi2 e;
        if (out_plane) {
            face_h(Ac);   // node partials of plane p
            reduce_y(p, Ac, q);
        }
        fail = __syncthreads_or(bad);   // z partners visible; ring slot t - 1 free
        if (!fail && tid == 0 && t - 1 + HRING < nst) issue(t - 1 + HRING);
        if (!fail && out_plane) {
            load_epi2<MODE>(smem + (t % HRING) * S::slot, w, l, e);
            emit(p, t, Ac, q, Uc, e);
        }
    };
    auto finish_last = [&](float (&Uc)[9], float2 (&Ac)[HF]) {   // plane nx: only elements nx - 1 touch it
        cur = nE + 1;
        wait_stage(nE + 1);
        float q[6];
        Epi2 e;
        face_h(Ac);
        reduce_y(E1, Ac, q);
        load_epi2<MODE>(smem + ((nE + 1) % HRING) * S::slot, w, l, e);
        fail = __syncthreads_or(bad);
        if (!fail) emit(E1, nE + 1, Ac, q, Uc, e);
    };

    float U0[9], U1[9];
    float2 F0[HF], A0[HF], F1[HF], A1[HF];
    wait_stage(0);
    load_face(0, raw, cxn);
    take_face(raw, U0, F0);
#pragma unroll
    for (int q = 0; q < HF; ++q) A0[q] = make_float2(0.f, 0.f);
    fail = __syncthreads_or(bad);
    {
        int t = 1;
        for (; !fail && t + 1 <= nE; t += 2) {
            step(t, U0, F0, A0, U1, F1, A1);
            if (!fail) step(t + 1, U1, F1, A1, U0, F0, A0);
        }
        if (!fail && t <= nE) {   // odd count: one more step, the state ends in set 1
            step(t, U0, F0, A0, U1, F1, A1);
            if (!fail && last_plane) finish_last(U1, A1);
        } else if (!fail && last_plane) {
            finish_last(U0, A0);
        }
    }
    if (fail && tid == 0) {
        for (int s = cur; s < issued; ++s)
            if (s != skip_stage) (void)mbar_wait_for(&bar[s % HRING], (uint32_t)((s / HRING) & 1), kHDrainNs);
        if (err) atomicExch(err, GPUTO_ERR_TIMEOUT);
    }
    cluster.sync();   // seam partials from the left neighbour have arrived
    if (!fail && r > 0) {   // node column jc0, from both sides of the seam
        const int np = P1 - P0;
        for (int idx = tid; idx < np * WZ; idx += NT) {
            const int pp = idx / WZ, ww = idx - pp * WZ;
            const int k = kc0 + ww, p = P0 + pp, at = idx * 3;
            if (!((ww >= 1 || zt == 0) && k <= g.nz)) continue;
            const long long base = L.at(p, jc0, k);
            float v[3], uu[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                v[d] = (s_own[at + d] + s_recv[at + d]) + (s_ownz[at + d] + s_recvz[at + d]);
                if (N::PRE)
                    uu[d] = hmul(hmul(prerelax, f[base + d]), rdiag[base + d]);
                else
                    uu[d] = (MODE == MODE_APPLY || N::D) ? ug[base + d] : 0.f;
            }
            h_store<float, MODE>(base, mask[g.node(p, jc0, k)], v, uu, f + base, rdiag + base, out, omega, dsum,
                                 Rd + base, zo + base, dsum2);
        }
    }
    if ((MODE == MODE_APPLY || MODE == MODE_JACOBI_DOT) && dot_partial) {
        constexpr bool PAIR = MODE == MODE_JACOBI_DOT;
        double *red = reinterpret_cast<double *>(smem + S::red_off);
        for (int o = 16; o > 0; o >>= 1) {
            dsum += __shfl_xor_sync(0xffffffffu, dsum, o);
            if (PAIR) dsum2 += __shfl_xor_sync(0xffffffffu, dsum2, o);
        }
        if (l == 0) {
            red[w] = dsum;
            red[WZ + w] = dsum2;
        }
        __syncthreads();
        if (tid == 0) {
            double v = 0.0, v2 = 0.0;
            for (int qq = 0; qq < WZ; ++qq) {
                v += red[qq];
                v2 += red[WZ + qq];
            }
            const long long cta = blockIdx.x + gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
            if (MODE == MODE_APPLY) {
                dot_partial[cta] = v;
            } else {
                dot_partial[2 * cta] = v;
                dot_partial[2 * cta + 1] = v2;
            }
        }
    }
}

// Warps (element rows along z) per CTA: FP32 8; FP64 4, so that more CTAs share an SM (the FP64 apply
// measured 126.8 against 132.0 us with 8, despite the extra overlapping row in four)
template <typename T> constexpr int hwz() { return sizeof(T) == 8 ? 4 : 8; }

// Row pitch of the padded mask copy: TMA needs 16-byte row strides.
long long hmask_pitch(const Grid &g) { return ((long long)g.ny + 1 + 15) & ~15LL; }

// z tiles of WZ element rows, overlapping by one row
int hztiles_wz(const Grid &g, int WZ)
{
    const int rest = g.nz + 1 - WZ;
    return 1 + (rest > 0 ? (rest + WZ - 2) / (WZ - 1) : 0);
}
template <typename T> int hztiles(const Grid &g) { return hztiles_wz(g, hwz<T>()); }

// Test hook for the bounded waits (gputo_debug_set_sweep_fault): the ring
// stage whose copies a launch leaves unissued (-1: none) and how long each
// wait of the march lasts before the CTA gives up (2 s by default).
struct SweepFaultHook {
    int skip_stage = -1;
    uint32_t wait_ns = 2000000000u;
};
std::mutex g_hook_mu;
SweepFaultHook g_hook;

SweepFaultHook sweep_fault_hook()
{
    std::lock_guard<std::mutex> lock(g_hook_mu);
    return g_hook;
}

struct HState {
    bool init = false, ok = false, ok2 = false;
    int resident[2][7][HMAXCY + 1] = {};   // [FP64?][mode][cluster size]: clusters resident on the device
    int resident2[7][HMAXCY + 1] = {};     // the same for the paired FP32 kernel (hsweep2_kernel)
};

HState &hstate(int dev)
{
    static HState st[64];
    return st[dev < 64 ? dev : 63];
}

// Node planes per x chunk: whole rounds of resident clusters, few overlapping
// elements, and a fixed cost per CTA of about four planes.
template <typename T>
int hchunk(const Grid &g, int mode, bool pairs = false)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const int cy = (g.ny + (pairs ? HY2 : HY) - 1) / (pairs ? HY2 : HY);
    const HState &hs = hstate(dev);
    const int res = cy <= HMAXCY ? (pairs ? hs.resident2[mode][cy] : hs.resident[sizeof(T) == 8][mode][cy]) : 0;
    if (res <= 0 || g.nx <= HTX) return g.nx <= HTX ? (g.nx > 0 ? g.nx : 1) : HTX;
    const long long nzt = pairs ? hztiles_wz(g, HWZ2) : hztiles<T>(g);
    long long best = -1;
    int bh = HTX;
    for (int ncx = (g.nx + HTX - 1) / HTX; ncx <= g.nx; ++ncx) {
        const int htx = (g.nx + ncx - 1) / ncx;
        const long long chunks = (g.nx + htx - 1) / htx;
        const long long rounds = (nzt * chunks + res - 1) / res;
        const long long cost = rounds * (htx + 1 + 4);
        if (best < 0 || cost < best) {
            best = cost;
            bh = htx;
        }
        if (htx == 1) break;
    }
    return bh;
}

// The x chunk of a launch: the caller's choice (an autotuned option, clamped
// to 1 .. HTX planes) or the heuristic above.
template <typename T>
int hsweep_chunk(const Grid &g, int mode, int xchunk, bool pairs = false)
{
    if (xchunk <= 0) return hchunk<T>(g, mode, pairs);
    int c = xchunk < HTX ? xchunk : HTX;
    return c < g.nx ? c : (g.nx > 0 ? g.nx : 1);
}

template <typename T>
dim3 hgrid(const Grid &g, int htx, bool pairs = false)
{
    const int cy = (g.ny + (pairs ? HY2 : HY) - 1) / (pairs ? HY2 : HY);
    const int ncx = g.nx > htx ? (g.nx + htx - 1) / htx : 1;
    return dim3((unsigned)cy, (unsigned)(pairs ? hztiles_wz(g, HWZ2) : hztiles<T>(g)), (unsigned)ncx);
}

template <typename T, int MODE>
int hlaunch(const Lay &L, const ELay &E, const HadamardKe &hk, const T *CX, const T *u, const T *f, const T *rdiag,
            const uint8_t *mask, const uint8_t *maskp, T *out, T omega, T prerelax, double *dot_partial,
            const int *done, int *err, cudaStream_t st, const double *Rd = nullptr, const T *zo = nullptr,
            double *ce = nullptr, double *dcv = nullptr, const double *dsK = nullptr, const T *uc = nullptr,
            const Lay *Lc = nullptr, int xchunk = 0)
{
    constexpr int WZ = hwz<T>();
    using N = HNeeds<MODE>;
    using S = HSmem<T, WZ, MODE>;
    const Grid &g = L.g;
    const uint64_t es = sizeof(T);
    // node-plane maps (u, f, diag) share one box: WZ + 1 rows of HUW values
    auto node_map = [&](CUtensorMap *m, const T *base) {
        return make_tmap_3d(m, base, (int)es, (uint64_t)L.pitch, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1,
                            L.pitch * es, L.pitch * es * (g.nz + 1), HUW, WZ + 1, 1);
    };
    CUtensorMap mu, md, mf, mc, mm, mr, mz;
    int s = node_map(&mu, N::PRE ? f : u);
    if (!s && N::DOT) {   // the FP64 residual and z_old, same boxes as the node planes
        s = make_tmap_3d(&mr, Rd, 8, (uint64_t)L.pitch, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1, L.pitch * 8,
                         L.pitch * 8 * (g.nz + 1), HUW, WZ + 1, 1);
        if (!s) s = node_map(&mz, zo);
    }
    if (!s && N::D) s = node_map(&md, rdiag);
    if (!s && N::F) s = node_map(&mf, f);
    if (!s)
        s = make_tmap_3d(&mc, CX, (int)es, (uint64_t)E.pitch, (uint64_t)E.g.nz, (uint64_t)E.g.nx, E.pitch * es,
                         E.pitch * es * E.g.nz, HY, WZ, 1);
    const uint64_t mp = hmask_pitch(g);
    if (!s)
        s = make_tmap_3d(&mm, maskp, 1, mp, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1, mp, mp * (g.nz + 1), HM, WZ, 1);
    // MODE_JACOBI_PRO: mr carries the coarse correction (level-1 layout, boxes
    // of HCZ rows x HCW values) and mz the Dirichlet bits with WZ + 1 rows
    if (!s && N::PRO) {
        const uint64_t ces = sizeof(T);
        s = make_tmap_3d(&mr, uc, (int)es, (uint64_t)Lc->pitch, (uint64_t)Lc->g.nz + 1, (uint64_t)Lc->g.nx + 1,
                         Lc->pitch * ces, Lc->pitch * ces * (Lc->g.nz + 1), HCW, HCZ, 1);
        if (!s)
            s = make_tmap_3d(&mz, maskp, 1, mp, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1, mp, mp * (g.nz + 1), HM,
                             WZ + 1, 1);
    }
    if (s) return s;
    if (!N::D) md = mu;
    if (!N::F) mf = mu;
    if (!N::DOT && !N::PRO) mr = mz = mu;
    const HC<T> hc = make_hc<T>(hk);
    const int htx = hsweep_chunk<T>(g, MODE, xchunk);
    const dim3 grid = hgrid<T>(g, htx);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(32 * WZ);
    cfg.dynamicSmemBytes = S::bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = grid.x;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const SweepFaultHook hook = sweep_fault_hook();
    GPUTO_CUDA(cudaLaunchKernelEx(&cfg, hsweep_kernel<T, MODE, WZ>, mu, md, mf, mc, mm, mr, mz, L, hc, htx, f, rdiag, mask,
                                  out, omega, prerelax, dot_partial, done, err, Rd, zo, hook.wait_ns, hook.skip_stage,
                                  ce, dcv, dsK, uc, Lc ? *Lc : L, u));
    count_launches(1);
    return GPUTO_OK;
}

// The paired FP32 sweep (hsweep2_kernel): the same maps with boxes of HY2
// element columns.
template <int MODE>
int hlaunch2(const Lay &L, const ELay &E, const HadamardKe &hk, const float *CX, const float *u, const float *f,
             const float *rdiag, const uint8_t *maskp, const uint8_t *mask, float *out, float omega, float prerelax,
             double *dot_partial, const int *done, int *err, cudaStream_t st, const double *Rd, const float *zo,
             int xchunk)
{
    constexpr int WZ = HWZ2;
    using N = HNeeds<MODE>;
    using S = HSmem2<MODE>;
    const Grid &g = L.g;
    const uint64_t es = sizeof(float);
    auto node_map = [&](CUtensorMap *m, const float *base) {
        return make_tmap_3d(m, base, (int)es, (uint64_t)L.pitch, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1,
                            L.pitch * es, L.pitch * es * (g.nz + 1), HUW2, WZ + 1, 1);
    };
    CUtensorMap mu, md, mf, mc, mm, mr, mz;
    int s = node_map(&mu, N::PRE ? f : u);
    if (!s && N::DOT) {
        s = make_tmap_3d(&mr, Rd, 8, (uint64_t)L.pitch, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1, L.pitch * 8,
                         L.pitch * 8 * (g.nz + 1), HUW2, WZ + 1, 1);
        if (!s) s = node_map(&mz, zo);
    }
    if (!s && N::D) s = node_map(&md, rdiag);
    if (!s && N::F) s = node_map(&mf, f);
    if (!s)
        s = make_tmap_3d(&mc, CX, (int)es, (uint64_t)E.pitch, (uint64_t)E.g.nz, (uint64_t)E.g.nx, E.pitch * es,
                         E.pitch * es * E.g.nz, HY2, WZ, 1);
    const uint64_t mp = hmask_pitch(g);
    if (!s)
        s = make_tmap_3d(&mm, maskp, 1, mp, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1, mp, mp * (g.nz + 1), HM2, WZ, 1);
    if (s) return s;
    if (!N::D) md = mu;
    if (!N::F) mf = mu;
    if (!N::DOT) mr = mz = mu;
    const HC<float2> hc = pair_hc(make_hc<float>(hk));
    const int htx = hsweep_chunk<float>(g, MODE, xchunk, true);
    const dim3 grid = hgrid<float>(g, htx, true);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(32 * WZ);
    cfg.dynamicSmemBytes = S::bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = grid.x;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const SweepFaultHook hook = sweep_fault_hook();
    GPUTO_CUDA(cudaLaunchKernelEx(&cfg, hsweep2_kernel<MODE>, mu, md, mf, mc, mm, mr, mz, L, hc, htx, f, rdiag, mask,
                                  out, omega, prerelax, dot_partial, done, err, Rd, zo, hook.wait_ns,
                                  hook.skip_stage, u));
    count_launches(1);
    return GPUTO_OK;
}

template <int MODE>
cudaError_t h2set_attr()
{
    return cudaFuncSetAttribute(hsweep2_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)HSmem2<MODE>::bytes);
}

template <int MODE>
int h2resident(int cy)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cy, 1, 1);
    cfg.blockDim = dim3(32 * HWZ2);
    cfg.dynamicSmemBytes = HSmem2<MODE>::bytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cy;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, hsweep2_kernel<MODE>, &cfg) != cudaSuccess) return 0;
    return n;
}

template <typename T, int MODE>
cudaError_t hset_attr()
{
    return cudaFuncSetAttribute(hsweep_kernel<T, MODE, hwz<T>()>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)HSmem<T, hwz<T>(), MODE>::bytes);
}

template <typename T>
cudaError_t hset_attrs()
{
    cudaError_t e;
    if ((e = hset_attr<T, MODE_APPLY>()) != cudaSuccess) return e;
    if ((e = hset_attr<T, MODE_DEFECT>()) != cudaSuccess) return e;
    if ((e = hset_attr<T, MODE_JACOBI>()) != cudaSuccess) return e;
    if constexpr (sizeof(T) == 4)
        if ((e = hset_attr<T, MODE_JACOBI_DOT>()) != cudaSuccess) return e;
    if constexpr (sizeof(T) == 8)
        if ((e = hset_attr<T, MODE_ENERGY>()) != cudaSuccess) return e;
    if ((e = hset_attr<T, MODE_JACOBI_PRO>()) != cudaSuccess) return e;
    return hset_attr<T, MODE_JACOBI_PRE>();
}

// Clusters of 'cy' CTAs of one kernel instance that the device holds at once
// (0: none fit).
template <typename T, int MODE>
int hresident(int cy)
{
    constexpr int WZ = hwz<T>();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cy, 1, 1);
    cfg.blockDim = dim3(32 * WZ);
    cfg.dynamicSmemBytes = HSmem<T, WZ, MODE>::bytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cy;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, hsweep_kernel<T, MODE, WZ>, &cfg) != cudaSuccess) return 0;
    return n;
}

template <typename T>
void hresident_all(HState &s, int cy)
{
    const int p = sizeof(T) == 8;
    s.resident[p][MODE_APPLY][cy] = hresident<T, MODE_APPLY>(cy);
    s.resident[p][MODE_DEFECT][cy] = hresident<T, MODE_DEFECT>(cy);
    s.resident[p][MODE_JACOBI][cy] = hresident<T, MODE_JACOBI>(cy);
    s.resident[p][MODE_JACOBI_PRE][cy] = hresident<T, MODE_JACOBI_PRE>(cy);
    if constexpr (sizeof(T) == 4) s.resident[p][MODE_JACOBI_DOT][cy] = hresident<T, MODE_JACOBI_DOT>(cy);
    if constexpr (sizeof(T) == 8) s.resident[p][MODE_ENERGY][cy] = hresident<T, MODE_ENERGY>(cy);
    s.resident[p][MODE_JACOBI_PRO][cy] = hresident<T, MODE_JACOBI_PRO>(cy);
}

__global__ void pad_mask_kernel(Grid g, const uint8_t *__restrict__ mask, uint8_t *__restrict__ maskp, long long mp)
{
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g.nnod()) return;
    const long long row = n / (g.ny + 1);
    maskp[row * mp + (n - row * (g.ny + 1))] = mask[n];
}

}  // namespace

bool hadamard_ke(const double *Ke, HadamardKe *hk)
{
    hk->ok = false;
    // S = T Ke T' with T[m][b] = (-1)^(px x_b + py y_b + pz z_b), m = 4 px + 2 py + pz
    double T8[8][8];
    for (int m = 0; m < 8; ++m)
        for (int b = 0; b < 8; ++b) {
            const int e = ((m >> 2) & 1) * local_x(b) + ((m >> 1) & 1) * local_y(b) + (m & 1) * local_z(b);
            T8[m][b] = (e & 1) ? -1.0 : 1.0;
        }
    static thread_local double S[24][24], tmp[24][24];
    for (int m = 0; m < 8; ++m)
        for (int d = 0; d < 3; ++d)
            for (int col = 0; col < 24; ++col) {
                double s = 0.0;
                for (int b = 0; b < 8; ++b) s += T8[m][b] * Ke[(3 * b + d) * 24 + col];
                tmp[3 * m + d][col] = s;
            }
    double big = 0.0;
    for (int row = 0; row < 24; ++row)
        for (int n = 0; n < 8; ++n)
            for (int d = 0; d < 3; ++d) {
                double s = 0.0;
                for (int b = 0; b < 8; ++b) s += tmp[row][3 * b + d] * T8[n][b];
                S[row][3 * n + d] = s;
                big = std::fmax(big, std::fabs(s));
            }
    if (!(big > 0.0)) return false;
    auto R = [](int m, int d) { return 3 * m + d; };
    const double a = S[R(1, 0)][R(1, 0)], b = S[R(1, 2)][R(1, 2)], c = S[R(1, 2)][R(2, 1)],
                 dd = S[R(3, 0)][R(3, 0)], e = S[R(3, 0)][R(5, 1)], f = S[R(3, 1)][R(3, 1)],
                 gg = S[R(3, 1)][R(5, 0)], h = S[R(7, 0)][R(7, 0)];
    static thread_local double M[24][24];
    for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) M[i][j] = 0.0;
    const int pa[3][2][2] = {{{1, 0}, {4, 2}}, {{1, 1}, {2, 2}}, {{2, 0}, {4, 1}}};
    for (auto &gp : pa)
        for (auto &x : gp)
            for (auto &y : gp) M[R(x[0], x[1])][R(y[0], y[1])] = a;
    const int tb[2][3][2] = {{{1, 2}, {2, 1}, {4, 0}}, {{3, 0}, {5, 1}, {6, 2}}};
    for (int q = 0; q < 2; ++q)
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                M[R(tb[q][i][0], tb[q][i][1])][R(tb[q][j][0], tb[q][j][1])] =
                    i == j ? (q ? dd : b) : (q ? e : c);
    const int pf[3][2][2] = {{{3, 1}, {5, 0}}, {{3, 2}, {6, 0}}, {{5, 2}, {6, 1}}};
    for (auto &gp : pf)
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) M[R(gp[i][0], gp[i][1])][R(gp[j][0], gp[j][1])] = i == j ? f : gg;
    for (int d = 0; d < 3; ++d) M[R(7, d)][R(7, d)] = h;
    double dev = 0.0;
    for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) dev = std::fmax(dev, std::fabs(S[i][j] - M[i][j]));
    if (!(dev <= 1e-12 * big)) return false;
    const double v[8] = {a, b, c, dd, e, f, gg, h};
    for (int q = 0; q < 8; ++q) hk->c[q] = v[q];
    hk->ok = true;
    return true;
}

int set_sweep_fault_hook(int skip_stage, unsigned wait_us)
{
    if (skip_stage < -1 || wait_us > 4000000u) {
        set_error("skip_stage must be >= -1 and wait_us at most 4,000,000");
        return GPUTO_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_hook_mu);
    g_hook.skip_stage = skip_stage;
    g_hook.wait_ns = wait_us ? wait_us * 1000u : SweepFaultHook{}.wait_ns;
    return GPUTO_OK;
}

int init_hsweep_kernels()
{
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    int dev = 0;
    GPUTO_CUDA(cudaGetDevice(&dev));
    HState &s = hstate(dev);
    if (s.init) return GPUTO_OK;
    s.init = true;
    if (hset_attrs<float>() != cudaSuccess || hset_attrs<double>() != cudaSuccess) {
        cudaGetLastError();
        return GPUTO_OK;   // the dense kernel serves every sweep
    }
    for (int cy = 1; cy <= HMAXCY; ++cy) {
        hresident_all<float>(s, cy);
        hresident_all<double>(s, cy);
    }
    cudaGetLastError();
    s.ok = true;
    if (h2set_attr<MODE_APPLY>() == cudaSuccess && h2set_attr<MODE_DEFECT>() == cudaSuccess &&
        h2set_attr<MODE_JACOBI>() == cudaSuccess && h2set_attr<MODE_JACOBI_PRE>() == cudaSuccess &&
        h2set_attr<MODE_JACOBI_DOT>() == cudaSuccess) {
        for (int cy = 1; cy <= HMAXCY; ++cy) {
            s.resident2[MODE_APPLY][cy] = h2resident<MODE_APPLY>(cy);
            s.resident2[MODE_DEFECT][cy] = h2resident<MODE_DEFECT>(cy);
            s.resident2[MODE_JACOBI][cy] = h2resident<MODE_JACOBI>(cy);
            s.resident2[MODE_JACOBI_PRE][cy] = h2resident<MODE_JACOBI_PRE>(cy);
            s.resident2[MODE_JACOBI_DOT][cy] = h2resident<MODE_JACOBI_DOT>(cy);
        }
        s.ok2 = true;
    }
    cudaGetLastError();   // without the paired kernel, hsweep_kernel serves the FP32 sweeps
    return GPUTO_OK;
}

template <typename T>
bool hsweep_fits(const Grid &g)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    const HState &s = hstate(dev);
    const int cy = (g.ny + HY - 1) / HY;
    if (!s.ok || cy < 1 || cy > HMAXCY || g.nx < 1 || g.nz < 1) return false;
    const int p = sizeof(T) == 8;
    for (int m = 0; m < (p ? 4 : 5); ++m)
        if (s.resident[p][m][cy] <= 0) return false;
    return true;
}

bool hsweep_pairs_fit(const Grid &g)
{
    int dev = 0;
    if (!hsweep_fits<float>(g) || cudaGetDevice(&dev) != cudaSuccess) return false;
    const HState &s = hstate(dev);
    const int cy = (g.ny + HY2 - 1) / HY2;
    if (!s.ok2 || cy > HMAXCY) return false;
    for (int m = 0; m < 5; ++m)
        if (s.resident2[m][cy] <= 0) return false;
    return true;
}

template <typename T>
int hsweep_blocks(const Grid &g, int mode, int xchunk, bool pairs)
{
    pairs = pairs && sizeof(T) == 4 && mode != MODE_ENERGY && mode != MODE_JACOBI_PRO && hsweep_pairs_fit(g);
    const dim3 gr = hgrid<T>(g, hsweep_chunk<T>(g, mode, xchunk, pairs), pairs);
    return (int)(gr.x * gr.y * gr.z);
}

long long hsweep_mask_bytes(const Grid &g) { return hmask_pitch(g) * (g.nz + 1) * (g.nx + 1); }

void launch_pad_mask(const Grid &g, const uint8_t *mask, uint8_t *maskp, cudaStream_t st)
{
    pad_mask_kernel<<<(unsigned)((g.nnod() + 255) / 256), 256, 0, st>>>(g, mask, maskp, hmask_pitch(g));
    count_launches(1);
}

template <typename T>
bool hsweep_pro_fits(const Grid &g)
{
    int dev = 0;
    if (!hsweep_fits<T>(g) || cudaGetDevice(&dev) != cudaSuccess) return false;
    return hstate(dev).resident[sizeof(T) == 8][MODE_JACOBI_PRO][(g.ny + HY - 1) / HY] > 0;
}
template bool hsweep_pro_fits<float>(const Grid &);
template bool hsweep_pro_fits<double>(const Grid &);

bool hsweep_energy_fits(const Grid &g)
{
    int dev = 0;
    if (!hsweep_fits<double>(g) || cudaGetDevice(&dev) != cudaSuccess) return false;
    return hstate(dev).resident[1][MODE_ENERGY][(g.ny + HY - 1) / HY] > 0;
}

int launch_hsweep_energy(const Lay &L, const ELay &E, const HadamardKe &hk, const double *CX, const double *u,
                         const double *f, const uint8_t *mask, const uint8_t *maskp, double *out, double *partial,
                         double *ce, double *dc, const double *dsK, int *err, cudaStream_t st)
{
    if (!ce || !partial || (dc && !dsK)) {
        set_error("the energy sweep needs ce, the partials, and dsK with dc");
        return GPUTO_ERR_ARG;
    }
    return hlaunch<double, MODE_ENERGY>(L, E, hk, CX, u, f, nullptr, mask, maskp, out, 1.0, 0.0, partial, nullptr,
                                        err, st, nullptr, nullptr, ce, dc, dsK);
}

__global__ void __launch_bounds__(256) sum_pairs_kernel(int nb, const double *__restrict__ partial,
                                                        double *__restrict__ out2)
{
    __shared__ double red[2][8];
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < nb; i += 256) {
        a += partial[2 * i];
        b += partial[2 * i + 1];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = a;
        red[1][threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double x = 0.0, y = 0.0;
        for (int q = 0; q < 8; ++q) {
            x += red[0][q];
            y += red[1][q];
        }
        out2[0] = x;
        out2[1] = y;
    }
}

void launch_sum_pairs(int nb, const double *partial, double *out2, cudaStream_t st)
{
    sum_pairs_kernel<<<1, 256, 0, st>>>(nb, partial, out2);
    count_launches(1);
}

template <typename T>
int launch_hsweep(int mode, const Lay &L, const ELay &E, const HadamardKe &hk, const T *CX, const T *u, const T *f,
                  const T *rdiag, const uint8_t *mask, const uint8_t *maskp, T *out, T omega, T prerelax,
                  double *dot_partial, const int *done, int *err, cudaStream_t st, const double *Rd, const T *zo,
                  const T *uc, const Lay *Lc, int xchunk, bool pairs)
{
    if constexpr (sizeof(T) == 4) {
        if (pairs && mode != MODE_JACOBI_PRO && hsweep_pairs_fit(L.g)) {
            switch (mode) {
            case MODE_JACOBI_DOT:
                if (!Rd || !zo || !dot_partial) {
                    set_error("a Jacobi sweep with dots needs the residual, z_old and the partials");
                    return GPUTO_ERR_ARG;
                }
                return hlaunch2<MODE_JACOBI_DOT>(L, E, hk, CX, u, f, rdiag, maskp, mask, out, omega, prerelax,
                                                 dot_partial, done, err, st, Rd, zo, xchunk);
            case MODE_APPLY:
                return hlaunch2<MODE_APPLY>(L, E, hk, CX, u, f, rdiag, maskp, mask, out, omega, prerelax, dot_partial,
                                            done, err, st, nullptr, nullptr, xchunk);
            case MODE_DEFECT:
                return hlaunch2<MODE_DEFECT>(L, E, hk, CX, u, f, rdiag, maskp, mask, out, omega, prerelax, nullptr,
                                             done, err, st, nullptr, nullptr, xchunk);
            case MODE_JACOBI:
                return hlaunch2<MODE_JACOBI>(L, E, hk, CX, u, f, rdiag, maskp, mask, out, omega, prerelax, nullptr,
                                             done, err, st, nullptr, nullptr, xchunk);
            default:
                return hlaunch2<MODE_JACOBI_PRE>(L, E, hk, CX, u, f, rdiag, maskp, mask, out, omega, prerelax,
                                                 nullptr, done, err, st, nullptr, nullptr, xchunk);
            }
        }
    }
    switch (mode) {
    case MODE_JACOBI_PRO:
        if (!uc || !Lc || Lc->g.nx * 2 != L.g.nx || Lc->g.ny * 2 != L.g.ny || Lc->g.nz * 2 != L.g.nz) {
            set_error("a Jacobi sweep with the prolongation needs the coarse correction and its layout");
            return GPUTO_ERR_ARG;
        }
        return hlaunch<T, MODE_JACOBI_PRO>(L, E, hk, CX, u, f, rdiag, mask, maskp, out, omega, prerelax, nullptr,
                                           done, err, st, nullptr, nullptr, nullptr, nullptr, nullptr, uc, Lc, xchunk);
    case MODE_JACOBI_DOT:
        if constexpr (sizeof(T) == 4) {
            if (!Rd || !zo || !dot_partial) {
                set_error("a Jacobi sweep with dots needs the residual, z_old and the partials");
                return GPUTO_ERR_ARG;
            }
            return hlaunch<T, MODE_JACOBI_DOT>(L, E, hk, CX, u, f, rdiag, mask, maskp, out, omega, prerelax,
                                               dot_partial, done, err, st, Rd, zo, nullptr, nullptr, nullptr, nullptr,
                                               nullptr, xchunk);
        }
        set_error("the Jacobi sweep with dots is FP32 only");
        return GPUTO_ERR_ARG;
    case MODE_APPLY:
        return hlaunch<T, MODE_APPLY>(L, E, hk, CX, u, f, rdiag, mask, maskp, out, omega, prerelax, dot_partial, done,
                                      err, st, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, xchunk);
    case MODE_DEFECT:
        return hlaunch<T, MODE_DEFECT>(L, E, hk, CX, u, f, rdiag, mask, maskp, out, omega, prerelax, nullptr, done,
                                       err, st, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, xchunk);
    case MODE_JACOBI:
        return hlaunch<T, MODE_JACOBI>(L, E, hk, CX, u, f, rdiag, mask, maskp, out, omega, prerelax, nullptr, done,
                                       err, st, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, xchunk);
    default:
        return hlaunch<T, MODE_JACOBI_PRE>(L, E, hk, CX, u, f, rdiag, mask, maskp, out, omega, prerelax, nullptr,
                                           done, err, st, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                           xchunk);
    }
}

template bool hsweep_fits<float>(const Grid &);
template bool hsweep_fits<double>(const Grid &);
template int hsweep_blocks<float>(const Grid &, int, int, bool);
template int hsweep_blocks<double>(const Grid &, int, int, bool);
template int launch_hsweep<float>(int, const Lay &, const ELay &, const HadamardKe &, const float *, const float *,
                                  const float *, const float *, const uint8_t *, const uint8_t *, float *, float,
                                  float, double *, const int *, int *, cudaStream_t, const double *, const float *,
                                  const float *, const Lay *, int, bool);
template int launch_hsweep<double>(int, const Lay &, const ELay &, const HadamardKe &, const double *,
                                   const double *, const double *, const double *, const uint8_t *,
                                   const uint8_t *, double *, double, double, double *, const int *, int *,
                                   cudaStream_t, const double *, const double *, const double *, const Lay *, int,
                                   bool);

}  // namespace gputo
