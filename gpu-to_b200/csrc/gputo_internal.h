// Internal declarations shared by the gputo kernels and the host solver.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "gputo.h"

namespace gputo {

constexpr int kMaxLevels = 12;

// Structured hex grid of nx*ny*nz elements (the reference's nelx, nely, nelz).
struct Grid {
    int nx, ny, nz;
    __host__ __device__ long long nnod() const { return (long long)(nx + 1) * (ny + 1) * (nz + 1); }
    __host__ __device__ long long ndof() const { return 3 * nnod(); }
    __host__ __device__ long long nel() const { return (long long)nx * ny * nz; }
    // node n = (nz+1)(ny+1) i + (ny+1) k + j   (mgcg1.cu:966)
    __host__ __device__ long long node(int i, int j, int k) const {
        return ((long long)(nz + 1) * (ny + 1)) * i + (long long)(ny + 1) * k + j;
    }
    // element e = nz ny i + ny k + j   (mgcg1.cu:980)
    __host__ __device__ long long elem(int i, int j, int k) const {
        return ((long long)nz * ny) * i + (long long)ny * k + j;
    }
};

// Row-padded storage of a level's nodal vectors.  Each (i,k) row of ny+1
// nodes (3(ny+1) values, dofs interleaved as in the reference) is padded to
// 'pitch' values, a multiple of 8, so that rows start on 64-byte boundaries:
// TMA needs 16-byte row strides, which 3(ny+1) values never give for odd
// ny+1.  Padding entries are zero and no kernel writes them.  Vectors cross
// the C ABI in the reference's dense layout and are packed / unpacked there.
struct Lay {
    Grid g;
    long long pitch;
    static long long pitch_for(const Grid &g) { return (3LL * (g.ny + 1) + 7) & ~7LL; }
    static Lay of(const Grid &g) { return Lay{g, pitch_for(g)}; }
    __host__ __device__ long long row(int i, int k) const { return ((long long)i * (g.nz + 1) + k) * pitch; }
    __host__ __device__ long long at(int i, int j, int k) const { return row(i, k) + 3LL * j; }
    __host__ __device__ long long size() const { return (long long)(g.nx + 1) * (g.nz + 1) * pitch; }
};

// Row-padded element arrays (CX for the TMA-tiled fine sweep): rows of ny
// elements padded to a multiple of 8.  Padding entries are zero.
struct ELay {
    Grid g;
    long long pitch;
    static ELay of(const Grid &g) { return ELay{g, ((long long)g.ny + 7) & ~7LL}; }
    __host__ __device__ long long at(int i, int j, int k) const { return ((long long)i * g.nz + k) * pitch + j; }
    __host__ __device__ long long size() const { return (long long)g.nx * g.nz * pitch; }
};

// Element-local node a -> (x,y,z) offset, reference order (mgcg1.c:621-624):
// 0:(0,0,0) 1:(1,0,0) 2:(1,1,0) 3:(0,1,0) 4:(0,0,1) 5:(1,0,1) 6:(1,1,1) 7:(0,1,1)
__host__ __device__ constexpr int local_x(int a) { return (a == 1 || a == 2 || a == 5 || a == 6) ? 1 : 0; }
__host__ __device__ constexpr int local_y(int a) { return (a == 2 || a == 3 || a == 6 || a == 7) ? 1 : 0; }
__host__ __device__ constexpr int local_z(int a) { return a >= 4 ? 1 : 0; }
__host__ __device__ constexpr int local_index(int x, int y, int z) { return 4 * z + (y == 0 ? x : 3 - x); }
// Packed lower-triangular index of the symmetric 24x24 element matrix
// (the 300-entry layout of mgcg1.cu:1302-1306).
__host__ __device__ constexpr int packed_index(int m, int n) {
    return m >= n ? (m * (m + 1)) / 2 + n : (n * (n + 1)) / 2 + m;
}

// Device-resident PCG scalars: the host never needs them inside an iteration.
struct PcgScalars {
    double res0;     // ||F||
    double rho_p;    // r'z of the previous iteration
    double pq;       // p'q
    double alpha;
    double rr;       // r'r after the update
    double rz;       // r'z after the preconditioner
    double rz_old;   // r'z_old, flexible (Polak-Ribiere) variant
    double beta;
    double relres;
    double tol;
    int iter;        // iterations completed
    int maxit;
    int done;        // 1 once converged or maxit reached
    int nit;         // reference's return value
    int status;      // gputo_status raised on the device (breakdown)
    int flexible;
    int x_pending;   // 1 between a residual update and the U update of the same iteration
};

// Per-level storage of the multigrid hierarchy.
template <typename T>
struct LevelBuf {
    Grid g;
    T *u0 = nullptr, *u1 = nullptr;  // smoother iterates (ping-pong)
    T *f = nullptr;                  // right-hand side of this level
    T *r = nullptr;                  // defect after pre-smoothing (restriction input)
    T *diag = nullptr;               // operator diagonal
    T *rdiag = nullptr;              // 1 / diag (0 where diag is 0): the sweeps multiply by it
    T *Apk = nullptr;                // packed element matrices, [300][nel] (levels >= 1)
    T *yq = nullptr;                 // level-1 element outputs, [24][nel] (matrix-free level 1)
    uint8_t *mask = nullptr;         // fixed-dof bits per node (bit d = dof d fixed)
};

// ---- error plumbing ------------------------------------------------------
void set_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);
#define GPUTO_CUDA(call)                                                     \
    do {                                                                     \
        cudaError_t _e = (call);                                             \
        if (_e != cudaSuccess) return ::gputo::cuda_status(_e, #call);       \
    } while (0)

// ---- host arrays (hostio.cpp) ----------------------------------------------
// Copies between a caller's (pageable) host array and the device through
// pinned chunks, host side split over a few threads; both return once the
// data has arrived.  host_call_buffer: a device buffer of at least 'count'
// doubles for slot 'slot' of the current device, kept between calls.  Hold
// host_io_mutex() around all three.
std::mutex &host_io_mutex();
int host_to_device(void *dst, const void *src, size_t bytes);
int device_to_host(void *dst, const void *src, size_t bytes);
double *host_call_buffer(int slot, size_t count, int *status);

// ---- kernel launchers (kernels_*.cu) --------------------------------------
// Level-0 element matrix in constant memory (FP64 and FP32 copies).
int upload_fine_ke(const double *Ke_host, cudaStream_t st);
// Unique id of the calling thread's current CUDA context (0 if none or the
// driver lacks cuCtxGetId).  Per-device caches of device state (constant
// memory contents, symbol addresses) key on it, so a cudaDeviceReset, which
// replaces the primary context, invalidates them.
unsigned long long current_context_id();
int upload_design_ke(const double *Ke_host, cudaStream_t st);
int upload_tc_ke(const double *Ke_host, cudaStream_t st);
int upload_tcsweep_ke(const double *Ke_host, cudaStream_t st);
// B^T D B w at one Gauss point (ix,iy,iz) of an h-cube, E = 1 (host).
void gauss_part(double nu, double h, int ix, int iy, int iz, double K[24][24]);
// Level-1 quadrature parts Kg[g] (packed 300 each) for nu, h = 2.
int upload_quadrature_parts(double nu, cudaStream_t st);

enum SweepMode { MODE_APPLY = 0, MODE_DEFECT = 1, MODE_JACOBI = 2, MODE_JACOBI_PRE = 3 };
// A Jacobi sweep of the FP32 fine level that also sums r'z and r'z_old (r the
// FP64 PCG residual, z its output, z_old the previous one) into per-CTA
// partial pairs: the mixed PCG's last smoothing sweep (Hadamard-basis kernel only).
constexpr int MODE_JACOBI_DOT = 4;
// The FP64 fine operator applied to a solution U, with the element energies
// in the same pass (Hadamard-basis kernel only): per-CTA partial pairs of
// |f - K u|^2 over the free dofs and sum CX_e u_e' Ke u_e, and ce_e (dc_e =
// dsK_e ce_e) written once per element.
constexpr int MODE_ENERGY = 5;
// The first damped-Jacobi sweep after a coarse-grid correction: u = u_pre +
// P e_c (trilinear prolongation, fixed dofs zeroed) is formed in the sweep's
// own node-plane tiles, so the prolongation pass and its write and re-read
// of u disappear (Hadamard-basis kernel only; same results bit for bit).
constexpr int MODE_JACOBI_PRO = 6;

// Fine level (K = sum CX_e Ke), FP64 and FP32 instantiations; CX padded (ELay),
// vectors padded (Lay).  'err' receives GPUTO_ERR_TIMEOUT if a bounded wait
// gives up.  Returns a status (tensor-map encoding can fail).
template <typename T>
int launch_fine_sweep(int mode, const Lay &L, const ELay &E, const T *CX, const T *u, const T *f,
                      const T *diag, const uint8_t *mask, T *out, T omega, T prerelax,
                      double *dot_partial, const int *done, int *err, cudaStream_t st);
// Level-1 quadrature operator applied matrix-free (L: level-1 layout, Ef: the
// fine element layout of the padded CX, yscratch: 24 values per level-1
// element, nu: Poisson ratio of the quadrature operator).
// Far-face nodes of a fine sweep only (kernels_fine.cu).
template <typename T>
int launch_fine_faces(int mode, const Lay &L, const ELay &E, const T *CX, const T *u, const T *f, const T *diag,
                      const uint8_t *mask, T *out, T omega, T prerelax, const int *done, cudaStream_t st);

// FP32 fine sweep with the element contraction on the tensor cores
// (kernels_tcsweep.cu).  parts: u and Ke each split into 1 or 2 BF16 parts.
// xchunk: node planes per CTA along x.
int init_tc_sweep_kernels();
int launch_tc_sweep(int parts, int mode, const Lay &L, const ELay &E, const float *CX, const float *u,
                    const float *f, const float *diag, const uint8_t *mask, float *out, float omega,
                    float prerelax, int xchunk, const int *done, int *err, cudaStream_t st);

template <typename T>
int launch_quad_sweep(int mode, const Lay &L, const ELay &Ef, const T *CX, const T *u, const T *f,
                      const T *rdiag, const uint8_t *mask, T *out, T omega, T prerelax, double nu,
                      T *yscratch, const int *done, int *err, cudaStream_t st);
void launch_diag_quad(const Lay &L, const double *CXf, double *diag, cudaStream_t st);
int upload_quadrature_fine(const double *kg_packed, cudaStream_t st);
// Level-2 Galerkin operator directly from the fine CX (level 1 not stored).
void launch_build_galerkin_from_quad(const Grid &g2, const double *CXfine, double *Apk, cudaStream_t st);
// Fine sweeps with Ke in its Hadamard basis (kernels_hsweep.cu).  hadamard_ke
// derives the eight constants of T Ke T from a cube element's Ke and returns
// false when Ke lacks that structure.  hsweep_fits: the grid suits the kernel
// (ny <= 256) and its clusters are resident on this device.
struct HadamardKe {
    bool ok = false;
    double c[8] = {};   // a, b, c, d, e, f, g, h
};
bool hadamard_ke(const double *Ke, HadamardKe *hk);
int init_hsweep_kernels();
// Test hook of the Hadamard-basis sweeps' bounded waits (see
// gputo_debug_set_sweep_fault in gputo.h).
int set_sweep_fault_hook(int skip_stage, unsigned wait_us);
template <typename T> bool hsweep_fits(const Grid &g);
// The paired FP32 sweep (two element columns per lane, ny <= 512) is built
// and resident on this device for g.
bool hsweep_pairs_fit(const Grid &g);
// CTAs (= partials) of a sweep; xchunk: node planes per x chunk (0: chosen
// from the device's resident clusters); pairs: the paired FP32 sweep where it
// fits.
template <typename T> int hsweep_blocks(const Grid &g, int mode = MODE_APPLY, int xchunk = 0, bool pairs = false);
// rdiag: 1/diag (launch_recip); maskp: the Dirichlet bytes with rows padded
// to 16 bytes (launch_pad_mask; hsweep_mask_bytes of storage).
// MODE_JACOBI_PRO: uc is the coarse correction in the layout Lc (level 1).
template <typename T>
int launch_hsweep(int mode, const Lay &L, const ELay &E, const HadamardKe &hk, const T *CX, const T *u, const T *f,
                  const T *rdiag, const uint8_t *mask, const uint8_t *maskp, T *out, T omega, T prerelax,
                  double *dot_partial, const int *done, int *err, cudaStream_t st, const double *Rd = nullptr,
                  const T *zo = nullptr, const T *uc = nullptr, const Lay *Lc = nullptr, int xchunk = 0,
                  bool pairs = false);
template <typename T> bool hsweep_pro_fits(const Grid &g);
// MODE_ENERGY sweep (FP64): out (optional) = f - K u with fixed rows zero,
// ce / dc in natural element order, partial pairs (|r|^2, sum CX ce) per CTA.
bool hsweep_energy_fits(const Grid &g);
int launch_hsweep_energy(const Lay &L, const ELay &E, const HadamardKe &hk, const double *CX, const double *u,
                         const double *f, const uint8_t *mask, const uint8_t *maskp, double *out, double *partial,
                         double *ce, double *dc, const double *dsK, int *err, cudaStream_t st);
// Sums the nb partial pairs in fixed order: out2[0] = sum of the first
// members, out2[1] = sum of the second.
void launch_sum_pairs(int nb, const double *partial, double *out2, cudaStream_t st);
long long hsweep_mask_bytes(const Grid &g);
void launch_pad_mask(const Grid &g, const uint8_t *mask, uint8_t *maskp, cudaStream_t st);
// Opt the tile kernels into their dynamic shared memory (call once per device).
int init_fine_kernels();
// Number of per-CTA partials a MODE_APPLY fine sweep writes.
int fine_sweep_blocks(const Grid &g);
// Coarse level (packed element matrices, natural element order).
template <typename T>
// The coarse-level sweeps take rdiag = 1/diag (LevelBuf::rdiag).
void launch_packed_sweep(int mode, const Lay &L, const T *Apk, const T *u, const T *f,
                         const T *rdiag, const uint8_t *mask, T *out, T omega, T prerelax,
                         const int *done, cudaStream_t st);

// Element-centric form of the same sweep (yscratch: 24 values per element).
template <typename T>
void launch_packed_sweep_ec(int mode, const Lay &L, const T *Apk, const T *u, const T *f, const T *rdiag,
                            const uint8_t *mask, T *out, T omega, T prerelax, T *yscratch,
                            const int *done, cudaStream_t st);
// Levels at least this many elements use the element-centric sweep.
constexpr long long kElementCentricMinElems = 16384;

template <typename T>
void launch_restrict(const Lay &Lc, const Lay &Lf, const T *rf, const uint8_t *maskc, T *fc,
                     const int *done, cudaStream_t st);
template <typename T>
void launch_prolong_add(const Lay &Lf, const Lay &Lc, const T *uc, const uint8_t *maskf, T *uf,
                        const int *done, cudaStream_t st);

void launch_diag_fine(const Lay &L, const double *CX, double *diag, cudaStream_t st);
template <typename T>
void launch_diag_packed(const Lay &L, const T *Apk, T *diag, cudaStream_t st);
// dense (reference layout) <-> padded, optionally negating y components
void launch_pack(const Lay &L, const double *dense, double *padded, int flip_y, cudaStream_t st);
void launch_unpack(const Lay &L, const double *padded, double *dense, int flip_y, cudaStream_t st);
template <typename T>
void launch_pack_cx(const ELay &E, const double *CX, T *padded, cudaStream_t st);
void launch_build_level1(const Grid &gc, const double *CXfine, double *Apk, cudaStream_t st);
void launch_build_galerkin(const Grid &gc, const double *Afine, double *Apk, cudaStream_t st);
void launch_coarsest_penalty(const Grid &g, const uint8_t *mask, double *Apk, cudaStream_t st);
void launch_assemble_dense(const Grid &g, const double *Apk, double *AQ, cudaStream_t st);
void launch_dense_fine(const Grid &g, const double *CX, double *Apk_tmp, cudaStream_t st);
// re-discretised hierarchy (mgcg9): coarse CX = 2 mean(children); fixed dofs
// of the dense coarsest matrix as zero rows/columns with 1e10 on the diagonal
void launch_coarse_cx(const Grid &gc, const double *CXf, double *CXc, cudaStream_t st);
void launch_dense_fix(const Grid &g, const uint8_t *mask, double *AQ, cudaStream_t st);
// Cholesky + explicit inverse of the lower factor; info[0] = 0 or bad pivot (1-based).
void launch_cholesky(int n, double *A, int *info, cudaStream_t st);
void launch_tri_inverse(int n, const double *L, double *Linv, double *LinvT, cudaStream_t st);
template <typename T>
void launch_coarse_solve(const Lay &L, const double *Linv, const double *LinvT, const T *b, T *x,
                         double *tmp, const int *done, cudaStream_t st);

void launch_mask_from_list(long long nnod, const double *fixed1b, int nfd, uint8_t *mask,
                           cudaStream_t st);
void launch_mask_restrict(const Grid &gc, const uint8_t *maskf, uint8_t *maskc, cudaStream_t st);
template <typename Tin, typename Tout>
void launch_convert(long long n, const Tin *in, Tout *out, const int *done, cudaStream_t st);
void launch_cast_f32(long long n, const double *in, float *out, cudaStream_t st);
// out = 1 / in (0 where in is 0), rounded once to T
template <typename T>
void launch_recip(long long n, const double *in, T *out, cudaStream_t st);

// PCG vector kernels (kernels_blas.cu).
int reduce_partials_capacity();
void launch_dot(long long n, const double *a, const double *b, double *partial, unsigned *ticket,
                PcgScalars *sc, int which, const int *done, cudaStream_t st);
// R32 (optional): also write float(R) there.
void launch_pcg_update(long long n, double *R, const double *Q, double *partial, unsigned *ticket, PcgScalars *sc,
                       cudaStream_t st, float *R32 = nullptr);
// Z: double, or float for the FP32 V-cycle output read directly.  Also
// applies the pending U += alpha P.
template <typename Z>
void launch_p_update(long long n, const Z *z, double *P, Z *Zold, double *U, PcgScalars *sc, cudaStream_t st);
// U += alpha P when a solve stopped with that update pending.
void launch_flush_x(long long n, double *U, const double *P, const PcgScalars *sc, cudaStream_t st);
template <typename Z>
void launch_dot2(long long n, const double *r, const Z *z, const Z *zold, double *partial, unsigned *ticket,
                 PcgScalars *sc, const int *done, cudaStream_t st);
void launch_pcg_init(long long n, const double *F, double *U, double *R, double *partial,
                     unsigned *ticket, PcgScalars *sc, double tol, int maxit, int flexible,
                     cudaStream_t st);
void launch_finish_apply_dot(int nblocks, double *partial, unsigned *ticket, PcgScalars *sc,
                             cudaStream_t st);
// r'z and r'z_old from the partial pairs of a MODE_JACOBI_DOT sweep, then the
// end-of-iteration scalars (beta, relres, convergence) as the two-dot kernel.
void launch_finish_dot2(int nblocks, const double *partial, PcgScalars *sc, cudaStream_t st);
void launch_copy(long long n, const double *a, double *b, const int *done, cudaStream_t st);
void launch_flip_y(long long nnod, double *U, cudaStream_t st);

// Design steps (kernels_design.cu).
void launch_element_energy(const Grid &g, const double *U, const double *CX, const double *dsK,
                           double *ce, double *dc, double *partial, unsigned *ticket,
                           double *compliance, cudaStream_t st);
// ce / dc / compliance with the element contraction on the tensor cores
// (tcgen05, BF16 splits, FP32 accumulate): kernels_tc.cu.
long long element_energy_tc_partials(const Grid &g);
bool element_energy_tc_fits(const Grid &g);   // 32-bit dof indexing
void launch_element_energy_tc(const Grid &g, const double *U, const double *CX, const double *dsK,
                              double *ce, double *dc, double *partial, double *compliance, int *err,
                              cudaStream_t st);
void launch_element_energy_blocks(const Grid &g, const double *U, const double *CX,
                                  const double *dsK, double *ce, double *dc, double *partial,
                                  unsigned *ticket, double *compliance, int nblocks,
                                  cudaStream_t st);
int launch_filter(const Grid &g, const double *in, const double *div, double *out, double rmin,
                  int normalize, cudaStream_t st);
void launch_simp(long long n, const double *x, double penal, double E0, double Emin, double *CX,
                 double *dsK, cudaStream_t st);
int oc_state_bytes();
int proj_state_bytes();
void launch_heaviside(long long n, const double *xt, double volfrac, double beta, double eta0, double *xphys,
                      double *dprj, double *partial, unsigned *ticket, void *state, int max_steps, cudaStream_t st);
void launch_mul(long long n, const double *a, const double *b, double *out, cudaStream_t st);
void launch_oc_update(long long n, const double *x, const double *dc, const double *dv0,
                      double volfrac, double move, double *ocp, double *xnew, double *partial,
                      unsigned *ticket, void *state, int max_steps, cudaStream_t st);

// Counter of kernel launches issued by this library (per process).
void count_launches(long long n);

// Programmatic dependent launch.  A kernel started with launch_pdl may begin
// while its predecessor in the stream is still finishing (its launch latency
// overlaps the predecessor's tail); it calls pdl_wait() before it touches
// memory, which returns once the predecessor has completed and its writes
// are visible.  A kernel that calls pdl_wait() but is launched normally is
// unaffected.
#if defined(__CUDACC__)
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Lets the next kernel in the stream launch before this one has finished (its
// pdl_wait() still waits for this kernel's completion).
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Grid of thread-per-node kernels, one row of CTAs per x node plane
// (blockIdx.y = i), so a thread finds (j, k) with one 32-bit division.
inline dim3 plane_grid(const Grid &g, int bs)
{
    const int per_plane = (g.ny + 1) * (g.nz + 1);
    return dim3((unsigned)((per_plane + bs - 1) / bs), (unsigned)(g.nx + 1));
}
__device__ __forceinline__ bool plane_ijk(const Grid &g, int &i, int &j, int &k)
{
    const unsigned m = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned ny1 = (unsigned)g.ny + 1u;
    if (m >= ny1 * ((unsigned)g.nz + 1u)) return false;
    i = (int)blockIdx.y;
    k = (int)(m / ny1);
    j = (int)(m - (unsigned)k * ny1);
    return true;
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args &&...args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}
#endif
long long launches_issued();

// ---------------------------------------------------------------------------
// learned coarse-grid correction (kernels_learned.cu)
// ---------------------------------------------------------------------------

// Node grid of the network, channels-first [C][X][Z][Y] (Y fastest).
struct NetDims {
    int X, Z, Y;
    __host__ __device__ long long n() const { return (long long)X * Z * Y; }
};

// The network's parameters, Adam state and activation buffers on one device.
struct Net {
    int device = 0;
    float *params = nullptr, *grads = nullptr, *m1 = nullptr, *m2 = nullptr;
    double *part = nullptr, *loss_acc = nullptr;   // loss reduction scratch, summed loss
    float *gscale = nullptr;
    float *act[5] = {};                            // act[0] = input (not owned), act[1..4] owned
    float *gA = nullptr, *gB = nullptr;            // gradient ping-pong, 64 channels each
    long long cap_n = 0, step = 0;
    std::vector<void *> owned;

    static long long num_params();
    static long long param_offset(int layer, bool bias);
    ~Net();
    int create(unsigned long long seed);
    int reserve(long long nodes);   // activation buffers (never inside a stream capture)
    // y = net(x) (y may be null: the output stays in act[4])
    int forward(const float *x, const NetDims &d, float *y, cudaStream_t st);
    // one sample's masked mean-square loss added to *loss_acc, its gradient to grads
    int accumulate(const float *x, const float *t, const float *m, const NetDims &d, cudaStream_t st);
    // gradient of the last forward's output in gA ([3][n]) -> added to grads
    int backward_from(const NetDims &d, cudaStream_t st);
    // Adam step with the mean gradient of nsamples accumulated samples; clears grads
    int adam(float lr, int nsamples, cudaStream_t st);
};

int init_net_kernels();
// Level-2 node features of the learned correction: log-density of the
// element scales, then the restricted residual in Jacobi-scaled units divided
// by its RMS (device s); dsq (optional) receives sqrt(diag), channels-first.
void launch_net_density(const Grid &g2, const Grid &gf, const double *CXf, float *dens2, cudaStream_t st);
void launch_net_features(const Lay &L2, const float *r2, const float *diag2, const float *dens2, float *x,
                         float *dsq, float *s, const int *done, cudaStream_t st);
void launch_net_output(const Lay &L2, const float *y, const float *diag2, const float *s, const uint8_t *mask2,
                       float *e2, const int *done, cudaStream_t st);
void launch_add_f2d(long long n, const float *e, double *z, const int *done, cudaStream_t st);
void launch_net_mask(const Grid &g2, const uint8_t *mask2, float *m, cudaStream_t st);
void launch_level2_inject(const Grid &g2, const Grid &gf, const double *v, float *out, cudaStream_t st);
// Energy loss of the correction: w = D^-1/2 y (padded), and with q = A2 w the
// output gradient gy = 2 (D^-1/2 q - g~) and loss += y'D^-1/2 q - 2 y'g~.
void launch_net_to_padded(const Lay &L2, const float *y, const float *diag2, const uint8_t *mask2, float *w,
                          cudaStream_t st);
void launch_net_energy_rhs(const Lay &L2, const float *v2, const float *diag2, const uint8_t *mask2, float scale,
                           float *gt, cudaStream_t st);
int launch_net_energy(const Lay &L2, const float *y, const float *q, const float *diag2, const float *gt,
                      const uint8_t *mask2, float *gy, double *part, int part_cap, double *loss_acc, cudaStream_t st);

}  // namespace gputo
