// Fine-level sweeps of the mixed-precision V-cycle with the element
// contraction on the 5th-generation tensor cores.
//
// The operator is the one of the CUDA-core tile kernels (K = sum_e CX_e Ke,
// node-centred result, Dirichlet rows zeroed; mgcg1.cu:941-997,1199-1264,
// 1326-1331), computed element-centred: Y_e = Ke u_e for a whole layer of
// elements as tcgen05 MMAs (BF16 operands, FP32 accumulation in TMEM), then
// scaled by CX_e in FP32 and gathered at the nodes in a fixed order.
//
// Layout that avoids an im2col of u.  A CTA owns a 32 (y) x 8 (z) block of
// nodes and marches along x over a chunk of node planes.  Each node plane of
// its halo (rows k0-1 .. k0+8) is kept in shared memory as BF16 with the
// three dofs padded to four (8 bytes per node), twice: an "even" copy that
// starts at node j0 and an "odd" copy that starts at node j0-1.  A 16-byte
// core-matrix row is then one element's two y-adjacent nodes: elements
// j0, j0+2, ... read the even copy, elements j0-1, j0+1, ... the odd copy, so
// the MMA's A operand for 4 element rows x 32 elements is read straight from
// the plane copies by the shared-memory descriptor (core groups of 8
// elements 128 bytes apart, the two z-rows of an element 512 bytes apart).
// One MMA with K = 16 covers an element's four nodes on one x face, a second
// MMA the other face.  The last element column (j0+31) falls outside this
// pattern and gets a small im2col tile of its own.
//
// Precision: u and Ke are split into SU and SK BF16 parts (SU = SK = 1 is a
// plain BF16 product, 2 adds the rounding remainder); all parts accumulate in
// FP32.  The sweep is a preconditioner inside flexible FP64 PCG, which keeps
// the solution and the convergence test in FP64.
#include <cuda_bf16.h>

#include <cstring>
#include <mutex>

#include "gputo_internal.h"
#include "tma.h"

namespace gputo {

namespace {
// The B operand (Ke split into SK BF16 parts) as the K-major core-matrix image
// the MMAs read, built on the host when Ke is uploaded: one 2 KB image per
// part, rows n = 4 a_out + d_out (d_out = 3 is zero padding), columns
// k = 16 h + 8 kc + 4 p + d <-> input node (x = h, y = p, z = kc), dof d.
__device__ uint4 gBimg1[128];   // SK = 1
__device__ uint4 gBimg2[256];   // SK = 2

uint16_t host_bf16_trunc(float v)
{
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return (uint16_t)(b >> 16);
}
float host_from_bf16(uint16_t h)
{
    const uint32_t b = (uint32_t)h << 16;
    float v;
    std::memcpy(&v, &b, 4);
    return v;
}
uint16_t host_bf16_rn(float v)   // round to nearest even (finite values)
{
    uint32_t b;
    std::memcpy(&b, &v, 4);
    return (uint16_t)((b + 0x7FFFu + ((b >> 16) & 1u)) >> 16);
}
}  // namespace

int upload_tcsweep_ke(const double *Ke_host, cudaStream_t st)
{
    // same split as the device's u: every part but the last truncates, the
    // last rounds the remainder to nearest
    uint16_t img1[32 * 32] = {}, img2[64 * 32] = {};
    auto off = [](int row, int col) { return ((row >> 3) * 4 + (col >> 3)) * 64 + (row & 7) * 8 + (col & 7); };
    for (int n = 0; n < 32; ++n)
        for (int k = 0; k < 32; ++k) {
            const int ao = n >> 2, dout = n & 3;
            const int h = k >> 4, kc = (k >> 3) & 1, p = (k >> 2) & 1, d = k & 3;
            if (dout == 3 || d == 3) continue;
            const float v = (float)Ke_host[(3 * ao + dout) * 24 + 3 * local_index(h, p, kc) + d];
            img1[off(n, k)] = host_bf16_rn(v);
            const uint16_t hi = host_bf16_trunc(v);
            img2[off(n, k)] = hi;
            img2[off(32 + n, k)] = host_bf16_rn(v - host_from_bf16(hi));
        }
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(gBimg1, img1, sizeof(img1), 0, cudaMemcpyHostToDevice, st));
    GPUTO_CUDA(cudaMemcpyToSymbolAsync(gBimg2, img2, sizeof(img2), 0, cudaMemcpyHostToDevice, st));
    GPUTO_CUDA(cudaStreamSynchronize(st));
    return GPUTO_OK;
}

namespace {

constexpr int SY = 32, SZ = 8;          // nodes per CTA in y, z
constexpr int SNT = 256;                // threads per CTA (one node of the block each)
constexpr int SUW = 104;                // FP32 u box width: values of nodes j0-1 .. j0+32 from 3(j0-1)-1
constexpr int SUOFF = 1;                // offset of node j0-1 in a box row
constexpr int SROWS = SZ + 2;           // node rows k0-1 .. k0+8
constexpr int SCW = 36, SCOFF = 3;      // CX box width; element j0-1 at SCOFF (16-byte aligned start)
constexpr int SCROWS = SZ + 1;          // element rows k0-1 .. k0+7
constexpr int EY = SY + 1;              // element columns j0-1 .. j0+31
constexpr int YSTR = 25;                // Y stride per element (24 + 1 against bank conflicts)
constexpr int NSTAGE = 3;               // plane ring depth
constexpr int ROWB = 512;               // bytes per BF16 node row: even copy 256 + odd copy 256
constexpr int PLANEB = SROWS * ROWB;    // bytes per BF16 plane copy (one part)
constexpr int FIXB = 16 * 64;           // im2col tile: rows 0..15 of 128 x 32 BF16 (see fix_off)
constexpr uint32_t kSweepPolls = 1u << 22;

// first element row of the three plane tiles (the third overlaps the second;
// only its last row is read back)
__host__ __device__ constexpr int tile_row0(int t) { return t == 0 ? 0 : (t == 1 ? 4 : 5); }

// Byte offset of (row, col) in a K-major BF16 operand with four 8x8 core
// matrices along K per 8-row group (K = 32): LBO 128, SBO 512.
__host__ __device__ constexpr uint32_t core_off(int row, int col)
{
    return (uint32_t)(((row >> 3) * 4 + (col >> 3)) * 128 + (row & 7) * 16 + (col & 7) * 2);
}

__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version (sm_100); base offset 0, no swizzle
    return d;
}

template <int N>
__host__ __device__ constexpr uint32_t instr_desc()
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// 32 consecutive TMEM columns of this warp's 32 lanes; the wait for the load
// is part of the same asm statement, so no use of v can precede it.
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr)
        : "memory");
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// Part `part` of an SP-way BF16 split of v: every part but the last keeps
// the top 8 significand bits of what remains (truncation, exact remainder);
// the last part rounds the remainder to nearest.
template <int SP>
__device__ __forceinline__ uint16_t bf16_part(float v, int part)
{
    float r = v;
#pragma unroll
    for (int s = 0; s < SP - 1; ++s) {
        if (s == part) return (uint16_t)(__float_as_uint(r) >> 16);
        r -= __uint_as_float(__float_as_uint(r) & 0xFFFF0000u);
    }
    return __bfloat16_as_ushort(__float2bfloat16_rn(r));
}

}  // namespace

template <int SU, int SK, bool PRE>
struct SweepSmem {
    static constexpr int N = 32;   // 8 nodes x (3 dofs + 1 pad); split products accumulate in place
    static constexpr size_t u_box = (size_t)SUW * SROWS * 4;         // FP32 plane box (bytes)
    static constexpr size_t c_box = (size_t)SCW * SCROWS * 4;        // FP32 CX layer box (bytes)
    static constexpr size_t u_slot = (u_box + 127) & ~size_t(127);   // TMA destinations: 128-byte aligned
    static constexpr size_t c_slot = (c_box + 127) & ~size_t(127);
    static constexpr size_t u_off = 0;
    static constexpr size_t d_off = u_off + NSTAGE * u_slot;         // diag planes (PRE)
    static constexpr size_t c_off = d_off + (PRE ? NSTAGE * u_slot : 0);
    static constexpr size_t a_off = c_off + NSTAGE * c_slot;              // two BF16 plane slots
    // The im2col tile holds 9 real rows (two 8-row core groups); the M = 128
    // MMA also reads groups 2..15, up to 8 KB further on.  Those rows' results
    // are never read back, so they may read whatever follows (B and Y): the
    // layout only guarantees that the reads stay inside this CTA's shared memory.
    static constexpr size_t fix_off = a_off + (size_t)2 * SU * PLANEB;
    static constexpr size_t b_off = fix_off + (size_t)SU * FIXB;
    static constexpr size_t y_off = b_off + (size_t)SK * 2048;
    static constexpr size_t y_bytes = (size_t)SCROWS * EY * YSTR * 4;
    static constexpr size_t bar_off = (y_off + y_bytes + 15) & ~size_t(15);
    static constexpr size_t bytes = bar_off + 8 * (NSTAGE + 1) + 16;
    static_assert(fix_off + (SU - 1) * FIXB + 256 + 15 * 512 + 256 <= bytes, "im2col junk rows leave the CTA");
    static constexpr uint32_t stage_tx = (uint32_t)(u_box * (PRE ? 2 : 1) + c_box);
};

template <int MODE, int SU, int SK>
__global__ void __launch_bounds__(SNT, 3)
tc_sweep_kernel(const __grid_constant__ CUtensorMap tm_u, const __grid_constant__ CUtensorMap tm_d,
                const __grid_constant__ CUtensorMap tm_c, Lay L, int xchunk, const float *__restrict__ f,
                const float *__restrict__ diag, const uint8_t *__restrict__ mask, float *__restrict__ out,
                float omega, float prerelax, const int *__restrict__ done, int *__restrict__ err)
{
    if (done && *done) return;
    constexpr bool PRE = (MODE == MODE_JACOBI_PRE);
    using S = SweepSmem<SU, SK, PRE>;
    constexpr int N = S::N;
    constexpr int TILE_COLS = N;        // TMEM columns per M tile (4 tiles)
    constexpr uint32_t TMEM_COLS = 128u;
    constexpr uint32_t IDESC = instr_desc<N>();
    extern __shared__ __align__(128) unsigned char smem[];
    float *su = reinterpret_cast<float *>(smem + S::u_off);
    float *sd = reinterpret_cast<float *>(smem + S::d_off);
    float *sc = reinterpret_cast<float *>(smem + S::c_off);
    unsigned char *sa = smem + S::a_off;
    unsigned char *sfix = smem + S::fix_off;
    unsigned char *sb = smem + S::b_off;
    float *ys = reinterpret_cast<float *>(smem + S::y_off);
    uint64_t *tbar = reinterpret_cast<uint64_t *>(smem + S::bar_off);   // NSTAGE TMA barriers
    uint64_t *mbar = tbar + NSTAGE;                                       // MMA completion
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mbar + 1);

    const Grid &g = L.g;
    const int j0 = blockIdx.x * SY, k0 = blockIdx.y * SZ;
    const int ia = blockIdx.z * xchunk;
    const int ib = min(ia + xchunk, g.nx);      // node planes ia .. ib-1 (plane nx: face kernel)
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ty = tid & 31, tz = tid >> 5;     // this thread's node in the block

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s <= NSTAGE; ++s) mbar_init(tbar + s, 1);
        fence_barrier_init();
    }
    // B image (built on the host) -> shared memory
    {
        const uint4 *bimg = SK == 1 ? gBimg1 : gBimg2;   // part k at byte 2048 k
        for (int idx = tid; idx < SK * 128; idx += SNT) reinterpret_cast<uint4 *>(sb)[idx] = bimg[idx];
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    // stage q (relative plane p = ia - 1 + q): u plane p (f for PRE, with
    // diag), CX layer p - 1, into ring slot q % NSTAGE
    auto issue_stage = [&](int q) {
        const int p = ia - 1 + q, s = q % NSTAGE;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive_expect_tx(tbar + s, S::stage_tx);
        const int cu = 3 * (j0 - 1) - SUOFF;
        tma_load_3d(reinterpret_cast<unsigned char *>(su) + s * S::u_slot, &tm_u, cu, k0 - 1, p, tbar + s);
        if (PRE) tma_load_3d(reinterpret_cast<unsigned char *>(sd) + s * S::u_slot, &tm_d, cu, k0 - 1, p, tbar + s);
        tma_load_3d(reinterpret_cast<unsigned char *>(sc) + s * S::c_slot, &tm_c, j0 - 1 - SCOFF, k0 - 1, p - 1,
                    tbar + s);
    };
    // wait for stage q; every thread returns the same answer
    auto wait_stage = [&](int q) -> bool {
        const bool ok = mbar_wait_bounded(tbar + (q % NSTAGE), (uint32_t)((q / NSTAGE) & 1), kSweepPolls);
        return !__syncthreads_or(!ok);
    };
    // FP32 plane of stage q -> its BF16 even/odd copies (and PRE's initial guess)
    auto convert_plane = [&](int q) {
        const int s = q % NSTAGE;
        float *pu = su + s * (S::u_slot / 4);
        if (PRE) {
            const float *pd = sd + s * (S::u_slot / 4);
            for (int idx = tid; idx < SUW * SROWS; idx += SNT) {
                const float dv = pd[idx];
                pu[idx] = dv != 0.f ? prerelax * pu[idx] / dv : 0.f;
            }
            __syncthreads();
        }
        constexpr int NYN = SY + 1;   // nodes j0-1 .. j0+31 feed the two copies
        for (int idx = tid; idx < SROWS * NYN; idx += SNT) {
            const int rho = idx / NYN, yn = idx - rho * NYN;
            const float *v = pu + rho * SUW + SUOFF + 3 * yn;
            const float vx = v[0], vy = v[1], vz = v[2];
#pragma unroll
            for (int part = 0; part < SU; ++part) {
                const uint32_t lo = (uint32_t)bf16_part<SU>(vx, part) | ((uint32_t)bf16_part<SU>(vy, part) << 16);
                const uint32_t hi = (uint32_t)bf16_part<SU>(vz, part);
                unsigned char *row = sa + ((size_t)(q & 1) * SU + part) * PLANEB + rho * ROWB;
                if (yn <= 31) *reinterpret_cast<uint2 *>(row + 256 + 8 * yn) = make_uint2(lo, hi);   // odd copy
                if (yn >= 1) *reinterpret_cast<uint2 *>(row + 8 * (yn - 1)) = make_uint2(lo, hi);    // even copy
            }
        }
    };

    // stages issued / consumed (the same on every thread) and whether an MMA
    // batch is outstanding: what an abort has to let finish
    int nissued = 2, nwaited = 0;
    int mma_pending = -1;
    if (tid == 0) {
        issue_stage(0);
        issue_stage(1);
    }
    bool alive = wait_stage(0);
    if (alive) {
        nwaited = 1;
        convert_plane(0);
    }

    // epilogue operands (f, diag, mask) of this thread's node in a plane, one
    // plane ahead of their use so that their latency hides behind a step
    const int jn = j0 + ty, kn = k0 + tz;
    const bool node_in = jn < g.ny && kn < g.nz;
    float fv[3] = {0.f, 0.f, 0.f}, dv[3] = {1.f, 1.f, 1.f}, fn[3], dn[3];
    unsigned mk = 0, mn = 0;
    auto load_epi = [&](int plane, float (&fo)[3], float (&dO)[3], unsigned &mo) {
        fo[0] = fo[1] = fo[2] = 0.f;
        dO[0] = dO[1] = dO[2] = 1.f;
        mo = 0;
        if (!node_in || plane >= ib) return;
        const long long b = L.at(plane, jn, kn);
        mo = mask[g.node(plane, jn, kn)];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (MODE != MODE_APPLY) fo[d] = f[b + d];
            if (MODE == MODE_JACOBI || MODE == MODE_JACOBI_PRE) dO[d] = diag[b + d];
        }
    };
    load_epi(ia, fv, dv, mk);

    float accp[3] = {0.f, 0.f, 0.f};   // contributions of the previous layer to this plane
    const int nsteps = ib - ia + 1;     // element layers ia-1 .. ib-1
    for (int q = 0; alive && q < nsteps; ++q) {
        const int l = ia - 1 + q;      // element layer between node planes l and l+1
        if (q >= 1) load_epi(l + 1, fn, dn, mn);
        if (q + 2 <= nsteps) {
            if (tid == 0) issue_stage(q + 2);
            nissued = q + 3;
        }
        if (!wait_stage(q + 1)) {
            alive = false;
            break;
        }
        nwaited = q + 2;
        convert_plane(q + 1);
        // im2col tile for element column j0+31: row r <-> element row r,
        // K chunk c = 2 h + kc <-> nodes (plane l+h, row r+kc, y j0+31 and j0+32)
        if (tid < SCROWS * 4) {
            const int r = tid >> 2, c = tid & 3, h = c >> 1, kc = c & 1;
            const float *pu = su + ((q + h) % NSTAGE) * (S::u_slot / 4) + (r + kc) * SUW + SUOFF + 3 * 32;
            float vv[8];
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                vv[4 * p] = pu[3 * p];
                vv[4 * p + 1] = pu[3 * p + 1];
                vv[4 * p + 2] = pu[3 * p + 2];
                vv[4 * p + 3] = 0.f;
            }
#pragma unroll
            for (int part = 0; part < SU; ++part) {
                uint32_t w[4];
#pragma unroll
                for (int e2 = 0; e2 < 4; ++e2)
                    w[e2] = (uint32_t)bf16_part<SU>(vv[2 * e2], part) |
                            ((uint32_t)bf16_part<SU>(vv[2 * e2 + 1], part) << 16);
                *reinterpret_cast<uint4 *>(sfix + part * FIXB + core_off(r, 8 * c)) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

        if (tid == 0) {
            // D_t = sum over u parts s, Ke parts k and x faces h of A(t, s, h) B_k(h)
            const uint32_t b0 = smem_u32(sb);
#pragma unroll
            for (int t = 0; t < 4; ++t) {
#pragma unroll
                for (int part = 0; part < SU; ++part)
#pragma unroll
                    for (int k = 0; k < SK; ++k)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            uint64_t da;
                            if (t < 3)
                                da = sdesc(smem_u32(sa + ((size_t)((q + h) & 1) * SU + part) * PLANEB +
                                                    tile_row0(t) * ROWB),
                                           ROWB, 128);
                            else
                                da = sdesc(smem_u32(sfix + part * FIXB + h * 256), 128, 512);
                            mma_bf16(tmem + t * TILE_COLS, da, sdesc(b0 + k * 2048 + h * 256, 128, 512), IDESC,
                                     (part | k | h) ? 1u : 0u);
                        }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(mbar))
                         : "memory");
        }

        const bool ok = mbar_wait_bounded(mbar, (uint32_t)(q & 1), kSweepPolls);
        if (__syncthreads_or(!ok)) {
            alive = false;
            mma_pending = q & 1;
            break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

        // TMEM -> Y (scaled by CX) in shared memory.  Warp w reads TMEM lanes
        // 32 (w % 4) ..; warps 0-3 tile 0, 4-7 tile 1, warp 3 also tile 2
        // (its last element row), warp 4 also the im2col tile.
        const float *cxs = sc + ((q + 1) % NSTAGE) * (S::c_slot / 4);
        auto readback = [&](int t) {
            const int rho = 32 * (warp & 3) + lane;
            int r, ey;
            if (t < 3) {
                const int zr = rho >> 5, grp = (rho >> 3) & 3, m8 = rho & 7;
                r = tile_row0(t) + zr;
                ey = grp < 2 ? 1 + 2 * (8 * grp + m8) : 2 * (8 * (grp - 2) + m8);
            } else {
                r = rho;
                ey = EY - 1;
            }
            float yv[32];
            tmem_ld32(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(t * TILE_COLS), yv);
            if (t == 3 && rho >= SCROWS) return;
            const float cx = cxs[r * SCW + SCOFF + ey];
            float *yo = ys + (r * EY + ey) * YSTR;
#pragma unroll
            for (int a = 0; a < 8; ++a)
#pragma unroll
                for (int d = 0; d < 3; ++d) yo[3 * a + d] = cx * yv[4 * a + d];
        };
        readback(warp < 4 ? 0 : 1);
        if (warp == 3) readback(2);
        if (warp == 4) readback(3);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();

        // node gather: this layer's x = 0 face completes plane l, its x = 1
        // face starts plane l+1
        float acc[3] = {accp[0], accp[1], accp[2]};
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            float t3[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int ez = 0; ez < 2; ++ez)
#pragma unroll
                for (int ey = 0; ey < 2; ++ey) {
                    const int a = local_index(side, 1 - ey, 1 - ez);
                    const float *yo = ys + ((tz + ez) * EY + ty + ey) * YSTR + 3 * a;
                    t3[0] += yo[0];
                    t3[1] += yo[1];
                    t3[2] += yo[2];
                }
            if (side == 0) {
                acc[0] += t3[0];
                acc[1] += t3[1];
                acc[2] += t3[2];
            } else {
                accp[0] = t3[0];
                accp[1] = t3[1];
                accp[2] = t3[2];
            }
        }
        if (l >= ia && node_in) {
            const long long base = L.at(l, jn, kn);
            const float *us = su + (q % NSTAGE) * (S::u_slot / 4) + (tz + 1) * SUW + SUOFF + 3 * (ty + 1);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const bool fixed = (mk >> d) & 1u;
                if (MODE == MODE_APPLY) {
                    out[base + d] = fixed ? 0.f : acc[d];
                } else if (MODE == MODE_DEFECT) {
                    out[base + d] = fixed ? 0.f : fv[d] - acc[d];
                } else {
                    const float rr = fixed ? 0.f : fv[d] - acc[d];
                    out[base + d] = us[d] + omega * rr / dv[d];
                }
            }
        }
        if (q >= 1) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                fv[d] = fn[d];
                dv[d] = dn[d];
            }
            mk = mn;
        }
        __syncthreads();   // Y and the ring slot of plane l are reused next step
    }
    if (!alive) {
        if (tid == 0 && err) atomicExch(err, GPUTO_ERR_TIMEOUT);
        // let outstanding MMAs and tile loads land before TMEM and shared
        // memory are released (bounded again)
        if (mma_pending >= 0) mbar_wait_bounded(mbar, (uint32_t)mma_pending, kSweepPolls);
        for (int q = nwaited; q < nissued; ++q)
            mbar_wait_bounded(tbar + (q % NSTAGE), (uint32_t)((q / NSTAGE) & 1), kSweepPolls);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

template <int MODE, int SU, int SK>
static cudaError_t tc_attr()
{
    return cudaFuncSetAttribute(tc_sweep_kernel<MODE, SU, SK>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)SweepSmem<SU, SK, MODE == MODE_JACOBI_PRE>::bytes);
}

template <int SU, int SK>
static cudaError_t tc_attrs()
{
    cudaError_t e;
    if ((e = tc_attr<MODE_APPLY, SU, SK>()) != cudaSuccess) return e;
    if ((e = tc_attr<MODE_DEFECT, SU, SK>()) != cudaSuccess) return e;
    if ((e = tc_attr<MODE_JACOBI, SU, SK>()) != cudaSuccess) return e;
    return tc_attr<MODE_JACOBI_PRE, SU, SK>();
}

int init_tc_sweep_kernels()
{
    static std::mutex mu;
    static bool done_dev[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && done_dev[dev]) return GPUTO_OK;
    GPUTO_CUDA((tc_attrs<1, 1>()));
    GPUTO_CUDA((tc_attrs<2, 2>()));
    if (dev < 64) done_dev[dev] = true;
    return GPUTO_OK;
}

template <int MODE, int SU, int SK>
static int launch_tc(const Lay &L, const ELay &E, const float *CX, const float *u, const float *f,
                     const float *diag, const uint8_t *mask, float *out, float omega, float prerelax, int xchunk,
                     const int *done, int *err, cudaStream_t st)
{
    constexpr bool PRE = (MODE == MODE_JACOBI_PRE);
    const Grid &g = L.g;
    CUtensorMap mu, md, mc;
    const float *src = PRE ? f : u;
    int s = make_tmap_3d(&mu, src, 4, (uint64_t)L.pitch, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1, L.pitch * 4,
                         L.pitch * 4 * (g.nz + 1), SUW, SROWS, 1);
    if (!s && PRE)
        s = make_tmap_3d(&md, diag, 4, (uint64_t)L.pitch, (uint64_t)g.nz + 1, (uint64_t)g.nx + 1, L.pitch * 4,
                         L.pitch * 4 * (g.nz + 1), SUW, SROWS, 1);
    if (!s)
        s = make_tmap_3d(&mc, CX, 4, (uint64_t)E.pitch, (uint64_t)E.g.nz, (uint64_t)E.g.nx, E.pitch * 4,
                         E.pitch * 4 * E.g.nz, SCW, SCROWS, 1);
    if (s) return s;
    if (!PRE) md = mu;
    const dim3 grid((g.ny + SY - 1) / SY, (g.nz + SZ - 1) / SZ, (g.nx + xchunk - 1) / xchunk);
    tc_sweep_kernel<MODE, SU, SK><<<grid, SNT, SweepSmem<SU, SK, PRE>::bytes, st>>>(
        mu, md, mc, L, xchunk, f, diag, mask, out, omega, prerelax, done, err);
    count_launches(1);
    return launch_fine_faces<float>(MODE, L, E, CX, u, f, diag, mask, out, omega, prerelax, done, st);
}

template <int SU, int SK>
static int launch_tc_modes(int mode, const Lay &L, const ELay &E, const float *CX, const float *u, const float *f,
                           const float *diag, const uint8_t *mask, float *out, float omega, float prerelax,
                           int xchunk, const int *done, int *err, cudaStream_t st)
{
    switch (mode) {
    case MODE_APPLY:
        return launch_tc<MODE_APPLY, SU, SK>(L, E, CX, u, f, diag, mask, out, omega, prerelax, xchunk, done, err, st);
    case MODE_DEFECT:
        return launch_tc<MODE_DEFECT, SU, SK>(L, E, CX, u, f, diag, mask, out, omega, prerelax, xchunk, done, err, st);
    case MODE_JACOBI:
        return launch_tc<MODE_JACOBI, SU, SK>(L, E, CX, u, f, diag, mask, out, omega, prerelax, xchunk, done, err, st);
    default:
        return launch_tc<MODE_JACOBI_PRE, SU, SK>(L, E, CX, u, f, diag, mask, out, omega, prerelax, xchunk, done, err,
                                                   st);
    }
}

int launch_tc_sweep(int parts, int mode, const Lay &L, const ELay &E, const float *CX, const float *u,
                    const float *f, const float *diag, const uint8_t *mask, float *out, float omega,
                    float prerelax, int xchunk, const int *done, int *err, cudaStream_t st)
{
    if (xchunk < 1) xchunk = 16;
    if (parts == 1)
        return launch_tc_modes<1, 1>(mode, L, E, CX, u, f, diag, mask, out, omega, prerelax, xchunk, done, err, st);
    return launch_tc_modes<2, 2>(mode, L, E, CX, u, f, diag, mask, out, omega, prerelax, xchunk, done, err, st);
}

}  // namespace gputo
