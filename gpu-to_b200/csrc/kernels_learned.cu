// The learned coarse-grid correction network: forward, backward and Adam
// kernels, written for this project (the reference has no learned part).
//
// Network (level-2 node grid, channels-first [C][X][Z][Y], Y fastest as in
// the solver's node order): three 3x3x3 convolutions 4 -> 16 -> 32 -> 64 with
// bias and ReLU, zero padding, then a 1x1x1 convolution 64 -> 3.  Weights are
// kept in FP32 for training and used rounded to BF16; activations and sums are
// FP32.  Flat parameter layout per layer: w[co][ci][tap] then b[co], tap =
// 9 (dx+1) + 3 (dz+1) + (dy+1).
//
// Convolutions are direct: one thread per node computes a chunk of output
// channels, the chunk's weights sit in shared memory and every thread of a
// warp reads the same weight at the same time (broadcast), the input reads
// are coalesced along Y.  Weight gradients are reduced per (co, ci) pair by
// one CTA in a fixed order, so training is deterministic.
#include <cuda_bf16.h>

#include <cmath>
#include <vector>

#include "gputo_internal.h"

namespace gputo {

namespace {

__host__ __device__ constexpr int net_ch(int l) { return l == 0 ? 4 : l == 1 ? 16 : l == 2 ? 32 : l == 3 ? 64 : 3; }
__host__ __device__ constexpr int net_k(int l) { return l == 3 ? 1 : 3; }

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

constexpr int kNetThreads = 128;

// Offset of tap t of a 3x3x3 stencil, and whether it stays inside the grid.
__device__ __forceinline__ bool tap_in(int t, int xi, int zi, int yi, const NetDims &d, long long &off)
{
    const int dx = t / 9 - 1, dz = (t / 3) % 3 - 1, dy = t % 3 - 1;
    off = ((long long)dx * d.Z + dz) * d.Y + dy;
    return (unsigned)(xi + dx) < (unsigned)d.X && (unsigned)(zi + dz) < (unsigned)d.Z && (unsigned)(yi + dy) < (unsigned)d.Y;
}

template <int CIN, int COT, int K, bool RELU>
__global__ void __launch_bounds__(kNetThreads)
conv_fwd_kernel(const float *__restrict__ x, const float *__restrict__ w, const float *__restrict__ b,
                float *__restrict__ y, NetDims d, int cout)
{
    constexpr int K3 = K * K * K;
    extern __shared__ float ws[];   // [CIN][K3][COT], BF16-rounded
    const int co0 = blockIdx.y * COT;
    for (int idx = threadIdx.x; idx < CIN * K3 * COT; idx += blockDim.x) {
        const int c = idx % COT, rest = idx / COT, t = rest % K3, ci = rest / K3;
        const int co = co0 + c;
        ws[idx] = co < cout ? bf16r(w[((long long)co * CIN + ci) * K3 + t]) : 0.f;
    }
    __syncthreads();
    const long long N = d.n();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int yi = (int)(n % d.Y);
    const long long r = n / d.Y;
    const int zi = (int)(r % d.Z), xi = (int)(r / d.Z);
    float acc[COT];
#pragma unroll
    for (int c = 0; c < COT; ++c) acc[c] = co0 + c < cout ? b[co0 + c] : 0.f;
    for (int ci = 0; ci < CIN; ++ci) {
        const float *xc = x + (long long)ci * N;
#pragma unroll
        for (int t = 0; t < K3; ++t) {
            long long off = 0;
            const bool in = K == 1 ? true : tap_in(t, xi, zi, yi, d, off);
            const float v = in ? xc[n + off] : 0.f;
            const float *wr = ws + (ci * K3 + t) * COT;
#pragma unroll
            for (int c = 0; c < COT; ++c) acc[c] = fmaf(wr[c], v, acc[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < COT; ++c)
        if (co0 + c < cout) y[(long long)(co0 + c) * N + n] = RELU ? fmaxf(acc[c], 0.f) : acc[c];
}

// gx[ci](n) = sum_co sum_tap w[co][ci][tap] g[co](n - offset(tap))
template <int COUT, int CIT, int K>
__global__ void __launch_bounds__(kNetThreads)
conv_bwd_data_kernel(const float *__restrict__ g, const float *__restrict__ w, float *__restrict__ gx, NetDims d,
                     int cin)
{
    constexpr int K3 = K * K * K;
    extern __shared__ float ws[];   // [COUT][K3][CIT]
    const int ci0 = blockIdx.y * CIT;
    for (int idx = threadIdx.x; idx < COUT * K3 * CIT; idx += blockDim.x) {
        const int c = idx % CIT, rest = idx / CIT, t = rest % K3, co = rest / K3;
        const int ci = ci0 + c;
        ws[idx] = ci < cin ? bf16r(w[((long long)co * cin + ci) * K3 + t]) : 0.f;
    }
    __syncthreads();
    const long long N = d.n();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    const int yi = (int)(n % d.Y);
    const long long r = n / d.Y;
    const int zi = (int)(r % d.Z), xi = (int)(r / d.Z);
    float acc[CIT];
#pragma unroll
    for (int c = 0; c < CIT; ++c) acc[c] = 0.f;
    for (int co = 0; co < COUT; ++co) {
        const float *gc = g + (long long)co * N;
#pragma unroll
        for (int t = 0; t < K3; ++t) {
            long long off = 0;
            // output node n - offset(t): the mirrored tap of n
            const bool in = K == 1 ? true : tap_in(K3 - 1 - t, xi, zi, yi, d, off);
            const float v = in ? gc[n + off] : 0.f;
            const float *wr = ws + (co * K3 + t) * CIT;
#pragma unroll
            for (int c = 0; c < CIT; ++c) acc[c] = fmaf(wr[c], v, acc[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < CIT; ++c)
        if (ci0 + c < cin) gx[(long long)(ci0 + c) * N + n] = acc[c];
}

// gw[co][ci][tap] += sum_n g[co](n) x[ci](n + offset(tap)): one CTA per (co, ci)
template <int K>
__global__ void __launch_bounds__(256)
conv_bwd_weight_kernel(const float *__restrict__ g, const float *__restrict__ x, float *__restrict__ gw, NetDims d,
                       int cin)
{
    constexpr int K3 = K * K * K;
    const int co = blockIdx.x / cin, ci = blockIdx.x % cin;
    const long long N = d.n();
    const float *gc = g + (long long)co * N, *xc = x + (long long)ci * N;
    float acc[K3];
#pragma unroll
    for (int t = 0; t < K3; ++t) acc[t] = 0.f;
    for (long long n = threadIdx.x; n < N; n += blockDim.x) {
        const float gv = gc[n];
        if (gv == 0.f) continue;
        const int yi = (int)(n % d.Y);
        const long long r = n / d.Y;
        const int zi = (int)(r % d.Z), xi = (int)(r / d.Z);
#pragma unroll
        for (int t = 0; t < K3; ++t) {
            long long off = 0;
            const bool in = K == 1 ? true : tap_in(t, xi, zi, yi, d, off);
            if (in) acc[t] = fmaf(gv, xc[n + off], acc[t]);
        }
    }
    __shared__ float red[8][K3];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int t = 0; t < K3; ++t) {
        float v = acc[t];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[wid][t] = v;
    }
    __syncthreads();
    if (threadIdx.x < K3) {
        float s = 0.f;
        for (int q = 0; q < 8; ++q) s += red[q][threadIdx.x];
        gw[((long long)co * cin + ci) * K3 + threadIdx.x] += s;
    }
}

// gb[co] += sum_n g[co](n)
__global__ void __launch_bounds__(256) bias_grad_kernel(const float *__restrict__ g, float *__restrict__ gb, NetDims d)
{
    const long long N = d.n();
    const float *gc = g + (long long)blockIdx.x * N;
    float v = 0.f;
    for (long long n = threadIdx.x; n < N; n += blockDim.x) v += gc[n];
    __shared__ float red[8];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int q = 0; q < 8; ++q) s += red[q];
        gb[blockIdx.x] += s;
    }
}

// g <- g where the layer's ReLU output is positive, else 0
__global__ void relu_mask_kernel(float *__restrict__ g, const float *__restrict__ y, long long n)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(y[i] > 0.f)) g[i] = 0.f;
}

// Masked mean square error of one sample: partial sums per CTA, then a
// single-CTA finish that also writes the gradient scale; fixed order.
__global__ void __launch_bounds__(256)
mse_partial_kernel(const float *__restrict__ y, const float *__restrict__ t, const float *__restrict__ m, long long n,
                   double *__restrict__ part)
{
    double s = 0.0, c = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double r = (double)y[i] - (double)t[i];
        s += (double)m[i] * r * r;
        c += (double)m[i];
    }
    __shared__ double rs[8], rc[8];
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) rs[threadIdx.x >> 5] = s, rc[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < 8; ++q) a += rs[q], b += rc[q];
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = b;
    }
}

__global__ void mse_finish_kernel(const double *__restrict__ part, int nb, double *__restrict__ loss_acc,
                                  float *__restrict__ gscale)
{
    if (threadIdx.x != 0) return;
    double a = 0.0, b = 0.0;
    for (int q = 0; q < nb; ++q) a += part[2 * q], b += part[2 * q + 1];
    const double den = b > 1.0 ? b : 1.0;
    *loss_acc += a / den;
    *gscale = (float)(2.0 / den);
}

__global__ void mse_grad_kernel(const float *__restrict__ y, const float *__restrict__ t, const float *__restrict__ m,
                                long long n, const float *__restrict__ gscale, float *__restrict__ g)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) g[i] = *gscale * m[i] * (y[i] - t[i]);
}

__global__ void adam_kernel(float *__restrict__ p, float *__restrict__ g, float *__restrict__ m1, float *__restrict__ m2,
                            long long n, float lr, float gscale, float bc1, float bc2)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] * gscale;
    const float a = 0.9f * m1[i] + 0.1f * gi;
    const float v = 0.999f * m2[i] + 0.001f * gi * gi;
    m1[i] = a;
    m2[i] = v;
    p[i] -= lr * (a / bc1) / (sqrtf(v / bc2) + 1e-8f);
    g[i] = 0.f;
}

template <int CIN, int COT, int K, bool RELU>
void launch_fwd(const float *x, const float *w, const float *b, float *y, const NetDims &d, int cout, cudaStream_t st)
{
    constexpr int K3 = K * K * K;
    const size_t smem = sizeof(float) * CIN * K3 * COT;
    const dim3 grid((unsigned)((d.n() + kNetThreads - 1) / kNetThreads), (unsigned)((cout + COT - 1) / COT));
    conv_fwd_kernel<CIN, COT, K, RELU><<<grid, kNetThreads, smem, st>>>(x, w, b, y, d, cout);
    count_launches(1);
}

template <int COUT, int CIT, int K>
void launch_bwd_data(const float *g, const float *w, float *gx, const NetDims &d, int cin, cudaStream_t st)
{
    constexpr int K3 = K * K * K;
    const size_t smem = sizeof(float) * COUT * K3 * CIT;
    const dim3 grid((unsigned)((d.n() + kNetThreads - 1) / kNetThreads), (unsigned)((cin + CIT - 1) / CIT));
    conv_bwd_data_kernel<COUT, CIT, K><<<grid, kNetThreads, smem, st>>>(g, w, gx, d, cin);
    count_launches(1);
}

}  // namespace

// ---------------------------------------------------------------------------
// Net: parameters, Adam state and activation buffers on one device
// ---------------------------------------------------------------------------

long long Net::num_params()
{
    long long s = 0;
    for (int l = 0; l < 4; ++l) s += (long long)net_ch(l + 1) * net_ch(l) * net_k(l) * net_k(l) * net_k(l) + net_ch(l + 1);
    return s;
}

long long Net::param_offset(int l, bool bias)
{
    long long o = 0;
    for (int q = 0; q < l; ++q) o += (long long)net_ch(q + 1) * net_ch(q) * net_k(q) * net_k(q) * net_k(q) + net_ch(q + 1);
    if (bias) o += (long long)net_ch(l + 1) * net_ch(l) * net_k(l) * net_k(l) * net_k(l);
    return o;
}

Net::~Net()
{
    for (void *p : owned) cudaFree(p);
    for (int l = 1; l <= 4; ++l) cudaFree(act[l]);
    cudaFree(gA);
    cudaFree(gB);
}

int Net::create(unsigned long long seed)
{
    GPUTO_CUDA(cudaGetDevice(&device));
    const long long np = num_params();
    for (float **p : {&params, &grads, &m1, &m2}) {
        GPUTO_CUDA(cudaMalloc(p, sizeof(float) * np));
        owned.push_back(*p);
        GPUTO_CUDA(cudaMemset(*p, 0, sizeof(float) * np));
    }
    GPUTO_CUDA(cudaMalloc(&part, sizeof(double) * 2 * 1024 + sizeof(double) + sizeof(float)));
    owned.push_back(part);
    loss_acc = part + 2 * 1024;   // part: 2048 doubles of reduction scratch
    gscale = reinterpret_cast<float *>(loss_acc + 1);
    // He-normal initial weights (last layer scaled by 0.1), zero biases;
    // a fixed generator so that a seed reproduces the network
    std::vector<float> h((size_t)np, 0.f);
    unsigned long long s = seed * 6364136223846793005ULL + 1442695040888963407ULL;
    auto uni = [&]() {
        s = s * 6364136223846793005ULL + 1442695040888963407ULL;
        return ((s >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < 4; ++l) {
        const long long nw = (long long)net_ch(l + 1) * net_ch(l) * net_k(l) * net_k(l) * net_k(l);
        const double std = std::sqrt(2.0 / ((double)net_ch(l) * net_k(l) * net_k(l) * net_k(l))) * (l == 3 ? 0.1 : 1.0);
        const long long o = param_offset(l, false);
        for (long long i = 0; i < nw; ++i) {
            const double u1 = uni(), u2 = uni();
            h[(size_t)(o + i)] = (float)(std * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
        }
    }
    GPUTO_CUDA(cudaMemcpy(params, h.data(), sizeof(float) * np, cudaMemcpyHostToDevice));
    return GPUTO_OK;
}

int Net::reserve(long long n)
{
    if (n <= cap_n) return GPUTO_OK;
    for (int l = 1; l <= 4; ++l) cudaFree(act[l]), act[l] = nullptr;
    cudaFree(gA), cudaFree(gB);
    gA = gB = nullptr;
    cap_n = 0;
    const int chs[5] = {4, 16, 32, 64, 3};
    for (int l = 1; l <= 4; ++l) GPUTO_CUDA(cudaMalloc(&act[l], sizeof(float) * chs[l] * n));
    GPUTO_CUDA(cudaMalloc(&gA, sizeof(float) * 64 * n));
    GPUTO_CUDA(cudaMalloc(&gB, sizeof(float) * 64 * n));
    cap_n = n;
    return GPUTO_OK;
}

int init_net_kernels()
{
    static bool done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && done[dev]) return GPUTO_OK;
    GPUTO_CUDA(cudaFuncSetAttribute(conv_fwd_kernel<32, 16, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    32 * 27 * 16 * 4));
    GPUTO_CUDA(cudaFuncSetAttribute(conv_bwd_data_kernel<64, 16, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    64 * 27 * 16 * 4));
    GPUTO_CUDA(cudaFuncSetAttribute(conv_bwd_data_kernel<32, 16, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    32 * 27 * 16 * 4));
    if (dev < 64) done[dev] = true;
    return GPUTO_OK;
}

int Net::forward(const float *x, const NetDims &d, float *y, cudaStream_t st)
{
    int s = reserve(d.n());
    if (s) return s;
    act[0] = const_cast<float *>(x);
    const float *p = params;
    launch_fwd<4, 16, 3, true>(x, p + param_offset(0, false), p + param_offset(0, true), act[1], d, 16, st);
    launch_fwd<16, 16, 3, true>(act[1], p + param_offset(1, false), p + param_offset(1, true), act[2], d, 32, st);
    launch_fwd<32, 16, 3, true>(act[2], p + param_offset(2, false), p + param_offset(2, true), act[3], d, 64, st);
    launch_fwd<64, 3, 1, false>(act[3], p + param_offset(3, false), p + param_offset(3, true), y ? y : act[4], d, 3,
                                st);
    return GPUTO_OK;
}

// Loss of one sample (x, target t, mask m) added to loss_acc, gradients
// added to grads.
int Net::accumulate(const float *x, const float *t, const float *m, const NetDims &d, cudaStream_t st)
{
    int s = forward(x, d, nullptr, st);
    if (s) return s;
    const long long N = d.n(), n3 = 3 * N;
    const int nb = (int)std::min<long long>(1024, (n3 + 255) / 256);
    mse_partial_kernel<<<nb, 256, 0, st>>>(act[4], t, m, n3, part);
    mse_finish_kernel<<<1, 32, 0, st>>>(part, nb, loss_acc, gscale);
    mse_grad_kernel<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(act[4], t, m, n3, gscale, gA);
    count_launches(3);
    return backward_from(d, st);
}

int Net::adam(float lr, int nsamples, cudaStream_t st)
{
    ++step;
    const float bc1 = 1.f - std::pow(0.9f, (float)step), bc2 = 1.f - std::pow(0.999f, (float)step);
    const long long np = num_params();
    adam_kernel<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(params, grads, m1, m2, np, lr,
                                                             1.f / (float)std::max(nsamples, 1), bc1, bc2);
    count_launches(1);
    return GPUTO_OK;
}

// ---------------------------------------------------------------------------
// level-2 features and the correction's way back to the fine grid
// ---------------------------------------------------------------------------

// Density feature at a level-2 node: mean element scale of the adjacent
// level-2 elements (each the mean of its fine elements), (log10 + 9) / 9.
__global__ void net_density_kernel(Grid g2, Grid gf, const double *__restrict__ CXf, float *__restrict__ dens2)
{
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= g2.nnod()) return;
    const int j = (int)(n % (g2.ny + 1));
    const long long r = n / (g2.ny + 1);
    const int k = (int)(r % (g2.nz + 1)), i = (int)(r / (g2.nz + 1));
    const int fx = gf.nx / g2.nx, fy = gf.ny / g2.ny, fz = gf.nz / g2.nz;
    double s = 0.0;
    int cnt = 0;
    for (int ex = i - 1; ex <= i; ++ex)
        for (int ez = k - 1; ez <= k; ++ez)
            for (int ey = j - 1; ey <= j; ++ey) {
                if (ex < 0 || ex >= g2.nx || ez < 0 || ez >= g2.nz || ey < 0 || ey >= g2.ny) continue;
                double c = 0.0;
                for (int a = 0; a < fx; ++a)
                    for (int b = 0; b < fz; ++b)
                        for (int q = 0; q < fy; ++q) c += CXf[gf.elem(ex * fx + a, ey * fy + q, ez * fz + b)];
                s += c / (fx * fy * fz);
                ++cnt;
            }
    const double m = cnt ? s / cnt : 1e-9;
    dens2[n] = (float)((log10(fmax(m, 1e-9)) + 9.0) / 9.0);
}

void launch_net_density(const Grid &g2, const Grid &gf, const double *CXf, float *dens2, cudaStream_t st)
{
    net_density_kernel<<<(unsigned)((g2.nnod() + 255) / 256), 256, 0, st>>>(g2, gf, CXf, dens2);
    count_launches(1);
}

// The network works in Jacobi-scaled units, in which the level-2 operator
// has a unit diagonal: input r~ = D^-1/2 r, output e~ with e = D^-1/2 e~,
// both divided by s = RMS of r~ (free dofs; fixed dofs have r = 0).  That
// keeps the stiffness contrast of SIMP designs (1e9 here) out of the values
// the network sees.

// s = RMS of D^-1/2 r2 (one CTA, fixed order)
__global__ void __launch_bounds__(1024) net_rms_kernel(Lay L2, const float *__restrict__ r2,
                                                     const float *__restrict__ diag2, float *__restrict__ s,
                                                     const int *__restrict__ done)
{
    if (done && *done) return;
    const Grid &g = L2.g;
    const long long nn = g.nnod();
    double acc = 0.0;
    for (long long n = threadIdx.x; n < nn; n += blockDim.x) {
        const int j = (int)(n % (g.ny + 1));
        const long long r = n / (g.ny + 1);
        const int k = (int)(r % (g.nz + 1)), i = (int)(r / (g.nz + 1));
        const long long b = L2.at(i, j, k);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double dv = diag2[b + d];
            if (dv > 0.0) acc += (double)r2[b + d] * r2[b + d] / dv;
        }
    }
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        const double rms = sqrt(t / (3.0 * (double)nn));
        *s = rms > 0.0 ? (float)rms : 1.f;
    }
}

__global__ void net_features_kernel(Lay L2, const float *__restrict__ r2, const float *__restrict__ diag2,
                                    const float *__restrict__ dens2, float *__restrict__ x, float *__restrict__ dsq,
                                    const float *__restrict__ s, const int *__restrict__ done)
{
    if (done && *done) return;
    const Grid &g = L2.g;
    const long long nn = g.nnod();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const int j = (int)(n % (g.ny + 1));
    const long long r = n / (g.ny + 1);
    const int k = (int)(r % (g.nz + 1)), i = (int)(r / (g.nz + 1));
    const float inv = 1.f / *s;
    const long long b = L2.at(i, j, k);
    x[n] = dens2[n];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float dv = diag2[b + d];
        const float sq = dv > 0.f ? sqrtf(dv) : 1.f;
        x[(1 + d) * nn + n] = r2[b + d] / sq * inv;
        if (dsq) dsq[d * nn + n] = sq;
    }
}

void launch_net_features(const Lay &L2, const float *r2, const float *diag2, const float *dens2, float *x,
                         float *dsq, float *s, const int *done, cudaStream_t st)
{
    net_rms_kernel<<<1, 1024, 0, st>>>(L2, r2, diag2, s, done);
    net_features_kernel<<<(unsigned)((L2.g.nnod() + 255) / 256), 256, 0, st>>>(L2, r2, diag2, dens2, x, dsq, s,
                                                                               done);
    count_launches(2);
}

// e2 = s D^-1/2 y at the free dofs of level 2, 0 at fixed dofs
__global__ void net_output_kernel(Lay L2, const float *__restrict__ y, const float *__restrict__ diag2,
                                  const float *__restrict__ s, const uint8_t *__restrict__ mask2,
                                  float *__restrict__ e2, const int *__restrict__ done)
{
    if (done && *done) return;
    const Grid &g = L2.g;
    const long long nn = g.nnod();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const int j = (int)(n % (g.ny + 1));
    const long long r = n / (g.ny + 1);
    const int k = (int)(r % (g.nz + 1)), i = (int)(r / (g.nz + 1));
    const unsigned m = mask2[n];
    const float sc = *s;
    const long long b = L2.at(i, j, k);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float dv = diag2[b + d];
        e2[b + d] = ((m >> d) & 1u) || !(dv > 0.f) ? 0.f : sc * y[d * nn + n] / sqrtf(dv);
    }
}

void launch_net_output(const Lay &L2, const float *y, const float *diag2, const float *s, const uint8_t *mask2,
                       float *e2, const int *done, cudaStream_t st)
{
    net_output_kernel<<<(unsigned)((L2.g.nnod() + 255) / 256), 256, 0, st>>>(L2, y, diag2, s, mask2, e2, done);
    count_launches(1);
}

__global__ void add_f2d_kernel(long long n, const float *__restrict__ e, double *__restrict__ z,
                               const int *__restrict__ done)
{
    if (done && *done) return;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] += (double)e[i];
}

void launch_add_f2d(long long n, const float *e, double *z, const int *done, cudaStream_t st)
{
    add_f2d_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, e, z, done);
    count_launches(1);
}

// Loss mask of the level-2 dofs: 1 free, 0 fixed, channels-first [3][n]
__global__ void net_mask_kernel(Grid g2, const uint8_t *__restrict__ mask2, float *__restrict__ m)
{
    const long long nn = g2.nnod();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const unsigned b = mask2[n];
#pragma unroll
    for (int d = 0; d < 3; ++d) m[d * nn + n] = ((b >> d) & 1u) ? 0.f : 1.f;
}

void launch_net_mask(const Grid &g2, const uint8_t *mask2, float *m, cudaStream_t st)
{
    net_mask_kernel<<<(unsigned)((g2.nnod() + 255) / 256), 256, 0, st>>>(g2, mask2, m);
    count_launches(1);
}

// Values of a fine dense vector (the reference's layout) at the level-2
// nodes (fine node (fx i, fy j, fz k)), channels-first [3][n]
__global__ void level2_inject_kernel(Grid g2, Grid gf, const double *__restrict__ v, float *__restrict__ out)
{
    const long long nn = g2.nnod();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const int j = (int)(n % (g2.ny + 1));
    const long long r = n / (g2.ny + 1);
    const int k = (int)(r % (g2.nz + 1)), i = (int)(r / (g2.nz + 1));
    const long long nf = gf.node(i * (gf.nx / g2.nx), j * (gf.ny / g2.ny), k * (gf.nz / g2.nz));
#pragma unroll
    for (int d = 0; d < 3; ++d) out[d * nn + n] = (float)v[3 * nf + d];
}

void launch_level2_inject(const Grid &g2, const Grid &gf, const double *v, float *out, cudaStream_t st)
{
    level2_inject_kernel<<<(unsigned)((g2.nnod() + 255) / 256), 256, 0, st>>>(g2, gf, v, out);
    count_launches(1);
}

// ---------------------------------------------------------------------------
// energy loss of the correction (level-2 operator A2 in the scaled units)
// ---------------------------------------------------------------------------
//
// With the correction c = s D^-1/2 y added after the V-cycle, the energy of
// the remaining error is, up to a constant, c'A2 c - 2 c'g2 with
// g2 = P'(r - A z) the twice-restricted post-V-cycle residual and A2 = P'AP
// the Galerkin level-2 operator.  Divided by s^2 this is
//   L = y'A~y - 2 y'g~,   A~ = D^-1/2 A2 D^-1/2,  g~ = D^-1/2 g2 / s,
// with gradient 2 (A~y - g~).  L(0) = 0: any learned correction lowers it.

// w = D^-1/2 y in the padded level-2 layout (0 at fixed dofs)
__global__ void net_to_padded_kernel(Lay L2, const float *__restrict__ y, const float *__restrict__ diag2,
                                     const uint8_t *__restrict__ mask2, float *__restrict__ w)
{
    const Grid &g = L2.g;
    const long long nn = g.nnod();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const int j = (int)(n % (g.ny + 1));
    const long long r = n / (g.ny + 1);
    const int k = (int)(r % (g.nz + 1)), i = (int)(r / (g.nz + 1));
    const unsigned m = mask2[n];
    const long long b = L2.at(i, j, k);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float dv = diag2[b + d];
        w[b + d] = ((m >> d) & 1u) || !(dv > 0.f) ? 0.f : y[d * nn + n] / sqrtf(dv);
    }
}

// gy = 2 (D^-1/2 q - g~), partial sums of y'(D^-1/2 q) - 2 y'g~ per CTA
__global__ void __launch_bounds__(256)
net_energy_kernel(Lay L2, const float *__restrict__ y, const float *__restrict__ q, const float *__restrict__ diag2,
                  const float *__restrict__ gt, const uint8_t *__restrict__ mask2, float *__restrict__ gy,
                  double *__restrict__ part)
{
    const Grid &g = L2.g;
    const long long nn = g.nnod();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (n < nn) {
        const int j = (int)(n % (g.ny + 1));
        const long long r = n / (g.ny + 1);
        const int k = (int)(r % (g.nz + 1)), i = (int)(r / (g.nz + 1));
        const unsigned m = mask2[n];
        const long long b = L2.at(i, j, k);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const float dv = diag2[b + d];
            const bool free_dof = !((m >> d) & 1u) && dv > 0.f;
            const float aq = free_dof ? q[b + d] / sqrtf(dv) : 0.f;
            const float gv = free_dof ? gt[d * nn + n] : 0.f;
            const float yv = free_dof ? y[d * nn + n] : 0.f;
            gy[d * nn + n] = 2.f * (aq - gv);
            acc += (double)yv * aq - 2.0 * (double)yv * gv;
        }
    }
    __shared__ double red[8];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += red[w];
        part[blockIdx.x] = s;
    }
}

__global__ void net_energy_finish_kernel(const double *__restrict__ part, int nb, double *__restrict__ loss_acc)
{
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int q = 0; q < nb; ++q) s += part[q];
    *loss_acc += s;
}

void launch_net_to_padded(const Lay &L2, const float *y, const float *diag2, const uint8_t *mask2, float *w,
                          cudaStream_t st)
{
    net_to_padded_kernel<<<(unsigned)((L2.g.nnod() + 255) / 256), 256, 0, st>>>(L2, y, diag2, mask2, w);
    count_launches(1);
}

int launch_net_energy(const Lay &L2, const float *y, const float *q, const float *diag2, const float *gt,
                      const uint8_t *mask2, float *gy, double *part, int part_cap, double *loss_acc, cudaStream_t st)
{
    const int nb = (int)((L2.g.nnod() + 255) / 256);
    if (nb > part_cap) {
        set_error("level-2 grid too large for the network loss scratch");
        return GPUTO_ERR_ARG;
    }
    net_energy_kernel<<<nb, 256, 0, st>>>(L2, y, q, diag2, gt, mask2, gy, part);
    net_energy_finish_kernel<<<1, 32, 0, st>>>(part, nb, loss_acc);
    count_launches(2);
    return GPUTO_OK;
}

// The backward pass from a given output gradient gA (3 channels); adds to grads.
int Net::backward_from(const NetDims &d, cudaStream_t st)
{
    const long long N = d.n();
    float *g = gA, *gn = gB;
    for (int l = 3; l >= 0; --l) {
        const int cin = net_ch(l), cout = net_ch(l + 1);
        float *gw = grads + param_offset(l, false), *gb = grads + param_offset(l, true);
        if (l < 3) {
            relu_mask_kernel<<<(unsigned)((cout * N + 255) / 256), 256, 0, st>>>(g, act[l + 1], cout * N);
            count_launches(1);
        }
        if (net_k(l) == 3)
            conv_bwd_weight_kernel<3><<<cout * cin, 256, 0, st>>>(g, act[l], gw, d, cin);
        else
            conv_bwd_weight_kernel<1><<<cout * cin, 256, 0, st>>>(g, act[l], gw, d, cin);
        bias_grad_kernel<<<cout, 256, 0, st>>>(g, gb, d);
        count_launches(2);
        if (l == 0) break;
        const float *w = params + param_offset(l, false);
        switch (l) {
        case 3: launch_bwd_data<3, 16, 1>(g, w, gn, d, 64, st); break;
        case 2: launch_bwd_data<64, 16, 3>(g, w, gn, d, 32, st); break;
        default: launch_bwd_data<32, 16, 3>(g, w, gn, d, 16, st); break;
        }
        std::swap(g, gn);
    }
    return GPUTO_OK;
}

// g~ = D^-1/2 v2 / s at the level-2 nodes, channels-first (0 at fixed dofs),
// for a padded level-2 vector v2
__global__ void net_energy_rhs_kernel(Lay L2, const float *__restrict__ v2, const float *__restrict__ diag2,
                                      const uint8_t *__restrict__ mask2, float scale, float *__restrict__ gt)
{
    const Grid &g = L2.g;
    const long long nn = g.nnod();
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const int j = (int)(n % (g.ny + 1));
    const long long r = n / (g.ny + 1);
    const int k = (int)(r % (g.nz + 1)), i = (int)(r / (g.nz + 1));
    const unsigned m = mask2[n];
    const long long b = L2.at(i, j, k);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float dv = diag2[b + d];
        gt[d * nn + n] = ((m >> d) & 1u) || !(dv > 0.f) ? 0.f : v2[b + d] / sqrtf(dv) / scale;
    }
}

void launch_net_energy_rhs(const Lay &L2, const float *v2, const float *diag2, const uint8_t *mask2, float scale,
                           float *gt, cudaStream_t st)
{
    net_energy_rhs_kernel<<<(unsigned)((L2.g.nnod() + 255) / 256), 256, 0, st>>>(L2, v2, diag2, mask2, scale, gt);
    count_launches(1);
}

}  // namespace gputo
