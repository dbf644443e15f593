// Compliance sensitivity for callers that cannot allocate device memory.
//
// gputo_compliance_sens_dev() creates its reduction scratch (per-CTA partial
// sums, a completion ticket, the compliance scalar) and a stream with
// cudaMalloc / cudaStreamCreate on its first call.  Some callers cannot let a
// library do that: hosts whose memory manager owns the whole device (a
// MATLAB gpuArray workspace, or a caching allocator that has reserved the
// free memory and must account for every byte), and real-time loops where
// the implicit device synchronisation of cudaMalloc / cudaFree is not
// allowed.  This entry point computes the same result with its scratch in a
// file-scope device array, so it allocates nothing at all.
#include "gputo_internal.h"

#include <mutex>

namespace gputo {

// One partial sum per CTA; each CTA covers kNoAllocElemsPerCta elements.
constexpr int kNoAllocSlots = 8192;
constexpr long long kNoAllocElemsPerCta = 2048;   // 256 threads x 8 elements
constexpr long long kNoAllocMaxElements = kNoAllocSlots * kNoAllocElemsPerCta;  // 16,777,216

struct NoAllocScratch {
    double partial[kNoAllocSlots];
    double compliance;
    unsigned ticket;
};

// The scratch every call shares (about 64 KB, held by every GPU that loads
// the library until the process exits).
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of the scratch, looked up once per device and context (host
// code must not use the symbol itself: on the host it only stands in for the
// device array).  A cudaDeviceReset replaces the device's primary context; the
// context id tells the cached address of the old one apart, and the lookup
// runs again.
static NoAllocScratch *noalloc_scratch_for_current_device(int *status)
{
    static std::mutex mu;
    static NoAllocScratch *addr[64] = {};
    static unsigned long long ctx_of[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) {
        *status = e != cudaSuccess ? cuda_status(e, "cudaGetDevice") : GPUTO_ERR_NO_DEVICE;
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long ctx = current_context_id();
    if (!addr[dev] || ctx == 0 || ctx != ctx_of[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            *status = cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
            return nullptr;
        }
        addr[dev] = static_cast<NoAllocScratch *>(p);
        ctx_of[dev] = current_context_id();   // the lookup made the context current
    }
    *status = GPUTO_OK;
    return addr[dev];
}

}  // namespace gputo

extern "C" int gputo_compliance_sens_noalloc_dev(const double *Ke0, const double *U,
                                                 const double *CX, const double *dsK, int nelx,
                                                 int nely, int nelz, double *ce, double *dc,
                                                 double *compliance, void *stream)
{
    using namespace gputo;
    if (!Ke0 || !U || nelx <= 0 || nely <= 0 || nelz <= 0 || (dc && !dsK) || (compliance && !CX))
        return GPUTO_ERR_ARG;
    const Grid g{nelx, nely, nelz};
    if (g.nel() > kNoAllocMaxElements) {
        set_error("gputo_compliance_sens_noalloc_dev: " + std::to_string(g.nel()) +
                  " elements exceed the 16,777,216-element limit of its fixed scratch; "
                  "use gputo_compliance_sens_dev for larger grids");
        return GPUTO_ERR_ARG;
    }
    int st = GPUTO_OK;
    NoAllocScratch *s = noalloc_scratch_for_current_device(&st);
    if (!s) return st;
    cudaStream_t strm = static_cast<cudaStream_t>(stream);
    st = upload_fine_ke(Ke0, strm);   // constant-memory copy: no allocation
    if (st) return st;
    // the completion ticket must start at zero; partials are overwritten
    GPUTO_CUDA(cudaMemsetAsync(&s->ticket, 0, sizeof(unsigned), strm));
    const int nb = (int)((g.nel() + kNoAllocElemsPerCta - 1) / kNoAllocElemsPerCta);
    launch_element_energy_blocks(g, U, CX, dsK, ce, dc, s->partial, &s->ticket,
                                 compliance ? &s->compliance : nullptr, nb, strm);
    if (compliance)
        GPUTO_CUDA(cudaMemcpyAsync(compliance, &s->compliance, sizeof(double),
                                   cudaMemcpyDeviceToHost, strm));
    GPUTO_CUDA(cudaStreamSynchronize(strm));
    GPUTO_CUDA(cudaGetLastError());
    return GPUTO_OK;
}
