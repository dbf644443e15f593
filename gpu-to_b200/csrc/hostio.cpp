// Host <-> device copies for the entry points that take host arrays (the MEX
// drop-ins and the host-buffer design steps), and the device workspace they
// reuse between calls.
//
// A caller's arrays are ordinary (pageable) memory.  Each copy goes through
// two pinned chunks of kChunk bytes: while the DMA engine moves one chunk,
// host threads copy the next one between the caller's array and the other
// pinned chunk.  The host-side copy is split over copy_threads() threads, so
// the copy is not limited by one core's memcpy bandwidth (environment
// variable GPUTO_COPY_THREADS, 1-64, read once; default kCopyThreads, at most
// the host's hardware threads).
//
// The device buffers are grown on demand and kept, so a design loop that calls
// these entry points does not allocate and free device memory every time
// (cudaFree also waits for the whole device).
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "gputo_internal.h"

namespace gputo {

namespace {

constexpr size_t kChunk = size_t(8) << 20;   // bytes per pinned chunk
constexpr int kCopyThreads = 4;              // default host threads per chunk copy
constexpr size_t kMinSplit = size_t(1) << 20;

// Runs job(i) for i in [0, parts) on a few persistent threads plus the caller.
class CopyPool {
  public:
    explicit CopyPool(int n)
    {
        for (int i = 0; i < n; ++i) workers_.emplace_back([this] { loop(); });
    }
    void run(int parts, const std::function<void(int)> &job)
    {
        std::unique_lock<std::mutex> lk(mu_);
        job_ = &job;
        parts_ = parts;
        next_ = 0;
        pending_ = parts;
        ++gen_;
        cv_.notify_all();
        lk.unlock();
        work();
        lk.lock();
        done_cv_.wait(lk, [this] { return pending_ == 0; });
        job_ = nullptr;
    }

  private:
    void work()
    {
        for (;;) {
            int i;
            const std::function<void(int)> *job;
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (!job_ || next_ >= parts_) return;
                i = next_++;
                job = job_;
            }
            (*job)(i);
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0) done_cv_.notify_all();
        }
    }
    void loop()
    {
        unsigned long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
            }
            work();
        }
    }
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)> *job_ = nullptr;
    int parts_ = 0, next_ = 0, pending_ = 0;
    unsigned long gen_ = 0;
    std::vector<std::thread> workers_;
};

int copy_threads()
{
    static const int n = [] {
        int v = kCopyThreads;
        if (const char *e = std::getenv("GPUTO_COPY_THREADS")) {
            const int a = std::atoi(e);
            if (a >= 1 && a <= 64) v = a;
        }
        const int hw = (int)std::thread::hardware_concurrency();
        return (hw > 0 && v > hw) ? hw : v;
    }();
    return n;
}

CopyPool &pool()
{
    // never destroyed: its threads wait on the pool until the process ends
    static CopyPool *p = new CopyPool(copy_threads() - 1);
    return *p;
}

void par_memcpy(void *dst, const void *src, size_t n)
{
    const int nt = copy_threads();
    if (n < kMinSplit || nt == 1) {
        std::memcpy(dst, src, n);
        return;
    }
    const size_t part = (n + nt - 1) / nt;
    const std::function<void(int)> job = [&](int i) {
        const size_t off = (size_t)i * part;
        if (off < n) std::memcpy((char *)dst + off, (const char *)src + off, std::min(part, n - off));
    };
    pool().run(nt, job);
}

struct Staging {
    void *pin[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    std::vector<double *> ws;
    std::vector<size_t> ws_cap;
    int init()
    {
        if (st) return GPUTO_OK;
        for (int b = 0; b < 2; ++b) {
            GPUTO_CUDA(cudaHostAlloc(&pin[b], kChunk, cudaHostAllocDefault));
            GPUTO_CUDA(cudaEventCreateWithFlags(&ev[b], cudaEventDisableTiming));
        }
        GPUTO_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        return GPUTO_OK;
    }
};

std::mutex g_io_mu;
Staging g_stage[64];

Staging *staging(int *status)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        *status = GPUTO_ERR_NO_DEVICE;
        return nullptr;
    }
    Staging &s = g_stage[dev];
    *status = s.init();
    return *status ? nullptr : &s;
}

}  // namespace

std::mutex &host_io_mutex() { return g_io_mu; }

int host_to_device(void *dst, const void *src, size_t bytes)
{
    int stt = GPUTO_OK;
    Staging *s = staging(&stt);
    if (!s) return stt;
    size_t off = 0;
    int last = -1;
    for (int k = 0; off < bytes; ++k, off += kChunk) {
        const int b = k & 1;
        const size_t n = std::min(kChunk, bytes - off);
        if (k >= 2) GPUTO_CUDA(cudaEventSynchronize(s->ev[b]));   // the DMA out of pin[b] has finished
        par_memcpy(s->pin[b], (const char *)src + off, n);
        GPUTO_CUDA(cudaMemcpyAsync((char *)dst + off, s->pin[b], n, cudaMemcpyHostToDevice, s->st));
        GPUTO_CUDA(cudaEventRecord(s->ev[b], s->st));
        last = b;
    }
    if (last >= 0) GPUTO_CUDA(cudaStreamSynchronize(s->st));
    return GPUTO_OK;
}

int device_to_host(void *dst, const void *src, size_t bytes)
{
    int stt = GPUTO_OK;
    Staging *s = staging(&stt);
    if (!s) return stt;
    size_t prev_off = 0, prev_n = 0;
    int prev_b = -1;
    size_t off = 0;
    for (int k = 0; off < bytes; ++k, off += kChunk) {
        const int b = k & 1;
        const size_t n = std::min(kChunk, bytes - off);
        GPUTO_CUDA(cudaMemcpyAsync(s->pin[b], (const char *)src + off, n, cudaMemcpyDeviceToHost, s->st));
        GPUTO_CUDA(cudaEventRecord(s->ev[b], s->st));
        if (prev_b >= 0) {   // copy the previous chunk out while this one moves
            GPUTO_CUDA(cudaEventSynchronize(s->ev[prev_b]));
            par_memcpy((char *)dst + prev_off, s->pin[prev_b], prev_n);
        }
        prev_b = b;
        prev_off = off;
        prev_n = n;
    }
    if (prev_b >= 0) {
        GPUTO_CUDA(cudaEventSynchronize(s->ev[prev_b]));
        par_memcpy((char *)dst + prev_off, s->pin[prev_b], prev_n);
    }
    return GPUTO_OK;
}

double *host_call_buffer(int slot, size_t count, int *status)
{
    Staging *s = staging(status);
    if (!s) return nullptr;
    if ((int)s->ws.size() <= slot) {
        s->ws.resize(slot + 1, nullptr);
        s->ws_cap.resize(slot + 1, 0);
    }
    if (s->ws_cap[slot] < count) {
        cudaFree(s->ws[slot]);
        s->ws[slot] = nullptr;
        s->ws_cap[slot] = 0;
        if (cudaMalloc(&s->ws[slot], sizeof(double) * count) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc failed for a host-call buffer");
            *status = GPUTO_ERR_OOM;
            return nullptr;
        }
        s->ws_cap[slot] = count;
    }
    *status = GPUTO_OK;
    return s->ws[slot];
}

}  // namespace gputo
