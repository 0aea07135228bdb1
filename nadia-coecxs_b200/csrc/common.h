// common.h -- error handling, device buffers and transform plans shared by
// the FP64 and FP32 paths of libnadia_b200.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "nadia_b200.h"

namespace nadia {

// A named range on the host timeline for profilers (Nsight tools show it;
// with no tool attached the calls do nothing).
struct Range {
    explicit Range(const char *name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range &) = delete;
    Range &operator=(const Range &) = delete;
};

// An error carried to the C ABI boundary, where it becomes a status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define NADIA_CUDA(call)                                                                  \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw ::nadia::Error(e_ == cudaErrorMemoryAllocation ? NADIA_ERR_NOMEM         \
                                                                 : NADIA_ERR_CUDA,         \
                                 std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

#define NADIA_REQUIRE(cond, code, msg)                                                    \
    do {                                                                                  \
        if (!(cond)) throw ::nadia::Error((code), (msg));                                 \
    } while (0)

// Bytes currently held by DevBuf allocations of this process (all devices).
inline std::atomic<long long> g_device_bytes{0};

// Device allocations come from the device's stream-ordered memory pool.  An
// allocation is ordered on the stream that is current for allocations on the
// calling thread (AllocScope; otherwise the thread's per-thread stream), and
// its release is a free ordered on that same stream: a reconstruction's
// buffers are freed behind the last work queued on its own stream, with no
// device-wide synchronisation (cudaFree waits for the whole device, which
// would stall every other reconstruction sharing the GPU).  A buffer is
// usable on any stream once alloc returns.  Rule for temporaries allocated
// outside a scope: release them only after the work that uses them is done.
inline thread_local cudaStream_t t_alloc_stream = cudaStreamPerThread;

struct AllocScope {
    cudaStream_t saved;
    explicit AllocScope(cudaStream_t s) : saved(t_alloc_stream) { t_alloc_stream = s; }
    ~AllocScope() { t_alloc_stream = saved; }
    AllocScope(const AllocScope &) = delete;
    AllocScope &operator=(const AllocScope &) = delete;
};

// keep freed pool memory for reuse instead of returning it to the driver
void retain_pool_memory();

// Owning device allocation.
template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t st = nullptr; // the stream its allocation and release are ordered on
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n), st(o.st) { o.p = nullptr; o.n = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept
    {
        if (this != &o) {
            release();
            p = o.p; n = o.n; st = o.st;
            o.p = nullptr; o.n = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count)
    {
        release();
        if (count) {
            retain_pool_memory();
            st = t_alloc_stream;
            NADIA_CUDA(cudaMallocAsync((void **)&p, count * sizeof(T), st));
            NADIA_CUDA(cudaStreamSynchronize(st));
        }
        n = count;
        g_device_bytes += (long long)(n * sizeof(T));
    }
    void release()
    {
        if (p) cudaFreeAsync(p, st);
        g_device_bytes -= (long long)(n * sizeof(T));
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
    explicit operator bool() const { return p != nullptr; }
};

// A stream owned by an object whose buffers are ordered on it: declared
// before those buffers, so it outlives their releases.
struct OwnedStream {
    cudaStream_t s = nullptr;
    OwnedStream() = default;
    OwnedStream(const OwnedStream &) = delete;
    OwnedStream &operator=(const OwnedStream &) = delete;
    ~OwnedStream()
    {
        if (s) cudaStreamDestroy(s);
    }
};

// Host-to-device copy that has landed when it returns.  A plain cudaMemcpy
// from pageable memory may return before its DMA completes, and the library's
// streams do not synchronise with the legacy default stream.
inline void upload_now(void *dst, const void *src, size_t bytes)
{
    NADIA_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    NADIA_CUDA(cudaStreamSynchronize(0));
}

constexpr int kMaxPasses = 40;
constexpr int kMaxRadix = 64;    // generic radices up to this keep their inputs in registers
constexpr int kMaxPrime = 1021;  // the largest prime factor a transform length may have

// Radix plan of a transform length: 8s, then the remaining 4 or 2, then odd
// primes in ascending order.  Returns the number of passes, or -1 when n has
// a prime factor above kMaxPrime.
inline int plan_radices(int n, int *radix)
{
    int p = 0;
    if (n < 1) return -1;
    while (n % 8 == 0) { radix[p++] = 8; n /= 8; }
    if (n % 4 == 0) { radix[p++] = 4; n /= 4; }
    if (n % 2 == 0) { radix[p++] = 2; n /= 2; }
    for (int f = 3; n > 1; f += 2) {
        while (n % f == 0) {
            if (f > kMaxPrime) return -1;
            radix[p++] = f;
            n /= f;
        }
    }
    return p;
}

// Transform plan passed to kernels by value.
struct FftPlan {
    int n;
    int np;
    int radix[kMaxPasses];
};

inline FftPlan make_plan(int n)
{
    FftPlan p{};
    p.n = n;
    p.np = plan_radices(n, p.radix);
    NADIA_REQUIRE(p.np >= 0, NADIA_ERR_INVALID,
                  "transform length " + std::to_string(n) + " has a prime factor above 1021");
    return p;
}

// Twiddle table W[t] = (cos, -sin)(2 pi t / n), computed in double on the host.
inline std::vector<double2> twiddles(int n)
{
    std::vector<double2> w((size_t)n);
    for (int t = 0; t < n; ++t) {
        double ang = (2.0 * M_PI * (double)t) / (double)n;
        w[t].x = cos(ang);
        w[t].y = -sin(ang);
    }
    return w;
}

} // namespace nadia
