// runtime.cu — error reporting, the library stream, allocation, argument
// staging and the kernel-launch counter of libggb_cuda.so.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "ggb_internal.h"

namespace ggb {

void fail_cuda(const char *what, cudaError_t e, const char *file, int line) {
    fprintf(stderr, "libggb_cuda: CUDA error in %s (%s:%d): %s\n", what, file, line, cudaGetErrorString(e));
    fflush(stderr);
    exit(1);
}

void fail_msg(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    fprintf(stderr, "libggb_cuda: ");
    vfprintf(stderr, fmt, ap);
    fprintf(stderr, "\n");
    va_end(ap);
    fflush(stderr);
    exit(1);
}

static std::atomic<long> g_launches{0};
void note_launch(long k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
long launch_count() { return g_launches.load(std::memory_order_relaxed); }

static std::mutex g_stream_mu;
static cudaStream_t g_own_stream = nullptr;
static cudaStream_t g_override = nullptr;
static int g_stream_dev = -1;
static int g_sms = 0;

bool have_device() {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

cudaStream_t stream() {
    if (g_override) return g_override;
    std::lock_guard<std::mutex> lk(g_stream_mu);
    if (!g_own_stream) {
        if (!have_device()) fail_msg("no CUDA device is available (this library has no CPU path)");
        GGB_CHECK(cudaStreamCreateWithFlags(&g_own_stream, cudaStreamNonBlocking));
        GGB_CHECK(cudaGetDevice(&g_stream_dev));
    }
    return g_own_stream;
}

int stream_device() {
    std::lock_guard<std::mutex> lk(g_stream_mu);
    return g_stream_dev;
}

void set_stream(cudaStream_t s) { g_override = s; }

void sync() {
    GGB_CHECK(cudaStreamSynchronize(stream()));
    stage_collect();
}

// ---- stage timing
static bool g_timing = false;
static cudaEvent_t g_ev[ST_N][2];
static bool g_pending[ST_N];
static double g_stage_ms[ST_N];
static long g_stage_n[ST_N];

void stage_begin(int s) {
    if (!g_timing) return;
    GGB_CHECK(cudaEventRecord(g_ev[s][0], stream()));
}

void stage_end(int s) {
    if (!g_timing) return;
    GGB_CHECK(cudaEventRecord(g_ev[s][1], stream()));
    g_pending[s] = true;
}

void stage_collect() {
    if (!g_timing) return;
    for (int s = 0; s < ST_N; s++)
        if (g_pending[s]) {
            float ms = 0;
            GGB_CHECK(cudaEventSynchronize(g_ev[s][1]));
            GGB_CHECK(cudaEventElapsedTime(&ms, g_ev[s][0], g_ev[s][1]));
            g_stage_ms[s] += ms;
            g_stage_n[s]++;
            g_pending[s] = false;
        }
}

int device_sm_count() {
    if (!g_sms) {
        int dev = 0;
        GGB_CHECK(cudaGetDevice(&dev));
        GGB_CHECK(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    return g_sms;
}

// Allocation-failure injection (ggb_inject_alloc_failure): while >= 0, the
// number of allocations that still succeed; the one after fails as if device
// memory were exhausted, without calling the allocator.
static std::atomic<long> g_allocs_left{-1};

static bool injected_failure() {
    long k = g_allocs_left.load();
    while (k >= 0) {
        if (k == 0) return true;
        if (g_allocs_left.compare_exchange_weak(k, k - 1)) return false;
    }
    return false;
}

void *dev_try_alloc(size_t bytes) {
    void *p = nullptr;
    if (!bytes) bytes = 16;
    if (injected_failure()) return nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    GGB_CHECK(cudaMemsetAsync(p, 0, bytes, stream()));
    return p;
}

void *dev_alloc(size_t bytes) {
    void *p = dev_try_alloc(bytes);
    if (!p) fail_msg("device memory allocation of %zu bytes failed", bytes);
    return p;
}

void dev_free(void *p) {
    if (p) GGB_CHECK(cudaFree(p));
}

void *managed_alloc(size_t bytes) {
    void *p = managed_try_alloc(bytes);
    if (!p) fail_msg("managed memory allocation of %zu bytes failed", bytes);
    return p;
}

void *managed_try_alloc(size_t bytes) {
    void *p = nullptr;
    if (!bytes) bytes = 16;
    if (injected_failure()) return nullptr;
    if (cudaMallocManaged(&p, bytes, cudaMemAttachGlobal) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    int dev = 0;
    GGB_CHECK(cudaGetDevice(&dev));
#if CUDART_VERSION >= 13000
    cudaMemLocation loc;
    loc.type = cudaMemLocationTypeDevice;
    loc.id = dev;
    cudaMemAdvise(p, bytes, cudaMemAdviseSetPreferredLocation, loc);
    cudaMemPrefetchAsync(p, bytes, loc, 0, stream());
#else
    cudaMemAdvise(p, bytes, cudaMemAdviseSetPreferredLocation, dev);
    cudaMemPrefetchAsync(p, bytes, dev, stream());
#endif
    cudaGetLastError();  // advice / prefetch are hints; ignore "not supported"
    GGB_CHECK(cudaMemsetAsync(p, 0, bytes, stream()));
    return p;
}

void managed_free(void *p) {
    if (p) GGB_CHECK(cudaFree(p));
}

static bool device_accessible(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

Staged::~Staged() {
    if (owned) cudaFree(dev);
}

void stage_in(Staged &s, const void *src, size_t bytes) {
    s.bytes = bytes;
    s.host = const_cast<void *>(src);
    if (device_accessible(src)) {
        s.dev = const_cast<void *>(src);
        s.owned = false;
        return;
    }
    GGB_CHECK(cudaMalloc(&s.dev, bytes ? bytes : 16));
    s.owned = true;
    GGB_CHECK(cudaMemcpyAsync(s.dev, src, bytes, cudaMemcpyHostToDevice, stream()));
}

void stage_out(Staged &s, void *dst, size_t bytes) {
    s.bytes = bytes;
    s.host = dst;
    if (device_accessible(dst)) {
        s.dev = dst;
        s.owned = false;
        return;
    }
    GGB_CHECK(cudaMalloc(&s.dev, bytes ? bytes : 16));
    s.owned = true;
}

void stage_finish(Staged &s) {
    if (s.owned) GGB_CHECK(cudaMemcpyAsync(s.host, s.dev, s.bytes, cudaMemcpyDeviceToHost, stream()));
    sync();
}

}  // namespace ggb

GGB_EXPORT long ggb_launch_count(void) { return ggb::launch_count(); }

// Host-side fault injection: after `after` more successful allocations every
// device / managed allocation of the library fails (after < 0: off).
GGB_EXPORT void ggb_inject_alloc_failure(long after) { ggb::g_allocs_left.store(after < 0 ? -1 : after); }

// Selects the CUDA device this library uses (before any other call).
GGB_EXPORT int ggb_set_device(int dev) { return cudaSetDevice(dev) == cudaSuccess ? 0 : -1; }

// Waits for all work issued by this library.
GGB_EXPORT void ggb_sync(void) { ggb::sync(); }

// Per-stage timing: enable/disable (resets the totals); read totals in ms and
// interval counts for the stages particles, advect, solve, velocity,
// max_speed, render binning, render tiles.
GGB_EXPORT void ggb_stage_timing(int on) {
    using namespace ggb;
    sync();
    if (on && !g_timing)
        for (int s = 0; s < ST_N; s++) {
            GGB_CHECK(cudaEventCreate(&g_ev[s][0]));
            GGB_CHECK(cudaEventCreate(&g_ev[s][1]));
        }
    for (int s = 0; s < ST_N; s++) {
        g_stage_ms[s] = 0;
        g_stage_n[s] = 0;
        g_pending[s] = false;
    }
    g_timing = on != 0;
}

GGB_EXPORT int ggb_stage_times(double *ms, long *count, int n) {
    using namespace ggb;
    sync();
    for (int s = 0; s < ST_N && s < n; s++) {
        ms[s] = g_stage_ms[s];
        count[s] = g_stage_n[s];
    }
    return ST_N;
}

// Wall-clock interval of the library stream measured with CUDA events.
static cudaEvent_t g_t0 = nullptr, g_t1 = nullptr;
GGB_EXPORT void ggb_timer_start(void) {
    if (!g_t0) {
        GGB_CHECK(cudaEventCreate(&g_t0));
        GGB_CHECK(cudaEventCreate(&g_t1));
    }
    GGB_CHECK(cudaEventRecord(g_t0, ggb::stream()));
}
GGB_EXPORT double ggb_timer_stop(void) {
    GGB_CHECK(cudaEventRecord(g_t1, ggb::stream()));
    GGB_CHECK(cudaEventSynchronize(g_t1));
    float ms = 0;
    GGB_CHECK(cudaEventElapsedTime(&ms, g_t0, g_t1));
    return ms;
}
