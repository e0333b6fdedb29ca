// noalloc.cu — ggb_remove_mean_noalloc: the area-weighted mean removal of
// fluid_remove_mean for callers that cannot allocate device memory.
//
// fluid_remove_mean allocates a small array of per-block partial sums with
// cudaMalloc on every call (and stages host buffers through cudaMalloc'd
// scratch).  Some callers cannot do that: code that runs in a process whose
// device memory is entirely reserved up front by another allocator (a
// framework's memory pool), and steady-state loops that must never call
// cudaMalloc / cudaFree because those calls synchronise the whole device.
// This variant keeps its scratch in a fixed, file-scope device array instead.
//
// The scratch array is shared by every call in the process and keeps the last
// call's partial sums; each call overwrites every slot it reads, so nothing has
// to start at zero.  Two calls whose GPU work overlaps (from two host threads)
// race on it and give wrong results.
#include <cstdio>
#include <mutex>

#include "ggb_internal.h"

namespace ggb {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocCellsPerBlock = 4096;  // 16 cells per thread
constexpr int kNoAllocMaxBlocks = 4096;      // scratch: 4096 partial sums + the mean (32 KB)
constexpr long kNoAllocMaxCells = (long)kNoAllocCellsPerBlock * kNoAllocMaxBlocks;  // 16,777,216

// The only scratch of the no-allocation entry point.  Host code must not use
// the symbol itself as a device address: its device address is obtained once
// per device with cudaGetSymbolAddress (see scratch_for_current_device).
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxBlocks + 1];

// partial[b] = sum over the cells of block b of area * f (FP64, fixed order)
__global__ void __launch_bounds__(kNoAllocThreads) k_noalloc_partials(int n, const float *area, const float *f,
                                                                     double *partial) {
    __shared__ double s_red[kNoAllocThreads / 32 + 2];
    const int c0 = blockIdx.x * kNoAllocCellsPerBlock;
    const int c1 = min(n, c0 + kNoAllocCellsPerBlock);
    double s = 0;
    for (int c = c0 + threadIdx.x; c < c1; c += kNoAllocThreads) s += (double)area[c] * f[c];
    double t = block_sum<kNoAllocThreads>(s, s_red);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// partial[nblocks] = the mean (one block, fixed order)
__global__ void __launch_bounds__(kNoAllocThreads) k_noalloc_mean(int nblocks, double total_area, double *partial) {
    __shared__ double s_red[kNoAllocThreads / 32 + 2];
    double s = 0;
    for (int b = threadIdx.x; b < nblocks; b += kNoAllocThreads) s += partial[b];
    double t = block_sum<kNoAllocThreads>(s, s_red);
    if (threadIdx.x == 0) partial[kNoAllocMaxBlocks] = t / total_area;
}

__global__ void __launch_bounds__(kNoAllocThreads) k_noalloc_subtract(int n, const double *partial, float *f) {
    const float m = (float)partial[kNoAllocMaxBlocks];
    const int c0 = blockIdx.x * kNoAllocCellsPerBlock;
    const int c1 = min(n, c0 + kNoAllocCellsPerBlock);
    for (int c = c0 + threadIdx.x; c < c1; c += kNoAllocThreads) f[c] -= m;
}

// Device address of the scratch array on the current device, looked up once
// per device (with that device current) and cached; nullptr on failure.
static double *scratch_for_current_device() {
    static std::mutex mu;
    static double *addr[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            fprintf(stderr, "ggb_remove_mean_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                    cudaGetErrorString(e));
            return nullptr;
        }
        addr[dev] = (double *)p;
    }
    return addr[dev];
}

}  // namespace ggb

using namespace ggb;

// See include/ggb_ext.h.  Returns 0; or -1 with a message on stderr and f
// unchanged when the grid is unknown, has more than 16,777,216 cells, lives on
// another device than the current one or the library stream's, f is not
// device or managed memory, or the scratch address cannot be obtained; or -1
// with f undefined when a launch or the final synchronisation fails.
GGB_EXPORT int ggb_remove_mean_noalloc(const CubeSphere *cs, float *f) {
    GridTables *t = grid_find(cs);
    if (!t) {
        fprintf(stderr, "ggb_remove_mean_noalloc: the grid was not created by this library's cs_init\n");
        return -1;
    }
    const int n = t->n;
    if ((long)n > kNoAllocMaxCells) {
        fprintf(stderr,
                "ggb_remove_mean_noalloc: %d cells exceed the fixed scratch of this entry point "
                "(at most %ld cells, N <= 1672); use fluid_remove_mean\n",
                n, kNoAllocMaxCells);
        return -1;
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        fprintf(stderr, "ggb_remove_mean_noalloc: no current CUDA device\n");
        return -1;
    }
    // the scratch address below is the current device's: the grid's tables and
    // the library stream must belong to that same device
    cudaStream_t s = stream();
    if (t->device != dev || stream_device() != dev) {
        fprintf(stderr,
                "ggb_remove_mean_noalloc: the current device (%d) differs from the grid's (%d) or the "
                "library stream's (%d)\n",
                dev, t->device, stream_device());
        return -1;
    }
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, f) != cudaSuccess ||
        (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged)) {
        cudaGetLastError();
        fprintf(stderr, "ggb_remove_mean_noalloc: the field must be device or managed memory "
                        "(host buffers would need staging, i.e. an allocation)\n");
        return -1;
    }
    double *scratch = scratch_for_current_device();
    if (!scratch) return -1;
    const int nb = (n + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock;
    k_noalloc_partials<<<nb, kNoAllocThreads, 0, s>>>(n, t->area, f, scratch);
    k_noalloc_mean<<<1, kNoAllocThreads, 0, s>>>(nb, t->total_area, scratch);
    k_noalloc_subtract<<<nb, kNoAllocThreads, 0, s>>>(n, scratch, f);
    note_launch(3);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        fprintf(stderr, "ggb_remove_mean_noalloc: %s\n", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}
