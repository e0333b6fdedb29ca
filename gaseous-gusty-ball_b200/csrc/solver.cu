// solver.cu — the Poisson solve K psi = -A omega as ONE persistent cooperative
// kernel: warm-started preconditioned conjugate gradients whose
// preconditioner is a symmetric multigrid V-cycle (damped-Jacobi smoother,
// bilinear prolongation P, restriction R = P^T, many-sweep Jacobi on the
// coarsest grid), with FP64 dot products and FP64 zero-mean projections.
//
// Upstream: src/fluid.c:41-160 (multigrid), :264-275 (mean), :290-358 (PCG).
// Two precisions share one kernel body (template parameter MP):
//   * plain (MP = false): the arithmetic of every vector update follows
//     upstream (FP32 vectors, FP64 accumulation of the stencil sums);
//   * mixed (MP = true): the V-cycle's level vectors and the coarse levels'
//     slot weights are stored in FP16, every stencil sum, restriction and
//     prolongation accumulates in FP32, and the outer CG is flexible
//     (Polak-Ribiere beta = r.(z - z_prev) / rz_prev), which tolerates the
//     preconditioner's rounding; psi, omega, r, p, z stay FP32 and the dots,
//     norms and mean projections stay FP64.  FP16 holds about five decimal
//     orders of magnitude, less than the spread of a residual across the
//     levels, so the mixed V-cycle runs on scaled vectors: its input is
//     multiplied by a power of two that brings its RMS near 1/16, restriction
//     carries a factor 1/4 and prolongation a factor 4 (so that every level's
//     right-hand side stays at the input's scale instead of growing 4x per
//     level), and the output is scaled back.  All factors are powers of two
//     (exact), and the V-cycle is linear, so they change nothing but the range.
// The schedule is this library's:
//   * phases are separated by a bounded grid-wide barrier instead of host loops;
//   * each block owns a contiguous range of cells of every level; a stencil
//     phase first computes the (transformed) neighbour value of every cell of
//     the range plus its halo once into shared memory (FP64 plain, FP32
//     mixed), then applies the stencil from shared memory;
//   * p = z + beta p and r - alpha Ap are recomputed inside K p and the level-0
//     pre-smooth, which saves two barriers per iteration;
//   * interior rows of R and P use index arithmetic (no CSR indirection);
//   * the V-cycle below the grid levels (N <= 16, at most 1536 cells) is a
//     fixed linear map, precomputed once as a dense matrix and applied by all
//     blocks from L2.
#include <algorithm>
#include <cstdio>
#include <type_traits>
#include <vector>

#include "ggb_internal.h"
#include "ggb_solver.h"

namespace ggb {

#include "solver_body.cuh"

// Many planets' solves in one cooperative launch: block b runs planet
// bmap[b].x's solve as block bmap[b].y of bmap[b].z (the planet's blocks are
// consecutive), with that planet's parameters, barrier, partial sums and
// result.  Planets finish independently.
template <bool MP>
__global__ void __launch_bounds__(kPB, 1) k_pcg_batch(const SolveParams *prm, const int4 *bmap) {
    __shared__ SolveParams sP;
    const int4 m = bmap[blockIdx.x];
    {
        const int *src = reinterpret_cast<const int *>(prm + m.x);
        int *dst = reinterpret_cast<int *>(&sP);
        for (int k = threadIdx.x; k < (int)(sizeof(SolveParams) / sizeof(int)); k += blockDim.x) dst[k] = src[k];
    }
    if (threadIdx.x == 0) {
        s_vgrid[0] = m.y;
        s_vgrid[1] = m.z;
    }
    __syncthreads();
    pcg_body<MP>(sP);
}

// ---- setup kernels -------------------------------------------------------

// Column j of the dense map of levels l0..nlev-1: the block's V-cycle applied
// to the unit vector e_j, stored row-major D[row][j] in FP64.
__global__ void __launch_bounds__(kPB, 1) k_dense_columns(SolveParams P, int l0, double *D) {
    extern __shared__ __align__(16) unsigned char dyn[];
    float *smem = reinterpret_cast<float *>(dyn);
    const int nd = P.L[l0].S.n;
    for (int j = blockIdx.x; j < nd; j += gridDim.x) {
        SmemLevel lv[kMaxLev];
        carve_smem(P, l0, smem, lv);
        BLOCK_LOOP(c, nd) lv[l0].b[c] = c == j ? 1.0f : 0.0f;
        __syncthreads();
        vcycle_block_smem(P, l0, lv);
        BLOCK_LOOP(c, nd) D[(size_t)c * nd + j] = lv[l0].xo[c];
        __syncthreads();
    }
}

// Coarse-major weights of the structured rows of R: rw16[q][c] = the weight of
// fine cell q (q = 4*dj + di of the 4x4 window) in row c, taken from the CSR
// row (which the structured check has verified to be that window in order).
__global__ void k_build_rw16(LevelDev F, LevelDev C, float *rw16) {
    const int Nc = C.S.N, nc = C.S.n;
    KERNEL_LOOP(c, nc) {
        int f, I, J;
        cell_fij(C.S, c, f, I, J);
        const bool inner = I >= 1 && J >= 1 && I + 2 <= Nc && J + 2 <= Nc;
        const int k0 = F.rstart[c];
        for (int q = 0; q < 16; q++) rw16[q * nc + c] = inner ? F.rw[k0 + q] : 0.f;
    }
}

// Counts rows of R / taps of P of a level pair that the structured path would
// take but that do not follow the structured index pattern.
__global__ void k_check_structured(LevelDev F, LevelDev C, int *bad) {
    const int Nf = F.S.N, Nc = C.S.N;
    KERNEL_LOOP(c, C.S.n) {
        int f, I, J;
        cell_fij(C.S, c, f, I, J);
        if (!(I >= 1 && J >= 1 && I + 2 <= Nc && J + 2 <= Nc)) continue;
        int k0 = F.rstart[c], k1 = F.rstart[c + 1];
        if (k1 - k0 != 16) {
            atomicAdd(bad, 1);
            continue;
        }
        const int base = (f * Nf + 2 * J - 1) * Nf + 2 * I - 1;
        for (int dj = 0; dj < 4; dj++)
            for (int di = 0; di < 4; di++) {
                const int i = base + dj * Nf + di, q = k0 + dj * 4 + di;
                const int k = (di <= 1 ? 1 : 0) + 2 * (dj <= 1 ? 1 : 0);
                if (F.ridx[q] != i || F.rw[q] != F.pw[4 * i + k]) atomicAdd(bad, 1);
            }
    }
    KERNEL_LOOP(i, F.S.n) {
        int f, fi, fj;
        cell_fij(F.S, i, f, fi, fj);
        const int I0 = (fi - 1) >> 1, J0 = (fj - 1) >> 1;
        if (!(I0 >= 0 && J0 >= 0 && I0 + 1 < Nc && J0 + 1 < Nc)) continue;
        const int t0 = (f * Nc + J0) * Nc + I0;
        if (F.ptap[4 * i] != t0 || F.ptap[4 * i + 1] != t0 + 1 || F.ptap[4 * i + 2] != t0 + Nc ||
            F.ptap[4 * i + 3] != t0 + Nc + 1)
            atomicAdd(bad, 1);
    }
}

// ---------------------------------------------------------------- host

int pcg_block_size() { return kPB; }

static unsigned long long *g_trace_dev = nullptr;
static int g_trace_cap = 0;
void solve_trace_target(unsigned long long **buf, int *cap) {
    *buf = g_trace_dev;
    *cap = g_trace_cap;
}

// Dynamic shared memory of a launch: the staged window, plus x, xo, b, r of
// every level run by block 0.
static size_t pcg_smem_bytes(const SolveParams &p) {
    size_t cells = 0;
    if (p.nlev >= 2 && !p.dense && !p.coarse_on_grid)
        for (int l = p.nlev_grid; l < p.nlev; l++) cells += p.L[l].S.n;
    if (p.nlev == 1 && !p.coarse_on_grid) cells = p.L[0].S.n;
    return kStageBytes + 4 * sizeof(float) * cells;
}

int pcg_max_blocks() { return 2 * device_sm_count(); }

// Largest level edge N whose staged window (a block's cells plus N + 1 on
// either side) leaves at least one block of threads' worth of cells per pass.
int pcg_max_grid_n() { return (kStageCap - kPB) / 2 - 1; }

// Threads per block of a single solve on a grid of edge N (the wide block
// where its window still leaves a block's worth of cells per pass).
static int pcg_threads(int N) { return N >= kWideMinN && N <= (kStageCap - kPBWide) / 2 - 1 ? kPBWide : kPB; }

// The 640-thread kernels and their diagnostic symbols (solver_wide.cu).
const void *pcg_wide_kernel(bool mixed);
void pcg_wide_trace_symbols(void **trace_n, void **stage_trace, void **stage_n, void **stage_all);

static const void *pcg_kernel(bool mixed, int threads) {
    if (threads == kPBWide) return pcg_wide_kernel(mixed);
    return mixed ? (const void *)k_pcg<true, kPB> : (const void *)k_pcg<false, kPB>;
}

// Device addresses of the diagnostic counters and pointers of both solve
// modules (k = 0: this one, k = 1: the 640-thread kernels').
struct TraceSyms {
    void *trace_n, *stage_trace, *stage_n, *stage_all;
};
static TraceSyms trace_syms(int k) {
    TraceSyms t{};
    if (k == 1) {
        pcg_wide_trace_symbols(&t.trace_n, &t.stage_trace, &t.stage_n, &t.stage_all);
    } else {
        GGB_CHECK(cudaGetSymbolAddress(&t.trace_n, g_trace_n));
        GGB_CHECK(cudaGetSymbolAddress(&t.stage_trace, g_stage_trace));
        GGB_CHECK(cudaGetSymbolAddress(&t.stage_n, g_stage_trace_n));
        GGB_CHECK(cudaGetSymbolAddress(&t.stage_all, g_stage_trace_all));
    }
    return t;
}

static void pcg_attributes() {
    static bool attr = false;
    if (!attr) {
        int dev = 0, optin = 0;
        GGB_CHECK(cudaGetDevice(&dev));
        GGB_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        for (int m = 0; m < 4; m++) {
            const void *k = pcg_kernel(m & 1, m & 2 ? kPBWide : kPB);
            cudaFuncAttributes fa;
            GGB_CHECK(cudaFuncGetAttributes(&fa, k));
            GGB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           optin - (int)fa.sharedSizeBytes));
        }
        GGB_CHECK(cudaFuncSetAttribute(k_dense_columns, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr = true;
    }
}

static int pcg_grid_for(size_t smem, bool mixed, int threads) {
    pcg_attributes();
    int per = 0;
    GGB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, pcg_kernel(mixed, threads), threads, smem));
    if (per < 1) fail_msg("the solve kernel cannot be resident on this device (%zu B shared memory)", smem);
    return device_sm_count() * std::min(per, 2);
}

int pcg_grid_size() { return pcg_grid_for(kStageBytes, false, kPB); }

// One solve launch; max_blocks > 0 caps its grid (batched planets: small
// grids take a share of the SMs so that several solves run at once).
void pcg_launch(const SolveParams &prm, cudaStream_t s, int max_blocks) {
    SolveParams p = prm;
    size_t smem = pcg_smem_bytes(p);
    void *args[] = {&p};
    const int threads = pcg_threads(p.L[0].S.N);
    int grid = pcg_grid_for(smem, p.mixed != 0, threads);
    if (max_blocks > 0) grid = std::max(1, std::min(grid, max_blocks));
    GGB_CHECK(cudaMemsetAsync(&p.bar->count, 0, sizeof(unsigned int), s));
    GGB_CHECK(
        cudaLaunchCooperativeKernel(pcg_kernel(p.mixed != 0, threads), dim3(grid), dim3(threads), args, smem, s));
    GGB_LAUNCHED();
}

// Blocks of one batched solve launch that can be resident at once (the
// launch's capacity), for the shared memory the planets' solves need.
int pcg_batch_capacity(size_t smem, bool mixed) {
    pcg_attributes();
    const void *k = mixed ? (const void *)k_pcg_batch<true> : (const void *)k_pcg_batch<false>;
    static bool attr[2] = {false, false};
    if (!attr[mixed]) {
        int dev = 0, optin = 0;
        GGB_CHECK(cudaGetDevice(&dev));
        GGB_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa;
        GGB_CHECK(cudaFuncGetAttributes(&fa, k));
        GGB_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
        attr[mixed] = true;
    }
    int per = 0;
    GGB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kPB, smem));
    return device_sm_count() * std::min(per, 2);
}

size_t pcg_launch_smem(const SolveParams &p) { return pcg_smem_bytes(p); }

// One cooperative launch of nblocks blocks solving every planet of a batch
// (dev_prm: the planets' parameters; dev_bmap: block -> planet, block of the
// planet, blocks of the planet).  The planets' barrier counters must be zero.
void pcg_launch_batch(const SolveParams *dev_prm, const int4 *dev_bmap, int nblocks, bool mixed, size_t smem,
                      cudaStream_t s) {
    const void *k = mixed ? (const void *)k_pcg_batch<true> : (const void *)k_pcg_batch<false>;
    void *args[] = {(void *)&dev_prm, (void *)&dev_bmap};
    GGB_CHECK(cudaLaunchCooperativeKernel(k, dim3(nblocks), dim3(kPB), args, smem, s));
    GGB_LAUNCHED();
}

// Coarse-major structured restriction weights of a level pair (after the check).
float *pcg_build_rw16(const LevelDev &F, const LevelDev &C) {
    float *rw16 = (float *)dev_alloc(sizeof(float) * 16 * (size_t)C.S.n);
    k_build_rw16<<<std::max(1u, std::min(grid_for(C.S.n, 256), 2048u)), 256, 0, stream()>>>(F, C, rw16);
    GGB_LAUNCHED();
    return rw16;
}

// Verifies the structured index pattern of a level pair's R / P (1 = usable).
int pcg_check_structured(const LevelDev &F, const LevelDev &C) {
    int *bad = (int *)dev_alloc(sizeof(int));
    k_check_structured<<<std::max(1u, std::min(grid_for(F.S.n, 256), 2048u)), 256, 0, stream()>>>(F, C, bad);
    GGB_LAUNCHED();
    int hb = 0;
    GGB_CHECK(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, stream()));
    GGB_CHECK(cudaStreamSynchronize(stream()));
    dev_free(bad);
    return hb == 0;
}

// The dense map of the V-cycle of levels l0..nlev-1 (nd x nd, FP64).
double *pcg_dense_map(const SolveParams &prm, int l0) {
    SolveParams p = prm;
    const int nd = p.L[l0].S.n;
    size_t cells = 0;
    for (int l = l0; l < p.nlev; l++) cells += p.L[l].S.n;
    size_t smem = 4 * sizeof(float) * cells;
    pcg_attributes();
    int grid = std::min(nd, 4 * device_sm_count());
    double *D = (double *)dev_alloc(sizeof(double) * nd * nd);
    k_dense_columns<<<grid, kPB, smem, stream()>>>(p, l0, D);
    GGB_LAUNCHED();
    GGB_CHECK(cudaStreamSynchronize(stream()));
    return D;
}

// ---- micro-benchmark of the grid barrier (additive entry point) ----------
// `rounds` barriers with a wait limit of limit_ns each; block `withhold`
// (-1: none) returns without arriving, so that the others' wait runs out:
// they raise the barrier's error flag, clear *ok and return.
__global__ void __launch_bounds__(kPB, 1) k_barrier_bench(GridBarrier *bar, int rounds, int *ok, int withhold,
                                                        unsigned long long limit_ns) {
    if ((int)blockIdx.x == withhold) return;
    for (int k = 0; k < rounds; k++)
        if (!grid_sync_limit(bar, limit_ns)) {
            if (threadIdx.x == 0) atomicExch(ok, 0);
            return;
        }
}

}  // namespace ggb

// One cooperative launch of `rounds` grid-wide barriers of the solve kernel's
// launch shape, each wait limited to limit_ms; block `withhold` (-1: none)
// never arrives.  Returns the launch's duration in ms (*ok = 1 when every
// barrier completed, 0 when the waits ran out and the kernel returned).
static double barrier_run(int rounds, int withhold, double limit_ms, int *ok_out) {
    using namespace ggb;
    GridBarrier *bar = (GridBarrier *)dev_alloc(sizeof(GridBarrier));
    int *ok = (int *)dev_alloc(sizeof(int));
    int one = 1;
    GGB_CHECK(cudaMemcpyAsync(ok, &one, sizeof(int), cudaMemcpyHostToDevice, stream()));
    int per = 0;
    GGB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_barrier_bench, kPB, 0));
    int grid = device_sm_count() * std::min(per, 2);
    unsigned long long limit_ns = (unsigned long long)(limit_ms * 1e6);
    cudaEvent_t e0, e1;
    GGB_CHECK(cudaEventCreate(&e0));
    GGB_CHECK(cudaEventCreate(&e1));
    void *args[] = {&bar, &rounds, &ok, &withhold, &limit_ns};
    GGB_CHECK(cudaEventRecord(e0, stream()));
    GGB_CHECK(cudaLaunchCooperativeKernel((const void *)k_barrier_bench, dim3(grid), dim3(kPB), args, 0, stream()));
    GGB_LAUNCHED();
    GGB_CHECK(cudaEventRecord(e1, stream()));
    GGB_CHECK(cudaEventSynchronize(e1));
    float ms = 0;
    GGB_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    int hok = 0;
    GGB_CHECK(cudaMemcpy(&hok, ok, sizeof(int), cudaMemcpyDeviceToHost));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    dev_free(bar);
    dev_free(ok);
    *ok_out = hok;
    return ms;
}

// Mean time of one grid-wide barrier of the solve kernel's launch shape, in
// microseconds (`rounds` barriers in one cooperative launch); -1 on timeout.
GGB_EXPORT double ggb_barrier_bench(int rounds) {
    int ok = 0;
    double ms = barrier_run(rounds, -1, 2000.0, &ok);
    return ok ? 1000.0 * ms / rounds : -1.0;
}

// Failure detection without a fault: one block of a cooperative launch never
// arrives at the grid barrier, the others wait limit_ms, raise the barrier's
// error flag and return.  Returns 1 when the waits ran out (0 if the barrier
// completed after all); *elapsed_ms gets the launch's duration.
GGB_EXPORT int ggb_barrier_timeout_probe(double limit_ms, double *elapsed_ms) {
    int ok = 1;
    double ms = barrier_run(1, 0, limit_ms, &ok);
    if (elapsed_ms) *elapsed_ms = ms;
    return ok ? 0 : 1;
}

// Diagnostics: the next solves record up to `cap` (mark, time in ns) pairs from
// block 0 (cap = 0 turns it off); ggb_solve_trace copies them out and returns
// how many were recorded.
GGB_EXPORT void ggb_solve_trace_enable(int cap) {
    using namespace ggb;
    sync();
    dev_free(g_trace_dev);
    g_trace_dev = cap > 0 ? (unsigned long long *)dev_alloc(sizeof(unsigned long long) * 2 * cap) : nullptr;
    g_trace_cap = cap > 0 ? cap : 0;
    int zero = 0;
    for (int k = 0; k < 2; k++) GGB_CHECK(cudaMemcpy(trace_syms(k).trace_n, &zero, sizeof(int), cudaMemcpyHostToDevice));
}

GGB_EXPORT int ggb_solve_trace(unsigned long long *out, int cap) {
    using namespace ggb;
    sync();
    int n = 0;
    for (int k = 0; k < 2; k++) {  // only the module whose kernel ran has records
        int m = 0;
        GGB_CHECK(cudaMemcpy(&m, trace_syms(k).trace_n, sizeof(int), cudaMemcpyDeviceToHost));
        n = std::max(n, m);
    }
    n = n < cap ? n : cap;
    if (n > 0) GGB_CHECK(cudaMemcpy(out, g_trace_dev, sizeof(unsigned long long) * 2 * n, cudaMemcpyDeviceToHost));
    return n;
}

// Diagnostics: enable = 1 makes block 0 of the next solves stamp the start
// (mark 1), window loaded (4), staged (2) and computed (3) points of every
// staged phase (mark, ns); enable = 2 makes
// every block stamp them (mark | block << 16, ns); enable = 0 stops and copies
// out up to cap records, returning their number.
GGB_EXPORT int ggb_stage_trace(int enable, unsigned long long *out, int cap) {
    using namespace ggb;
    sync();
    static unsigned long long *buf = nullptr;
    int n = 0;
    if (!enable) {
        unsigned long long *null = nullptr;
        for (int k = 0; k < 2; k++) {  // only the module whose kernel ran has records
            const TraceSyms t = trace_syms(k);
            int m = 0;
            GGB_CHECK(cudaMemcpy(&m, t.stage_n, sizeof(int), cudaMemcpyDeviceToHost));
            n = std::max(n, m);
            GGB_CHECK(cudaMemcpy(t.stage_trace, &null, sizeof(null), cudaMemcpyHostToDevice));
        }
        n = n < cap ? n : cap;
        n = n < 4096 ? n : 4096;
        if (n > 0 && buf) GGB_CHECK(cudaMemcpy(out, buf, sizeof(unsigned long long) * 2 * n, cudaMemcpyDeviceToHost));
        return n;
    }
    if (!buf) buf = (unsigned long long *)dev_alloc(sizeof(unsigned long long) * 2 * 4096);
    const int all = enable == 2;
    for (int k = 0; k < 2; k++) {
        const TraceSyms t = trace_syms(k);
        GGB_CHECK(cudaMemcpy(t.stage_trace, &buf, sizeof(buf), cudaMemcpyHostToDevice));
        GGB_CHECK(cudaMemcpy(t.stage_n, &n, sizeof(int), cudaMemcpyHostToDevice));
        GGB_CHECK(cudaMemcpy(t.stage_all, &all, sizeof(int), cudaMemcpyHostToDevice));
    }
    return 0;
}
