// solver.cu — the Poisson solve K psi = -A omega as ONE persistent cooperative
// kernel: warm-started preconditioned conjugate gradients whose
// preconditioner is a symmetric multigrid V-cycle (damped-Jacobi smoother,
// bilinear prolongation P, restriction R = P^T, many-sweep Jacobi on the
// coarsest grid), with FP64 dot products and FP64 zero-mean projections.
//
// Upstream: src/fluid.c:41-160 (multigrid), :264-275 (mean), :290-358 (PCG).
// The arithmetic of every vector update follows upstream (FP32 vectors, FP64
// accumulation); the schedule is this library's:
//   * phases are separated by a bounded grid-wide barrier instead of host loops;
//   * each block owns a contiguous range of cells of every level; a stencil
//     phase first computes the (transformed) neighbour value of every cell of
//     the range plus its halo once, in FP64, into shared memory, then applies
//     the stencil with FP64 weights (no FP32/FP64 conversion per link);
//   * p = z + beta p and r - alpha Ap are recomputed inside K p and the level-0
//     pre-smooth, which saves two barriers per iteration;
//   * interior rows of R and P use index arithmetic (no CSR indirection);
//   * the V-cycle below the grid levels (N <= 16, at most 1536 cells) is a
//     fixed linear map, precomputed once as a dense matrix and applied by all
//     blocks from L2.
#include <algorithm>
#include <cstdio>
#include <vector>

#include "ggb_internal.h"
#include "ggb_solver.h"

namespace ggb {

constexpr int kPB = 512;            // threads per block of the persistent kernel
constexpr double kOmegaJ = 0.8;     // upstream MG_OMEGA
constexpr double kCorrScale = 1.0;  // upstream MG_CORR_SCALE
constexpr int kStageCap = 3584;     // cells of a block's staged window (value + 4 slot weights FP64, 3 FP32 own inputs)
constexpr int kRingCap = 1024;      // boundary-ring cells of one staged sub-range (their off-face link sums)
constexpr int kStageWords = kStageCap * 5 + (kStageCap * 3 + 1) / 2 + kRingCap;  // in doubles
constexpr size_t kStageBytes = (size_t)kStageWords * sizeof(double);

enum { RED_BB = 0, RED_RR, RED_PAP, RED_RZ, RED_MEAN, RED_AREA, RED_N };

// Phase trace (diagnostics): block 0, thread 0 records (mark, %globaltimer).
__device__ int g_trace_n;
__device__ __forceinline__ void trace_mark(const SolveParams &P, int mark) {
    if (P.trace && blockIdx.x == 0 && threadIdx.x == 0) {
        int k = g_trace_n;
        if (k < P.trace_cap) {
            P.trace[2 * k] = (unsigned long long)mark;
            P.trace[2 * k + 1] = globaltimer_ns();
            g_trace_n = k + 1;
        }
    }
}

#define GRID_LOOP(c, n) for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < (n); c += gridDim.x * blockDim.x)
#define BLOCK_LOOP(c, n) for (int c = threadIdx.x; c < (n); c += blockDim.x)
#define SYNC_OR(fail)                    \
    do {                                 \
        if (!grid_sync(P.bar)) fail;     \
    } while (0)

struct Red {
    double v[kPB / 32 + 2];
};

__device__ __forceinline__ void put_partial(const SolveParams &P, int which, double v, double *s_red) {
    double t = block_sum<kPB>(v, s_red);
    if (threadIdx.x == 0) P.part[which * gridDim.x + blockIdx.x] = t;
}
__device__ __forceinline__ double get_total(const SolveParams &P, int which, double *s_red) {
    return sum_partials<kPB>(P.part + which * gridDim.x, gridDim.x, s_red);
}

// ---- staged stencil phases ------------------------------------------------

// This block's contiguous range of a level's n = 6 N^2 cells (face-major).
// With at least 6 blocks every face gets a whole number of blocks (face f:
// blocks [f nb / 6, (f + 1) nb / 6)) and splits its cells evenly among them,
// so that no range holds the boundary rows of two faces: a range straddling a
// face edge has twice the boundary-ring cells, which takes a second link pass
// (or, at N = 512, another sub-range) and makes that block the phase's last.
// Fewer blocks split the cells evenly.
__device__ __forceinline__ void block_range(int n, int N, int &c0, int &c1) {
    const int nb = gridDim.x, b = blockIdx.x;
    if (nb < 6) {
        c0 = (int)(((long long)n * b) / nb);
        c1 = (int)(((long long)n * (b + 1)) / nb);
        return;
    }
    int f = 0;
    while (f < 5 && b >= ((f + 1) * nb) / 6) f++;
    const int b0 = (f * nb) / 6, m = ((f + 1) * nb) / 6 - b0;
    const long long nf = (long long)N * N;
    c0 = (int)(f * nf + nf * (b - b0) / m);
    c1 = (int)(f * nf + nf * (b - b0 + 1) / m);
}

__device__ unsigned long long *g_stage_trace;  // diagnostics: block 0 stamps staging / compute ends
__device__ int g_stage_trace_n;
__device__ int g_stage_trace_all;  // 1: every block records, mark | block << 16
__device__ __forceinline__ void stage_mark(int mark) {
    unsigned long long *t = g_stage_trace;
    if (!t || threadIdx.x != 0) return;
    if (g_stage_trace_all) {
        const int k = atomicAdd(&g_stage_trace_n, 1);
        if (k < 4096) {
            t[2 * k] = (unsigned long long)(mark | (blockIdx.x << 16));
            t[2 * k + 1] = globaltimer_ns();
        }
    } else if (blockIdx.x == 0) {
        int k = g_stage_trace_n;
        if (k < 4096) {
            t[2 * k] = (unsigned long long)mark;
            t[2 * k + 1] = globaltimer_ns();
            g_stage_trace_n = k + 1;
        }
    }
}

// Inputs of a cell of the block's own range: a, b, c are staged in shared
// memory for the compute loop; d stays in the staging thread (for commit).
struct Own {
    float a, b, c, d;
};

// cell(c, x, wE, wN, wNE, wNW, rsum, r0, o) for every cell c of this block's
// range of a level.  Over the stencil window of the current sub-range, x[k] =
// load(k, mine, o) and the four slot weights are staged (FP64) in shared
// memory; for the cells of the sub-range (mine) load also fills o, whose a, b,
// c are staged too, and commit(k, o) then performs the cell's side effects
// (global stores) after the loads of the pass are issued.  load must not
// store.  The links that leave a face (boundary-ring cells) are summed while
// staging as well: rsum[ring rank - r0] = sum_k w_k (x(c) - x(nb_k)), one
// thread per ring cell.  All global loads happen while staging, where they are
// independent, so the compute loop reads shared memory only.  Ends with a
// block barrier.
template <class Load, class Commit, class Cell>
__device__ __forceinline__ void staged(const StencilDev &S, double *buf, Load load, Commit commit, Cell cell) {
    const int N = S.N, n = S.n, nring = S.nring, bs = blockDim.x, tid = threadIdx.x;
    int c0, c1;
    block_range(n, N, c0, c1);
    const int halo = N + 1;
    const int sub = kStageCap - 2 * halo;
    double *bx = buf, *b0 = buf + kStageCap, *b1 = buf + 2 * kStageCap, *b2 = buf + 3 * kStageCap,
           *b3 = buf + 4 * kStageCap;
    float *oa = reinterpret_cast<float *>(buf + 5 * kStageCap), *ob = oa + kStageCap, *oc = ob + kStageCap;
    double *rs = buf + kStageWords - kRingCap;
    const double *wd = S.wslot_d;
    stage_mark(1);
    for (int s0 = c0; s0 < c1;) {
        int s1 = min(c1, s0 + sub);
        const int r0 = ring_rank_below(s0, N, nring);
        int r1 = ring_rank_below(s1, N, nring);
        if (r1 - r0 > kRingCap) {  // end the sub-range before its (kRingCap+1)-th ring cell
            r1 = r0 + kRingCap;
            int f, i, j;
            ring_cell_of_rank(r1, N, nring, f, i, j);
            s1 = (f * N + j) * N + i;
        }
        const int w0 = s0 - halo, w1 = s1 + halo;  // cells outside [0, n) stage as zeros
        // The ring tables are in ring-rank order: this sub-range's boundary-ring
        // cells are rows r0..r1-1, one thread per ring cell.  The first row of
        // each thread (its eight links as two 16-byte loads each) and its own
        // value are fetched before the window loop so that their latency
        // overlaps it.
        const int nr = r1 - r0;
        const int4 *rn4 = reinterpret_cast<const int4 *>(S.ring_nb) + 2 * (size_t)r0;
        const float4 *rw4 = reinterpret_cast<const float4 *>(S.ring_w) + 2 * (size_t)r0;
        int4 fo0 = make_int4(-1, -1, -1, -1), fo1 = fo0;
        float4 fw0 = make_float4(0.f, 0.f, 0.f, 0.f), fw1 = fw0;
        double fvc = 0;
        if (tid < nr) {
            fo0 = __ldg(rn4 + 2 * tid);
            fo1 = __ldg(rn4 + 2 * tid + 1);
            fw0 = __ldg(rw4 + 2 * tid);
            fw1 = __ldg(rw4 + 2 * tid + 1);
            int f, i, j;
            ring_cell_of_rank(r0 + tid, N, nring, f, i, j);
            Own none;
            fvc = load((f * N + j) * N + i, false, none);
        }
        // window: values and slot weights, two cells per thread per pass with
        // every global load of both issued before any shared-memory store
        for (int k = w0 + tid; k < w1; k += 2 * bs) {
            const int k2 = k + bs;
            const bool two = k2 < w1;
            const bool in1 = k >= s0 && k < s1, in2 = two && k2 >= s0 && k2 < s1;
            Own o1{0.f, 0.f, 0.f, 0.f}, o2{0.f, 0.f, 0.f, 0.f};
            double e1 = 0, n1 = 0, ne1 = 0, nw1 = 0, v1 = 0;
            if (k >= 0 && k < n) {
                e1 = __ldg(wd + k);
                n1 = __ldg(wd + n + k);
                ne1 = __ldg(wd + 2 * n + k);
                nw1 = __ldg(wd + 3 * n + k);
                v1 = load(k, in1, o1);
            }
            double e2 = 0, n2 = 0, ne2 = 0, nw2 = 0, v2 = 0;
            if (two && k2 >= 0 && k2 < n) {
                e2 = __ldg(wd + k2);
                n2 = __ldg(wd + n + k2);
                ne2 = __ldg(wd + 2 * n + k2);
                nw2 = __ldg(wd + 3 * n + k2);
                v2 = load(k2, in2, o2);
            }
            if (in1) commit(k, o1);
            if (in2) commit(k2, o2);
            int q = k - w0;
            bx[q] = v1;
            b0[q] = e1;
            b1[q] = n1;
            b2[q] = ne1;
            b3[q] = nw1;
            if (in1) {
                oa[k - s0] = o1.a;
                ob[k - s0] = o1.b;
                oc[k - s0] = o1.c;
            }
            if (two) {
                q = k2 - w0;
                bx[q] = v2;
                b0[q] = e2;
                b1[q] = n2;
                b2[q] = ne2;
                b3[q] = nw2;
            }
            if (in2) {
                oa[k2 - s0] = o2.a;
                ob[k2 - s0] = o2.b;
                oc[k2 - s0] = o2.c;
            }
        }
        stage_mark(4);
        // off-face links of each ring cell: all present neighbour values
        // requested at once, summed in link order
        for (int q = tid; q < nr; q += bs) {
            int4 o0, o1;
            float4 w0v, w1v;
            double vc;
            if (q == tid) {
                o0 = fo0;
                o1 = fo1;
                w0v = fw0;
                w1v = fw1;
                vc = fvc;
            } else {
                o0 = __ldg(rn4 + 2 * q);
                o1 = __ldg(rn4 + 2 * q + 1);
                w0v = __ldg(rw4 + 2 * q);
                w1v = __ldg(rw4 + 2 * q + 1);
                int f, i, j;
                ring_cell_of_rank(r0 + q, N, nring, f, i, j);
                Own none;
                vc = load((f * N + j) * N + i, false, none);
            }
            const int o[8] = {o0.x, o0.y, o0.z, o0.w, o1.x, o1.y, o1.z, o1.w};
            const float w[8] = {w0v.x, w0v.y, w0v.z, w0v.w, w1v.x, w1v.y, w1v.z, w1v.w};
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                Own none;
                v[k] = o[k] >= 0 ? load(o[k], false, none) : vc;
            }
            double t = 0;
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (o[k] >= 0) t += (double)w[k] * (vc - v[k]);
            rs[q] = t;
        }
        __syncthreads();
        stage_mark(2);
        // two independent cells in flight per thread: one cell's dependent
        // chain (shared loads, FP64 sum, conversions) leaves the issue slots
        // idle with 16 warps per SM
#pragma unroll 2
        for (int c = s0 + tid; c < s1; c += bs) {
            Own o;
            o.a = oa[c - s0];
            o.b = ob[c - s0];
            o.c = oc[c - s0];
            cell(c, bx - w0, b0 - w0, b1 - w0, b2 - w0, b3 - w0, rs, r0, o);
        }
        __syncthreads();
        stage_mark(3);
        s0 = s1;
    }
}

#define STAGED_ARGS                                                                                             \
    const double *x, const double *wE, const double *wN, const double *wNE, const double *wNW, const double *rsum, \
        int r0, Own o
#define APPLY(S, c, xc) apply_k_smem(S, c, xc, x, wE, wN, wNE, wNW, rsum, r0)

// The pre-smoothed iterate from 0 at cell k: w D^-1 b.
__device__ __forceinline__ float presmooth_x(const LevelDev &L, int k, float b) {
    return (float)(kOmegaJ * __ldg(L.dinv + k) * b);
}

// (R r_fine) at coarse cell c.  Interior coarse cells gather their 4x4 fine
// window in the CSR row order (fine index ascending) with the P weights; the
// others use the CSR rows.
__device__ __forceinline__ float restrict_value(const LevelDev &F, const LevelDev &C, int c) {
    const int Nc = C.S.N, Nf = F.S.N;
    int f, I, J;
    cell_fij(C.S, c, f, I, J);
    double acc = 0;
    if (F.structured && I >= 1 && J >= 1 && I + 2 <= Nc && J + 2 <= Nc) {
        const float *r = F.r;
        const int base = (f * Nf + 2 * J - 1) * Nf + 2 * I - 1;
        const int nc = C.S.n;
        float wv[16], rv[16];
#pragma unroll
        for (int dj = 0; dj < 4; dj++)
#pragma unroll
            for (int di = 0; di < 4; di++) {
                const int i = base + dj * Nf + di;
                wv[dj * 4 + di] = __ldg(F.rw16 + (dj * 4 + di) * nc + c);
                rv[dj * 4 + di] = r[i];
            }
#pragma unroll
        for (int q = 0; q < 16; q++) acc += (double)(wv[q] * rv[q]);
    } else {
        const int k0 = __ldg(F.rstart + c), k1 = __ldg(F.rstart + c + 1);
        for (int k = k0; k < k1; k++) acc += (double)(__ldg(F.rw + k) * F.r[__ldg(F.ridx + k)]);
    }
    return (float)acc;
}
__device__ __forceinline__ void restrict_cell(const LevelDev &F, const LevelDev &C, int c) {
    C.b[c] = restrict_value(F, C, c);
}

// x_fine + P xo_coarse at fine cell i.  Interior fine cells compute their 2x2
// coarse taps.
__device__ __forceinline__ float prolong_value(const LevelDev &F, const LevelDev &C, int i) {
    const int Nf = F.S.N, Nc = C.S.N;
    const float4 w = __ldg(reinterpret_cast<const float4 *>(F.pw) + i);
    const float *xc = C.xo;
    int t0, t1, t2, t3;
    int f, fi, fj;
    cell_fij(F.S, i, f, fi, fj);
    const int I0 = (fi - 1) >> 1, J0 = (fj - 1) >> 1;
    if (F.structured && I0 >= 0 && J0 >= 0 && I0 + 1 < Nc && J0 + 1 < Nc) {
        t0 = (f * Nc + J0) * Nc + I0;
        t1 = t0 + 1;
        t2 = t0 + Nc;
        t3 = t0 + Nc + 1;
    } else {
        const int4 t = __ldg(reinterpret_cast<const int4 *>(F.ptap) + i);
        t0 = t.x;
        t1 = t.y;
        t2 = t.z;
        t3 = t.w;
    }
    const float s = w.x * xc[t0] + w.y * xc[t1] + w.z * xc[t2] + w.w * xc[t3];
    return F.x[i] + (float)(kCorrScale * s);
}
__device__ __forceinline__ void prolong_cell(const LevelDev &F, const LevelDev &C, int i) {
    F.x[i] = prolong_value(F, C, i);
}

// Pre-smooth of a level from x = 0 with right-hand side b: x = w D^-1 b,
// r = b - K x.
__device__ __forceinline__ void phase_presmooth(const LevelDev &L, const float *b, double *buf) {
    auto load = [&](int k, bool mine, Own &o) -> double {
        const float bk = b[k];
        if (mine) o.a = bk;
        return (double)presmooth_x(L, k, bk);
    };
    auto commit = [&](int, const Own &) {};
    staged(L.S, buf, load, commit, [&](int c, STAGED_ARGS) {
        const float bc = o.a;
        const float xc = (float)x[c];  // = presmooth_x(L, c, bc)
        const double kx = APPLY(L.S, c, (double)xc);
        L.x[c] = xc;
        L.r[c] = (float)(bc - kx);
    });
}

// Prolongation C -> L fused with L's post-smooth: x = x_L + P xo_C is formed on
// the fly over the staged window (never stored), then xo = x + w D^-1 (b - K x);
// returns sum dotr . xo when dotr != nullptr.  Same arithmetic as a separate
// prolongation pass followed by the post-smooth, one grid barrier fewer.
__device__ __forceinline__ double phase_prolong_postsmooth(const LevelDev &L, const LevelDev &C, const float *b,
                                                           float *xo, const float *dotr, double *buf) {
    double s = 0;
    auto load = [&](int k, bool mine, Own &o) -> double {
        if (mine) {
            o.a = b[k];
            o.b = __ldg(L.dinv + k);
            o.c = dotr ? dotr[k] : 0.f;
        }
        return (double)prolong_value(L, C, k);
    };
    auto commit = [&](int, const Own &) {};
    staged(L.S, buf, load, commit, [&](int c, STAGED_ARGS) {
        const float xc = (float)x[c];
        const float rc = (float)(o.a - APPLY(L.S, c, (double)xc));
        const float out = xc + (float)(kOmegaJ * o.b * rc);
        xo[c] = out;
        s += (double)o.c * out;
    });
    return s;
}

// One damped-Jacobi sweep src -> dst with per-link conversions (small levels).
__device__ __forceinline__ float jacobi_cell(const StencilDev &S, const float *dinv, const float *b, const float *src,
                                             float *dst, int c) {
    auto X = [&](int k) -> double { return (double)src[k]; };
    float xc = src[c];
    float rc = (float)(b[c] - apply_k(S, c, (double)xc, X));
    float out = xc + (float)(kOmegaJ * __ldg(dinv + c) * rc);
    dst[c] = out;
    return out;
}

// ---- the coarse levels inside one block (setup of the dense map, fallback) --

struct SmemLevel {
    float *x, *xo, *b, *r;
};

__device__ void carve_smem(const SolveParams &P, int l0, float *smem, SmemLevel *lv) {
    float *q = smem;
    for (int l = l0; l < P.nlev; l++) {
        int n = P.L[l].S.n;
        lv[l].x = q;
        lv[l].xo = q + n;
        lv[l].b = q + 2 * n;
        lv[l].r = q + 3 * n;
        q += 4 * n;
    }
}

// Coarsest level: `sweeps` Jacobi sweeps from 0; result in V.xo.  When every
// cell has its own thread, the cell's links, 1/diag and b stay in registers.
__device__ void coarsest_smem(const LevelDev &L, const SmemLevel &V, int sweeps) {
    const int n = L.S.n;
    BLOCK_LOOP(c, n) V.x[c] = 0.f;
    __syncthreads();
    float *src = V.x, *dst = V.xo;
    if (n <= (int)blockDim.x) {
        const int c = threadIdx.x;
        int nb[kMaxNb];
        float wv[kMaxNb];
        float bc = 0.f, dv = 0.f;
        if (c < n) {
            cell_links(L.S, c, nb, wv);
            bc = V.b[c];
            dv = __ldg(L.dinv + c);
        }
        for (int s = 0; s < sweeps; s++) {
            if (c < n) {
                float xc = src[c];
                double xd = xc, acc = 0;
#pragma unroll
                for (int k = 0; k < kMaxNb; k++) acc += (double)wv[k] * (xd - (double)src[nb[k]]);
                float rc = (float)(bc - acc);
                dst[c] = xc + (float)(kOmegaJ * dv * rc);
            }
            __syncthreads();
            float *t = src;
            src = dst;
            dst = t;
        }
    } else {
        for (int s = 0; s < sweeps; s++) {
            BLOCK_LOOP(c, n) jacobi_cell(L.S, L.dinv, V.b, src, dst, c);
            __syncthreads();
            float *t = src;
            src = dst;
            dst = t;
        }
    }
    if (src != V.xo) {
        BLOCK_LOOP(c, n) V.xo[c] = src[c];
        __syncthreads();
    }
}

// Levels l0..nlev-1 of the V-cycle inside this block, on vectors in shared
// memory.  b of level l0 is lv[l0].b on entry; xo of level l0 is written to
// `out` (global memory).
__device__ void vcycle_block_smem(const SolveParams &P, int l0, SmemLevel *lv, float *out) {
    const int last = P.nlev - 1;
    for (int l = l0; l < last; l++) {
        LevelDev L = P.L[l];
        L.x = lv[l].x;
        L.r = lv[l].r;
        const float *b = lv[l].b;
        BLOCK_LOOP(c, L.S.n) {
            auto X = [&](int k) -> double { return (double)(float)(kOmegaJ * __ldg(L.dinv + k) * b[k]); };
            float bc = b[c];
            float xc = (float)(kOmegaJ * __ldg(L.dinv + c) * bc);
            double kx = apply_k(L.S, c, (double)xc, X);
            L.x[c] = xc;
            L.r[c] = (float)(bc - kx);
        }
        __syncthreads();
        LevelDev C = P.L[l + 1];
        C.b = lv[l + 1].b;
        BLOCK_LOOP(c, C.S.n) restrict_cell(L, C, c);
        __syncthreads();
    }
    coarsest_smem(P.L[last], lv[last], P.coarse_sweeps);
    for (int l = last - 1; l >= l0; l--) {
        LevelDev L = P.L[l];
        L.x = lv[l].x;
        LevelDev C = P.L[l + 1];
        C.xo = lv[l + 1].xo;
        BLOCK_LOOP(i, L.S.n) prolong_cell(L, C, i);
        __syncthreads();
        BLOCK_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, lv[l].b, lv[l].x, lv[l].xo, c);
        __syncthreads();
    }
    BLOCK_LOOP(c, P.L[l0].S.n) out[c] = lv[l0].xo[c];
    __syncthreads();
}

// ---- the V-cycle after level 0's pre-smooth --------------------------------

// The rest of z = V(r) once level 0's pre-smooth (x, r of level 0) is complete
// and visible.  Ends with rz = r . z published; returns false on abort.
__device__ bool vcycle_rest(const SolveParams &P, const float *r, double *s_red, double *buf, float *smem) {
    const int G = P.nlev_grid;
    // down
    for (int l = 0; l < G; l++) {
        const LevelDev &L = P.L[l];
        if (l > 0) {
            phase_presmooth(L, L.b, buf);
            trace_mark(P, 100 + l);
            SYNC_OR(return false);
        }
        GRID_LOOP(c, P.L[l + 1].S.n) restrict_cell(L, P.L[l + 1], c);
        trace_mark(P, 300 + l);
        SYNC_OR(return false);
    }
    // below the grid levels: the dense map, or block 0
    if (P.dense) {
        const LevelDev &C = P.L[G];
        const int nd = P.nd, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int gw = blockIdx.x * (blockDim.x >> 5) + warp, nw = gridDim.x * (blockDim.x >> 5);
        for (int row = gw; row < nd; row += nw) {
            const double *d = P.dense + (size_t)row * nd;
            double acc = 0;
            for (int j = lane; j < nd; j += 32) acc += __ldg(d + j) * (double)C.b[j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) C.xo[row] = (float)acc;
        }
        trace_mark(P, 500);
        SYNC_OR(return false);
    } else if (!P.coarse_on_grid) {
        if (blockIdx.x == 0) {
            SmemLevel lv[kMaxLev];
            carve_smem(P, G, smem, lv);
            BLOCK_LOOP(c, P.L[G].S.n) lv[G].b[c] = P.L[G].b[c];
            __syncthreads();
            vcycle_block_smem(P, G, lv, P.L[G].xo);
        }
        trace_mark(P, 500);
        SYNC_OR(return false);
    } else {
        // the coarsest level is large (nlev_grid == nlev - 1): sweep it grid-wide
        const LevelDev &L = P.L[P.nlev - 1];
        GRID_LOOP(c, L.S.n) L.x[c] = 0.f;
        SYNC_OR(return false);
        float *src = L.x, *dst = L.xo;
        for (int s = 0; s < P.coarse_sweeps; s++) {
            GRID_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, L.b, src, dst, c);
            SYNC_OR(return false);
            float *t = src;
            src = dst;
            dst = t;
        }
        if (src != L.xo) {
            GRID_LOOP(c, L.S.n) L.xo[c] = src[c];
            SYNC_OR(return false);
        }
    }
    // up: prolongation fused with each grid level's post-smooth
    for (int l = G - 1; l >= 0; l--) {
        const LevelDev &L = P.L[l];
        if (l > 0) {
            phase_prolong_postsmooth(L, P.L[l + 1], L.b, L.xo, nullptr, buf);
            trace_mark(P, 900 + l);
            SYNC_OR(return false);
        } else {
            double s = phase_prolong_postsmooth(L, P.L[1], r, P.z, r, buf);
            put_partial(P, RED_RZ, s, s_red);
            trace_mark(P, 900);
            SYNC_OR(return false);
        }
    }
    return true;
}

// z = V(r) for a single-level hierarchy (level 0 is the coarsest grid).
__device__ bool single_level(const SolveParams &P, const float *r, double *s_red, float *smem) {
    const LevelDev &L = P.L[0];
    if (!P.coarse_on_grid) {
        if (blockIdx.x == 0) {
            SmemLevel lv[kMaxLev];
            carve_smem(P, 0, smem, lv);
            BLOCK_LOOP(c, L.S.n) lv[0].b[c] = r[c];
            __syncthreads();
            coarsest_smem(L, lv[0], P.coarse_sweeps);
            BLOCK_LOOP(c, L.S.n) L.xo[c] = lv[0].xo[c];
        }
    } else {
        GRID_LOOP(c, L.S.n) L.x[c] = 0.f;
        SYNC_OR(return false);
        float *src = L.x, *dst = L.xo;
        for (int s = 0; s < P.coarse_sweeps; s++) {
            GRID_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, r, src, dst, c);
            SYNC_OR(return false);
            float *t = src;
            src = dst;
            dst = t;
        }
        if (src != L.xo) {
            GRID_LOOP(c, L.S.n) L.xo[c] = src[c];
        }
    }
    SYNC_OR(return false);
    double s = 0;
    GRID_LOOP(c, L.S.n) {
        float z = L.xo[c];
        P.z[c] = z;
        s += (double)r[c] * z;
    }
    put_partial(P, RED_RZ, s, s_red);
    return grid_sync(P.bar);
}

__global__ void __launch_bounds__(kPB, 1) k_pcg(SolveParams P) {
    __shared__ Red sh;
    extern __shared__ __align__(16) unsigned char dyn[];
    double *buf = reinterpret_cast<double *>(dyn);               // staged window
    float *smem = reinterpret_cast<float *>(dyn + kStageBytes);  // block-0 levels
    double *s_red = sh.v;
    const LevelDev &L0 = P.L[0];
    const StencilDev &S0 = L0.S;
    const int n = S0.n;
    const bool mg = P.nlev >= 2;
    const bool single = P.nlev == 1;
    float *r = P.r, *rn = P.r2, *p = P.p, *pn = P.p2;
    double bb, rr, rz = 0, tol2, beta = 0, m2;
    int it = 0;
    bool first = true, ok = true;

    // zero-mean projection of omega (FP64 sum), upstream src/fluid.c:264-275
    if (P.remove_mean) {
        double s = 0;
        GRID_LOOP(c, n) s += (double)__ldg(P.area + c) * P.omega[c];
        put_partial(P, RED_MEAN, s, s_red);
        SYNC_OR(goto aborted);
        float m = (float)(get_total(P, RED_MEAN, s_red) / P.total_area);
        GRID_LOOP(c, n) P.omega[c] -= m;  // read back below only at the own cell
    }

    // FP64 projection that makes the singular system consistent: the stored
    // FP32 omega keeps a residual area-weighted mean m2 (the FP32 rounding of
    // the subtracted mean); b = -A (omega - m2) is formed in FP64 so that
    // sum b = 0 to double precision.  Without it the constant mode of the
    // residual stays at the FP32 rounding level and CG diverges once the
    // residual reaches it.
    {
        double s = 0, sa = 0;
        GRID_LOOP(c, n) {
            double a = __ldg(P.area + c);
            s += a * P.omega[c];
            sa += a;
        }
        put_partial(P, RED_MEAN, s, s_red);
        put_partial(P, RED_AREA, sa, s_red);
        SYNC_OR(goto aborted);
        m2 = get_total(P, RED_MEAN, s_red) / get_total(P, RED_AREA, s_red);
    }

    // r = b - K psi, b = -A (omega - m2)
    {
        double sb = 0, sr = 0;
        const float *psi = P.psi;
        auto load = [&](int k, bool mine, Own &o) -> double {
            if (mine) {
                o.a = P.omega[k];
                o.b = __ldg(P.area + k);
            }
            return (double)psi[k];
        };
        auto commit = [&](int, const Own &) {};
        staged(S0, buf, load, commit, [&](int c, STAGED_ARGS) {
            double b = -(double)o.b * ((double)o.a - m2);
            double ri = b - APPLY(S0, c, x[c]);
            r[c] = (float)ri;
            sb += b * b;
            sr += ri * ri;
        });
        put_partial(P, RED_BB, sb, s_red);
        put_partial(P, RED_RR, sr, s_red);
    }
    SYNC_OR(goto aborted);
    bb = get_total(P, RED_BB, s_red);
    rr = get_total(P, RED_RR, s_red);
    if (bb == 0.0) {
        GRID_LOOP(c, n) P.psi[c] = 0.f;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            P.res->iters = 0;
            P.res->relres = 0;
            P.res->status = 0;
            P.res->r_final = 0;
        }
        return;
    }
    tol2 = P.tol * P.tol * bb;

    // z = M^-1 r, rz
    if (rr > tol2) {
        if (mg) {
            phase_presmooth(L0, r, buf);
            SYNC_OR(goto aborted);
            ok = vcycle_rest(P, r, s_red, buf, smem);
        } else if (single) {
            ok = single_level(P, r, s_red, smem);
        } else {
            double s = 0;
            GRID_LOOP(c, n) {
                float z = __ldg(L0.dinv + c) * r[c];
                P.z[c] = z;
                s += (double)r[c] * z;
            }
            put_partial(P, RED_RZ, s, s_red);
            ok = grid_sync(P.bar);
        }
        if (!ok) goto aborted;
        rz = get_total(P, RED_RZ, s_red);
    }

    while (rr > tol2 && it < P.maxit) {
        // p = z (first) or z + beta p;  Ap = K p;  pAp
        {
            const float *z = P.z;
            const float *po = p;
            const bool fst = first;
            const double be = beta;
            auto pnew = [&](int k) -> float { return fst ? z[k] : (float)(z[k] + be * po[k]); };
            auto load = [&](int k, bool, Own &) -> double { return (double)pnew(k); };
            auto commit = [&](int, const Own &) {};
            double s = 0;
            float *pw = pn, *ap = P.Ap;
            staged(S0, buf, load, commit, [&](int c, STAGED_ARGS) {
                const float pc = (float)x[c];
                const double a = APPLY(S0, c, (double)pc);
                pw[c] = pc;
                ap[c] = (float)a;
                s += a * pc;
            });
            put_partial(P, RED_PAP, s, s_red);
            float *t = p;
            p = pn;
            pn = t;
            first = false;
        }
        trace_mark(P, 10);
        SYNC_OR(goto aborted);
        trace_mark(P, 11);
        {
            double pAp = get_total(P, RED_PAP, s_red);
            if (pAp <= 0) break;
            const double alpha = rz / pAp;
            const float *Ap = P.Ap;
            const float *ro = r;
            const float *pp = p;
            double s = 0, sz = 0;
            float *rw_ = rn;
            if (mg) {
                // psi += alpha p; r' = r - alpha Ap; level-0 pre-smooth of r'
                auto rnew = [&](int k) -> float { return (float)(ro[k] - alpha * Ap[k]); };
                // mine: r, Ap of the cell staged; p and psi kept for commit,
                // which does psi += alpha p (nothing else reads psi)
                auto load = [&](int k, bool mine, Own &o) -> double {
                    if (mine) {
                        o.a = ro[k];
                        o.b = Ap[k];
                        o.c = pp[k];
                        o.d = P.psi[k];
                    }
                    return (double)presmooth_x(L0, k, rnew(k));
                };
                auto commit = [&](int k, const Own &o) { P.psi[k] = o.d + (float)(alpha * o.c); };
                staged(S0, buf, load, commit, [&](int c, STAGED_ARGS) {
                    const double ri = o.a - alpha * o.b;
                    const float rc = (float)ri;
                    rw_[c] = rc;
                    s += ri * ri;
                    const float xc = (float)x[c];  // = presmooth_x(L0, c, rc)
                    const double kx = APPLY(S0, c, (double)xc);
                    L0.x[c] = xc;
                    L0.r[c] = (float)(rc - kx);
                });
            } else {
                GRID_LOOP(c, n) {
                    P.psi[c] += (float)(alpha * pp[c]);
                    double ri = ro[c] - alpha * Ap[c];
                    float rc = (float)ri;
                    rw_[c] = rc;
                    s += ri * ri;
                    if (!single) {
                        float z = __ldg(L0.dinv + c) * rc;
                        P.z[c] = z;
                        sz += (double)rc * z;
                    }
                }
                if (!single) put_partial(P, RED_RZ, sz, s_red);
            }
            put_partial(P, RED_RR, s, s_red);
            float *t = r;
            r = rn;
            rn = t;
        }
        it++;
        trace_mark(P, 12);
        SYNC_OR(goto aborted);
        trace_mark(P, 13);
        rr = get_total(P, RED_RR, s_red);
        if (rr <= tol2) break;
        if (mg)
            ok = vcycle_rest(P, r, s_red, buf, smem);
        else if (single)
            ok = single_level(P, r, s_red, smem);
        if (!ok) goto aborted;
        {
            double rznew = get_total(P, RED_RZ, s_red);
            beta = rznew / rz;
            rz = rznew;
        }
    }

    // zero-mean projection of psi
    SYNC_OR(goto aborted);
    {
        double s = 0;
        GRID_LOOP(c, n) s += (double)__ldg(P.area + c) * P.psi[c];
        put_partial(P, RED_MEAN, s, s_red);
    }
    SYNC_OR(goto aborted);
    {
        float m = (float)(get_total(P, RED_MEAN, s_red) / P.total_area);
        GRID_LOOP(c, n) P.psi[c] -= m;
        // leave the final residual / direction in the caller's r / p buffers
        if (r != P.r) GRID_LOOP(c, n) P.r[c] = r[c];
        if (p != P.p) GRID_LOOP(c, n) P.p[c] = p[c];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.res->iters = it;
        P.res->relres = sqrt(rr / bb);
        P.res->status = 0;
        P.res->r_final = 0;
    }
    return;

aborted:
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.res->iters = it;
        P.res->relres = -1.0;
        P.res->status = 1;
    }
}

// ---- setup kernels -------------------------------------------------------

// Column j of the dense map of levels l0..nlev-1: the block's V-cycle applied
// to the unit vector e_j, stored row-major D[row][j] in FP64.
__global__ void __launch_bounds__(kPB, 1) k_dense_columns(SolveParams P, int l0, float *colbuf, double *D) {
    extern __shared__ __align__(16) unsigned char dyn[];
    float *smem = reinterpret_cast<float *>(dyn);
    const int nd = P.L[l0].S.n;
    for (int j = blockIdx.x; j < nd; j += gridDim.x) {
        SmemLevel lv[kMaxLev];
        carve_smem(P, l0, smem, lv);
        BLOCK_LOOP(c, nd) lv[l0].b[c] = c == j ? 1.0f : 0.0f;
        __syncthreads();
        float *col = colbuf + (size_t)blockIdx.x * nd;
        vcycle_block_smem(P, l0, lv, col);
        BLOCK_LOOP(c, nd) D[(size_t)c * nd + j] = col[c];
        __syncthreads();
    }
}

// Coarse-major weights of the structured rows of R: rw16[q][c] = the weight of
// fine cell q (q = 4*dj + di of the 4x4 window) in row c, taken from the CSR
// row (which the structured check has verified to be that window in order).
__global__ void k_build_rw16(LevelDev F, LevelDev C, float *rw16) {
    const int Nc = C.S.N, nc = C.S.n;
    GRID_LOOP(c, nc) {
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
    GRID_LOOP(c, C.S.n) {
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
    GRID_LOOP(i, F.S.n) {
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

static void pcg_attributes() {
    static bool attr = false;
    if (!attr) {
        int dev = 0, optin = 0;
        GGB_CHECK(cudaGetDevice(&dev));
        GGB_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa;
        GGB_CHECK(cudaFuncGetAttributes(&fa, k_pcg));
        GGB_CHECK(cudaFuncSetAttribute(k_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       optin - (int)fa.sharedSizeBytes));
        GGB_CHECK(cudaFuncSetAttribute(k_dense_columns, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr = true;
    }
}

static int pcg_grid_for(size_t smem) {
    pcg_attributes();
    int per = 0;
    GGB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg, kPB, smem));
    if (per < 1) fail_msg("the solve kernel cannot be resident on this device (%zu B shared memory)", smem);
    return device_sm_count() * std::min(per, 2);
}

int pcg_grid_size() { return pcg_grid_for(kStageBytes); }

// One solve launch; max_blocks > 0 caps its grid (batched planets: small
// grids take a share of the SMs so that several solves run at once).
void pcg_launch(const SolveParams &prm, cudaStream_t s, int max_blocks) {
    SolveParams p = prm;
    size_t smem = pcg_smem_bytes(p);
    void *args[] = {&p};
    int grid = pcg_grid_for(smem);
    if (max_blocks > 0) grid = std::max(1, std::min(grid, max_blocks));
    GGB_CHECK(cudaMemsetAsync(&p.bar->count, 0, sizeof(unsigned int), s));
    GGB_CHECK(cudaLaunchCooperativeKernel((const void *)k_pcg, dim3(grid), dim3(kPB), args, smem, s));
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
    float *colbuf = (float *)dev_alloc(sizeof(float) * (size_t)grid * nd);
    k_dense_columns<<<grid, kPB, smem, stream()>>>(p, l0, colbuf, D);
    GGB_LAUNCHED();
    GGB_CHECK(cudaStreamSynchronize(stream()));
    dev_free(colbuf);
    return D;
}

// ---- micro-benchmark of the grid barrier (additive entry point) ----------
__global__ void __launch_bounds__(kPB, 1) k_barrier_bench(GridBarrier *bar, int rounds, int *ok) {
    for (int k = 0; k < rounds; k++)
        if (!grid_sync(bar)) {
            if (threadIdx.x == 0) atomicExch(ok, 0);
            return;
        }
}

}  // namespace ggb

// Mean time of one grid-wide barrier of the solve kernel's launch shape, in
// microseconds (`rounds` barriers in one cooperative launch); -1 on timeout.
GGB_EXPORT double ggb_barrier_bench(int rounds) {
    using namespace ggb;
    GridBarrier *bar = (GridBarrier *)dev_alloc(sizeof(GridBarrier));
    int *ok = (int *)dev_alloc(sizeof(int));
    int one = 1;
    GGB_CHECK(cudaMemcpyAsync(ok, &one, sizeof(int), cudaMemcpyHostToDevice, stream()));
    int per = 0;
    GGB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_barrier_bench, kPB, 0));
    int grid = device_sm_count() * std::min(per, 2);
    cudaEvent_t e0, e1;
    GGB_CHECK(cudaEventCreate(&e0));
    GGB_CHECK(cudaEventCreate(&e1));
    void *args[] = {&bar, &rounds, &ok};
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
    return hok ? 1000.0 * ms / rounds : -1.0;
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
    GGB_CHECK(cudaMemcpyToSymbol(g_trace_n, &zero, sizeof(int)));
}

GGB_EXPORT int ggb_solve_trace(unsigned long long *out, int cap) {
    using namespace ggb;
    sync();
    int n = 0;
    GGB_CHECK(cudaMemcpyFromSymbol(&n, g_trace_n, sizeof(int)));
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
        GGB_CHECK(cudaMemcpyFromSymbol(&n, g_stage_trace_n, sizeof(int)));
        n = n < cap ? n : cap;
        n = n < 4096 ? n : 4096;
        if (n > 0 && buf) GGB_CHECK(cudaMemcpy(out, buf, sizeof(unsigned long long) * 2 * n, cudaMemcpyDeviceToHost));
        unsigned long long *null = nullptr;
        GGB_CHECK(cudaMemcpyToSymbol(g_stage_trace, &null, sizeof(null)));
        return n;
    }
    if (!buf) buf = (unsigned long long *)dev_alloc(sizeof(unsigned long long) * 2 * 4096);
    GGB_CHECK(cudaMemcpyToSymbol(g_stage_trace, &buf, sizeof(buf)));
    GGB_CHECK(cudaMemcpyToSymbol(g_stage_trace_n, &n, sizeof(int)));
    const int all = enable == 2;
    GGB_CHECK(cudaMemcpyToSymbol(g_stage_trace_all, &all, sizeof(int)));
    return 0;
}
