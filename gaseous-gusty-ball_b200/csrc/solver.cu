// solver.cu — the Poisson solve K psi = -A omega as ONE persistent cooperative
// kernel: warm-started preconditioned conjugate gradients whose
// preconditioner is a symmetric multigrid V-cycle (damped-Jacobi smoother,
// bilinear prolongation P, restriction R = P^T, many-sweep Jacobi on the
// coarsest grid), with FP64 dot products and FP64 zero-mean projections.
//
// Upstream: src/fluid.c:41-160 (multigrid), :264-275 (mean), :290-358 (PCG).
// The arithmetic of every vector update follows upstream (FP32 vectors, FP64
// accumulation); the schedule is this library's: phases are separated by a
// bounded grid-wide barrier instead of host loops, the neighbour values of a
// freshly updated vector are recomputed on the fly where that saves a
// barrier (p = z + beta p inside K p; r - alpha Ap inside the level-0
// pre-smooth), and the small coarse levels run inside thread block 0.
#include <algorithm>
#include <cstdio>

#include "ggb_internal.h"
#include "ggb_solver.h"

namespace ggb {

constexpr int kPB = 512;           // threads per block of the persistent kernel
constexpr double kOmegaJ = 0.8;    // upstream MG_OMEGA
constexpr double kCorrScale = 1.0; // upstream MG_CORR_SCALE

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

// ---- per-cell pieces of the V-cycle -------------------------------------

// Pre-smooth from x = 0 with right-hand side b: x = w D^-1 b, r = b - K x
// (x at the neighbours recomputed from b).
template <class B>
__device__ __forceinline__ void presmooth_cell(const LevelDev &L, int c, B bval) {
    const float *dv = L.dinv;
    auto X = [&](int k) -> double { return (double)(float)(kOmegaJ * __ldg(dv + k) * bval(k)); };
    float bc = bval(c);
    float xc = (float)(kOmegaJ * __ldg(dv + c) * bc);
    double kx = apply_k(L.S, c, (double)xc, X);
    L.x[c] = xc;
    L.r[c] = (float)(bc - kx);
}

// b_coarse[c] = sum over row c of R of rw * r_fine.
__device__ __forceinline__ void restrict_cell(const LevelDev &F, const LevelDev &C, int c) {
    int k0 = __ldg(F.rstart + c), k1 = __ldg(F.rstart + c + 1);
    double acc = 0;
    int k = k0;
    for (; k + 4 <= k1; k += 4) {  // four independent gathers per round
        int i0 = __ldg(F.ridx + k), i1 = __ldg(F.ridx + k + 1), i2 = __ldg(F.ridx + k + 2), i3 = __ldg(F.ridx + k + 3);
        float w0 = __ldg(F.rw + k), w1 = __ldg(F.rw + k + 1), w2 = __ldg(F.rw + k + 2), w3 = __ldg(F.rw + k + 3);
        float r0 = F.r[i0], r1 = F.r[i1], r2 = F.r[i2], r3 = F.r[i3];
        acc += (double)(w0 * r0);
        acc += (double)(w1 * r1);
        acc += (double)(w2 * r2);
        acc += (double)(w3 * r3);
    }
    for (; k < k1; k++) acc += (double)(__ldg(F.rw + k) * F.r[__ldg(F.ridx + k)]);
    C.b[c] = (float)acc;
}

// x_fine += P xo_coarse.
__device__ __forceinline__ void prolong_cell(const LevelDev &F, const LevelDev &C, int i) {
    const int *t = F.ptap + 4 * i;
    const float *w = F.pw + 4 * i;
    const float *xc = C.xo;
    float s = __ldg(w) * xc[__ldg(t)] + __ldg(w + 1) * xc[__ldg(t + 1)] + __ldg(w + 2) * xc[__ldg(t + 2)] +
              __ldg(w + 3) * xc[__ldg(t + 3)];
    F.x[i] += (float)(kCorrScale * s);
}

// One damped-Jacobi sweep src -> dst: dst = src + w D^-1 (b - K src).
__device__ __forceinline__ float jacobi_cell(const StencilDev &S, const float *dinv, const float *b, const float *src,
                                             float *dst, int c) {
    auto X = [&](int k) -> double { return (double)src[k]; };
    float xc = src[c];
    float rc = (float)(b[c] - apply_k(S, c, (double)xc, X));
    float out = xc + (float)(kOmegaJ * __ldg(dinv + c) * rc);
    dst[c] = out;
    return out;
}

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

// ---- the coarse levels inside block 0, vectors in shared memory ----------
// Levels l0..nlev-1 have at most kBlockCells cells in total; each gets x, xo,
// b, r slices of the dynamic shared memory.  The operator tables stay in
// global memory (read-only, L1-cached).

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
// cell has its own thread, the cell's links, 1/diag and b stay in registers
// for all sweeps (the level has ~100 cells and 60 sweeps are latency-bound).
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

// Levels l0..nlev-1 of the V-cycle inside this block.  Reads b of level l0
// from global memory and writes xo of level l0 back to global memory.
__device__ void vcycle_block(const SolveParams &P, int l0, float *smem) {
    SmemLevel lv[kMaxLev];
    carve_smem(P, l0, smem, lv);
    const int last = P.nlev - 1;
    BLOCK_LOOP(c, P.L[l0].S.n) lv[l0].b[c] = P.L[l0].b[c];
    __syncthreads();
    for (int l = l0; l < last; l++) {
        LevelDev L = P.L[l];
        L.x = lv[l].x;
        L.r = lv[l].r;
        const float *b = lv[l].b;
        BLOCK_LOOP(c, L.S.n) presmooth_cell(L, c, [&](int k) -> float { return b[k]; });
        __syncthreads();
        trace_mark(P, 2000 + l);
        LevelDev C = P.L[l + 1];
        C.b = lv[l + 1].b;
        BLOCK_LOOP(c, C.S.n) restrict_cell(L, C, c);
        __syncthreads();
        trace_mark(P, 2100 + l);
    }
    coarsest_smem(P.L[last], lv[last], P.coarse_sweeps);
    trace_mark(P, 2200);
    for (int l = last - 1; l >= l0; l--) {
        LevelDev L = P.L[l];
        L.x = lv[l].x;
        LevelDev C = P.L[l + 1];
        C.xo = lv[l + 1].xo;
        BLOCK_LOOP(i, L.S.n) prolong_cell(L, C, i);
        __syncthreads();
        trace_mark(P, 2300 + l);
        float *xo = l == l0 ? P.L[l0].xo : lv[l].xo;  // level l0's result goes to global memory
        BLOCK_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, lv[l].b, lv[l].x, xo, c);
        __syncthreads();
        trace_mark(P, 2400 + l);
    }
    if (l0 == last) {
        BLOCK_LOOP(c, P.L[last].S.n) P.L[last].xo[c] = lv[last].xo[c];
        __syncthreads();
    }
}

// The rest of z = V(r) once level 0's pre-smooth (x, r of level 0) is complete
// and visible.  Ends with rz = r . z published; returns false on abort.
__device__ bool vcycle_rest(const SolveParams &P, const float *r, double *s_red, float *smem) {
    const int G = P.nlev_grid;
    const int last = P.nlev - 1;
    // down: restrict level 0, then pre-smooth + restrict the other grid levels
    for (int l = 0; l < G; l++) {
        const LevelDev &L = P.L[l];
        if (l > 0) {
            GRID_LOOP(c, L.S.n) presmooth_cell(L, c, [&](int k) -> float { return L.b[k]; });
            trace_mark(P, 100 + l);
            if (!grid_sync(P.bar)) return false;
            trace_mark(P, 200 + l);
        }
        GRID_LOOP(c, P.L[l + 1].S.n) restrict_cell(L, P.L[l + 1], c);
        trace_mark(P, 300 + l);
        if (!grid_sync(P.bar)) return false;
        trace_mark(P, 400 + l);
    }
    // the coarse part
    if (!P.coarse_on_grid) {
        if (blockIdx.x == 0) vcycle_block(P, G, smem);
        trace_mark(P, 500);
        if (!grid_sync(P.bar)) return false;
        trace_mark(P, 600);
    } else {
        // G == last: the coarsest level is large, sweep it grid-wide
        const LevelDev &L = P.L[last];
        GRID_LOOP(c, L.S.n) L.x[c] = 0.f;
        if (!grid_sync(P.bar)) return false;
        float *src = L.x, *dst = L.xo;
        for (int s = 0; s < P.coarse_sweeps; s++) {
            GRID_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, L.b, src, dst, c);
            if (!grid_sync(P.bar)) return false;
            float *t = src;
            src = dst;
            dst = t;
        }
        if (src != L.xo) {
            GRID_LOOP(c, L.S.n) L.xo[c] = src[c];
            if (!grid_sync(P.bar)) return false;
        }
    }
    // up: prolong + post-smooth; level 0 writes z and the rz partial
    for (int l = G - 1; l >= 0; l--) {
        const LevelDev &L = P.L[l];
        GRID_LOOP(i, L.S.n) prolong_cell(L, P.L[l + 1], i);
        trace_mark(P, 700 + l);
        if (!grid_sync(P.bar)) return false;
        trace_mark(P, 800 + l);
        if (l > 0) {
            GRID_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, L.b, L.x, L.xo, c);
            trace_mark(P, 900 + l);
            if (!grid_sync(P.bar)) return false;
            trace_mark(P, 1000 + l);
        } else {
            double s = 0;
            GRID_LOOP(c, L.S.n) {
                float z = jacobi_cell(L.S, L.dinv, r, L.x, P.z, c);
                s += (double)r[c] * z;
            }
            put_partial(P, RED_RZ, s, s_red);
            if (!grid_sync(P.bar)) return false;
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
        if (!grid_sync(P.bar)) return false;
        float *src = L.x, *dst = L.xo;
        for (int s = 0; s < P.coarse_sweeps; s++) {
            GRID_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, r, src, dst, c);
            if (!grid_sync(P.bar)) return false;
            float *t = src;
            src = dst;
            dst = t;
        }
        if (src != L.xo) {
            GRID_LOOP(c, L.S.n) L.xo[c] = src[c];
        }
    }
    if (!grid_sync(P.bar)) return false;
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
    extern __shared__ float smem[];
    double *s_red = sh.v;
    const LevelDev &L0 = P.L[0];
    const StencilDev &S0 = L0.S;
    const int n = S0.n;
    const bool mg = P.nlev >= 2;
    const bool single = P.nlev == 1;
    float *r = P.r, *rn = P.r2, *p = P.p, *pn = P.p2;
    double bb, rr, rz = 0, tol2, beta = 0;
    int it = 0;
    bool first = true, ok = true;

    // zero-mean projection of omega (FP64 sum), upstream src/fluid.c:264-275
    if (P.remove_mean) {
        double s = 0;
        GRID_LOOP(c, n) s += (double)__ldg(P.area + c) * P.omega[c];
        put_partial(P, RED_MEAN, s, s_red);
        if (!grid_sync(P.bar)) goto aborted;
        float m = (float)(get_total(P, RED_MEAN, s_red) / P.total_area);
        GRID_LOOP(c, n) P.omega[c] -= m;  // read back below only at the own cell
    }

    // FP64 projection that makes the singular system consistent: the stored
    // FP32 omega keeps a residual area-weighted mean m2 (the FP32 rounding of
    // the subtracted mean); b = -A (omega - m2) is formed in FP64 so that
    // sum b = 0 to double precision.  Without it the constant mode of the
    // residual stays at the FP32 rounding level and CG diverges once the
    // residual reaches it.
    double m2;
    {
        double s = 0, sa = 0;
        GRID_LOOP(c, n) {
            double a = __ldg(P.area + c);
            s += a * P.omega[c];
            sa += a;
        }
        put_partial(P, RED_MEAN, s, s_red);
        put_partial(P, RED_AREA, sa, s_red);
        if (!grid_sync(P.bar)) goto aborted;
        m2 = get_total(P, RED_MEAN, s_red) / get_total(P, RED_AREA, s_red);
    }

    // r = b - K psi, b = -A (omega - m2)
    {
        double sb = 0, sr = 0;
        const float *psi = P.psi;
        auto X = [&](int k) -> double { return (double)psi[k]; };
        GRID_LOOP(c, n) {
            double b = -(double)__ldg(P.area + c) * ((double)P.omega[c] - m2);
            double ri = b - apply_k(S0, c, (double)psi[c], X);
            r[c] = (float)ri;
            sb += b * b;
            sr += ri * ri;
        }
        put_partial(P, RED_BB, sb, s_red);
        put_partial(P, RED_RR, sr, s_red);
    }
    if (!grid_sync(P.bar)) goto aborted;
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
            GRID_LOOP(c, n) presmooth_cell(L0, c, [&](int k) -> float { return r[k]; });
            if (!grid_sync(P.bar)) goto aborted;
            ok = vcycle_rest(P, r, s_red, smem);
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
            auto PN = [&](int k) -> float { return fst ? z[k] : (float)(z[k] + be * po[k]); };
            auto X = [&](int k) -> double { return (double)PN(k); };
            double s = 0;
            GRID_LOOP(c, n) {
                float pc = PN(c);
                double a = apply_k(S0, c, (double)pc, X);
                pn[c] = pc;
                P.Ap[c] = (float)a;
                s += a * pc;
            }
            put_partial(P, RED_PAP, s, s_red);
            float *t = p;
            p = pn;
            pn = t;
            first = false;
        }
        trace_mark(P, 10);
        if (!grid_sync(P.bar)) goto aborted;
        trace_mark(P, 11);
        {
            double pAp = get_total(P, RED_PAP, s_red);
            if (pAp <= 0) break;
            const double alpha = rz / pAp;
            const float *Ap = P.Ap;
            const float *ro = r;
            double s = 0, sz = 0;
            if (mg) {
                // psi += alpha p; r' = r - alpha Ap; level-0 pre-smooth of r'
                auto RN = [&](int k) -> float { return (float)(ro[k] - alpha * Ap[k]); };
                GRID_LOOP(c, n) {
                    P.psi[c] += (float)(alpha * p[c]);
                    double ri = ro[c] - alpha * Ap[c];
                    rn[c] = (float)ri;
                    s += ri * ri;
                    presmooth_cell(L0, c, RN);
                }
            } else {
                GRID_LOOP(c, n) {
                    P.psi[c] += (float)(alpha * p[c]);
                    double ri = ro[c] - alpha * Ap[c];
                    float rc = (float)ri;
                    rn[c] = rc;
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
        if (!grid_sync(P.bar)) goto aborted;
        trace_mark(P, 13);
        rr = get_total(P, RED_RR, s_red);
        if (rr <= tol2) break;
        if (mg)
            ok = vcycle_rest(P, r, s_red, smem);
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
    if (!grid_sync(P.bar)) goto aborted;
    {
        double s = 0;
        GRID_LOOP(c, n) s += (double)__ldg(P.area + c) * P.psi[c];
        put_partial(P, RED_MEAN, s, s_red);
    }
    if (!grid_sync(P.bar)) goto aborted;
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

// ---------------------------------------------------------------- host

int pcg_block_size() { return kPB; }

static unsigned long long *g_trace_dev = nullptr;
static int g_trace_cap = 0;
void solve_trace_target(unsigned long long **buf, int *cap) {
    *buf = g_trace_dev;
    *cap = g_trace_cap;
}

// Dynamic shared memory of a launch: x, xo, b, r of every level run by block 0.
static size_t pcg_smem_bytes(const SolveParams &p) {
    size_t cells = 0;
    if (p.nlev >= 2 && !p.coarse_on_grid)
        for (int l = p.nlev_grid; l < p.nlev; l++) cells += p.L[l].S.n;
    if (p.nlev == 1 && !p.coarse_on_grid) cells = p.L[0].S.n;
    return 4 * sizeof(float) * cells;
}

int pcg_max_blocks() { return 2 * device_sm_count(); }

static int pcg_grid_for(size_t smem) {
    static bool attr = false;
    if (!attr) {
        GGB_CHECK(cudaFuncSetAttribute(k_pcg, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr = true;
    }
    int per = 0;
    GGB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg, kPB, smem));
    if (per < 1) fail_msg("the solve kernel cannot be resident on this device (%zu B shared memory)", smem);
    return device_sm_count() * std::min(per, 2);
}

int pcg_grid_size() { return pcg_grid_for(0); }

void pcg_launch(const SolveParams &prm, cudaStream_t s) {
    SolveParams p = prm;
    size_t smem = pcg_smem_bytes(p);
    void *args[] = {&p};
    GGB_CHECK(cudaLaunchCooperativeKernel((const void *)k_pcg, dim3(pcg_grid_for(smem)), dim3(kPB), args, smem, s));
    GGB_LAUNCHED();
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
