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

enum { RED_BB = 0, RED_RR, RED_PAP, RED_RZ, RED_MEAN, RED_N };

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
    for (int k = k0; k < k1; k++) acc += (double)(__ldg(F.rw + k) * F.r[__ldg(F.ridx + k)]);
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

// Coarsest level: `sweeps` Jacobi sweeps from 0 inside this block, result in L.xo.
__device__ void coarsest_block(const LevelDev &L, const float *b, int sweeps) {
    const int n = L.S.n;
    BLOCK_LOOP(c, n) L.x[c] = 0.f;
    __syncthreads();
    float *src = L.x, *dst = L.xo;
    for (int s = 0; s < sweeps; s++) {
        BLOCK_LOOP(c, n) jacobi_cell(L.S, L.dinv, b, src, dst, c);
        __syncthreads();
        float *t = src;
        src = dst;
        dst = t;
    }
    if (src != L.xo) {
        BLOCK_LOOP(c, n) L.xo[c] = src[c];
        __syncthreads();
    }
}

// Levels l0..nlev-1 of the V-cycle inside this block; b of level l0 is set.
__device__ void vcycle_block(const SolveParams &P, int l0, const float *b_top) {
    const int last = P.nlev - 1;
    for (int l = l0; l < last; l++) {
        const LevelDev &L = P.L[l];
        const float *b = (l == l0 && b_top) ? b_top : L.b;
        BLOCK_LOOP(c, L.S.n) presmooth_cell(L, c, [&](int k) -> float { return b[k]; });
        __syncthreads();
        BLOCK_LOOP(c, P.L[l + 1].S.n) restrict_cell(L, P.L[l + 1], c);
        __syncthreads();
    }
    coarsest_block(P.L[last], (last == l0 && b_top) ? b_top : P.L[last].b, P.coarse_sweeps);
    for (int l = last - 1; l >= l0; l--) {
        const LevelDev &L = P.L[l];
        const float *b = (l == l0 && b_top) ? b_top : L.b;
        BLOCK_LOOP(i, L.S.n) prolong_cell(L, P.L[l + 1], i);
        __syncthreads();
        BLOCK_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, b, L.x, L.xo, c);
        __syncthreads();
    }
}

// The rest of z = V(r) once level 0's pre-smooth (x, r of level 0) is complete
// and visible.  Ends with rz = r . z published; returns false on abort.
__device__ bool vcycle_rest(const SolveParams &P, const float *r, double *s_red) {
    const int G = P.nlev_grid;
    const int last = P.nlev - 1;
    // down: restrict level 0, then pre-smooth + restrict the other grid levels
    for (int l = 0; l < G; l++) {
        const LevelDev &L = P.L[l];
        if (l > 0) {
            GRID_LOOP(c, L.S.n) presmooth_cell(L, c, [&](int k) -> float { return L.b[k]; });
            if (!grid_sync(P.bar)) return false;
        }
        GRID_LOOP(c, P.L[l + 1].S.n) restrict_cell(L, P.L[l + 1], c);
        if (!grid_sync(P.bar)) return false;
    }
    // the coarse part
    if (!P.coarse_on_grid) {
        if (blockIdx.x == 0) vcycle_block(P, G, nullptr);
        if (!grid_sync(P.bar)) return false;
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
        if (!grid_sync(P.bar)) return false;
        if (l > 0) {
            GRID_LOOP(c, L.S.n) jacobi_cell(L.S, L.dinv, L.b, L.x, L.xo, c);
            if (!grid_sync(P.bar)) return false;
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
__device__ bool single_level(const SolveParams &P, const float *r, double *s_red) {
    const LevelDev &L = P.L[0];
    if (!P.coarse_on_grid) {
        if (blockIdx.x == 0) {
            coarsest_block(L, r, P.coarse_sweeps);
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

    // r = b - K psi, b = -A omega
    {
        double sb = 0, sr = 0;
        const float *psi = P.psi;
        auto X = [&](int k) -> double { return (double)psi[k]; };
        GRID_LOOP(c, n) {
            double b = -(double)__ldg(P.area + c) * P.omega[c];
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
            ok = vcycle_rest(P, r, s_red);
        } else if (single) {
            ok = single_level(P, r, s_red);
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
        if (!grid_sync(P.bar)) goto aborted;
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
        if (!grid_sync(P.bar)) goto aborted;
        rr = get_total(P, RED_RR, s_red);
        if (rr <= tol2) break;
        if (mg)
            ok = vcycle_rest(P, r, s_red);
        else if (single)
            ok = single_level(P, r, s_red);
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

int pcg_grid_size() {
    static int g = 0;
    if (!g) {
        int per = 0;
        GGB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pcg, kPB, 0));
        if (per < 1) fail_msg("the solve kernel cannot be resident on this device");
        g = device_sm_count() * std::min(per, 2);
    }
    return g;
}

void pcg_launch(const SolveParams &prm, cudaStream_t s) {
    SolveParams p = prm;
    void *args[] = {&p};
    GGB_CHECK(cudaLaunchCooperativeKernel((const void *)k_pcg, dim3(pcg_grid_size()), dim3(kPB), args, 0, s));
    GGB_LAUNCHED();
}

}  // namespace ggb
