// fluid.cu — the fluid.h entry points of libggb_cuda.so: discrete operators,
// the multigrid hierarchy, the Poisson solve launch, velocity from the stream
// function and the BFECC semi-Lagrangian vorticity step.
//
// Upstream: src/fluid.c.  Public arrays of Fluid are managed memory updated in
// place by the kernels below; every entry point synchronises before returning.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "ggb_internal.h"
#include "ggb_solver.h"

namespace ggb {

int pcg_grid_size();
int pcg_max_blocks();
int pcg_max_grid_n();
int pcg_block_size();
void pcg_launch(const SolveParams &prm, cudaStream_t s, int max_blocks = 0);
int pcg_check_structured(const LevelDev &F, const LevelDev &C);
float *pcg_build_rw16(const LevelDev &F, const LevelDev &C);
double *pcg_dense_map(const SolveParams &prm, int l0);

constexpr int kB = 256;

// ------------------------------------------------------------ operators

// upstream src/fluid.c:214-230
__global__ void k_divergence(int n, const float *pos, const unsigned char *nnb, const int *nbr, const float *elen,
                             const float *area, const float *vel, float *div) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D3 p = load3(pos + 3 * i), ui = load3(vel + 3 * i);
        double s = 0;
        for (int k = 0; k < nnb[i]; k++) {
            int j = nbr[kMaxNb * i + k];
            D3 nrm = normalize(sub(load3(pos + 3 * j), p));
            D3 um = add(ui, load3(vel + 3 * j));
            s += elen[kMaxNb * i + k] * 0.5 * dot(um, nrm);
        }
        div[i] = (float)(s / area[i]);
    }
}

// upstream src/fluid.c:233-250
__global__ void k_curl(int n, const float *pos, const unsigned char *nnb, const int *nbr, const float *elen,
                       const float *area, const float *vel, float *omega) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D3 p = load3(pos + 3 * i);
        D3 wi = cross(load3(vel + 3 * i), p);
        double s = 0;
        for (int k = 0; k < nnb[i]; k++) {
            int j = nbr[kMaxNb * i + k];
            D3 pj = load3(pos + 3 * j);
            D3 wj = cross(load3(vel + 3 * j), pj);
            D3 nrm = normalize(sub(pj, p));
            s += elen[kMaxNb * i + k] * 0.5 * dot(add(wi, wj), nrm);
        }
        omega[i] = (float)(s / area[i]);
    }
}

// y = sum_j w (x_j - x_i) / A_i on the face-tiled layout; upstream src/fluid.c:252-262
__global__ void k_laplacian(StencilDev S, const float *area, const float *x, float *y) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.n; i += gridDim.x * blockDim.x) {
        auto X = [&](int k) -> double { return (double)x[k]; };
        double kx = apply_k(S, i, (double)x[i], X);
        y[i] = (float)(-kx / area[i]);
    }
}

// Per-block FP64 partials of sum A f, then a one-block fixed-order total.
__global__ void k_wsum_partial(int n, const float *area, const float *f, double *part) {
    __shared__ double s_red[kB / 32 + 2];
    double s = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        s += (double)area[i] * f[i];
    double t = block_sum<kB>(s, s_red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void k_remove_mean(int n, const double *part, int nparts, double total_area, float *f) {
    __shared__ double s_red[kB / 32 + 2];
    double s = sum_partials<kB>(part, nparts, s_red);
    float m = (float)(s / total_area);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) f[i] -= m;
}

// u = p x sum_k gc_k (psi_j - psi_i); upstream src/fluid.c:361-376
__device__ __forceinline__ void velocity_body(int n, const float *pos, const unsigned char *nnb, const int *nbr, const float *gc,
                           const float *psi, float *vel, int vb_, int vnb_) {
    for (int i = vb_ * blockDim.x + threadIdx.x; i < n; i += vnb_ * blockDim.x) {
        D3 p = load3(pos + 3 * i), g = d3(0, 0, 0);
        double pi = psi[i];
        const int m = nnb[i];
        // the cell's 8 neighbour slots and 24 coefficients (rows padded to
        // kMaxNb, 16-byte aligned) as 16-byte loads; unrolled over the slots
        // so that the psi gathers are in flight together; the sum keeps the
        // order k = 0..m-1
        static_assert(kMaxNb == 8, "a row is two int4 slots and six float4 coefficients");
        const int4 *n4 = reinterpret_cast<const int4 *>(nbr + (size_t)kMaxNb * i);
        const float4 *g4 = reinterpret_cast<const float4 *>(gc + (size_t)3 * kMaxNb * i);
        const int4 na = __ldg(n4), nb = __ldg(n4 + 1);
        const int jj[kMaxNb] = {na.x, na.y, na.z, na.w, nb.x, nb.y, nb.z, nb.w};
        float gv[3 * kMaxNb];
#pragma unroll
        for (int u = 0; u < 6; u++) {
            const float4 q = __ldg(g4 + u);
            gv[4 * u] = q.x;
            gv[4 * u + 1] = q.y;
            gv[4 * u + 2] = q.z;
            gv[4 * u + 3] = q.w;
        }
#pragma unroll
        for (int k = 0; k < kMaxNb; k++) {
            if (k < m) g = add(g, scale(d3(gv[3 * k], gv[3 * k + 1], gv[3 * k + 2]), psi[jj[k]] - pi));
        }
        store3(vel + 3 * i, cross(p, g));
    }
}
__global__ void k_velocity(int n, const float *pos, const unsigned char *nnb, const int *nbr, const float *gc,
                           const float *psi, float *vel) {
    velocity_body(n, pos, nnb, nbr, gc, psi, vel, blockIdx.x, gridDim.x);
}

// max |u|^2 (formed in FP32 like upstream src/fluid.c:480-491) into *out as the
// bits of a non-negative float, so that the unsigned atomicMax orders them; one
// atomic per block.
__device__ __forceinline__ void max_speed2_body(int n, const float *vel, unsigned int *out, int vb_, int vnb_) {
    __shared__ float s_m[kB / 32];
    float m = 0.f;
    for (int i = vb_ * blockDim.x + threadIdx.x; i < n; i += vnb_ * blockDim.x) {
        const float *v = vel + 3 * i;
        float s = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        m = fmaxf(m, s);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) s_m[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < kB / 32 ? s_m[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) atomicMax(out, __float_as_uint(m));
    }
}
__global__ void __launch_bounds__(kB) k_max_speed2(int n, const float *vel, unsigned int *out) {
    max_speed2_body(n, vel, out, blockIdx.x, gridDim.x);
}

// The application driver's CFL step on the device (upstream src/main.c:422-426):
// dt = cfl h / max(vmax, 1e-6), vmax the square root of k_max_speed2's maximum.
__global__ void k_cfl_dt(const unsigned int *vmax_bits, double cfl, double h, double *dt) {
    const double vmax = sqrt((double)__uint_as_float(*vmax_bits));
    *dt = cfl * h / (vmax > 1e-6 ? vmax : 1e-6);
}

// ------------------------------------------------------------ advection

// Absolute vorticity q0 = omega + 2 Omega y of cell j, as FP32 (upstream
// src/fluid.c:435-437).
__device__ __forceinline__ float q0_of(const float *omega, const float *pos, double two_omega, int j) {
    return (float)(__ldg(omega + j) + two_omega * __ldg(pos + 3 * j + 1));
}

// Midpoint backtraces (backward and, for BFECC, forward), q0 = omega + 2 Omega y
// and the first resample q1 = q0 at the backward departure point, in one pass
// (upstream src/fluid.c:397-414, 435-441).  q0 at the four taps is formed from
// omega and the positions instead of being read back from q0, which this
// kernel is writing; the sample point is the departure point as stored
// (FP32), so q1 equals a separate resample of the stored q0 bit for bit.
// dt: the time step, or *dtp when dtp is not null (a device-side CFL step).
__device__ __forceinline__ void departures_body(GridDev g, const float *pos, const float *vel, const float *omega, double dt_in,
                             const double *dtp, double two_omega, int forward, float *dep_b, float *dep_f,
                             float *q0, float *q1, int vb_, int vnb_) {
    const double dt = dtp ? *dtp : dt_in;
    for (int i = vb_ * blockDim.x + threadIdx.x; i < g.n; i += vnb_ * blockDim.x) {
        D3 p = load3(pos + 3 * i), u = load3(vel + 3 * i);
        D3 pm = sphere_move(p, u, -0.5 * dt);
        D3 um = tangent(sample_vec(g, vel, pm), p);
        float *db = dep_b + 3 * i;
        store3(db, sphere_move(p, um, -dt));
        if (forward) {
            pm = sphere_move(p, u, 0.5 * dt);
            um = tangent(sample_vec(g, vel, pm), p);
            store3(dep_f + 3 * i, sphere_move(p, um, dt));
        }
        q0[i] = q0_of(omega, pos, two_omega, i);
        int idx[4];
        double wt[4];
        taps(g, load3(db), idx, wt);
        q1[i] = (float)(wt[0] * q0_of(omega, pos, two_omega, idx[0]) + wt[1] * q0_of(omega, pos, two_omega, idx[1]) +
                        wt[2] * q0_of(omega, pos, two_omega, idx[2]) + wt[3] * q0_of(omega, pos, two_omega, idx[3]));
    }
}
__global__ void k_departures(GridDev g, const float *pos, const float *vel, const float *omega, double dt_in,
                             const double *dtp, double two_omega, int forward, float *dep_b, float *dep_f,
                             float *q0, float *q1) {
    departures_body(g, pos, vel, omega, dt_in, dtp, two_omega, forward, dep_b, dep_f, q0, q1, blockIdx.x, gridDim.x);
}

// dst = src sampled at dep; with `correct`, dst = q0 + 0.5 (q0 - dst)
// (the BFECC corrected source, upstream src/fluid.c:445-448).
__device__ __forceinline__ void resample_body(GridDev g, const float *src, const float *dep, const float *q0, int correct, float *dst, int vb_, int vnb_) {
    for (int i = vb_ * blockDim.x + threadIdx.x; i < g.n; i += vnb_ * blockDim.x) {
        float v = (float)sample_scalar(g, src, load3(dep + 3 * i));
        if (correct) {
            float q = q0[i];
            v = q + 0.5f * (q - v);
        }
        dst[i] = v;
    }
}
__global__ void k_resample(GridDev g, const float *src, const float *dep, const float *q0, int correct, float *dst) {
    resample_body(g, src, dep, q0, correct, dst, blockIdx.x, gridDim.x);
}

// Limited resample of the corrected source at dep_b (clamped to the range of
// q0 over the same taps), then back to relative vorticity and relaxation
// toward the band state.  upstream src/fluid.c:449-474
// relax: the relaxation factor, or 1 - exp(-forcing *dtp) when dtp is not null.
__device__ __forceinline__ void limit_relax_body(GridDev g, const float *pos, const float *dep_b, const float *q0, const float *q2,
                              int bfecc, double two_omega, double relax_in, const double *dtp, double forcing,
                              const float *omega_band, float *q1, float *omega, int vb_, int vnb_) {
    const double relax = dtp ? (forcing > 0 ? 1.0 - exp(-forcing * *dtp) : 0.0) : relax_in;
    for (int i = vb_ * blockDim.x + threadIdx.x; i < g.n; i += vnb_ * blockDim.x) {
        float qn;
        if (bfecc) {
            int idx[4];
            double wt[4];
            taps(g, load3(dep_b + 3 * i), idx, wt);
            double v = 0, lo = 1e30, hi = -1e30;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                v += wt[k] * q2[idx[k]];
                double o = q0[idx[k]];
                lo = o < lo ? o : lo;
                hi = o > hi ? o : hi;
            }
            v = v < lo ? lo : v;
            v = v > hi ? hi : v;
            qn = (float)v;
            q1[i] = qn;
        } else {
            qn = q1[i];
        }
        double w = qn - two_omega * pos[3 * i + 1];
        w += relax * (omega_band[i] - w);
        omega[i] = (float)w;
    }
}
__global__ void k_limit_relax(GridDev g, const float *pos, const float *dep_b, const float *q0, const float *q2,
                              int bfecc, double two_omega, double relax_in, const double *dtp, double forcing,
                              const float *omega_band, float *q1, float *omega) {
    limit_relax_body(g, pos, dep_b, q0, q2, bfecc, two_omega, relax_in, dtp, forcing, omega_band, q1, omega, blockIdx.x, gridDim.x);
}

// ---------------------------------------------- batched stages (all planets)
// One launch per stage for every planet of a batch: block b runs the stage's
// body for planet map[b].x as block map[b].y of map[b].z, with that planet's
// arguments; the arithmetic per cell is the per-planet kernels'.

__global__ void __launch_bounds__(kB) k_max_speed2_batch(const PlanetStepDev *pl, const int4 *map) {
    const int4 m = map[blockIdx.x];
    const PlanetStepDev &P = pl[m.x];
    max_speed2_body(P.g.n, P.vel, P.vmax, m.y, m.z);
}

// dt of every planet (one thread each), k_cfl_dt's expression
__global__ void k_cfl_dt_batch(const PlanetStepDev *pl, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const PlanetStepDev &P = pl[i];
    const double vmax = sqrt((double)__uint_as_float(*P.vmax));
    *P.dt = P.cfl * P.g.h / (vmax > 1e-6 ? vmax : 1e-6);
}

__global__ void k_departures_batch(const PlanetStepDev *pl, const int4 *map) {
    const int4 m = map[blockIdx.x];
    const PlanetStepDev &P = pl[m.x];
    departures_body(P.g, P.pos, P.vel, P.omega, 0.0, P.dt, P.two_omega, P.bfecc, P.dep_b, P.dep_f, P.q0, P.q1, m.y,
                    m.z);
}

__global__ void k_resample_batch(const PlanetStepDev *pl, const int4 *map) {
    const int4 m = map[blockIdx.x];
    const PlanetStepDev &P = pl[m.x];
    if (!P.bfecc) return;
    resample_body(P.g, P.q1, P.dep_f, P.q0, 1, P.q2, m.y, m.z);
}

__global__ void k_limit_relax_batch(const PlanetStepDev *pl, const int4 *map) {
    const int4 m = map[blockIdx.x];
    const PlanetStepDev &P = pl[m.x];
    limit_relax_body(P.g, P.pos, P.dep_b, P.q0, P.q2, P.bfecc, P.two_omega, 0.0, P.dt, P.forcing, P.omega_band, P.q1,
                     P.omega, m.y, m.z);
}

__global__ void k_velocity_batch(const PlanetStepDev *pl, const int4 *map) {
    const int4 m = map[blockIdx.x];
    const PlanetStepDev &P = pl[m.x];
    velocity_body(P.g.n, P.pos, P.nnb, P.nbr, P.gc, P.psi, P.vel, m.y, m.z);
}

// ------------------------------------------------------------ multigrid setup

// Fine cell i -> bilinear taps on the coarse grid at its (FP32-stored) centre.
// upstream src/fluid.c:70-79
__global__ void k_ptaps(int nf, const float *fine_pos, GridDev coarse, int *ptap, float *pw, int *rcount) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
        int idx[4];
        double wt[4];
        taps(coarse, load3(fine_pos + 3 * i), idx, wt);
        for (int k = 0; k < 4; k++) {
            ptap[4 * i + k] = idx[k];
            pw[4 * i + k] = (float)wt[k];
            atomicAdd(rcount + idx[k], 1);  // row counts; exclusive scan gives the row starts
        }
    }
}

// Exclusive prefix sum in place over a[0..n] (one block; setup only).
__global__ void k_scan_inplace(int n, int *a) {
    __shared__ int s_tot[1024];
    const int T = blockDim.x, t = threadIdx.x;
    int chunk = (n + T - 1) / T, lo = min(n, t * chunk), hi = min(n, lo + chunk);
    int s = 0;
    for (int k = lo; k < hi; k++) s += a[k];
    s_tot[t] = s;
    __syncthreads();
    if (t == 0) {
        int acc = 0;
        for (int k = 0; k < T; k++) {
            int v = s_tot[k];
            s_tot[k] = acc;
            acc += v;
        }
    }
    __syncthreads();
    int acc = s_tot[t];
    for (int k = lo; k < hi; k++) {
        int v = a[k];
        a[k] = acc;
        acc += v;
    }
}

__global__ void k_rfill(int nf, const int *ptap, const int *rstart, int *cursor, int *rkey) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x)
        for (int k = 0; k < 4; k++) {
            int c = ptap[4 * i + k];
            int slot = atomicAdd(cursor + c, 1);
            rkey[rstart[c] + slot] = 4 * i + k;
        }
}

// Sort each row by (fine cell, tap) — the fill order of upstream src/fluid.c:88-95.
__global__ void k_rsort(int nc, const int *rstart, int *rkey, const float *pw, int *ridx, float *rw) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        int a = rstart[c], b = rstart[c + 1];
        for (int u = a + 1; u < b; u++) {
            int key = rkey[u], v = u - 1;
            while (v >= a && rkey[v] > key) {
                rkey[v + 1] = rkey[v];
                v--;
            }
            rkey[v + 1] = key;
        }
        for (int u = a; u < b; u++) {
            ridx[u] = rkey[u] >> 2;
            rw[u] = pw[rkey[u]];
        }
    }
}

// FP16 copy of a level's slot weights (mixed-precision V-cycle).
__global__ void k_to_half(size_t n, const float *src, __half *dst) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = __float2half_rn(src[i]);
}

// ------------------------------------------------------------ private state

struct FluidPriv {
    MGLevel lev[kMaxLev];  // public view; first member (Fluid::lev points here)
    GridTables *grid0 = nullptr;
    GridTables coarse[kMaxLev];
    int nlev = 0;
    int *ptap[kMaxLev] = {}, *rstart[kMaxLev] = {}, *ridx[kMaxLev] = {};
    float *pw[kMaxLev] = {}, *rw[kMaxLev] = {};
    float *lx[kMaxLev] = {}, *lxo[kMaxLev] = {}, *lb[kMaxLev] = {}, *lr[kMaxLev] = {};
    float *r2 = nullptr, *p2 = nullptr;
    double *part = nullptr;
    double *wpart = nullptr;
    GridBarrier *bar = nullptr;
    SolveResult *res = nullptr;
    SolveResult *res_host = nullptr;
    unsigned int *vmax_bits = nullptr;
    unsigned int *vmax_host = nullptr;
    int structured[kMaxLev] = {};  // level l -> l+1 transfers follow the index pattern
    float *rw16[kMaxLev] = {};     // coarse-major structured restriction weights
    double *dense = nullptr;       // dense map of the V-cycle below the grid levels
    int nd = 0;
    int last_flags = 0;            // kSolve* bits of the last solve
    // mixed-precision solve (ggb_fluid_set_precision): FP16 level vectors,
    // FP16 slot weights of the coarse levels, the previous z
    int mixed = 0;
    __half *hx[kMaxLev] = {}, *hxo[kMaxLev] = {}, *hb[kMaxLev] = {}, *hr[kMaxLev] = {};
    __half *wh[kMaxLev] = {};
    float *z2 = nullptr;
};

static FluidPriv *priv_of(const Fluid *F) {
    if (!F->lev) fail_msg("Fluid %p was not initialised by this library's fluid_init", (const void *)F);
    return reinterpret_cast<FluidPriv *>(F->lev);
}

static StencilDev stencil_of(const GridTables *t) {
    StencilDev s;
    s.wslot_h = nullptr;
    s.N = t->N;
    s.n = t->n;
    s.nring = t->nring;
    s.lgN = -1;
    for (int l = 0; l < 31; l++)
        if ((1 << l) == t->N) s.lgN = l;
    s.wslot = t->wslot;
    s.wslot_d = t->wslot_d;
    s.ring_nb = t->ring_nb;
    s.ring_w = t->ring_w;
    return s;
}

static unsigned blocks_for(int n) { return std::max(1u, std::min<unsigned>(grid_for(n, kB), 148u * 16u)); }

static void build_levels(Fluid *F, FluidPriv *Pv) {
    cudaStream_t s = stream();
    int N = F->cs->N, nlev = 1;
    while ((N >> nlev) >= 4 && ((N >> (nlev - 1)) % 2) == 0) nlev++;
    if (nlev > kMaxLev) nlev = kMaxLev;
    Pv->nlev = nlev;
    for (int l = 1; l < nlev; l++) {
        GridTables *C = &Pv->coarse[l];
        if (grid_build(C, N >> l, false) != 0) fail_msg("multigrid level %d (N=%d) failed", l, N >> l);
        const GridTables *Fg = l == 1 ? Pv->grid0 : &Pv->coarse[l - 1];
        int nf = Fg->n, nc = C->n;
        int L = l - 1;
        Pv->ptap[L] = (int *)dev_alloc(sizeof(int) * 4 * nf);
        Pv->pw[L] = (float *)dev_alloc(sizeof(float) * 4 * nf);
        Pv->rstart[L] = (int *)dev_alloc(sizeof(int) * (nc + 1));
        Pv->ridx[L] = (int *)dev_alloc(sizeof(int) * 4 * nf);
        Pv->rw[L] = (float *)dev_alloc(sizeof(float) * 4 * nf);
        int *cursor = (int *)dev_alloc(sizeof(int) * nc);
        int *rkey = (int *)dev_alloc(sizeof(int) * 4 * nf);
        k_ptaps<<<blocks_for(nf), kB, 0, s>>>(nf, Fg->pos, C->dev(), Pv->ptap[L], Pv->pw[L], Pv->rstart[L]);
        GGB_LAUNCHED();
        k_scan_inplace<<<1, 1024, 0, s>>>(nc + 1, Pv->rstart[L]);
        GGB_LAUNCHED();
        k_rfill<<<blocks_for(nf), kB, 0, s>>>(nf, Pv->ptap[L], Pv->rstart[L], cursor, rkey);
        GGB_LAUNCHED();
        k_rsort<<<blocks_for(nc), kB, 0, s>>>(nc, Pv->rstart[L], rkey, Pv->pw[L], Pv->ridx[L], Pv->rw[L]);
        GGB_LAUNCHED();
        GGB_CHECK(cudaStreamSynchronize(s));
        dev_free(cursor);
        dev_free(rkey);
    }
    for (int l = 0; l < nlev; l++) {
        int n = l == 0 ? Pv->grid0->n : Pv->coarse[l].n;
        Pv->lx[l] = (float *)dev_alloc(sizeof(float) * n);
        Pv->lxo[l] = (float *)dev_alloc(sizeof(float) * n);
        Pv->lb[l] = (float *)dev_alloc(sizeof(float) * n);
        Pv->lr[l] = (float *)dev_alloc(sizeof(float) * n);
    }
    F->nlev = nlev;
    for (int l = 0; l < nlev; l++) {
        MGLevel *M = &Pv->lev[l];
        memset(M, 0, sizeof(*M));
        const GridTables *t = l == 0 ? Pv->grid0 : &Pv->coarse[l];
        M->cs.N = t->N;
        M->cs.ncells = t->n;
        M->cs.h = t->h;
        M->cs.total_area = t->total_area;
    }
}

constexpr int kBlockLevelMax = 1536;  // levels up to N=16 form the dense coarse map

static SolveParams solve_params(Fluid *F, FluidPriv *Pv, int remove_mean, int maxit) {
    if (F->cs->N > pcg_max_grid_n())
        fail_msg("grids with N > %d exceed the solve kernel's staged window (N = %d)", pcg_max_grid_n(), F->cs->N);
    SolveParams P;
    memset(&P, 0, sizeof(P));
    const bool mg = F->prm.multigrid != 0;
    P.nlev = mg ? Pv->nlev : 0;
    P.coarse_sweeps = 60;
    P.remove_mean = remove_mean;
    P.maxit = maxit;
    P.tol = F->prm.cg_tol;
    P.total_area = Pv->grid0->total_area;
    for (int l = 0; l < (mg ? Pv->nlev : 1); l++) {
        const GridTables *t = l == 0 ? Pv->grid0 : &Pv->coarse[l];
        LevelDev &L = P.L[l];
        L.S = stencil_of(t);
        L.dinv = t->dinv;
        if (Pv->mixed) {
            L.S.wslot_h = Pv->wh[l];
            L.x = Pv->hx[l];
            L.xo = Pv->hxo[l];
            L.b = Pv->hb[l];
            L.r = Pv->hr[l];
        } else {
            L.x = Pv->lx[l];
            L.xo = Pv->lxo[l];
            L.b = Pv->lb[l];
            L.r = Pv->lr[l];
        }
        if (l + 1 < Pv->nlev) {
            L.ptap = Pv->ptap[l];
            L.pw = Pv->pw[l];
            L.rstart = Pv->rstart[l];
            L.ridx = Pv->ridx[l];
            L.rw = Pv->rw[l];
            L.structured = Pv->structured[l];
            L.rw16 = Pv->rw16[l];
        }
    }
    if (mg && Pv->nlev >= 2) {
        int G = 0;
        while (G < Pv->nlev - 1 && P.L[G].S.n > kBlockLevelMax) G++;
        if (G < 1) G = 1;
        P.nlev_grid = G;
        P.coarse_on_grid = (G == Pv->nlev - 1 && P.L[Pv->nlev - 1].S.n > kBlockLevelMax) ? 1 : 0;
    } else if (mg) {
        P.nlev_grid = 0;
        P.coarse_on_grid = P.L[0].S.n > kBlockLevelMax ? 1 : 0;
    }
    P.area = F->cs->area;
    P.omega = F->omega;
    P.psi = F->psi;
    P.r = F->r;
    P.r2 = Pv->r2;
    P.p = F->p;
    P.p2 = Pv->p2;
    P.Ap = F->Ap;
    P.z = F->z;
    P.mixed = Pv->mixed;
    P.z2 = Pv->z2;
    P.part = Pv->part;
    P.bar = Pv->bar;
    P.res = Pv->res;
    if (mg && Pv->dense) {
        P.dense = Pv->dense;
        P.nd = Pv->nd;
    }
    return P;
}

// Structured-transfer flags and the dense coarse map (after build_levels).
static void finish_levels(Fluid *F, FluidPriv *Pv) {
    SolveParams P = solve_params(F, Pv, 0, 1);
    P.mixed = 0;
    for (int l = 0; l + 1 < Pv->nlev; l++) {
        LevelDev Fl = P.L[l], C = P.L[l + 1];
        Fl.structured = 0;
        Pv->structured[l] = pcg_check_structured(Fl, C);
        if (Pv->structured[l]) Pv->rw16[l] = pcg_build_rw16(Fl, C);
    }
    if (Pv->nlev >= 2) {
        P = solve_params(F, Pv, 0, 1);  // with the structured flags
        int G = P.nlev_grid;
        if (G < Pv->nlev && P.L[G].S.n <= kBlockLevelMax) {
            Pv->dense = pcg_dense_map(P, G);
            Pv->nd = P.L[G].S.n;
        }
    }
}

void solve_trace_target(unsigned long long **buf, int *cap);

// Launch the solve and read back its result into F (sync).
// Queues a solve (at most max_blocks blocks when > 0) and the copy of its
// result; solve_collect reads the result after a synchronisation.
static void solve_launch(Fluid *F, FluidPriv *Pv, int remove_mean, int maxit, int max_blocks) {
    SolveParams P = solve_params(F, Pv, remove_mean, maxit);
    solve_trace_target(&P.trace, &P.trace_cap);
    cudaStream_t s = stream();
    stage_begin(ST_SOLVE);
    pcg_launch(P, s, max_blocks);
    stage_end(ST_SOLVE);
    GGB_CHECK(cudaMemcpyAsync(Pv->res_host, Pv->res, sizeof(SolveResult), cudaMemcpyDeviceToHost, s));
}

static int solve_collect(Fluid *F, FluidPriv *Pv) {
    const SolveResult &R = *Pv->res_host;
    Pv->last_flags = R.flags;
    if (R.status != 0) fail_msg("Poisson solve aborted: a grid barrier timed out");
    F->cg_iters = R.iters;
    F->cg_relres = R.relres;
    return R.iters;
}

static int run_solve(Fluid *F, FluidPriv *Pv, int remove_mean, int maxit) {
    solve_launch(F, Pv, remove_mean, maxit, 0);
    GGB_CHECK(cudaStreamSynchronize(stream()));
    stage_collect();
    return solve_collect(F, Pv);
}

}  // namespace ggb

using namespace ggb;

// ------------------------------------------------------------ public API

GGB_EXPORT void fluid_divergence(const CubeSphere *cs, const float *vel, float *div) {
    GridTables *t = grid_lookup(cs);
    Staged in, out;
    stage_in(in, vel, sizeof(float) * 3 * t->n);
    stage_out(out, div, sizeof(float) * t->n);
    k_divergence<<<blocks_for(t->n), kB, 0, stream()>>>(t->n, t->pos, t->nnb, t->nbr, t->elen, t->area,
                                                        (const float *)in.dev, (float *)out.dev);
    GGB_LAUNCHED();
    stage_finish(out);
}

GGB_EXPORT void fluid_curl(const CubeSphere *cs, const float *vel, float *omega) {
    GridTables *t = grid_lookup(cs);
    Staged in, out;
    stage_in(in, vel, sizeof(float) * 3 * t->n);
    stage_out(out, omega, sizeof(float) * t->n);
    k_curl<<<blocks_for(t->n), kB, 0, stream()>>>(t->n, t->pos, t->nnb, t->nbr, t->elen, t->area,
                                                  (const float *)in.dev, (float *)out.dev);
    GGB_LAUNCHED();
    stage_finish(out);
}

GGB_EXPORT void fluid_laplacian(const CubeSphere *cs, const float *x, float *y) {
    GridTables *t = grid_lookup(cs);
    Staged in, out;
    stage_in(in, x, sizeof(float) * t->n);
    stage_out(out, y, sizeof(float) * t->n);
    k_laplacian<<<blocks_for(t->n), kB, 0, stream()>>>(stencil_of(t), t->area, (const float *)in.dev,
                                                       (float *)out.dev);
    GGB_LAUNCHED();
    stage_finish(out);
}

GGB_EXPORT void fluid_remove_mean(const CubeSphere *cs, float *f) {
    GridTables *t = grid_lookup(cs);
    Staged io;
    stage_in(io, f, sizeof(float) * t->n);
    unsigned nb = std::min(blocks_for(t->n), 1024u);
    double *part = (double *)dev_alloc(sizeof(double) * nb);
    k_wsum_partial<<<nb, kB, 0, stream()>>>(t->n, t->area, (const float *)io.dev, part);
    GGB_LAUNCHED();
    k_remove_mean<<<blocks_for(t->n), kB, 0, stream()>>>(t->n, part, nb, t->total_area, (float *)io.dev);
    GGB_LAUNCHED();
    if (io.owned) {
        io.bytes = sizeof(float) * t->n;
        stage_finish(io);
    } else {
        sync();
    }
    dev_free(part);
}

GGB_EXPORT int fluid_init(Fluid *F, const CubeSphere *cs, const FluidParams *prm) {
    memset(F, 0, sizeof(*F));
    FluidPriv *Pv = new FluidPriv();
    Pv->grid0 = grid_lookup(cs);
    F->cs = cs;
    F->prm = *prm;
    size_t n = cs->ncells;
    float **fields[] = {&F->omega, &F->omega_band, &F->psi, &F->q0, &F->q1, &F->q2,
                        &F->r, &F->p, &F->Ap, &F->z, &F->dinv};
    for (float **f : fields) *f = (float *)managed_alloc(sizeof(float) * n);
    F->vel = (float *)managed_alloc(sizeof(float) * 3 * n);
    F->dep_b = (float *)managed_alloc(sizeof(float) * 3 * n);
    F->dep_f = (float *)managed_alloc(sizeof(float) * 3 * n);
    Pv->r2 = (float *)dev_alloc(sizeof(float) * n);
    Pv->p2 = (float *)dev_alloc(sizeof(float) * n);
    GGB_CHECK(cudaMemcpyAsync(F->dinv, Pv->grid0->dinv, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream()));
    F->lev = Pv->lev;
    if (prm->multigrid) {
        build_levels(F, Pv);
        finish_levels(F, Pv);
    } else {
        Pv->nlev = 0;
        Pv->lx[0] = (float *)dev_alloc(sizeof(float) * n);
        Pv->lxo[0] = (float *)dev_alloc(sizeof(float) * n);
        Pv->lb[0] = (float *)dev_alloc(sizeof(float) * n);
        Pv->lr[0] = (float *)dev_alloc(sizeof(float) * n);
        F->nlev = 0;
    }
    Pv->part = (double *)dev_alloc(sizeof(double) * 8 * pcg_max_blocks());
    Pv->wpart = (double *)dev_alloc(sizeof(double) * 1024);
    Pv->bar = (GridBarrier *)dev_alloc(sizeof(GridBarrier));
    Pv->res = (SolveResult *)dev_alloc(sizeof(SolveResult));
    Pv->vmax_bits = (unsigned int *)dev_alloc(sizeof(unsigned int));
    GGB_CHECK(cudaMallocHost(&Pv->res_host, sizeof(SolveResult)));
    GGB_CHECK(cudaMallocHost(&Pv->vmax_host, sizeof(unsigned int)));
    sync();
    return 0;
}

GGB_EXPORT void fluid_free(Fluid *F) {
    if (!F->lev) {
        memset(F, 0, sizeof(*F));
        return;
    }
    FluidPriv *Pv = priv_of(F);
    sync();
    float *fields[] = {F->omega, F->omega_band, F->psi, F->vel, F->q0, F->q1, F->q2,
                       F->dep_b, F->dep_f, F->r, F->p, F->Ap, F->z, F->dinv};
    for (float *f : fields) managed_free(f);
    for (int l = 0; l < kMaxLev; l++) {
        if (l >= 1 && Pv->coarse[l].n) grid_release(&Pv->coarse[l]);
        dev_free(Pv->ptap[l]);
        dev_free(Pv->pw[l]);
        dev_free(Pv->rstart[l]);
        dev_free(Pv->ridx[l]);
        dev_free(Pv->rw[l]);
        dev_free(Pv->rw16[l]);
        dev_free(Pv->lx[l]);
        dev_free(Pv->lxo[l]);
        dev_free(Pv->lb[l]);
        dev_free(Pv->lr[l]);
        dev_free(Pv->hx[l]);
        dev_free(Pv->hxo[l]);
        dev_free(Pv->hb[l]);
        dev_free(Pv->hr[l]);
        dev_free(Pv->wh[l]);
    }
    dev_free(Pv->z2);
    dev_free(Pv->r2);
    dev_free(Pv->p2);
    dev_free(Pv->part);
    dev_free(Pv->wpart);
    dev_free(Pv->bar);
    dev_free(Pv->res);
    dev_free(Pv->vmax_bits);
    dev_free(Pv->dense);
    cudaFreeHost(Pv->res_host);
    cudaFreeHost(Pv->vmax_host);
    delete Pv;
    memset(F, 0, sizeof(*F));
}

// Status bits of the last solve of F (kSolve* in ggb_solver.h; see ggb_ext.h).
GGB_EXPORT int ggb_solve_flags(const Fluid *F) { return priv_of(F)->last_flags; }

// Switches the Poisson solve of F between the plain form (mixed = 0: FP32
// vectors, FP64 stencil accumulation, the upstream CG) and the mixed-precision
// form (mixed = 1: FP16 V-cycle vectors and coarse slot weights, FP32
// accumulation, flexible CG).  The buffers of the mixed form are allocated on
// the first switch.  Returns 0, or -1 for a fluid without multigrid.
GGB_EXPORT int ggb_fluid_set_precision(Fluid *F, int mixed) {
    FluidPriv *Pv = priv_of(F);
    if (!mixed) {
        Pv->mixed = 0;
        return 0;
    }
    if (!F->prm.multigrid || Pv->nlev < 1) {
        fprintf(stderr, "ggb_fluid_set_precision: the mixed-precision solve needs the multigrid preconditioner\n");
        return -1;
    }
    if (!Pv->z2) {
        cudaStream_t s = stream();
        for (int l = 0; l < Pv->nlev; l++) {
            const GridTables *t = l == 0 ? Pv->grid0 : &Pv->coarse[l];
            const size_t n = t->n;
            Pv->hx[l] = (__half *)dev_alloc(sizeof(__half) * n);
            Pv->hxo[l] = (__half *)dev_alloc(sizeof(__half) * n);
            Pv->hb[l] = (__half *)dev_alloc(sizeof(__half) * n);
            Pv->hr[l] = (__half *)dev_alloc(sizeof(__half) * n);
            if (l >= 1) {
                Pv->wh[l] = (__half *)dev_alloc(sizeof(__half) * 4 * n);
                k_to_half<<<blocks_for((int)std::min<size_t>(4 * n, 1u << 30)), kB, 0, s>>>(4 * n, t->wslot, Pv->wh[l]);
                GGB_LAUNCHED();
            }
        }
        Pv->z2 = (float *)dev_alloc(sizeof(float) * F->cs->ncells);
        sync();
    }
    Pv->mixed = 1;
    return 0;
}

GGB_EXPORT int fluid_solve_psi(Fluid *F) {
    FluidPriv *Pv = priv_of(F);
    return run_solve(F, Pv, 0, F->prm.cg_maxit);
}

static void launch_velocity(Fluid *F, FluidPriv *Pv) {
    const GridTables *t = Pv->grid0;
    stage_begin(ST_VELOCITY);
    k_velocity<<<blocks_for(t->n), kB, 0, stream()>>>(t->n, t->pos, t->nnb, t->nbr, t->gc, F->psi, F->vel);
    GGB_LAUNCHED();
    stage_end(ST_VELOCITY);
}

GGB_EXPORT void fluid_compute_velocity(Fluid *F) {
    launch_velocity(F, priv_of(F));
    sync();
}

// upstream src/fluid.c:378-395
GGB_EXPORT void fluid_set_state(Fluid *F, const float *vel_initial, const float *vel_band) {
    FluidPriv *Pv = priv_of(F);
    const CubeSphere *cs = F->cs;
    size_t n = cs->ncells;
    fluid_curl(cs, vel_initial, F->omega);
    fluid_remove_mean(cs, F->omega);
    if (vel_band) {
        fluid_curl(cs, vel_band, F->omega_band);
        fluid_remove_mean(cs, F->omega_band);
    } else {
        GGB_CHECK(cudaMemsetAsync(F->omega_band, 0, sizeof(float) * n, stream()));
    }
    GGB_CHECK(cudaMemsetAsync(F->psi, 0, sizeof(float) * n, stream()));
    int keep = F->prm.cg_maxit;
    int cold = keep * 20 > 20000 ? keep * 20 : 20000;
    run_solve(F, Pv, 0, cold);
    launch_velocity(F, Pv);
    sync();
}

// upstream src/fluid.c:424-478, before the solve: departures, BFECC
// resampling, limiter and relaxation (dt, or *dtp on the device when dtp is
// not null).
static void advect_launch(Fluid *F, FluidPriv *Pv, double dt, const double *dtp) {
    const GridTables *t = Pv->grid0;
    cudaStream_t s = stream();
    double two_omega = 2.0 * F->prm.rotation;
    int bfecc = F->prm.bfecc != 0;
    GridDev g = t->dev();
    unsigned nb = blocks_for(t->n);
    stage_begin(ST_ADVECT);
    k_departures<<<nb, kB, 0, s>>>(g, t->pos, F->vel, F->omega, dt, dtp, two_omega, bfecc, F->dep_b, F->dep_f,
                                   F->q0, F->q1);
    GGB_LAUNCHED();
    if (bfecc) {
        k_resample<<<nb, kB, 0, s>>>(g, F->q1, F->dep_f, F->q0, 1, F->q2);
        GGB_LAUNCHED();
    }
    double relax = F->prm.forcing > 0 ? 1.0 - exp(-F->prm.forcing * dt) : 0.0;
    k_limit_relax<<<nb, kB, 0, s>>>(g, t->pos, F->dep_b, F->q0, F->q2, bfecc, two_omega, relax, dtp, F->prm.forcing,
                                    F->omega_band, F->q1, F->omega);
    GGB_LAUNCHED();
    stage_end(ST_ADVECT);
}

// The body of fluid_step without its synchronisation (the solve on at most
// max_blocks blocks when > 0).
static void step_launch(Fluid *F, FluidPriv *Pv, double dt, const double *dtp, int max_blocks) {
    advect_launch(F, Pv, dt, dtp);
    solve_launch(F, Pv, 1, F->prm.cg_maxit, max_blocks);
    launch_velocity(F, Pv);
}

GGB_EXPORT void fluid_step(Fluid *F, double dt) {
    FluidPriv *Pv = priv_of(F);
    step_launch(F, Pv, dt, nullptr, 0);
    sync();
    solve_collect(F, Pv);
}

// ---- the batched step's pieces (no synchronisation; see batch.cu) --------
namespace ggb {

// dt_dev = the driver's CFL step from the current velocity, on the device.
void fluid_cfl_dt_launch(const Fluid *F, double cfl, double *dt_dev) {
    FluidPriv *Pv = priv_of(F);
    cudaStream_t s = stream();
    const int n = F->cs->ncells;
    GGB_CHECK(cudaMemsetAsync(Pv->vmax_bits, 0, sizeof(unsigned int), s));
    k_max_speed2<<<std::min(blocks_for(n), 2u * device_sm_count()), kB, 0, s>>>(n, F->vel, Pv->vmax_bits);
    GGB_LAUNCHED();
    k_cfl_dt<<<1, 1, 0, s>>>(Pv->vmax_bits, cfl, F->cs->h, dt_dev);
    GGB_LAUNCHED();
}

void fluid_step_queue(Fluid *F, const double *dt_dev, int max_blocks) {
    step_launch(F, priv_of(F), 0.0, dt_dev, max_blocks);
}

void fluid_step_collect(Fluid *F) { solve_collect(F, priv_of(F)); }

unsigned batch_cell_blocks(int n) { return blocks_for(n); }

void fluid_step_dev(Fluid *F, double cfl, double *dt_dev, unsigned int *vmax_dev, PlanetStepDev *out) {
    FluidPriv *Pv = priv_of(F);
    const GridTables *t = Pv->grid0;
    PlanetStepDev &d = *out;
    d.g = t->dev();
    d.pos = t->pos;
    d.nnb = t->nnb;
    d.nbr = t->nbr;
    d.gc = t->gc;
    d.vel = F->vel;
    d.omega = F->omega;
    d.omega_band = F->omega_band;
    d.psi = F->psi;
    d.q0 = F->q0;
    d.q1 = F->q1;
    d.q2 = F->q2;
    d.dep_b = F->dep_b;
    d.dep_f = F->dep_f;
    d.two_omega = 2.0 * F->prm.rotation;
    d.forcing = F->prm.forcing;
    d.cfl = cfl;
    d.bfecc = F->prm.bfecc != 0;
    d.dt = dt_dev;
    d.vmax = vmax_dev;
}

void batch_cfl_launch(const PlanetStepDev *pl, int n, const int4 *map, int nb, unsigned int *vmax_all) {
    cudaStream_t s = stream();
    GGB_CHECK(cudaMemsetAsync(vmax_all, 0, sizeof(unsigned int) * n, s));
    k_max_speed2_batch<<<nb, kB, 0, s>>>(pl, map);
    GGB_LAUNCHED();
    k_cfl_dt_batch<<<grid_for(n, 128), 128, 0, s>>>(pl, n);
    GGB_LAUNCHED();
}

void batch_advect_launch(const PlanetStepDev *pl, const int4 *map, int nb, bool any_bfecc) {
    cudaStream_t s = stream();
    k_departures_batch<<<nb, kB, 0, s>>>(pl, map);
    GGB_LAUNCHED();
    if (any_bfecc) {
        k_resample_batch<<<nb, kB, 0, s>>>(pl, map);
        GGB_LAUNCHED();
    }
    k_limit_relax_batch<<<nb, kB, 0, s>>>(pl, map);
    GGB_LAUNCHED();
}

void batch_velocity_launch(const PlanetStepDev *pl, const int4 *map, int nb) {
    k_velocity_batch<<<nb, kB, 0, stream()>>>(pl, map);
    GGB_LAUNCHED();
}

void fluid_result_queue(Fluid *F) {
    FluidPriv *Pv = priv_of(F);
    GGB_CHECK(cudaMemcpyAsync(Pv->res_host, Pv->res, sizeof(SolveResult), cudaMemcpyDeviceToHost, stream()));
}

// The batched step around one batched solve launch: fluid_advect_queue, then
// the solve (its parameters from fluid_step_solve_params; bar: the barrier the
// batched launch gives this planet), then fluid_result_velocity_queue.
void fluid_advect_queue(Fluid *F, const double *dt_dev) { advect_launch(F, priv_of(F), 0.0, dt_dev); }

void fluid_step_solve_params(Fluid *F, GridBarrier *bar, SolveParams *out) {
    FluidPriv *Pv = priv_of(F);
    *out = solve_params(F, Pv, 1, F->prm.cg_maxit);
    out->bar = bar;
}

int fluid_solve_mixed(const Fluid *F) { return priv_of(F)->mixed; }

// Device time of F's last collected solve, in seconds.
double fluid_last_solve_seconds(const Fluid *F) { return 1e-9 * (double)priv_of(F)->res_host->ns; }

void fluid_result_velocity_queue(Fluid *F) {
    FluidPriv *Pv = priv_of(F);
    GGB_CHECK(cudaMemcpyAsync(Pv->res_host, Pv->res, sizeof(SolveResult), cudaMemcpyDeviceToHost, stream()));
    launch_velocity(F, Pv);
}

}  // namespace ggb

GGB_EXPORT double fluid_max_speed(const Fluid *F) {
    FluidPriv *Pv = priv_of(F);
    cudaStream_t s = stream();
    int n = F->cs->ncells;
    stage_begin(ST_MAXSPEED);
    GGB_CHECK(cudaMemsetAsync(Pv->vmax_bits, 0, sizeof(unsigned int), s));
    k_max_speed2<<<std::min(blocks_for(n), 2u * device_sm_count()), kB, 0, s>>>(n, F->vel, Pv->vmax_bits);
    GGB_LAUNCHED();
    stage_end(ST_MAXSPEED);
    GGB_CHECK(cudaMemcpyAsync(Pv->vmax_host, Pv->vmax_bits, sizeof(unsigned int), cudaMemcpyDeviceToHost, s));
    GGB_CHECK(cudaStreamSynchronize(s));
    stage_collect();
    float m;
    memcpy(&m, Pv->vmax_host, sizeof(m));
    return sqrt((double)m);
}

