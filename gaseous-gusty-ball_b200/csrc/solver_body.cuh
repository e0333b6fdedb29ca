// solver_body.cuh — the device code of the persistent solve kernel k_pcg
// (constants, staged stencil phases, V-cycle, PCG body), included inside a
// namespace by solver.cu (the 512-thread kernel and everything else) and by
// solver_wide.cu (the 640-thread kernel).  Two translation units keep the
// compiler's inlining and register allocation of each kernel independent of
// the other: with both block sizes in one unit the 512-thread plain kernel
// lost its inlined V-cycle and ran 20 % slower.
//
// Upstream: src/fluid.c:41-160 (multigrid), :264-275 (mean), :290-358 (PCG).
// Must be included after ggb_internal.h and ggb_solver.h, inside a namespace.

constexpr int kPB = 512;            // threads per block of the persistent kernel
constexpr int kPBWide = 640;        // ... for grids from kWideMinN on (more loads in flight per SM)
constexpr int kWideMinN = 384;      // measured: 512 threads faster at N = 256, 640 at N = 512
constexpr int kRedBlock = 1024;     // block size the reductions are written for (absent warps add zeros)
constexpr double kOmegaJ = 0.8;     // upstream MG_OMEGA
constexpr double kCorrScale = 1.0;  // upstream MG_CORR_SCALE
constexpr int kStageCap = 3584;     // cells of a block's staged window (value + 4 slot weights FP64, 3 FP32 own inputs)
constexpr int kRingCap = 1024;      // boundary-ring cells of one staged sub-range (their off-face link sums)
constexpr int kStageWords = kStageCap * 5 + (kStageCap * 3 + 1) / 2 + kRingCap;  // in doubles
constexpr size_t kStageBytes = (size_t)kStageWords * sizeof(double);
static_assert((kStageCap * 3) % 2 == 0, "the ring sums follow the own-input arrays on an 8-byte boundary");

enum { RED_BB = 0, RED_RR, RED_PAP, RED_RZ, RED_MEAN, RED_AREA, RED_RZO, RED_N };

// Storage (V) and accumulation (A) types of the two precisions.
template <bool MP>
struct Prec {
    using V = float;
    using A = double;
};
template <>
struct Prec<true> {
    using V = __half;
    using A = float;
};

__device__ __forceinline__ float ldv(const float *p, int k) { return p[k]; }
__device__ __forceinline__ float ldv(const __half *p, int k) { return __half2float(p[k]); }
__device__ __forceinline__ void stv(float *p, int k, float v) { p[k] = v; }
__device__ __forceinline__ void stv(__half *p, int k, float v) { p[k] = __float2half_rn(v); }
// store and return the stored value
__device__ __forceinline__ float stv_get(float *p, int k, float v) {
    p[k] = v;
    return v;
}
__device__ __forceinline__ float stv_get(__half *p, int k, float v) {
    const __half h = __float2half_rn(v);
    p[k] = h;
    return __half2float(h);
}
// v as the storage type would hold it (rounded to FP16 in the mixed solve)
template <bool MP>
__device__ __forceinline__ float as_stored(float v) {
    return MP ? __half2float(__float2half_rn(v)) : v;
}
template <bool MP>
__device__ __forceinline__ typename Prec<MP>::V *lv(void *p) {
    return static_cast<typename Prec<MP>::V *>(p);
}

// Scale factors of the mixed V-cycle's transfers (1 in the plain solve).
template <bool MP>
__device__ __forceinline__ float restrict_scale() {
    return MP ? 0.25f : 1.0f;
}
template <bool MP>
__device__ __forceinline__ float prolong_scale() {
    return MP ? 4.0f : 1.0f;
}

// Slot weight at index q (= s * n + cell) of a level's FP64 (plain), FP16
// (mixed, when present) or FP32 slot table, as the stencil's accumulation type.
template <bool MP>
__device__ __forceinline__ typename Prec<MP>::A slot_w(const double *wd, const float *wf, const __half *wh, int q) {
    if (MP) {
        if (wh) return __half2float(wh[q]);
        return __ldg(wf + q);
    }
    return __ldg(wd + q);
}

// The block's place in its solve's grid (its "virtual grid"): the whole
// launch for a single solve (blockIdx.x of gridDim.x), or the share of the
// blocks of a batched launch that one planet's solve runs on.
__shared__ int s_vgrid[2];
__device__ __forceinline__ int vb() { return s_vgrid[0]; }
__device__ __forceinline__ int vnb() { return s_vgrid[1]; }

// Phase trace (diagnostics): block 0, thread 0 records (mark, %globaltimer).
__device__ int g_trace_n;
__device__ __forceinline__ void trace_mark(const SolveParams &P, int mark) {
    if (P.trace && vb() == 0 && threadIdx.x == 0) {
        int k = g_trace_n;
        if (k < P.trace_cap) {
            P.trace[2 * k] = (unsigned long long)mark;
            P.trace[2 * k + 1] = globaltimer_ns();
            g_trace_n = k + 1;
        }
    }
}

// GRID_LOOP: over the block's virtual grid (only inside k_pcg / k_pcg_batch,
// which set it); KERNEL_LOOP: over the launch's real grid (set-up kernels).
#define GRID_LOOP(c, n) for (int c = vb() * blockDim.x + threadIdx.x; c < (n); c += vnb() * blockDim.x)
#define KERNEL_LOOP(c, n) for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < (n); c += gridDim.x * blockDim.x)
#define BLOCK_LOOP(c, n) for (int c = threadIdx.x; c < (n); c += blockDim.x)
#define SYNC_OR(fail)              \
    do {                           \
        if (!vsync(P)) fail;       \
    } while (0)

struct Red {
    double v[kRedBlock / 32 + 2];
};

// Barrier of the blocks of one solve (a block barrier when the solve has one block).
__device__ __forceinline__ bool vsync(const SolveParams &P) {
    if (vnb() == 1) {
        __syncthreads();
        return true;
    }
    return grid_sync_nb(P.bar, (unsigned)vnb(), kBarrierTimeoutNs);
}

__device__ __forceinline__ void put_partial(const SolveParams &P, int which, double v, double *s_red) {
    double t = block_sum<kRedBlock>(v, s_red);
    if (threadIdx.x == 0) P.part[which * vnb() + vb()] = t;
}
__device__ __forceinline__ double get_total(const SolveParams &P, int which, double *s_red) {
    return sum_partials<kRedBlock>(P.part + which * vnb(), vnb(), s_red);
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
    const int nb = vnb(), b = vb();
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
// load(k, mine, o) and the four slot weights are staged (accumulation type A:
// FP64 plain, FP32 mixed) in shared memory; for the cells of the sub-range
// (mine) load also fills o, whose a, b, c are staged too, and commit(k, o)
// then performs the cell's side effects (global stores) after the loads of
// the pass are issued.  load must not store.  The links that leave a face
// (boundary-ring cells) are summed while staging as well: rsum[ring rank - r0]
// = sum_k w_k (x(c) - x(nb_k)), one thread per ring cell.  All global loads
// happen while staging, where they are independent, so the compute loop reads
// shared memory only.  Ends with a block barrier.
template <bool MP, class Load, class Commit, class Cell>
__device__ __forceinline__ void staged(const StencilDev &S, double *raw, Load load, Commit commit, Cell cell) {
    using A = typename Prec<MP>::A;
    const int N = S.N, n = S.n, nring = S.nring, bs = blockDim.x, tid = threadIdx.x;
    int c0, c1;
    block_range(n, N, c0, c1);
    const int halo = N + 1;
    const int sub = kStageCap - 2 * halo;
    A *buf = reinterpret_cast<A *>(raw);
    A *bx = buf, *b0 = buf + kStageCap, *b1 = buf + 2 * kStageCap, *b2 = buf + 3 * kStageCap, *b3 = buf + 4 * kStageCap;
    float *oa = reinterpret_cast<float *>(buf + 5 * kStageCap), *ob = oa + kStageCap, *oc = ob + kStageCap;
    A *rs = reinterpret_cast<A *>(oc + kStageCap);
    // the slot tables, read once into registers (not per window cell)
    const double *wd = S.wslot_d;
    const float *wf = S.wslot;
    const __half *wh = S.wslot_h;
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
        A fvc = 0;
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
            A e1 = 0, n1 = 0, ne1 = 0, nw1 = 0, v1 = 0;
            if (k >= 0 && k < n) {
                e1 = slot_w<MP>(wd, wf, wh, k);
                n1 = slot_w<MP>(wd, wf, wh, n + k);
                ne1 = slot_w<MP>(wd, wf, wh, 2 * n + k);
                nw1 = slot_w<MP>(wd, wf, wh, 3 * n + k);
                v1 = load(k, in1, o1);
            }
            A e2 = 0, n2 = 0, ne2 = 0, nw2 = 0, v2 = 0;
            if (two && k2 >= 0 && k2 < n) {
                e2 = slot_w<MP>(wd, wf, wh, k2);
                n2 = slot_w<MP>(wd, wf, wh, n + k2);
                ne2 = slot_w<MP>(wd, wf, wh, 2 * n + k2);
                nw2 = slot_w<MP>(wd, wf, wh, 3 * n + k2);
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
            A vc;
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
            A v[8];
#pragma unroll
            for (int k = 0; k < 8; k++) {
                Own none;
                v[k] = o[k] >= 0 ? load(o[k], false, none) : vc;
            }
            A t = 0;
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (o[k] >= 0) t += (A)w[k] * (vc - v[k]);
            rs[q] = t;
        }
        __syncthreads();
        stage_mark(2);
        // two independent cells in flight per thread: one cell's dependent
        // chain (shared loads, sum, conversions) leaves the issue slots idle
        // with 16 warps per SM
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

#define STAGED_ARGS                                                                                            \
    const typename Prec<MP>::A *x, const typename Prec<MP>::A *wE, const typename Prec<MP>::A *wN,           \
        const typename Prec<MP>::A *wNE, const typename Prec<MP>::A *wNW, const typename Prec<MP>::A *rsum, \
        int r0, Own o
#define APPLY(S, c, xc) apply_k_smem(S, c, xc, x, wE, wN, wNE, wNW, rsum, r0)

// The pre-smoothed iterate from 0 at cell k: w D^-1 b (as stored).
template <bool MP>
__device__ __forceinline__ float presmooth_x(const LevelDev &L, int k, float b) {
    if (MP) return as_stored<true>(0.8f * __ldg(L.dinv + k) * b);
    return (float)(kOmegaJ * __ldg(L.dinv + k) * b);
}

// (R r_fine) at coarse cell c (times 1/4 in the mixed V-cycle).  Interior
// coarse cells gather their 4x4 fine window in the CSR row order (fine index
// ascending) with the P weights; the others use the CSR rows.
template <bool MP>
__device__ __forceinline__ float restrict_value(const LevelDev &F, const LevelDev &C, int c) {
    using A = typename Prec<MP>::A;
    const int Nc = C.S.N, Nf = F.S.N;
    const auto *r = lv<MP>(F.r);
    int f, I, J;
    cell_fij(C.S, c, f, I, J);
    A acc = 0;
    if (F.structured && I >= 1 && J >= 1 && I + 2 <= Nc && J + 2 <= Nc) {
        const int base = (f * Nf + 2 * J - 1) * Nf + 2 * I - 1;
        const int nc = C.S.n;
        float wv[16], rv[16];
#pragma unroll
        for (int dj = 0; dj < 4; dj++)
#pragma unroll
            for (int di = 0; di < 4; di++) {
                const int i = base + dj * Nf + di;
                wv[dj * 4 + di] = __ldg(F.rw16 + (dj * 4 + di) * nc + c);
                rv[dj * 4 + di] = ldv(r, i);
            }
#pragma unroll
        for (int q = 0; q < 16; q++) acc += (A)(wv[q] * rv[q]);
    } else {
        const int k0 = __ldg(F.rstart + c), k1 = __ldg(F.rstart + c + 1);
        for (int k = k0; k < k1; k++) acc += (A)(__ldg(F.rw + k) * ldv(r, __ldg(F.ridx + k)));
    }
    return (float)acc * restrict_scale<MP>();
}
template <bool MP>
__device__ __forceinline__ void restrict_cell(const LevelDev &F, const LevelDev &C, int c) {
    stv(lv<MP>(C.b), c, restrict_value<MP>(F, C, c));
}

// x_fine + P xo_coarse (times 4 in the mixed V-cycle) at fine cell i.
// Interior fine cells compute their 2x2 coarse taps.
template <bool MP>
__device__ __forceinline__ float prolong_value(const LevelDev &F, const LevelDev &C, int i) {
    const int Nf = F.S.N, Nc = C.S.N;
    (void)Nf;
    const float4 w = __ldg(reinterpret_cast<const float4 *>(F.pw) + i);
    const auto *xc = lv<MP>(C.xo);
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
    const float s = w.x * ldv(xc, t0) + w.y * ldv(xc, t1) + w.z * ldv(xc, t2) + w.w * ldv(xc, t3);
    if (MP) return ldv(lv<MP>(F.x), i) + 4.0f * s;
    return ldv(lv<MP>(F.x), i) + (float)(kCorrScale * s);
}

// Pre-smooth of a level from x = 0 with right-hand side bscale * b:
// x = w D^-1 b, r = b - K x.
template <bool MP, class TB>
__device__ __forceinline__ void phase_presmooth(const LevelDev &L, const TB *b, float bscale, double *buf) {
    using A = typename Prec<MP>::A;
    auto load = [&](int k, bool mine, Own &o) -> A {
        const float bk = MP ? ldv(b, k) * bscale : ldv(b, k);
        if (mine) o.a = bk;
        return (A)presmooth_x<MP>(L, k, bk);
    };
    auto commit = [&](int, const Own &) {};
    auto *lx = lv<MP>(L.x);
    auto *lr = lv<MP>(L.r);
    staged<MP>(L.S, buf, load, commit, [&](int c, STAGED_ARGS) {
        const float bc = o.a;
        const float xc = (float)x[c];  // = presmooth_x(L, c, bc)
        const A kx = APPLY(L.S, c, (A)xc);
        stv(lx, c, xc);
        stv(lr, c, (float)(bc - kx));
    });
}

// Prolongation C -> L fused with L's post-smooth: x = x_L + P xo_C is formed on
// the fly over the staged window (never stored), then xo = x + w D^-1 (b - K x)
// with b = bscale * b_in, stored as oscale * xo; returns sum dotr . (oscale xo)
// in s (and sum dotr . zold in so) when dotr != nullptr.  Same arithmetic as a
// separate prolongation pass followed by the post-smooth, one grid barrier fewer.
template <bool MP, class TB, class TO>
__device__ __forceinline__ void phase_prolong_postsmooth(const LevelDev &L, const LevelDev &C, const TB *b,
                                                         float bscale, TO *xo, float oscale, const float *dotr,
                                                         const float *zold, double &s, double &so, double *buf) {
    using A = typename Prec<MP>::A;
    auto load = [&](int k, bool mine, Own &o) -> A {
        if (mine) {
            o.a = MP ? ldv(b, k) * bscale : ldv(b, k);
            o.b = __ldg(L.dinv + k);
            o.c = dotr ? dotr[k] : 0.f;
            if (MP) o.d = zold ? zold[k] : 0.f;
        }
        return (A)prolong_value<MP>(L, C, k);
    };
    double so_ = 0;
    auto commit = [&](int, const Own &o) {
        if (MP) so_ += (double)o.c * o.d;
    };
    staged<MP>(L.S, buf, load, commit, [&](int c, STAGED_ARGS) {
        const float xc = (float)x[c];
        const float rc = (float)(o.a - APPLY(L.S, c, (A)xc));
        float out;
        if (MP)
            out = (xc + 0.8f * o.b * rc) * oscale;
        else
            out = xc + (float)(kOmegaJ * o.b * rc);
        s += (double)o.c * stv_get(xo, c, out);
    });
    so = so_;
}

// One damped-Jacobi sweep src -> dst with per-link conversions (small levels).
template <bool MP>
__device__ __forceinline__ float jacobi_cell(const StencilDev &S, const float *dinv, const typename Prec<MP>::V *b,
                                             const typename Prec<MP>::V *src, typename Prec<MP>::V *dst, int c) {
    auto X = [&](int k) -> double { return (double)ldv(src, k); };
    float xc = ldv(src, c);
    float rc = (float)(ldv(b, c) - apply_k(S, c, (double)xc, X));
    float out = xc + (float)(kOmegaJ * __ldg(dinv + c) * rc);
    stv(dst, c, out);
    return out;
}

// ---- the coarse levels inside one block (setup of the dense map, fallback) --
// Always FP32 vectors in shared memory with the plain arithmetic: the V-cycle
// of these levels maps b_l0 to xo_l0 the same way in both precisions (the
// mixed transfer factors 1/4 and 4 cancel within it).

struct SmemLevel {
    float *x, *xo, *b, *r;
};

__device__ void carve_smem(const SolveParams &P, int l0, float *smem, SmemLevel *lv_) {
    float *q = smem;
    for (int l = l0; l < P.nlev; l++) {
        int n = P.L[l].S.n;
        lv_[l].x = q;
        lv_[l].xo = q + n;
        lv_[l].b = q + 2 * n;
        lv_[l].r = q + 3 * n;
        q += 4 * n;
    }
}

// Coarsest level: `sweeps` Jacobi sweeps from 0; result in V.xo.  When every
// cell has its own thread, the cell's links, 1/diag and b stay in registers.
__device__ __forceinline__ void coarsest_smem(const LevelDev &L, const SmemLevel &V, int sweeps) {
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
            BLOCK_LOOP(c, n) jacobi_cell<false>(L.S, L.dinv, V.b, src, dst, c);
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
// memory.  b of level l0 is lv[l0].b on entry; xo of level l0 is left in
// lv[l0].xo.  Always inlined (with coarsest_smem): a call that takes the
// solve's parameters by reference makes the compiler copy the whole
// parameter block of the kernel to local memory, and every parameter read of
// every phase then goes through it (measured: the solve 40 % slower).
__device__ __forceinline__ void vcycle_block_smem(const SolveParams &P, int l0, SmemLevel *lv_) {
    const int last = P.nlev - 1;
    for (int l = l0; l < last; l++) {
        LevelDev L = P.L[l];
        L.x = lv_[l].x;
        L.r = lv_[l].r;
        const float *b = lv_[l].b;
        float *lx = lv_[l].x, *lr = lv_[l].r;
        BLOCK_LOOP(c, L.S.n) {
            auto X = [&](int k) -> double { return (double)(float)(kOmegaJ * __ldg(L.dinv + k) * b[k]); };
            float bc = b[c];
            float xc = (float)(kOmegaJ * __ldg(L.dinv + c) * bc);
            double kx = apply_k(L.S, c, (double)xc, X);
            lx[c] = xc;
            lr[c] = (float)(bc - kx);
        }
        __syncthreads();
        LevelDev C = P.L[l + 1];
        C.b = lv_[l + 1].b;
        BLOCK_LOOP(c, C.S.n) restrict_cell<false>(L, C, c);
        __syncthreads();
    }
    coarsest_smem(P.L[last], lv_[last], P.coarse_sweeps);
    for (int l = last - 1; l >= l0; l--) {
        LevelDev L = P.L[l];
        L.x = lv_[l].x;
        LevelDev C = P.L[l + 1];
        C.xo = lv_[l + 1].xo;
        BLOCK_LOOP(i, L.S.n) lv_[l].x[i] = prolong_value<false>(L, C, i);
        __syncthreads();
        BLOCK_LOOP(c, L.S.n) jacobi_cell<false>(L.S, L.dinv, lv_[l].b, lv_[l].x, lv_[l].xo, c);
        __syncthreads();
    }
}

// ---- the V-cycle after level 0's pre-smooth --------------------------------

// The rest of z = V(r) once level 0's pre-smooth (x, r of level 0) is complete
// and visible; the V-cycle ran on s0 * r (s0 = 1 in the plain solve).  Ends
// with rz = r . z (and, mixed, r . z_prev) published; returns false on abort.
template <bool MP>
__device__ bool vcycle_rest(const SolveParams &P, const float *r, float s0, float *z, const float *zold,
                            double *s_red, double *buf, float *smem) {
    const int G = P.nlev_grid;
    // down
    for (int l = 0; l < G; l++) {
        const LevelDev &L = P.L[l];
        if (l > 0) {
            phase_presmooth<MP>(L, lv<MP>(L.b), 1.0f, buf);
            trace_mark(P, 100 + l);
            SYNC_OR(return false);
        }
        GRID_LOOP(c, P.L[l + 1].S.n) restrict_cell<MP>(L, P.L[l + 1], c);
        trace_mark(P, 300 + l);
        SYNC_OR(return false);
    }
    // below the grid levels: the dense map, or block 0
    if (P.dense) {
        const LevelDev &C = P.L[G];
        const auto *cb = lv<MP>(C.b);
        auto *cx = lv<MP>(C.xo);
        const int nd = P.nd, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int gw = vb() * (blockDim.x >> 5) + warp, nw = vnb() * (blockDim.x >> 5);
        for (int row = gw; row < nd; row += nw) {
            const double *d = P.dense + (size_t)row * nd;
            double acc = 0;
            for (int j = lane; j < nd; j += 32) acc += __ldg(d + j) * (double)ldv(cb, j);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) stv(cx, row, (float)acc);
        }
        trace_mark(P, 500);
        SYNC_OR(return false);
    } else if (!P.coarse_on_grid) {
        if (vb() == 0) {
            SmemLevel lvs[kMaxLev];
            carve_smem(P, G, smem, lvs);
            const auto *gb = lv<MP>(P.L[G].b);
            BLOCK_LOOP(c, P.L[G].S.n) lvs[G].b[c] = ldv(gb, c);
            __syncthreads();
            vcycle_block_smem(P, G, lvs);
            auto *gx = lv<MP>(P.L[G].xo);
            BLOCK_LOOP(c, P.L[G].S.n) stv(gx, c, lvs[G].xo[c]);
        }
        trace_mark(P, 500);
        SYNC_OR(return false);
    } else {
        // the coarsest level is large (nlev_grid == nlev - 1): sweep it grid-wide
        const LevelDev &L = P.L[P.nlev - 1];
        auto *lx = lv<MP>(L.x), *lxo = lv<MP>(L.xo);
        const auto *lb = lv<MP>(L.b);
        GRID_LOOP(c, L.S.n) stv(lx, c, 0.f);
        SYNC_OR(return false);
        auto *src = lx, *dst = lxo;
        for (int s = 0; s < P.coarse_sweeps; s++) {
            GRID_LOOP(c, L.S.n) jacobi_cell<MP>(L.S, L.dinv, lb, src, dst, c);
            SYNC_OR(return false);
            auto *t = src;
            src = dst;
            dst = t;
        }
        if (src != lxo) {
            GRID_LOOP(c, L.S.n) lxo[c] = src[c];
            SYNC_OR(return false);
        }
    }
    // up: prolongation fused with each grid level's post-smooth
    for (int l = G - 1; l >= 0; l--) {
        const LevelDev &L = P.L[l];
        double s = 0, so = 0;
        if (l > 0) {
            phase_prolong_postsmooth<MP>(L, P.L[l + 1], lv<MP>(L.b), 1.0f, lv<MP>(L.xo), 1.0f, nullptr, nullptr, s, so,
                                         buf);
            trace_mark(P, 900 + l);
            SYNC_OR(return false);
        } else {
            phase_prolong_postsmooth<MP>(L, P.L[1], r, s0, z, 1.0f / s0, r, zold, s, so, buf);
            put_partial(P, RED_RZ, s, s_red);
            if (MP) put_partial(P, RED_RZO, so, s_red);
            trace_mark(P, 900);
            SYNC_OR(return false);
        }
    }
    return true;
}

// z = V(r) for a single-level hierarchy (level 0 is the coarsest grid); the
// sweeps run on s0 * r (s0 = 1 in the plain solve).
template <bool MP>
__device__ bool single_level(const SolveParams &P, const float *r, float s0, float *z, const float *zold,
                             double *s_red, float *smem) {
    const LevelDev &L = P.L[0];
    auto *lx = lv<MP>(L.x), *lxo = lv<MP>(L.xo);
    auto *lb = lv<MP>(L.b);
    if (!P.coarse_on_grid) {
        if (vb() == 0) {
            SmemLevel lvs[kMaxLev];
            carve_smem(P, 0, smem, lvs);
            BLOCK_LOOP(c, L.S.n) lvs[0].b[c] = r[c];
            __syncthreads();
            coarsest_smem(L, lvs[0], P.coarse_sweeps);
            BLOCK_LOOP(c, L.S.n) stv(lxo, c, MP ? lvs[0].xo[c] * s0 : lvs[0].xo[c]);
        }
    } else {
        GRID_LOOP(c, L.S.n) {
            stv(lx, c, 0.f);
            stv(lb, c, MP ? r[c] * s0 : r[c]);
        }
        SYNC_OR(return false);
        auto *src = lx, *dst = lxo;
        for (int s = 0; s < P.coarse_sweeps; s++) {
            GRID_LOOP(c, L.S.n) jacobi_cell<MP>(L.S, L.dinv, lb, src, dst, c);
            SYNC_OR(return false);
            auto *t = src;
            src = dst;
            dst = t;
        }
        if (src != lxo) {
            GRID_LOOP(c, L.S.n) lxo[c] = src[c];
        }
    }
    SYNC_OR(return false);
    double s = 0, so = 0;
    const float inv = 1.0f / s0;
    GRID_LOOP(c, L.S.n) {
        if (zold) so += (double)r[c] * zold[c];
        float zc = MP ? ldv(lxo, c) * inv : ldv(lxo, c);
        z[c] = zc;
        s += (double)r[c] * zc;
    }
    put_partial(P, RED_RZ, s, s_red);
    if (MP) put_partial(P, RED_RZO, so, s_red);
    return vsync(P);
}

// Power of two that brings a residual of squared norm rr over n cells to an
// RMS near 1/16 (the mixed V-cycle's input scale; 1 in the plain solve).
template <bool MP>
__device__ __forceinline__ float vscale(double rr, int n) {
    if (!MP || !(rr > 0) || !isfinite(rr)) return 1.0f;
    const int e = ilogb(sqrt(rr / n));
    return ldexpf(1.0f, max(-100, min(100, -4 - e)));
}

// The whole solve for the SolveParams of this block's planet, on the block's
// virtual grid (vb(), vnb()).
template <bool MP>
__device__ __forceinline__ void pcg_body(const SolveParams &P) {
    __shared__ Red sh;
    extern __shared__ __align__(16) unsigned char dyn[];
    double *buf = reinterpret_cast<double *>(dyn);               // staged window
    float *smem = reinterpret_cast<float *>(dyn + kStageBytes);  // block-0 levels
    double *s_red = sh.v;
    // the warp slots of warps this block does not have stay zero (ordered
    // before the first read by the first block sum's barriers)
    if (threadIdx.x < kRedBlock / 32) s_red[threadIdx.x] = 0.0;
    using A = typename Prec<MP>::A;
    const LevelDev &L0 = P.L[0];
    const StencilDev &S0 = L0.S;
    const int n = S0.n;
    const bool mg = P.nlev >= 2;
    const bool single = P.nlev == 1;
    float *r = P.r, *rn = P.r2, *p = P.p, *pn = P.p2;
    float *z = P.z, *zo = MP ? P.z2 : nullptr;  // mixed: z / z2 ping-pong (the previous z for the flexible beta)
    double bb, rr, rz = 0, tol2, beta = 0, m2;
    int it = 0, flags = 0;
    bool first = true, ok = true;
    float s0 = 1.0f;
    const unsigned long long t_begin = threadIdx.x == 0 ? globaltimer_ns() : 0ull;

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
        auto load = [&](int k, bool mine, Own &o) -> A {
            if (mine) {
                o.a = P.omega[k];
                o.b = __ldg(P.area + k);
            }
            return (A)psi[k];
        };
        auto commit = [&](int, const Own &) {};
        staged<MP>(S0, buf, load, commit, [&](int c, STAGED_ARGS) {
            double b = -(double)o.b * ((double)o.a - m2);
            double ri = b - (double)APPLY(S0, c, x[c]);
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
    if (!isfinite(bb) || !isfinite(rr)) flags |= kSolveNonFinite;
    if (bb == 0.0) {
        GRID_LOOP(c, n) P.psi[c] = 0.f;
        if (vb() == 0 && threadIdx.x == 0) {
            P.res->iters = 0;
            P.res->relres = 0;
            P.res->status = 0;
            P.res->r_final = 0;
            P.res->flags = flags;
            P.res->ns = globaltimer_ns() - t_begin;
        }
        return;
    }
    tol2 = P.tol * P.tol * bb;

    // z = M^-1 r, rz
    if (rr > tol2) {
        if (mg) {
            s0 = vscale<MP>(rr, n);
            phase_presmooth<MP>(L0, r, s0, buf);
            SYNC_OR(goto aborted);
            ok = vcycle_rest<MP>(P, r, s0, z, nullptr, s_red, buf, smem);
        } else if (single) {
            s0 = vscale<MP>(rr, n);
            ok = single_level<MP>(P, r, s0, z, nullptr, s_red, smem);
        } else {
            double s = 0;
            GRID_LOOP(c, n) {
                float zc = __ldg(L0.dinv + c) * r[c];
                z[c] = zc;
                s += (double)r[c] * zc;
            }
            put_partial(P, RED_RZ, s, s_red);
            ok = vsync(P);
        }
        if (!ok) goto aborted;
        rz = get_total(P, RED_RZ, s_red);
        if (!isfinite(rz)) flags |= kSolveNonFinite;
    }

    while (rr > tol2 && it < P.maxit) {
        // p = z (first) or z + beta p;  Ap = K p;  pAp
        {
            const float *zz = z;
            const float *po = p;
            const bool fst = first;
            const double be = beta;
            auto pnew = [&](int k) -> float { return fst ? zz[k] : (float)(zz[k] + be * po[k]); };
            auto load = [&](int k, bool, Own &) -> A { return (A)pnew(k); };
            auto commit = [&](int, const Own &) {};
            double s = 0;
            float *pw = pn, *ap = P.Ap;
            staged<MP>(S0, buf, load, commit, [&](int c, STAGED_ARGS) {
                const float pc = (float)x[c];
                const A a = APPLY(S0, c, (A)pc);
                pw[c] = pc;
                ap[c] = (float)a;
                s += (double)a * pc;
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
            if (!isfinite(pAp)) flags |= kSolveNonFinite;
            if (pAp <= 0) {
                flags |= kSolveBreakdown;
                break;
            }
            const double alpha = rz / pAp;
            const float *Ap = P.Ap;
            const float *ro = r;
            const float *pp = p;
            double s = 0, sz = 0;
            float *rw_ = rn;
            if (mg) {
                // the previous r's scale (the new r is not reduced yet)
                s0 = vscale<MP>(rr, n);
                const float sc = s0;
                // psi += alpha p; r' = r - alpha Ap; level-0 pre-smooth of r'
                auto rnew = [&](int k) -> float { return (float)(ro[k] - alpha * Ap[k]); };
                // mine: r, Ap of the cell staged; p and psi kept for commit,
                // which does psi += alpha p (nothing else reads psi)
                auto load = [&](int k, bool mine, Own &o) -> A {
                    if (mine) {
                        o.a = ro[k];
                        o.b = Ap[k];
                        o.c = pp[k];
                        o.d = P.psi[k];
                    }
                    return (A)presmooth_x<MP>(L0, k, MP ? rnew(k) * sc : rnew(k));
                };
                auto commit = [&](int k, const Own &o) { P.psi[k] = o.d + (float)(alpha * o.c); };
                auto *l0x = lv<MP>(L0.x);
                auto *l0r = lv<MP>(L0.r);
                staged<MP>(S0, buf, load, commit, [&](int c, STAGED_ARGS) {
                    const double ri = o.a - alpha * o.b;
                    const float rc = (float)ri;
                    rw_[c] = rc;
                    s += ri * ri;
                    const float xc = (float)x[c];  // = presmooth_x(L0, c, rc * sc)
                    const A kx = APPLY(S0, c, (A)xc);
                    stv(l0x, c, xc);
                    stv(l0r, c, (float)((MP ? rc * sc : rc) - kx));
                });
            } else {
                GRID_LOOP(c, n) {
                    P.psi[c] += (float)(alpha * pp[c]);
                    double ri = ro[c] - alpha * Ap[c];
                    float rc = (float)ri;
                    rw_[c] = rc;
                    s += ri * ri;
                    if (!single) {
                        float zc = __ldg(L0.dinv + c) * rc;
                        z[c] = zc;
                        sz += (double)rc * zc;
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
        if (!isfinite(rr)) flags |= kSolveNonFinite;
        if (rr <= tol2) break;
        if (MP && (mg || single)) {  // the new z goes to the other buffer; zo keeps the previous one
            float *t = z;
            z = zo;
            zo = t;
        }
        if (mg)
            ok = vcycle_rest<MP>(P, r, s0, z, MP ? zo : nullptr, s_red, buf, smem);
        else if (single) {
            s0 = vscale<MP>(rr, n);
            ok = single_level<MP>(P, r, s0, z, MP ? zo : nullptr, s_red, smem);
        }
        if (!ok) goto aborted;
        {
            double rznew = get_total(P, RED_RZ, s_red);
            if (!isfinite(rznew)) flags |= kSolveNonFinite;
            if (MP && (mg || single))
                beta = (rznew - get_total(P, RED_RZO, s_red)) / rz;  // Polak-Ribiere
            else
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
        // leave the final residual / direction / preconditioned residual in the caller's buffers
        if (r != P.r) GRID_LOOP(c, n) P.r[c] = r[c];
        if (p != P.p) GRID_LOOP(c, n) P.p[c] = p[c];
        if (z != P.z) GRID_LOOP(c, n) P.z[c] = z[c];
    }
    if (it >= P.maxit && rr > tol2) flags |= kSolveMaxit;
    if (vb() == 0 && threadIdx.x == 0) {
        P.res->iters = it;
        P.res->relres = sqrt(rr / bb);
        P.res->status = 0;
        P.res->r_final = 0;
        P.res->flags = flags;
        P.res->ns = globaltimer_ns() - t_begin;
    }
    return;

aborted:
    if (vb() == 0 && threadIdx.x == 0) {
        P.res->iters = it;
        P.res->relres = -1.0;
        P.res->status = 1;
        P.res->flags = flags | kSolveTimeout;
    }
}

// One solve on the whole grid, TPB threads per block.
template <bool MP, int TPB>
__global__ void __launch_bounds__(TPB, 1) k_pcg(const __grid_constant__ SolveParams P) {
    if (threadIdx.x == 0) {
        s_vgrid[0] = blockIdx.x;
        s_vgrid[1] = gridDim.x;
    }
    __syncthreads();
    pcg_body<MP>(P);
}
