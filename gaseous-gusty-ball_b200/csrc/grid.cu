// grid.cu — the equiangular cubed-sphere grid on the GPU: cell centres, exact
// spherical-Voronoi cells (FP64 half-plane clipping in each cell's gnomonic
// plane), reciprocal-link symmetrisation, Laplacian weights, least-squares
// gradient coefficients, and this library's face-tiled operator layout.
// Also the host-side point-location API of cubesphere.h.
//
// Algorithm (upstream src/cubesphere.c:157-359, restated per cell):
//   candidates: the 5x5 cell window around the cell, ghost cells resolved to
//   the real cell containing their extended centre; clip a 8h box by the
//   bisector half-plane of every candidate; edges become links (neighbour,
//   length), the polygon fan gives the area; keep the <= 8 longest links
//   longer than 1e-4 h; keep only reciprocal links with averaged lengths;
//   w = len / centre angle; gradient coefficients from the weighted 2x2 normal
//   equations in the local (e1, e2) frame with weights len / d^3.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "ggb_internal.h"

namespace ggb {

constexpr int kMaxPV = 32;  // a 4-gon clipped by <= 24 half-planes has <= 28 vertices
constexpr int kBlk = 128;

struct PV {
    double a, b;
    int lab;
};

__device__ __forceinline__ void decode(int c, int N, int &f, int &i, int &j) {
    int nn = N * N;
    f = c / nn;
    int rem = c - f * nn;
    j = rem / N;
    i = rem - j * N;
}

__global__ void k_positions(int N, double h, float *pos) {
    int n = 6 * N * N;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int f, i, j;
        decode(c, N, f, i, j);
        store3(pos + 3 * c, centre_dir(f, i, j, h));
    }
}

// Ring of one-deep ghost cells around each face (4N+4 per face).
__global__ void k_ghost_table(int N, double h, int *ghost) {
    int per = 4 * N + 4;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 6 * per; t += gridDim.x * blockDim.x) {
        int f = t / per, r = t - f * per, i, j;
        if (r < N + 2) {
            j = -1;
            i = r - 1;
        } else if (r < 2 * (N + 2)) {
            j = N;
            i = r - (N + 2) - 1;
        } else if (r < 2 * (N + 2) + N) {
            i = -1;
            j = r - 2 * (N + 2);
        } else {
            i = N;
            j = r - 2 * (N + 2) - N;
        }
        ghost[t] = ghost_cell_direct(f, i, j, N, h);
    }
}

__device__ __forceinline__ double tri_area(D3 a, D3 b, D3 c) {
    double num = fabs(dot(a, cross(b, c)));
    double den = 1.0 + dot(a, b) + dot(b, c) + dot(c, a);
    return 2.0 * atan2(num, den);
}

__device__ int clip(const PV *in, int n, PV *out, double A, double B, double C, int lab) {
    int m = 0;
    for (int k = 0; k < n; k++) {
        PV v0 = in[k], v1 = in[k + 1 == n ? 0 : k + 1];
        double f0 = A * v0.a + B * v0.b + C;
        double f1 = A * v1.a + B * v1.b + C;
        bool in0 = f0 >= 0, in1 = f1 >= 0;
        if (in0 && m < kMaxPV) out[m++] = v0;
        if (in0 != in1) {
            double t = f0 / (f0 - f1);
            PV I;
            I.a = v0.a + t * (v1.a - v0.a);
            I.b = v0.b + t * (v1.b - v0.b);
            I.lab = in0 ? lab : v0.lab;
            if (m < kMaxPV) out[m++] = I;
        }
    }
    return m;
}

// Per cell: Voronoi links (<= 8 longest above 1e-4 h), area.
__global__ void __launch_bounds__(kBlk) k_voronoi(int N, double h, const float *pos, float *area, double *area64,
                                                  unsigned char *nnb, int *nbr, float *rawlen, int *open_count) {
    int n = 6 * N * N;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int f, i, j;
        decode(c, N, f, i, j);
        D3 p = load3(pos + 3 * c);
        // e1 = normalize(tangent(right_f, p)), e2 = p x e1
        D3 right;
        switch (f) {
            case 0: right = d3(1, 0, 0); break;
            case 1: right = d3(0, 0, -1); break;
            case 2: right = d3(-1, 0, 0); break;
            case 3: right = d3(0, 0, 1); break;
            default: right = d3(1, 0, 0); break;
        }
        D3 e1 = normalize(tangent(right, p));
        D3 e2 = cross(p, e1);

        int cand[24], nc = 0;
        for (int dj = -2; dj <= 2; dj++)
            for (int di = -2; di <= 2; di++) {
                if (!di && !dj) continue;
                int q = ghost_cell_direct(f, i + di, j + dj, N, h);
                bool dup = q == c;
                for (int k = 0; k < nc; k++) dup |= cand[k] == q;
                if (!dup) cand[nc++] = q;
            }

        PV bufA[kMaxPV], bufB[kMaxPV];
        PV *poly = bufA, *tmp = bufB;
        double S = 4 * h;
        int m = 4;
        poly[0].a = -S; poly[0].b = -S; poly[0].lab = -1;
        poly[1].a = S;  poly[1].b = -S; poly[1].lab = -1;
        poly[2].a = S;  poly[2].b = S;  poly[2].lab = -1;
        poly[3].a = -S; poly[3].b = S;  poly[3].lab = -1;
        for (int k = 0; k < nc; k++) {
            D3 q = load3(pos + 3 * cand[k]);
            D3 mv = sub(p, q);
            m = clip(poly, m, tmp, dot(e1, mv), dot(e2, mv), dot(p, mv), cand[k]);
            PV *t = poly;
            poly = tmp;
            tmp = t;
        }

        int lnb[24];
        double llen[24];
        int nl = 0, open = 0;
        double ar = 0;
        for (int k = 0; k < m; k++) {
            PV v0 = poly[k], v1 = poly[k + 1 == m ? 0 : k + 1];
            D3 V0 = normalize(add(p, add(scale(e1, v0.a), scale(e2, v0.b))));
            D3 V1 = normalize(add(p, add(scale(e1, v1.a), scale(e2, v1.b))));
            ar += tri_area(p, V0, V1);
            if (v0.lab < 0) {
                open = 1;
                continue;
            }
            double L = angle(V0, V1);
            int l = 0;
            while (l < nl && lnb[l] != v0.lab) l++;
            if (l < nl)
                llen[l] += L;
            else if (nl < 24) {
                lnb[nl] = v0.lab;
                llen[nl] = L;
                nl++;
            }
        }
        // stable sort, longest first
        for (int a = 1; a < nl; a++) {
            int xb = lnb[a];
            double xl = llen[a];
            int b = a - 1;
            while (b >= 0 && llen[b] < xl) {
                lnb[b + 1] = lnb[b];
                llen[b + 1] = llen[b];
                b--;
            }
            lnb[b + 1] = xb;
            llen[b + 1] = xl;
        }
        double minlen = 1e-4 * h;
        int kept = 0;
        while (kept < nl && kept < kMaxNb && llen[kept] >= minlen) {
            nbr[kMaxNb * c + kept] = lnb[kept];
            rawlen[kMaxNb * c + kept] = (float)llen[kept];
            kept++;
        }
        for (int k = kept; k < kMaxNb; k++) {
            nbr[kMaxNb * c + k] = -1;
            rawlen[kMaxNb * c + k] = 0.f;
        }
        nnb[c] = (unsigned char)kept;
        area[c] = (float)ar;
        area64[c] = ar;
        if (open) atomicAdd(open_count, 1);
    }
}

// Reciprocal links only; averaged lengths (-1 marks a dropped link).
__global__ void k_symmetrize(int N, double h, const unsigned char *nnb, const int *nbr, const float *rawlen,
                             float *symlen, int *asym_count) {
    int n = 6 * N * N;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        for (int k = 0; k < nnb[c]; k++) {
            int o = nbr[kMaxNb * c + k], back = -1;
            for (int kk = 0; kk < nnb[o]; kk++)
                if (nbr[kMaxNb * o + kk] == c) back = kk;
            double l = rawlen[kMaxNb * c + k];
            if (back < 0) {
                if (l > 1e-2 * h) atomicAdd(asym_count, 1);
                symlen[kMaxNb * c + k] = -1.0f;
            } else {
                symlen[kMaxNb * c + k] = (float)(0.5 * (l + rawlen[kMaxNb * o + back]));
            }
        }
    }
}

// Final links: weights, edge lengths, gradient coefficients, 1/diag.
__global__ void k_weights(int N, const float *pos, unsigned char *nnb, int *nbr, const float *symlen, float *w,
                          float *elen, float *gc, float *dinv) {
    int n = 6 * N * N;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        D3 p = load3(pos + 3 * c);
        int nb[kMaxNb], m = 0;
        double ln[kMaxNb];
        int cnt = nnb[c];
        for (int k = 0; k < cnt; k++)
            if (symlen[kMaxNb * c + k] >= 0) {
                nb[m] = nbr[kMaxNb * c + k];
                ln[m] = symlen[kMaxNb * c + k];
                m++;
            }
        nnb[c] = (unsigned char)m;
        int f = c / (N * N);
        D3 right;
        switch (f) {
            case 0: right = d3(1, 0, 0); break;
            case 1: right = d3(0, 0, -1); break;
            case 2: right = d3(-1, 0, 0); break;
            case 3: right = d3(0, 0, 1); break;
            default: right = d3(1, 0, 0); break;
        }
        D3 e1 = normalize(tangent(right, p));
        D3 e2 = cross(p, e1);
        double M00 = 0, M01 = 0, M11 = 0, tx[kMaxNb], ty[kMaxNb], wk[kMaxNb];
        double wsum = 0;
        for (int k = 0; k < m; k++) {
            D3 q = load3(pos + 3 * nb[k]);
            double d = angle(p, q);
            float wf = (float)(ln[k] / d);
            nbr[kMaxNb * c + k] = nb[k];
            w[kMaxNb * c + k] = wf;
            elen[kMaxNb * c + k] = (float)ln[k];
            wsum += wf;
            D3 t = tangent(sub(q, p), p);
            tx[k] = dot(t, e1);
            ty[k] = dot(t, e2);
            wk[k] = ln[k] / (d * d * d);
            M00 += wk[k] * tx[k] * tx[k];
            M01 += wk[k] * tx[k] * ty[k];
            M11 += wk[k] * ty[k] * ty[k];
        }
        double det = M00 * M11 - M01 * M01;
        double i00 = M11 / det, i01 = -M01 / det, i11 = M00 / det;
        for (int k = 0; k < m; k++) {
            double c1 = wk[k] * (i00 * tx[k] + i01 * ty[k]);
            double c2 = wk[k] * (i01 * tx[k] + i11 * ty[k]);
            store3(gc + 3 * (kMaxNb * c + k), add(scale(e1, c1), scale(e2, c2)));
        }
        for (int k = m; k < kMaxNb; k++) {
            nbr[kMaxNb * c + k] = -1;
            w[kMaxNb * c + k] = 0.f;
            elen[kMaxNb * c + k] = 0.f;
            gc[3 * (kMaxNb * c + k) + 0] = 0.f;
            gc[3 * (kMaxNb * c + k) + 1] = 0.f;
            gc[3 * (kMaxNb * c + k) + 2] = 0.f;
        }
        dinv[c] = (float)(1.0 / wsum);
    }
}

// Face-tiled layout: direction slots for on-face links inside the 3x3 box;
// everything else of a ring cell goes to its ring list.  `bad` counts
// interior cells with a link outside their 3x3 box (the layout requires 0)
// and slot pairs whose two weights differ.
__global__ void k_slots(int N, const unsigned char *nnb, const int *nbr, const float *w, float *wslot, int *ring_nb,
                        float *ring_w, int *bad) {
    int n = 6 * N * N, nring = N == 1 ? 1 : 4 * N - 4;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        int f, i, j;
        decode(c, N, f, i, j);
        bool ring = i == 0 || j == 0 || i == N - 1 || j == N - 1;
        int r = ring ? f * nring + ring_rank_in_face(i, j, N) : -1;
        int nx = 0;
        for (int k = 0; k < nnb[c]; k++) {
            int o = nbr[kMaxNb * c + k];
            float wk = w[kMaxNb * c + k];
            int fo, io, jo;
            decode(o, N, fo, io, jo);
            int di = io - i, dj = jo - j;
            bool box = fo == f && di >= -1 && di <= 1 && dj >= -1 && dj <= 1;
            if (box) {
                int s = -1;
                if (di == 1 && dj == 0) s = 0;
                else if (di == 0 && dj == 1) s = 1;
                else if (di == 1 && dj == 1) s = 2;
                else if (di == -1 && dj == 1) s = 3;
                if (s >= 0) {
                    wslot[s * n + c] = wk;
                } else {
                    // opposite direction: the neighbour's slot must hold the same weight
                    const int *nbo = nbr + kMaxNb * o;
                    float wo = -1.f;
                    for (int kk = 0; kk < nnb[o]; kk++)
                        if (nbo[kk] == c) wo = w[kMaxNb * o + kk];
                    if (wo != wk) atomicAdd(bad, 1);
                }
            } else if (ring) {
                ring_nb[r * kMaxNb + nx] = o;
                ring_w[r * kMaxNb + nx] = wk;
                nx++;
            } else {
                atomicAdd(bad, 1);
            }
        }
        if (ring)
            for (int k = nx; k < kMaxNb; k++) {
                ring_nb[r * kMaxNb + k] = -1;
                ring_w[r * kMaxNb + k] = 0.f;
            }
    }
}

__global__ void k_to_double(size_t n, const float *src, double *dst) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

__global__ void k_sum_area(int n, const double *a, double *out) {
    // one block, fixed order
    __shared__ double s_red[kBlk / 32 + 2];
    double v = 0;
    for (int c = threadIdx.x; c < n; c += kBlk) v += a[c];
    double t = block_sum<kBlk>(v, s_red);
    if (threadIdx.x == 0) *out = t;
}

static void *talloc(bool managed, size_t bytes) { return managed ? managed_try_alloc(bytes) : dev_try_alloc(bytes); }
static void tfree(bool managed, void *p) {
    if (managed)
        managed_free(p);
    else
        dev_free(p);
}

int grid_build(GridTables *t, int N, bool managed) {
    if (N < 1 || N > 16384) {
        fprintf(stderr, "cs_init: unsupported N %d\n", N);
        return -1;
    }
    if (!have_device()) {
        fprintf(stderr, "cs_init: no CUDA device is available (libggb_cuda has no CPU path)\n");
        return -1;
    }
    cudaStream_t s = stream();
    int n = 6 * N * N;
    GGB_CHECK(cudaGetDevice(&t->device));
    t->N = N;
    t->n = n;
    t->h = (kPi / 2) / N;
    t->managed = managed;
    t->nring = ring_count(N);
    t->pos = (float *)talloc(managed, sizeof(float) * 3 * n);
    t->area = (float *)talloc(managed, sizeof(float) * n);
    t->nnb = (unsigned char *)talloc(managed, n);
    t->nbr = (int *)talloc(managed, sizeof(int) * kMaxNb * n);
    t->w = (float *)talloc(managed, sizeof(float) * kMaxNb * n);
    t->elen = (float *)talloc(managed, sizeof(float) * kMaxNb * n);
    t->gc = (float *)talloc(managed, sizeof(float) * 3 * kMaxNb * n);
    t->ghost = (int *)dev_try_alloc(sizeof(int) * 6 * (4 * N + 4));
    t->wslot = (float *)dev_try_alloc(sizeof(float) * 4 * n);
    t->wslot_d = (double *)dev_try_alloc(sizeof(double) * 4 * n);
    t->ring_nb = (int *)dev_try_alloc(sizeof(int) * kMaxNb * 6 * t->nring);
    t->ring_w = (float *)dev_try_alloc(sizeof(float) * kMaxNb * 6 * t->nring);
    t->dinv = (float *)dev_try_alloc(sizeof(float) * n);
    float *rawlen = (float *)dev_try_alloc(sizeof(float) * kMaxNb * n);
    float *symlen = (float *)dev_try_alloc(sizeof(float) * kMaxNb * n);
    double *area64 = (double *)dev_try_alloc(sizeof(double) * n);
    int *counters = (int *)dev_try_alloc(sizeof(int) * 4);
    double *tot = (double *)dev_try_alloc(sizeof(double));
    const void *all[] = {t->pos,   t->area,    t->nnb,   t->nbr,    t->w,    t->elen,   t->gc,     t->ghost, t->wslot,
                         t->wslot_d, t->ring_nb, t->ring_w, t->dinv, rawlen, symlen, area64, counters, tot};
    for (const void *q : all)
        if (!q) {
            fprintf(stderr, "cs_init: N=%d: device memory allocation failed\n", N);
            dev_free(rawlen);
            dev_free(symlen);
            dev_free(area64);
            dev_free(counters);
            dev_free(tot);
            grid_release(t);
            return -1;
        }

    unsigned gb = std::min<unsigned>(grid_for(n, kBlk), 148u * 64u);
    k_positions<<<gb, kBlk, 0, s>>>(N, t->h, t->pos);
    GGB_LAUNCHED();
    k_ghost_table<<<grid_for(6 * (4 * N + 4), kBlk), kBlk, 0, s>>>(N, t->h, t->ghost);
    GGB_LAUNCHED();
    k_voronoi<<<gb, kBlk, 0, s>>>(N, t->h, t->pos, t->area, area64, t->nnb, t->nbr, rawlen, counters + 0);
    GGB_LAUNCHED();
    k_symmetrize<<<gb, kBlk, 0, s>>>(N, t->h, t->nnb, t->nbr, rawlen, symlen, counters + 1);
    GGB_LAUNCHED();
    k_weights<<<gb, kBlk, 0, s>>>(N, t->pos, t->nnb, t->nbr, symlen, t->w, t->elen, t->gc, t->dinv);
    GGB_LAUNCHED();
    k_slots<<<gb, kBlk, 0, s>>>(N, t->nnb, t->nbr, t->w, t->wslot, t->ring_nb, t->ring_w, counters + 2);
    GGB_LAUNCHED();
    k_to_double<<<gb, kBlk, 0, s>>>((size_t)4 * n, t->wslot, t->wslot_d);
    GGB_LAUNCHED();
    k_sum_area<<<1, kBlk, 0, s>>>(n, area64, tot);
    GGB_LAUNCHED();
    int hc[4];
    GGB_CHECK(cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, s));
    GGB_CHECK(cudaMemcpyAsync(&t->total_area, tot, sizeof(double), cudaMemcpyDeviceToHost, s));
    GGB_CHECK(cudaStreamSynchronize(s));
    t->open_cells = hc[0];
    t->asym_count = hc[1];
    dev_free(rawlen);
    dev_free(symlen);
    dev_free(area64);
    dev_free(counters);
    dev_free(tot);
    if (hc[2] != 0) {
        fprintf(stderr, "cs_init: N=%d: %d links do not fit the face-tiled stencil layout\n", N, hc[2]);
        grid_release(t);
        return -1;
    }
    if (t->asym_count) fprintf(stderr, "cs_init: warning: %d non-reciprocal Voronoi links\n", t->asym_count);
    if (t->open_cells) fprintf(stderr, "cs_init: warning: %d open Voronoi cells\n", t->open_cells);
    return 0;
}

void grid_release(GridTables *t) {
    bool m = t->managed;
    tfree(m, t->pos);
    tfree(m, t->area);
    tfree(m, t->nnb);
    tfree(m, t->nbr);
    tfree(m, t->w);
    tfree(m, t->elen);
    tfree(m, t->gc);
    dev_free(t->ghost);
    dev_free(t->wslot);
    dev_free(t->wslot_d);
    dev_free(t->ring_nb);
    dev_free(t->ring_w);
    dev_free(t->dinv);
    *t = GridTables();
}

// ------------------------------------------------------------ registry
static std::mutex g_reg_mu;
static std::vector<GridTables *> g_reg;

GridTables *grid_find(const CubeSphere *cs) {
    if (!cs) return nullptr;
    std::lock_guard<std::mutex> lk(g_reg_mu);
    for (GridTables *t : g_reg)
        if (t->pos == cs->pos && cs->pos) return t;
    return nullptr;
}

GridTables *grid_lookup(const CubeSphere *cs) {
    GridTables *t = grid_find(cs);
    if (!t) fail_msg("grid %p (N=%d) was not created by this library's cs_init", (const void *)cs, cs ? cs->N : -1);
    return t;
}

}  // namespace ggb

using namespace ggb;

// ------------------------------------------------------------ public API

GGB_EXPORT const vec3 cs_face_center[6] = {{0, 0, 1}, {1, 0, 0}, {0, 0, -1}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
GGB_EXPORT const vec3 cs_face_right[6] = {{1, 0, 0}, {0, 0, -1}, {-1, 0, 0}, {0, 0, 1}, {1, 0, 0}, {1, 0, 0}};
GGB_EXPORT const vec3 cs_face_up[6] = {{0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

GGB_EXPORT int cs_init(CubeSphere *cs, int N) {
    memset(cs, 0, sizeof(*cs));
    GridTables *t = new GridTables();
    if (grid_build(t, N, true) != 0) {
        delete t;
        return -1;
    }
    cs->N = N;
    cs->ncells = t->n;
    cs->h = t->h;
    cs->pos = t->pos;
    cs->area = t->area;
    cs->nnb = t->nnb;
    cs->nbr = t->nbr;
    cs->w = t->w;
    cs->elen = t->elen;
    cs->gc = t->gc;
    cs->total_area = t->total_area;
    cs->asym_count = t->asym_count;
    cs->open_cells = t->open_cells;
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_reg.push_back(t);
    return 0;
}

GGB_EXPORT void cs_free(CubeSphere *cs) {
    GridTables *t = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_reg_mu);
        for (size_t k = 0; k < g_reg.size(); k++)
            if (cs->pos && g_reg[k]->pos == cs->pos) {
                t = g_reg[k];
                g_reg.erase(g_reg.begin() + k);
                break;
            }
    }
    if (t) {
        sync();
        grid_release(t);
        delete t;
    }
    memset(cs, 0, sizeof(*cs));
}

// Host point location: the same FP64 arithmetic as the device helpers
// (upstream src/cubesphere.c:12-111), for callers working on the host.
GGB_EXPORT int cs_face_of(vec3 d) { return face_of(d3(d.x, d.y, d.z)); }

GGB_EXPORT vec3 cs_face_ab_to_dir(int f, double a, double b) {
    vec3 off = v3_add(v3_scale(cs_face_right[f], tan(a)), v3_scale(cs_face_up[f], tan(b)));
    return v3_normalize(v3_add(cs_face_center[f], off));
}

GGB_EXPORT void cs_locate(const CubeSphere *cs, vec3 d, int *f, double *x, double *y) {
    int face = cs_face_of(d);
    double dc = v3_dot(d, cs_face_center[face]);
    double u = v3_dot(d, cs_face_right[face]) / dc;
    double v = v3_dot(d, cs_face_up[face]) / dc;
    *f = face;
    *x = (atan(u) + kPi / 4) / cs->h - 0.5;
    *y = (atan(v) + kPi / 4) / cs->h - 0.5;
}

static int host_clamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

GGB_EXPORT int cs_cell_of(const CubeSphere *cs, vec3 d) {
    int f;
    double x, y;
    cs_locate(cs, d, &f, &x, &y);
    int i = host_clamp((int)floor(x + 0.5), 0, cs->N - 1), j = host_clamp((int)floor(y + 0.5), 0, cs->N - 1);
    return (f * cs->N + j) * cs->N + i;
}

static int host_tap(const CubeSphere *cs, int f, int i, int j) {
    int N = cs->N;
    if (i >= 0 && j >= 0 && i < N && j < N) return (f * N + j) * N + i;
    return cs_cell_of(cs, cs_face_ab_to_dir(f, -kPi / 4 + (i + 0.5) * cs->h, -kPi / 4 + (j + 0.5) * cs->h));
}

GGB_EXPORT void cs_taps(const CubeSphere *cs, vec3 p, int idx[4], double wt[4]) {
    int f;
    double x, y;
    cs_locate(cs, p, &f, &x, &y);
    int i0 = (int)floor(x), j0 = (int)floor(y);
    double fx = x - i0, fy = y - j0;
    for (int k = 0; k < 4; k++) idx[k] = host_tap(cs, f, i0 + (k & 1), j0 + (k >> 1));
    wt[0] = (1 - fx) * (1 - fy);
    wt[1] = fx * (1 - fy);
    wt[2] = (1 - fx) * fy;
    wt[3] = fx * fy;
}

GGB_EXPORT double cs_sample_scalar(const CubeSphere *cs, const float *fld, vec3 p) {
    int idx[4];
    double wt[4];
    cs_taps(cs, p, idx, wt);
    sync();
    return wt[0] * fld[idx[0]] + wt[1] * fld[idx[1]] + wt[2] * fld[idx[2]] + wt[3] * fld[idx[3]];
}

GGB_EXPORT vec3 cs_sample_vec(const CubeSphere *cs, const float *fld3, vec3 p) {
    int idx[4];
    double wt[4];
    cs_taps(cs, p, idx, wt);
    sync();
    vec3 r = v3(0, 0, 0);
    for (int k = 0; k < 4; k++) r = v3_add(r, v3_scale(v3_load(fld3 + 3 * idx[k]), wt[k]));
    return v3_tangent(r, p);
}

// ------------------------------------------------------------ batched lookups
// Additive entry points: the device-side point location used inside the
// advection / particle kernels, for n directions at once.

namespace ggb {
__global__ void k_cell_of(GridDev g, int n, const double *dirs, int *out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        out[k] = cell_of(d3(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]), g.N, g.h);
}
__global__ void k_taps_batch(GridDev g, int n, const double *dirs, int *idx, double *wt) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        taps(g, d3(dirs[3 * k], dirs[3 * k + 1], dirs[3 * k + 2]), idx + 4 * k, wt + 4 * k);
}
// Bad entries of the public arrays of a grid (ggb_grid_validate): area,
// weights and edge lengths must be finite and positive on every link, counts
// at most kMaxNb, neighbours in range and not the cell itself.
__global__ void k_validate(int n, const float *area, const unsigned char *nnb, const int *nbr, const float *w,
                           const float *elen, unsigned long long *bad) {
    unsigned long long b = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const float a = area[c];
        b += !(isfinite(a) && a > 0.f);
        int m = nnb[c];
        if (m > kMaxNb) {
            b++;
            m = kMaxNb;
        }
        for (int k = 0; k < m; k++) {
            const int j = nbr[(size_t)kMaxNb * c + k];
            const float q = w[(size_t)kMaxNb * c + k], e = elen[(size_t)kMaxNb * c + k];
            b += (j < 0 || j >= n || j == c);
            b += !(isfinite(q) && q > 0.f);
            b += !(isfinite(e) && e > 0.f);
        }
    }
    for (int o = 16; o > 0; o >>= 1) b += __shfl_xor_sync(0xffffffffu, b, o);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(bad, b);
}

}  // namespace ggb

GGB_EXPORT long ggb_grid_validate(const CubeSphere *cs) {
    GridTables *t = grid_lookup(cs);
    unsigned long long *bad = (unsigned long long *)dev_alloc(sizeof(unsigned long long));
    k_validate<<<std::max(1u, std::min(grid_for(t->n, 256), 4096u)), 256, 0, stream()>>>(t->n, t->area, t->nnb,
                                                                                      t->nbr, t->w, t->elen, bad);
    GGB_LAUNCHED();
    unsigned long long h = 0;
    GGB_CHECK(cudaMemcpyAsync(&h, bad, sizeof(h), cudaMemcpyDeviceToHost, stream()));
    sync();
    dev_free(bad);
    return (long)h;
}

// out[k] = cs_cell_of(cs, dirs[k]) computed on the GPU (dirs: n*3 doubles).
GGB_EXPORT void ggb_cell_of_batch(const CubeSphere *cs, const double *dirs, int n, int *out) {
    if (n <= 0) return;
    GridTables *t = grid_lookup(cs);
    Staged in, o;
    stage_in(in, dirs, sizeof(double) * 3 * (size_t)n);
    stage_out(o, out, sizeof(int) * (size_t)n);
    k_cell_of<<<std::max(1u, std::min(grid_for(n, 256), 4096u)), 256, 0, stream()>>>(t->dev(), n,
                                                                                  (const double *)in.dev, (int *)o.dev);
    GGB_LAUNCHED();
    stage_finish(o);
}

// cs_taps for n directions on the GPU (idx: n*4 ints, wt: n*4 doubles).
GGB_EXPORT void ggb_taps_batch(const CubeSphere *cs, const double *dirs, int n, int *idx, double *wt) {
    if (n <= 0) return;
    GridTables *t = grid_lookup(cs);
    Staged in, oi, ow;
    stage_in(in, dirs, sizeof(double) * 3 * (size_t)n);
    stage_out(oi, idx, sizeof(int) * 4 * (size_t)n);
    stage_out(ow, wt, sizeof(double) * 4 * (size_t)n);
    k_taps_batch<<<std::max(1u, std::min(grid_for(n, 256), 4096u)), 256, 0, stream()>>>(
        t->dev(), n, (const double *)in.dev, (int *)oi.dev, (double *)ow.dev);
    GGB_LAUNCHED();
    stage_finish(oi);
    stage_finish(ow);
}
