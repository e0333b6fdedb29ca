// ggb_stencil.cuh — the spherical-Voronoi operator K x = sum_j w_ij (x_i - x_j)
// on the face-tiled layout (direction slots + boundary-ring lists), for any
// way of producing the neighbour values (a stored vector or a value computed
// on the fly from other vectors).
#pragma once

#include "ggb_device.cuh"

namespace ggb {

struct StencilDev {
    int N, n, nring;
    const float *wslot;   // [4][n]: E, N, NE, NW weights (0 = no link)
    const int *ring_nb;   // [6*nring][8], -1 terminated
    const float *ring_w;  // [6*nring][8]
};

__device__ __forceinline__ int ring_slot(int f, int i, int j, int N, int nring) {
    int r;
    if (j == 0) r = i;
    else if (j == N - 1) r = N + i;
    else if (i == 0) r = 2 * N + (j - 1);
    else r = 2 * N + (N - 2) + (j - 1);
    return f * nring + r;
}

__device__ __forceinline__ void cell_fij(int c, int N, int &f, int &i, int &j) {
    int nn = N * N;
    f = c / nn;
    int rem = c - f * nn;
    j = rem / N;
    i = rem - j * N;
}

// sum over the links of cell c of w * (xc - X(nb)), accumulated in double.
// X(k) returns the neighbour value as a double.  Interior cells (not on the
// face's boundary ring) take a branch-free path: all eight direction weights
// and neighbour values are loaded unconditionally (absent links have weight 0),
// so the loads issue together instead of as a chain of dependent branches.
template <class X>
__device__ __forceinline__ double apply_k(const StencilDev &S, int c, double xc, X X_) {
    const int N = S.N, n = S.n;
    int f, i, j;
    cell_fij(c, N, f, i, j);
    const float *ws = S.wslot;
    if (i > 0 && j > 0 && i + 1 < N && j + 1 < N) {
        const float w0 = __ldg(ws + c), w1 = __ldg(ws + n + c), w2 = __ldg(ws + 2 * n + c),
                    w3 = __ldg(ws + 3 * n + c), w4 = __ldg(ws + c - 1), w5 = __ldg(ws + n + c - N),
                    w6 = __ldg(ws + 2 * n + c - N - 1), w7 = __ldg(ws + 3 * n + c - N + 1);
        const double x0 = X_(c + 1), x1 = X_(c + N), x2 = X_(c + N + 1), x3 = X_(c + N - 1), x4 = X_(c - 1),
                     x5 = X_(c - N), x6 = X_(c - N - 1), x7 = X_(c - N + 1);
        double s = (double)w0 * (xc - x0);
        s += (double)w1 * (xc - x1);
        s += (double)w2 * (xc - x2);
        s += (double)w3 * (xc - x3);
        s += (double)w4 * (xc - x4);
        s += (double)w5 * (xc - x5);
        s += (double)w6 * (xc - x6);
        s += (double)w7 * (xc - x7);
        return s;
    }
    const bool e = i + 1 < N, w = i > 0, up = j + 1 < N, dn = j > 0;
    double s = 0;
    float q;
    if (e && (q = __ldg(ws + c)) != 0.f) s += (double)q * (xc - X_(c + 1));
    if (up && (q = __ldg(ws + n + c)) != 0.f) s += (double)q * (xc - X_(c + N));
    if (e && up && (q = __ldg(ws + 2 * n + c)) != 0.f) s += (double)q * (xc - X_(c + N + 1));
    if (w && up && (q = __ldg(ws + 3 * n + c)) != 0.f) s += (double)q * (xc - X_(c + N - 1));
    if (w && (q = __ldg(ws + c - 1)) != 0.f) s += (double)q * (xc - X_(c - 1));
    if (dn && (q = __ldg(ws + n + c - N)) != 0.f) s += (double)q * (xc - X_(c - N));
    if (w && dn && (q = __ldg(ws + 2 * n + c - N - 1)) != 0.f) s += (double)q * (xc - X_(c - N - 1));
    if (e && dn && (q = __ldg(ws + 3 * n + c - N + 1)) != 0.f) s += (double)q * (xc - X_(c - N + 1));
    int r = ring_slot(f, i, j, N, S.nring);
    const int *rn = S.ring_nb + r * kMaxNb;
    const float *rw = S.ring_w + r * kMaxNb;
    for (int k = 0; k < kMaxNb; k++) {
        int o = __ldg(rn + k);
        if (o < 0) break;
        s += (double)__ldg(rw + k) * (xc - X_(o));
    }
    return s;
}

// The links of cell c as up to 8 (neighbour, weight) pairs; unused pairs have
// weight 0 and neighbour c.  For loops that apply one cell's stencil many times.
__device__ __forceinline__ void cell_links(const StencilDev &S, int c, int nb[kMaxNb], float wv[kMaxNb]) {
    const int N = S.N, n = S.n;
    int f, i, j;
    cell_fij(c, N, f, i, j);
    const float *ws = S.wslot;
    int m = 0;
    auto put = [&](int o, float q) {
        if (q != 0.f && m < kMaxNb) {
            nb[m] = o;
            wv[m] = q;
            m++;
        }
    };
    if (i + 1 < N) put(c + 1, __ldg(ws + c));
    if (j + 1 < N) put(c + N, __ldg(ws + n + c));
    if (i + 1 < N && j + 1 < N) put(c + N + 1, __ldg(ws + 2 * n + c));
    if (i > 0 && j + 1 < N) put(c + N - 1, __ldg(ws + 3 * n + c));
    if (i > 0) put(c - 1, __ldg(ws + c - 1));
    if (j > 0) put(c - N, __ldg(ws + n + c - N));
    if (i > 0 && j > 0) put(c - N - 1, __ldg(ws + 2 * n + c - N - 1));
    if (i + 1 < N && j > 0) put(c - N + 1, __ldg(ws + 3 * n + c - N + 1));
    if (!(i > 0 && j > 0 && i + 1 < N && j + 1 < N)) {
        int r = ring_slot(f, i, j, N, S.nring);
        for (int k = 0; k < kMaxNb; k++) {
            int o = __ldg(S.ring_nb + r * kMaxNb + k);
            if (o < 0) break;
            put(o, __ldg(S.ring_w + r * kMaxNb + k));
        }
    }
    for (int k = m; k < kMaxNb; k++) {
        nb[k] = c;
        wv[k] = 0.f;
    }
}

}  // namespace ggb
