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
// X(k) returns the neighbour value as a double.
template <class X>
__device__ __forceinline__ double apply_k(const StencilDev &S, int c, double xc, X X_) {
    const int N = S.N, n = S.n;
    int f, i, j;
    cell_fij(c, N, f, i, j);
    const float *ws = S.wslot;
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
    if (!(e && w && up && dn)) {
        int r = ring_slot(f, i, j, N, S.nring);
        const int *rn = S.ring_nb + r * kMaxNb;
        const float *rw = S.ring_w + r * kMaxNb;
        for (int k = 0; k < kMaxNb; k++) {
            int o = __ldg(rn + k);
            if (o < 0) break;
            s += (double)__ldg(rw + k) * (xc - X_(o));
        }
    }
    return s;
}

}  // namespace ggb
