// ggb_stencil.cuh — the spherical-Voronoi operator K x = sum_j w_ij (x_i - x_j)
// on the face-tiled layout (direction slots + boundary-ring lists), for any
// way of producing the neighbour values (a stored vector or a value computed
// on the fly from other vectors).
#pragma once

#include <cuda_fp16.h>

#include "ggb_device.cuh"

namespace ggb {

struct StencilDev {
    int N, n, nring;
    int lgN;              // log2(N) when N is a power of two, else -1
    const float *wslot;   // [4][n]: E, N, NE, NW weights (0 = no link)
    const double *wslot_d;  // the same in FP64
    const __half *wslot_h;  // the same in FP16 (mixed-precision V-cycle, levels >= 1), or nullptr
    const int *ring_nb;   // [6*nring][8], -1 terminated
    const float *ring_w;  // [6*nring][8]
};

// Row of the ring tables for boundary-ring cell (f, i, j): the tables are in
// cell order (ring rank), so the ring cells of a cell range own one contiguous
// block of rows.
__device__ __forceinline__ int ring_slot(int f, int i, int j, int N, int nring) {
    return f * nring + ring_rank_in_face(i, j, N);
}

__device__ __forceinline__ void cell_fij(int c, int N, int &f, int &i, int &j) {
    int nn = N * N;
    f = c / nn;
    int rem = c - f * nn;
    j = rem / N;
    i = rem - j * N;
}

// cell_fij for a level's stencil: shifts and masks when N is a power of two
// (an integer division takes some twenty instructions), the division otherwise.
__device__ __forceinline__ void cell_fij(const StencilDev &S, int c, int &f, int &i, int &j) {
    const int l = S.lgN;
    if (l >= 0) {
        f = c >> (2 * l);
        const int rem = c & ((1 << (2 * l)) - 1);
        j = rem >> l;
        i = rem & ((1 << l) - 1);
    } else {
        cell_fij(c, S.N, f, i, j);
    }
}

// The links of a boundary-ring cell that leave the face: all eight (neighbour,
// weight) pairs are loaded with two vector loads each, then every present
// neighbour value is requested at once (two dependent rounds in total instead
// of one per link).
template <class X>
__device__ __forceinline__ double ring_extras(const StencilDev &S, int f, int i, int j, double xc, X X_) {
    const int r = ring_slot(f, i, j, S.N, S.nring);
    const int4 *rn4 = reinterpret_cast<const int4 *>(S.ring_nb + r * kMaxNb);
    const float4 *rw4 = reinterpret_cast<const float4 *>(S.ring_w + r * kMaxNb);
    const int4 n0 = __ldg(rn4), n1 = __ldg(rn4 + 1);
    const float4 q0 = __ldg(rw4), q1 = __ldg(rw4 + 1);
    const int o[8] = {n0.x, n0.y, n0.z, n0.w, n1.x, n1.y, n1.z, n1.w};
    const float q[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = o[k] >= 0 ? X_(o[k]) : xc;
    double s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (o[k] >= 0) s += (double)q[k] * (xc - v[k]);
    return s;
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
    cell_fij(S, c, f, i, j);
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
    return s + ring_extras(S, f, i, j, xc, X_);
}

// Boundary-ring cells in cell order: the number of ring cells with index
// below c (c in [0, n]), and the cell of ring rank R.
__device__ __forceinline__ int ring_rank_below(int c, int N, int nring) {
    int f, i, j;
    cell_fij(c, N, f, i, j);
    return f * nring + ring_rank_in_face(i, j, N);
}
__device__ __forceinline__ void ring_cell_of_rank(int R, int N, int nring, int &f, int &i, int &j) {
    f = R / nring;
    const int q = R - f * nring;
    if (q < N) {
        j = 0;
        i = q;
    } else if (q < 3 * N - 4) {
        const int m = q - N;
        j = 1 + (m >> 1);
        i = (m & 1) ? N - 1 : 0;
    } else {
        j = N - 1;
        i = q - (3 * N - 4);
    }
}

// K at cell c with the window's values x[k] and FP64 slot weights w0..w3[k]
// all staged in shared memory (indexed by cell; the window spans [c - N - 1,
// c + N + 1] for every cell c of the block's range, zero-filled where it
// runs past the ends of the grid).  One branch-free formula serves every
// cell: a slot whose link would leave the face has weight 0 in the layout
// (also where the neighbouring index wraps to another row or face), so its
// term adds an exact zero.  A boundary-ring cell adds the staged sum of its
// links that leave the face, rsum[ring rank - r0].
template <class A>
__device__ __forceinline__ A apply_k_smem(const StencilDev &S, int c, A xc, const A *x, const A *wE, const A *wN,
                                          const A *wNE, const A *wNW, const A *rsum, int r0) {
    const int N = S.N;
    int f, i, j;
    cell_fij(S, c, f, i, j);
    A s = wE[c] * (xc - x[c + 1]);
    s += wN[c] * (xc - x[c + N]);
    s += wNE[c] * (xc - x[c + N + 1]);
    s += wNW[c] * (xc - x[c + N - 1]);
    s += wE[c - 1] * (xc - x[c - 1]);
    s += wN[c - N] * (xc - x[c - N]);
    s += wNE[c - N - 1] * (xc - x[c - N - 1]);
    s += wNW[c - N + 1] * (xc - x[c - N + 1]);
    if (i == 0 || j == 0 || i == N - 1 || j == N - 1) s += rsum[f * S.nring + ring_rank_in_face(i, j, N) - r0];
    return s;
}

// The links of cell c as up to 8 (neighbour, weight) pairs; unused pairs have
// weight 0 and neighbour c.  For loops that apply one cell's stencil many times.
__device__ __forceinline__ void cell_links(const StencilDev &S, int c, int nb[kMaxNb], float wv[kMaxNb]) {
    const int N = S.N, n = S.n;
    int f, i, j;
    cell_fij(S, c, f, i, j);
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
