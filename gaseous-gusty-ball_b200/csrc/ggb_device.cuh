// ggb_device.cuh — device-side geometry helpers shared by all kernels of
// libggb_cuda.so: double-precision 3-vectors, the cube-face projections,
// point location / bilinear taps on the equiangular cubed sphere, great-circle
// motion, a bounded grid-wide barrier and fixed-order FP64 block reductions.
//
// Expression order follows the upstream host code (src/vec3.h, src/cubesphere.c
// of gaseous-gusty-ball) so that FP64 results agree with it to rounding and the
// integer outcomes (face, cell, tap indices) agree exactly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ggb {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxNb = 8;

struct D3 {
    double x, y, z;
};

__host__ __device__ __forceinline__ D3 d3(double x, double y, double z) {
    D3 r;
    r.x = x;
    r.y = y;
    r.z = z;
    return r;
}
__host__ __device__ __forceinline__ D3 add(D3 a, D3 b) { return d3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ D3 sub(D3 a, D3 b) { return d3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ D3 scale(D3 a, double k) { return d3(a.x * k, a.y * k, a.z * k); }
__host__ __device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return d3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double len(D3 a) { return sqrt(dot(a, a)); }
__device__ __forceinline__ D3 normalize(D3 a) {
    double l = len(a);
    return l > 0.0 ? scale(a, 1.0 / l) : a;
}
__host__ __device__ __forceinline__ D3 tangent(D3 v, D3 n) { return sub(v, scale(n, dot(v, n))); }
__device__ __forceinline__ double angle(D3 a, D3 b) { return atan2(len(cross(a, b)), dot(a, b)); }

__device__ __forceinline__ D3 load3(const float *p) { return d3(p[0], p[1], p[2]); }
__device__ __forceinline__ void store3(float *p, D3 a) {
    p[0] = (float)a.x;
    p[1] = (float)a.y;
    p[2] = (float)a.z;
}

// Great-circle motion of unit p along the tangent part of v for time s.
__device__ __forceinline__ D3 sphere_move(D3 p, D3 v, double s) {
    D3 t = tangent(v, p);
    double sp = len(t);
    if (sp < 1e-300) return p;
    double th = sp * s;
    double sn, cs;
    sincos(th, &sn, &cs);
    return normalize(add(scale(p, cs), scale(t, sn / sp)));
}

// ---------------------------------------------------------------- faces
// Face f: centre c, right r, up u (face 0 = +Z, 1 = +X, 2 = -Z, 3 = -X,
// 4 = +Y, 5 = -Y).  Every component is 0 or +-1, so the dot products of the
// generic form reduce exactly to a signed coordinate; they are written that way.

__host__ __device__ __forceinline__ int face_of(D3 d) {
    double ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
    if (ax >= ay && ax >= az) return d.x > 0 ? 1 : 3;
    if (ay >= az) return d.y > 0 ? 4 : 5;
    return d.z > 0 ? 0 : 2;
}

// (d.c, d.r, d.u) for face f.
__host__ __device__ __forceinline__ void face_proj(int f, D3 d, double &dc, double &dr, double &du) {
    switch (f) {
        case 0: dc = d.z; dr = d.x; du = d.y; break;
        case 1: dc = d.x; dr = -d.z; du = d.y; break;
        case 2: dc = -d.z; dr = -d.x; du = d.y; break;
        case 3: dc = -d.x; dr = d.z; du = d.y; break;
        case 4: dc = d.y; dr = d.x; du = -d.z; break;
        default: dc = -d.y; dr = d.x; du = d.z; break;
    }
}

// c + (r*ta + u*tb) for face f (exact: each component is 1, +-ta or +-tb).
__host__ __device__ __forceinline__ D3 face_point(int f, double ta, double tb) {
    switch (f) {
        case 0: return d3(ta, tb, 1.0);
        case 1: return d3(1.0, tb, -ta);
        case 2: return d3(-ta, tb, -1.0);
        case 3: return d3(-1.0, tb, ta);
        case 4: return d3(ta, 1.0, -tb);
        default: return d3(ta, -1.0, tb);
    }
}

__device__ __forceinline__ D3 face_ab_to_dir(int f, double a, double b) {
    return normalize(face_point(f, tan(a), tan(b)));
}

// Equiangular cell-centre direction of (possibly off-face) cell (i, j).
__device__ __forceinline__ D3 centre_dir(int f, int i, int j, double h) {
    return face_ab_to_dir(f, -kPi / 4 + (i + 0.5) * h, -kPi / 4 + (j + 0.5) * h);
}

// Continuous cell coordinates (cell centres at integers).
__device__ __forceinline__ void locate(D3 d, double h, int &f, double &x, double &y) {
    f = face_of(d);
    double dc, dr, du;
    face_proj(f, d, dc, dr, du);
    double u = dr / dc, v = du / dc;
    x = (atan(u) + kPi / 4) / h - 0.5;
    y = (atan(v) + kPi / 4) / h - 0.5;
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

__device__ __forceinline__ int cell_of(D3 d, int N, double h) {
    int f;
    double x, y;
    locate(d, h, f, x, y);
    int i = clampi((int)floor(x + 0.5), 0, N - 1);
    int j = clampi((int)floor(y + 0.5), 0, N - 1);
    return (f * N + j) * N + i;
}

// Real cell of ghost (i, j) on face f computed from scratch (setup kernels).
__device__ __forceinline__ int ghost_cell_direct(int f, int i, int j, int N, double h) {
    if (i >= 0 && j >= 0 && i < N && j < N) return (f * N + j) * N + i;
    return cell_of(centre_dir(f, i, j, h), N, h);
}

// Position of boundary-ring cell (i, j) among its face's ring cells in cell
// order: row 0, then the two end cells of every middle row, then row N-1.
// For any cell it is the number of the face's ring cells before it.
__host__ __device__ __forceinline__ int ring_rank_in_face(int i, int j, int N) {
    return j == 0 ? i : (j < N - 1 ? N + 2 * (j - 1) + (i > 0) : 3 * N - 4 + i);
}

// Index of ghost (i, j), i, j in [-1, N], into a face's ring table of 4N+4 entries.
__host__ __device__ __forceinline__ int ghost_ring_index(int i, int j, int N) {
    if (j == -1) return i + 1;
    if (j == N) return (N + 2) + i + 1;
    if (i == -1) return 2 * (N + 2) + j;
    return 2 * (N + 2) + N + j;  // i == N
}

// Grid descriptor passed by value to kernels.
struct GridDev {
    int N;
    int n;                 // 6*N*N
    double h;
    const int *ghost;      // [6*(4N+4)] real cell of each one-deep ghost cell
};

__device__ __forceinline__ int tap_cell(const GridDev &g, int f, int i, int j) {
    int N = g.N;
    if (i >= 0 && j >= 0 && i < N && j < N) return (f * N + j) * N + i;
    return g.ghost[f * (4 * N + 4) + ghost_ring_index(i, j, N)];
}

// Bilinear taps at p; upstream src/cubesphere.c:68-92.
__device__ __forceinline__ void taps(const GridDev &g, D3 p, int idx[4], double wt[4]) {
    int f;
    double x, y;
    locate(p, g.h, f, x, y);
    int N = g.N;
    // x, y lie in [-0.5, N-0.5] for any unit vector; the clamp only guards the
    // table reads against non-finite input
    int i0 = clampi((int)floor(x), -1, N - 1), j0 = clampi((int)floor(y), -1, N - 1);
    double fx = x - i0, fy = y - j0;
    if (i0 >= 0 && j0 >= 0 && i0 + 1 < N && j0 + 1 < N) {
        int b = (f * N + j0) * N + i0;
        idx[0] = b;
        idx[1] = b + 1;
        idx[2] = b + N;
        idx[3] = b + N + 1;
    } else {
        idx[0] = tap_cell(g, f, i0, j0);
        idx[1] = tap_cell(g, f, i0 + 1, j0);
        idx[2] = tap_cell(g, f, i0, j0 + 1);
        idx[3] = tap_cell(g, f, i0 + 1, j0 + 1);
    }
    wt[0] = (1 - fx) * (1 - fy);
    wt[1] = fx * (1 - fy);
    wt[2] = (1 - fx) * fy;
    wt[3] = fx * fy;
}

__device__ __forceinline__ double sample_scalar(const GridDev &g, const float *fld, D3 p) {
    int idx[4];
    double wt[4];
    taps(g, p, idx, wt);
    return wt[0] * __ldg(fld + idx[0]) + wt[1] * __ldg(fld + idx[1]) + wt[2] * __ldg(fld + idx[2]) +
           wt[3] * __ldg(fld + idx[3]);
}

__device__ __forceinline__ D3 sample_vec(const GridDev &g, const float *fld3, D3 p) {
    int idx[4];
    double wt[4];
    taps(g, p, idx, wt);
    D3 r = d3(0, 0, 0);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float *q = fld3 + 3 * idx[k];
        r = add(r, scale(d3(__ldg(q), __ldg(q + 1), __ldg(q + 2)), wt[k]));
    }
    return tangent(r, p);
}

// ---------------------------------------------------------------- barrier
// Grid-wide barrier for cooperative (co-resident) launches.  Every wait is
// bounded: after kBarrierTimeoutNs the waiting block raises `err` and returns
// false, and every later barrier returns false at once, so a kernel can never
// spin forever.
struct GridBarrier {
    unsigned int count;  // arrivals since the launch began (zeroed by the host before each launch)
    int err;             // sticky: a barrier timed out
};

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int *p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_volatile_i32(const int *p) { return *(volatile const int *)p; }

__device__ __forceinline__ unsigned int atom_add_acq_rel_u32(unsigned int *p, unsigned int v) {
    unsigned int old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// Returns true when all blocks arrived; false on timeout (limit_ns after the
// first 64 polls) or an error raised by another block.  `count` counts
// arrivals since the launch began (the host zeroes it before every launch):
// thread 0 arrives with one acq_rel atomic
// after a block barrier (so every write of the block before the barrier is
// released), and the barrier is complete when the count reaches the next
// multiple of the number of blocks, which the waiters poll with acquire loads.
// The arrival is the first global access of a barrier (no generation or error
// read before it); the error flag and the timeout are checked every 64 polls.
// nb: the number of blocks that meet at this barrier (the whole grid, or the
// blocks of one solve inside a batched launch).
__device__ __forceinline__ bool grid_sync_nb(GridBarrier *bar, unsigned int nb, unsigned long long limit_ns) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int old = atom_add_acq_rel_u32(&bar->count, 1u);
        const unsigned int target = (old / nb + 1u) * nb;
        int ok = 1;
        unsigned long long t0 = 0;
        unsigned int polls = 0;
        while ((int)(ld_acquire_u32(&bar->count) - target) < 0) {
            if ((++polls & 63u) == 0) {
                if (ld_volatile_i32(&bar->err) != 0) {
                    ok = 0;
                    break;
                }
                const unsigned long long t = globaltimer_ns();
                if (polls == 64u) {
                    t0 = t;
                } else if (t - t0 > limit_ns) {
                    atomicExch(&bar->err, 1);
                    ok = 0;
                    break;
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}
__device__ __forceinline__ bool grid_sync_limit(GridBarrier *bar, unsigned long long limit_ns) {
    return grid_sync_nb(bar, gridDim.x * gridDim.y * gridDim.z, limit_ns);
}
__device__ __forceinline__ bool grid_sync(GridBarrier *bar) { return grid_sync_limit(bar, kBarrierTimeoutNs); }

// ------------------------------------------------------------ reductions
// Block sum of one double per thread, returned to every thread.  The
// combination order depends only on thread indices, so it is deterministic.
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double *s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    double t = 0;
    if (warp == 0) {
        t = lane < BLOCK / 32 ? s_red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) s_red[BLOCK / 32] = t;
    }
    __syncthreads();
    return s_red[BLOCK / 32];
}

// Sum of `count` per-block partials, in a fixed order, returned to every thread.
template <int BLOCK>
__device__ __forceinline__ double sum_partials(const double *part, int count, double *s_red) {
    double v = 0;
    if (threadIdx.x < 32) {
        for (int k = threadIdx.x; k < count; k += 32) v += *(volatile const double *)(part + k);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) s_red[BLOCK / 32 + 1] = v;
    }
    __syncthreads();
    double r = s_red[BLOCK / 32 + 1];
    __syncthreads();
    return r;
}

}  // namespace ggb
