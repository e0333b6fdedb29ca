// render.cu — the render.h entry points of libggb_cuda.so: tent-filtered,
// "over"-blended, globally fading particle-trail splatting into the six
// cube-face images.
//
// Upstream: src/render.c.  Per texel the composite must apply the splat
// samples in ascending (particle index, sample k) order (upstream records are
// binned thread-major over contiguous particle ranges, src/render.c:156-218).
// This library reaches the same per-texel order without a global sort:
//   1. count:  every particle counts the 32x32 texel tiles its arc touches
//              (bounding box of its sample footprints per face) — atomics;
//   2. scan:   tile offsets (one block);
//   3. fill:   every particle appends its index to the lists of those tiles;
//   4. tiles:  one block per tile sorts its list (bitonic, ascending index),
//              expands the samples of those particles that fall on the tile
//              in (index, k) order, bins them per texel, sorts each texel's
//              (short) list by sample order and applies the blends in order
//              to the tile held in shared memory.
// The pending renormalisation of render_fade is fused into step 4.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "ggb_internal.h"

namespace ggb {

constexpr int kT = 32;              // tile edge in texels
constexpr int kTB = 256;            // threads per tile block
constexpr int kSortCap = 2048;      // tile lists up to this length sort in shared memory
constexpr int kChunk = kTB;         // particles expanded per chunk
constexpr int kSampleCap = 2048;    // samples binned per window
constexpr int kEntryCap = 8192;     // (sample, texel) entries per window
constexpr int kMaxSamples = 4096;   // upstream cap on samples per arc

struct RenderPriv {
    int R = 0, ntx = 0, ntiles = 0;
    unsigned *tile_count = nullptr, *tile_start = nullptr, *tile_fill = nullptr;
    unsigned *list = nullptr;
    size_t list_cap = 0;
    unsigned *slow_tiles = nullptr;  // tiles left to the sorted path
    unsigned *slow_count = nullptr;
    unsigned *total_host = nullptr;
    bool pending = false;
    float pending_scale = 1.f;
    float *mirror = nullptr;
    std::atomic<unsigned long> dev_gen{1}, mirror_gen{0};
    std::mutex mu;
};

static RenderPriv *rpriv(const Render *r) {
    if (!r->tr) fail_msg("Render %p was not initialised by this library's render_init", (const void *)r);
    return reinterpret_cast<RenderPriv *>(r->tr);
}

struct SplatCfg {
    int R, ntx;
    float rad, invrad, invg, alpha;
    double spacing;
    int renorm;
    float scale;
};

// Sample k of the arc a -> b (chord lerp, normalised), FP64 with the
// contraction pattern of the upstream build.
__device__ __forceinline__ D3 arc_point(D3 a, D3 b, int k, int ns) {
    double tt = (double)k / ns, s = 1 - tt;
    D3 v = d3(__fma_rn(a.x, s, __dmul_rn(b.x, tt)), __fma_rn(a.y, s, __dmul_rn(b.y, tt)),
              __fma_rn(a.z, s, __dmul_rn(b.z, tt)));
    double l = sqrt(__fma_rn(v.z, v.z, __fma_rn(v.x, v.x, __dmul_rn(v.y, v.y))));
    return l > 0.0 ? scale(v, 1.0 / l) : v;
}

__device__ __forceinline__ int arc_samples(D3 a, D3 b, double spacing) {
    int ns = (int)ceil(angle(a, b) / spacing);
    return ns < 1 ? 1 : (ns > kMaxSamples ? kMaxSamples : ns);
}

// Projection of d on face f: false when the face is not used for d
// (d.c < 0.5).  px, py as upstream src/render.c:92-98.
__device__ __forceinline__ bool face_px(int f, D3 d, int R, float &px, float &py) {
    double dc, dr, du;
    face_proj(f, d, dc, dr, du);
    if (dc < 0.5) return false;
    double u = dr / dc, v = du / dc;
    px = (float)__fma_rn((u + 1.0) * 0.5, (double)R, -0.5);
    py = (float)__fma_rn((1.0 - v) * 0.5, (double)R, -0.5);
    return true;
}

struct Box {
    int xlo, xhi, ylo, yhi;
};

// Clamped texel footprint of a sample; empty when xlo > xhi or ylo > yhi.
__device__ __forceinline__ Box footprint(float px, float py, float rad, int R) {
    Box b;
    b.xlo = max(0, (int)ceilf(px - rad));
    b.xhi = min(R - 1, (int)floorf(px + rad));
    b.ylo = max(0, (int)ceilf(py - rad));
    b.yhi = min(R - 1, (int)floorf(py + rad));
    return b;
}

// Tiles (per face bounding box of the non-empty footprints) touched by one
// particle's arc; calls emit(tile) for each.
template <class Emit>
__device__ __forceinline__ void arc_tiles(const SplatCfg &C, D3 a, D3 b, Emit emit) {
    int ns = arc_samples(a, b, C.spacing);
    int tlo[6][2], thi[6][2];
    for (int f = 0; f < 6; f++) {
        tlo[f][0] = tlo[f][1] = 1 << 30;
        thi[f][0] = thi[f][1] = -1;
    }
    for (int k = 1; k <= ns; k++) {
        D3 d = arc_point(a, b, k, ns);
        for (int f = 0; f < 6; f++) {
            float px, py;
            if (!face_px(f, d, C.R, px, py)) continue;
            Box bx = footprint(px, py, C.rad, C.R);
            if (bx.xlo > bx.xhi || bx.ylo > bx.yhi) continue;
            tlo[f][0] = min(tlo[f][0], bx.xlo / kT);
            thi[f][0] = max(thi[f][0], bx.xhi / kT);
            tlo[f][1] = min(tlo[f][1], bx.ylo / kT);
            thi[f][1] = max(thi[f][1], bx.yhi / kT);
        }
    }
    for (int f = 0; f < 6; f++)
        for (int ty = tlo[f][1]; ty <= thi[f][1]; ty++)
            for (int tx = tlo[f][0]; tx <= thi[f][0]; tx++) emit((f * C.ntx + ty) * C.ntx + tx);
}

// Conservative tile set of an arc for binning (a superset of arc_tiles).  The
// samples are normalised chord points of the great-circle arc a -> b; on a
// face whose hemisphere holds both endpoints the gnomonic image of that arc is
// the segment between the endpoint images, so the bounding box of the two
// endpoint footprints (plus a margin) covers every sample footprint.  A face
// is skipped when neither endpoint is near it: along an arc of angle theta,
// d.c exceeds the larger endpoint value by at most a factor 1/cos(theta/2),
// so no sample reaches d.c >= 0.5.  Long arcs and arcs leaving a face's
// hemisphere take the exact per-sample path.
template <class Emit>
__device__ __forceinline__ void arc_tiles_bound(const SplatCfg &C, D3 a, D3 b, Emit emit) {
    // FP32 is enough for a bound: the projections carry a 0.05-texel margin
    // and the face test a 1e-3 margin, far above FP32 rounding.
    const float ax = (float)a.x, ay = (float)a.y, az = (float)a.z, bx = (float)b.x, by = (float)b.y, bz = (float)b.z;
    const float la = sqrtf(ax * ax + ay * ay + az * az), lb = sqrtf(bx * bx + by * by + bz * bz);
    const float cth = (ax * bx + ay * by + az * bz) / (la * lb);
    if (!(cth > 0.9f)) {  // theta > ~0.45 rad (or degenerate input): exact path
        arc_tiles(C, a, b, emit);
        return;
    }
    const float half_cos = sqrtf(0.5f * (1.0f + cth));  // cos(theta / 2)
    const float Rf = (float)C.R;
    for (int f = 0; f < 6; f++) {
        float ca, ra, ua, cb, rb, ub;
        switch (f) {
            case 0: ca = az; ra = ax; ua = ay; cb = bz; rb = bx; ub = by; break;
            case 1: ca = ax; ra = -az; ua = ay; cb = bx; rb = -bz; ub = by; break;
            case 2: ca = -az; ra = -ax; ua = ay; cb = -bz; rb = -bx; ub = by; break;
            case 3: ca = -ax; ra = az; ua = ay; cb = -bx; rb = bz; ub = by; break;
            case 4: ca = ay; ra = ax; ua = -az; cb = by; rb = bx; ub = -bz; break;
            default: ca = -ay; ra = ax; ua = az; cb = -by; rb = bx; ub = bz; break;
        }
        if (fmaxf(ca / la, cb / lb) < 0.5f * half_cos - 1e-3f) continue;
        if (ca <= 0.05f * la || cb <= 0.05f * lb) {
            // rare: an endpoint near or behind the face's horizon; exact samples for this arc
            arc_tiles(C, a, b, emit);
            return;
        }
        float pxa = (ra / ca + 1.0f) * 0.5f * Rf - 0.5f, pya = (1.0f - ua / ca) * 0.5f * Rf - 0.5f;
        float pxb = (rb / cb + 1.0f) * 0.5f * Rf - 0.5f, pyb = (1.0f - ub / cb) * 0.5f * Rf - 0.5f;
        float m = C.rad + 0.05f;
        float x0 = fminf(pxa, pxb) - m, x1 = fmaxf(pxa, pxb) + m;
        float y0 = fminf(pya, pyb) - m, y1 = fmaxf(pya, pyb) + m;
        if (x1 < 0.f || y1 < 0.f || x0 > Rf - 1.f || y0 > Rf - 1.f) continue;
        int tx0 = max(0, (int)floorf(x0)) / kT, tx1 = min(C.R - 1, (int)floorf(x1)) / kT;
        int ty0 = max(0, (int)floorf(y0)) / kT, ty1 = min(C.R - 1, (int)floorf(y1)) / kT;
        for (int ty = ty0; ty <= ty1; ty++)
            for (int tx = tx0; tx <= tx1; tx++) emit((f * C.ntx + ty) * C.ntx + tx);
    }
}

__global__ void k_rd_count(int n, SplatCfg C, const float *prev, const float *pos, unsigned *tile_count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D3 a = load3(prev + 3 * (size_t)i), b = load3(pos + 3 * (size_t)i);
        arc_tiles_bound(C, a, b, [&](int t) { atomicAdd(tile_count + t, 1u); });
    }
}

__global__ void k_rd_fill(int n, SplatCfg C, const float *prev, const float *pos, const unsigned *tile_start,
                          unsigned *tile_fill, unsigned *list) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D3 a = load3(prev + 3 * (size_t)i), b = load3(pos + 3 * (size_t)i);
        arc_tiles_bound(C, a, b, [&](int t) {
            unsigned slot = atomicAdd(tile_fill + t, 1u);
            if (tile_start[t] + slot < tile_start[t + 1]) list[tile_start[t] + slot] = (unsigned)i;
        });
    }
}

// Exclusive scan of cnt[0..n) into start[0..n] (one block).
__global__ void k_tile_scan(int n, const unsigned *cnt, unsigned *start, unsigned *total) {
    __shared__ unsigned s_tot[1024];
    const int T = blockDim.x, t = threadIdx.x;
    int chunk = (n + T - 1) / T, lo = min(n, t * chunk), hi = min(n, lo + chunk);
    unsigned s = 0;
    for (int k = lo; k < hi; k++) s += cnt[k];
    s_tot[t] = s;
    __syncthreads();
    if (t == 0) {
        unsigned acc = 0;
        for (int k = 0; k < T; k++) {
            unsigned v = s_tot[k];
            s_tot[k] = acc;
            acc += v;
        }
        start[n] = acc;
        *total = acc;
    }
    __syncthreads();
    unsigned acc = s_tot[t];
    for (int k = lo; k < hi; k++) {
        start[k] = acc;
        acc += cnt[k];
    }
}

// Ascending sort of a[0..n) by the whole block (all-ascending bitonic network;
// indices >= n act as +infinity).  `a` may be shared or global memory.
__device__ void block_sort(unsigned *a, int n) {
    int P = 1;
    while (P < n) P <<= 1;
    for (int k = 2; k <= P; k <<= 1) {
        int half = k >> 1;
        for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
            int lo = (t / half) * k + (t % half);
            int hi = lo ^ (k - 1);
            if (hi < n) {
                unsigned x = a[lo], y = a[hi];
                if (x > y) {
                    a[lo] = y;
                    a[hi] = x;
                }
            }
        }
        __syncthreads();
        for (int j = half >> 1; j > 0; j >>= 1) {
            for (int t = threadIdx.x; t < P / 2; t += blockDim.x) {
                int lo = (t / j) * 2 * j + (t % j);
                int hi = lo + j;
                if (hi < n) {
                    unsigned x = a[lo], y = a[hi];
                    if (x > y) {
                        a[lo] = y;
                        a[hi] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Exclusive block scan of one int per thread (kTB threads); returns the total.
__device__ __forceinline__ int block_excl_scan(int v, int &excl, int *s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < kTB / 32 ? s_w[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kTB / 32) s_w[lane] = w;
    }
    __syncthreads();
    int before = warp ? s_w[warp - 1] : 0;
    int total = s_w[kTB / 32 - 1];
    excl = before + x - v;
    __syncthreads();
    return total;
}

struct TileSmem {
    float4 tex[kT * kT];
    unsigned keys[kSortCap];
    float4 col[kChunk];
    float2 spos[kSampleCap];
    unsigned short sp[kSampleCap];
    int cnt[kT * kT];
    int start[kT * kT];
    unsigned short ent[kEntryCap];
    int scan_w[kTB / 32];
};

// One block per tile; see the file comment.
__global__ void __launch_bounds__(kTB) k_rd_tiles(SplatCfg C, const float *prev, const float *pos, const float *col,
                                                  const unsigned *tile_start, unsigned *list, float *buf,
                                                  const unsigned *tiles, const unsigned *ntiles_p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TileSmem &S = *reinterpret_cast<TileSmem *>(smem_raw);
    if (blockIdx.x >= *ntiles_p) return;
    const int tile = (int)tiles[blockIdx.x];
    const int R = C.R, ntx = C.ntx;
    const int f = tile / (ntx * ntx), rem = tile - f * ntx * ntx, ty = rem / ntx, tx = rem - ty * ntx;
    const int x0 = tx * kT, y0 = ty * kT;
    const int tw = min(kT, R - x0), th = min(kT, R - y0);
    const unsigned lstart = tile_start[tile];
    const int cnt = (int)(tile_start[tile + 1] - lstart);
    if (cnt == 0 && !C.renorm) return;
    float4 *face = reinterpret_cast<float4 *>(buf) + (size_t)f * R * R;

    for (int t = threadIdx.x; t < kT * kT; t += kTB) {
        int lx = t % kT, ly = t / kT;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (lx < tw && ly < th) {
            v = face[(size_t)(y0 + ly) * R + x0 + lx];
            if (C.renorm) {
                v.x *= C.scale;
                v.y *= C.scale;
                v.z *= C.scale;
                v.w *= C.scale;
            }
        }
        S.tex[t] = v;
    }

    // particle list of this tile, ascending
    const unsigned *keys;
    if (cnt <= kSortCap) {
        for (int t = threadIdx.x; t < cnt; t += kTB) S.keys[t] = list[lstart + t];
        __syncthreads();
        block_sort(S.keys, cnt);
        keys = S.keys;
    } else {
        block_sort(list + lstart, cnt);
        keys = list + lstart;
    }
    __syncthreads();

    const float rad = C.rad, invrad = C.invrad, invg = C.invg;
    // texels with positive tent weight per axis: < 2 rad + 1 (rounding of invrad included)
    const int fpmax = (2 * (int)ceilf(rad) + 1) * (2 * (int)ceilf(rad) + 1);
    const int win = max(1, min(kSampleCap, kEntryCap / max(1, fpmax)));

    for (int c0 = 0; c0 < cnt; c0 += kChunk) {
        const int t = threadIdx.x;
        const bool valid = c0 + t < cnt;
        D3 a = d3(0, 0, 0), b = d3(0, 0, 0);
        int ns = 0, mine = 0;
        if (valid) {
            unsigned pidx = keys[c0 + t];
            a = load3(prev + 3 * (size_t)pidx);
            b = load3(pos + 3 * (size_t)pidx);
            S.col[t] = reinterpret_cast<const float4 *>(col)[pidx];
            ns = arc_samples(a, b, C.spacing);
            for (int k = 1; k <= ns; k++) {
                float px, py;
                if (!face_px(f, arc_point(a, b, k, ns), R, px, py)) continue;
                Box bx = footprint(px, py, rad, R);
                if (bx.xlo > bx.xhi || bx.ylo > bx.yhi) continue;
                if (bx.xhi < x0 || bx.xlo >= x0 + tw || bx.yhi < y0 || bx.ylo >= y0 + th) continue;
                mine++;
            }
        }
        int first;
        const int M = block_excl_scan(mine, first, S.scan_w);
        for (int w0 = 0; w0 < M; w0 += win) {
            const int w1 = min(M, w0 + win);
            // samples of this window, in (particle, k) order
            if (valid && mine > 0 && first < w1 && first + mine > w0) {
                int s = first;
                for (int k = 1; k <= ns && s < w1; k++) {
                    float px, py;
                    if (!face_px(f, arc_point(a, b, k, ns), R, px, py)) continue;
                    Box bx = footprint(px, py, rad, R);
                    if (bx.xlo > bx.xhi || bx.ylo > bx.yhi) continue;
                    if (bx.xhi < x0 || bx.xlo >= x0 + tw || bx.yhi < y0 || bx.ylo >= y0 + th) continue;
                    if (s >= w0) {
                        S.spos[s - w0] = make_float2(px, py);
                        S.sp[s - w0] = (unsigned short)t;
                    }
                    s++;
                }
            }
            for (int q = threadIdx.x; q < kT * kT; q += kTB) S.cnt[q] = 0;
            __syncthreads();
            const int ws = w1 - w0;
            // count texel entries
            for (int s = threadIdx.x; s < ws; s += kTB) {
                float2 pp = S.spos[s];
                Box bx = footprint(pp.x, pp.y, rad, R);
                int xa = max(bx.xlo, x0), xb = min(bx.xhi, x0 + tw - 1);
                int ya = max(bx.ylo, y0), yb = min(bx.yhi, y0 + th - 1);
                for (int y = ya; y <= yb; y++) {
                    float wy = __fmaf_rn(-fabsf((float)y - pp.y), invrad, 1.0f);
                    if (wy <= 0) continue;
                    for (int x = xa; x <= xb; x++) {
                        float wx = __fmaf_rn(-fabsf((float)x - pp.x), invrad, 1.0f);
                        if (wx <= 0) continue;
                        atomicAdd(&S.cnt[(y - y0) * kT + (x - x0)], 1);
                    }
                }
            }
            __syncthreads();
            // texel offsets (each thread scans 4 consecutive texels)
            {
                int base = threadIdx.x * 4;
                int c4[4], sum = 0;
                for (int u = 0; u < 4; u++) {
                    c4[u] = S.cnt[base + u];
                    sum += c4[u];
                }
                int ex;
                block_excl_scan(sum, ex, S.scan_w);
                for (int u = 0; u < 4; u++) {
                    S.start[base + u] = ex;
                    ex += c4[u];
                    S.cnt[base + u] = 0;
                }
            }
            __syncthreads();
            // fill entries (order within a texel fixed below)
            for (int s = threadIdx.x; s < ws; s += kTB) {
                float2 pp = S.spos[s];
                Box bx = footprint(pp.x, pp.y, rad, R);
                int xa = max(bx.xlo, x0), xb = min(bx.xhi, x0 + tw - 1);
                int ya = max(bx.ylo, y0), yb = min(bx.yhi, y0 + th - 1);
                for (int y = ya; y <= yb; y++) {
                    float wy = __fmaf_rn(-fabsf((float)y - pp.y), invrad, 1.0f);
                    if (wy <= 0) continue;
                    for (int x = xa; x <= xb; x++) {
                        float wx = __fmaf_rn(-fabsf((float)x - pp.x), invrad, 1.0f);
                        if (wx <= 0) continue;
                        int q = (y - y0) * kT + (x - x0);
                        int slot = atomicAdd(&S.cnt[q], 1);
                        S.ent[S.start[q] + slot] = (unsigned short)s;
                    }
                }
            }
            __syncthreads();
            // per texel: order its samples, then blend (upstream src/render.c:135-151)
            for (int q = threadIdx.x; q < kT * kT; q += kTB) {
                int e0 = S.start[q], m = S.cnt[q];
                if (!m) continue;
                unsigned short *e = S.ent + e0;
                for (int u = 1; u < m; u++) {
                    unsigned short key = e[u];
                    int v = u - 1;
                    while (v >= 0 && e[v] > key) {
                        e[v + 1] = e[v];
                        v--;
                    }
                    e[v + 1] = key;
                }
                const float xf = (float)(x0 + q % kT), yf = (float)(y0 + q / kT);
                float4 d = S.tex[q];
                for (int u = 0; u < m; u++) {
                    int s = e[u];
                    float2 pp = S.spos[s];
                    float4 c = S.col[S.sp[s]];
                    float w0 = C.alpha * c.w;
                    float wy = __fmaf_rn(-fabsf(yf - pp.y), invrad, 1.0f);
                    float wx = __fmaf_rn(-fabsf(xf - pp.x), invrad, 1.0f);
                    float w = __fmul_rn(__fmul_rn(w0, wx), wy);
                    float keep = 1.0f - w, add = __fmul_rn(w, invg);
                    d.x = __fmaf_rn(d.x, keep, __fmul_rn(add, c.x));
                    d.y = __fmaf_rn(d.y, keep, __fmul_rn(add, c.y));
                    d.z = __fmaf_rn(d.z, keep, __fmul_rn(add, c.z));
                    d.w = __fmaf_rn(d.w, keep, add);
                }
                S.tex[q] = d;
            }
            __syncthreads();
        }
    }

    for (int t = threadIdx.x; t < kT * kT; t += kTB) {
        int lx = t % kT, ly = t / kT;
        if (lx < tw && ly < th) face[(size_t)(y0 + ly) * R + x0 + lx] = S.tex[t];
    }
}

// ---- fast per-tile path ------------------------------------------------
// One pass over the tile's particles expands each arc's samples on this tile
// (FP64, as upstream) and drops every (sample, texel) pair with positive tent
// weight straight into that texel's fixed-size entry slots.  Each entry
// carries the sample's global order key (particle index, k), and each texel
// sorts its few entries by that key before blending, so neither the tile's
// particle list nor the samples need any order.  A tile whose particles,
// samples or per-texel entries exceed the fixed buffers is left untouched and
// queued for k_rd_tiles (the sorted, windowed path).
constexpr int kFastParticles = 512;
constexpr int kFastSamples = 1536;
constexpr int kTexelSlots = 12;

struct FastSmem {
    float4 col[kFastParticles];
    float2 spos[kFastSamples];
    unsigned long long skey[kFastSamples];
    unsigned short sslot[kFastSamples];
    unsigned short ent[kT * kT * kTexelSlots];
    int tcnt[kT * kT];
    int nsamp, overflow;
};

__global__ void __launch_bounds__(kTB) k_rd_tiles_fast(SplatCfg C, const float *prev, const float *pos,
                                                       const float *col, const unsigned *tile_start,
                                                       const unsigned *list, float *buf, unsigned *slow_tiles,
                                                       unsigned *slow_count) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    FastSmem &S = *reinterpret_cast<FastSmem *>(smem_raw);
    const int tile = blockIdx.x;
    const int R = C.R, ntx = C.ntx;
    const int f = tile / (ntx * ntx), rem = tile - f * ntx * ntx, ty = rem / ntx, tx = rem - ty * ntx;
    const int x0 = tx * kT, y0 = ty * kT;
    const int tw = min(kT, R - x0), th = min(kT, R - y0);
    const unsigned lstart = tile_start[tile];
    const int cnt = (int)(tile_start[tile + 1] - lstart);
    if (cnt == 0 && !C.renorm) return;
    if (cnt > kFastParticles) {
        if (threadIdx.x == 0) slow_tiles[atomicAdd(slow_count, 1u)] = (unsigned)tile;
        return;
    }
    if (threadIdx.x == 0) {
        S.nsamp = 0;
        S.overflow = 0;
    }
    for (int q = threadIdx.x; q < kT * kT; q += kTB) S.tcnt[q] = 0;
    __syncthreads();
    const float rad = C.rad, invrad = C.invrad, invg = C.invg;
    for (int u = threadIdx.x; u < cnt; u += kTB) {
        unsigned pidx = list[lstart + u];
        D3 a = load3(prev + 3 * (size_t)pidx), b = load3(pos + 3 * (size_t)pidx);
        S.col[u] = reinterpret_cast<const float4 *>(col)[pidx];
        int ns = arc_samples(a, b, C.spacing);
        for (int k = 1; k <= ns; k++) {
            float px, py;
            if (!face_px(f, arc_point(a, b, k, ns), R, px, py)) continue;
            Box bx = footprint(px, py, rad, R);
            int xa = max(bx.xlo, x0), xb = min(bx.xhi, x0 + tw - 1);
            int ya = max(bx.ylo, y0), yb = min(bx.yhi, y0 + th - 1);
            if (xa > xb || ya > yb) continue;
            int sidx = atomicAdd(&S.nsamp, 1);
            if (sidx >= kFastSamples) {
                S.overflow = 1;
                break;
            }
            S.spos[sidx] = make_float2(px, py);
            S.skey[sidx] = ((unsigned long long)pidx << 13) | (unsigned)k;
            S.sslot[sidx] = (unsigned short)u;
            for (int y = ya; y <= yb; y++) {
                float wy = __fmaf_rn(-fabsf((float)y - py), invrad, 1.0f);
                if (wy <= 0) continue;
                for (int x = xa; x <= xb; x++) {
                    float wx = __fmaf_rn(-fabsf((float)x - px), invrad, 1.0f);
                    if (wx <= 0) continue;
                    int q = (y - y0) * kT + (x - x0);
                    int slot = atomicAdd(&S.tcnt[q], 1);
                    if (slot < kTexelSlots)
                        S.ent[q * kTexelSlots + slot] = (unsigned short)sidx;
                    else
                        S.overflow = 1;
                }
            }
        }
    }
    __syncthreads();
    if (S.overflow) {
        if (threadIdx.x == 0) slow_tiles[atomicAdd(slow_count, 1u)] = (unsigned)tile;
        return;  // tile untouched; the sorted path redoes it
    }
    // per texel: order by (particle, k), then blend (upstream src/render.c:135-151)
    float4 *face = reinterpret_cast<float4 *>(buf) + (size_t)f * R * R;
    for (int q = threadIdx.x; q < kT * kT; q += kTB) {
        const int lx = q % kT, ly = q / kT;
        const int m = S.tcnt[q];
        if (lx >= tw || ly >= th || (m == 0 && !C.renorm)) continue;
        float4 *dp = face + (size_t)(y0 + ly) * R + x0 + lx;
        float4 d = *dp;
        if (C.renorm) {
            d.x *= C.scale;
            d.y *= C.scale;
            d.z *= C.scale;
            d.w *= C.scale;
        }
        unsigned short *e = S.ent + q * kTexelSlots;
        for (int u = 1; u < m; u++) {
            unsigned short key = e[u];
            unsigned long long kk = S.skey[key];
            int v = u - 1;
            while (v >= 0 && S.skey[e[v]] > kk) {
                e[v + 1] = e[v];
                v--;
            }
            e[v + 1] = key;
        }
        const float xf = (float)(x0 + lx), yf = (float)(y0 + ly);
        for (int u = 0; u < m; u++) {
            int sdx = e[u];
            float2 pp = S.spos[sdx];
            float4 c = S.col[S.sslot[sdx]];
            float w0 = C.alpha * c.w;
            float wy = __fmaf_rn(-fabsf(yf - pp.y), invrad, 1.0f);
            float wx = __fmaf_rn(-fabsf(xf - pp.x), invrad, 1.0f);
            float w = __fmul_rn(__fmul_rn(w0, wx), wy);
            float keep = 1.0f - w, add = __fmul_rn(w, invg);
            d.x = __fmaf_rn(d.x, keep, __fmul_rn(add, c.x));
            d.y = __fmaf_rn(d.y, keep, __fmul_rn(add, c.y));
            d.z = __fmaf_rn(d.z, keep, __fmul_rn(add, c.z));
            d.w = __fmaf_rn(d.w, keep, add);
        }
        *dp = d;
    }
}

// Buffer renormalisation on its own (a second renormalisation falling due
// before the next deposit).
__global__ void k_scale(size_t n, float s, float *buf) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        buf[i] *= s;
}

static SplatCfg splat_cfg(const Render *r, const RenderPriv *Pv) {
    SplatCfg C;
    C.R = r->R;
    C.ntx = Pv->ntx;
    C.rad = r->radius;
    C.invrad = 1.0f / r->radius;
    C.invg = (float)(1.0 / r->g);
    C.alpha = r->alpha;
    C.spacing = 0.7 / r->R;
    C.renorm = Pv->pending ? 1 : 0;
    C.scale = Pv->pending_scale;
    return C;
}

static void flush_pending(Render *r, RenderPriv *Pv) {
    if (!Pv->pending) return;
    size_t n = (size_t)6 * r->R * r->R * 4;
    k_scale<<<148 * 8, 256, 0, stream()>>>(n, Pv->pending_scale, r->buf);
    GGB_LAUNCHED();
    Pv->pending = false;
    Pv->pending_scale = 1.f;
    Pv->dev_gen++;
}

void render_deposit_launch(Render *r, const Particles *P, bool sync_total) {
    RenderPriv *Pv = rpriv(r);
    cudaStream_t s = stream();
    SplatCfg C = splat_cfg(r, Pv);
    int n = P->n;
    stage_begin(ST_BIN);
    GGB_CHECK(cudaMemsetAsync(Pv->tile_count, 0, sizeof(unsigned) * Pv->ntiles, s));
    GGB_CHECK(cudaMemsetAsync(Pv->tile_fill, 0, sizeof(unsigned) * Pv->ntiles, s));
    unsigned nb = (unsigned)std::max(1, std::min(n / 256 + 1, 148 * 16));
    if (n > 0) {
        k_rd_count<<<nb, 256, 0, s>>>(n, C, P->prev, P->pos, Pv->tile_count);
        GGB_LAUNCHED();
    }
    k_tile_scan<<<1, 1024, 0, s>>>(Pv->ntiles, Pv->tile_count, Pv->tile_start, Pv->tile_count + Pv->ntiles);
    GGB_LAUNCHED();
    (void)sync_total;
    GGB_CHECK(cudaMemcpyAsync(Pv->total_host, Pv->tile_count + Pv->ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    stage_end(ST_BIN);
    GGB_CHECK(cudaStreamSynchronize(s));
    size_t need = *Pv->total_host;
    if (need > Pv->list_cap) {
        dev_free(Pv->list);
        Pv->list_cap = need + need / 4 + 1024;
        Pv->list = (unsigned *)dev_alloc(sizeof(unsigned) * Pv->list_cap);
    }
    stage_begin(ST_TILES);
    if (n > 0) {
        k_rd_fill<<<nb, 256, 0, s>>>(n, C, P->prev, P->pos, Pv->tile_start, Pv->tile_fill, Pv->list);
        GGB_LAUNCHED();
    }
    GGB_CHECK(cudaMemsetAsync(Pv->slow_count, 0, sizeof(unsigned), s));
    k_rd_tiles_fast<<<Pv->ntiles, kTB, sizeof(FastSmem), s>>>(C, P->prev, P->pos, P->col, Pv->tile_start, Pv->list,
                                                               r->buf, Pv->slow_tiles, Pv->slow_count);
    GGB_LAUNCHED();
    k_rd_tiles<<<Pv->ntiles, kTB, sizeof(TileSmem), s>>>(C, P->prev, P->pos, P->col, Pv->tile_start, Pv->list,
                                                           r->buf, Pv->slow_tiles, Pv->slow_count);
    GGB_LAUNCHED();
    stage_end(ST_TILES);
    Pv->pending = false;
    Pv->pending_scale = 1.f;
    Pv->dev_gen++;
}

static void refresh_mirror(const Render *r, RenderPriv *Pv) {
    if (Pv->mirror_gen.load() == Pv->dev_gen.load()) return;
    std::lock_guard<std::mutex> lk(Pv->mu);
    unsigned long g = Pv->dev_gen.load();
    if (Pv->mirror_gen.load() == g) return;
    size_t bytes = sizeof(float) * 6 * (size_t)r->R * r->R * 4;
    if (!Pv->mirror) GGB_CHECK(cudaMallocHost(&Pv->mirror, bytes));
    GGB_CHECK(cudaMemcpyAsync(Pv->mirror, r->buf, bytes, cudaMemcpyDeviceToHost, stream()));
    GGB_CHECK(cudaStreamSynchronize(stream()));
    Pv->mirror_gen.store(g);
}

}  // namespace ggb

using namespace ggb;

GGB_EXPORT int render_init(Render *r, int R, float radius, float alpha) {
    memset(r, 0, sizeof(*r));
    if (R < 1) {
        fprintf(stderr, "render: bad resolution %d\n", R);
        return -1;
    }
    if (!have_device()) {
        fprintf(stderr, "render: no CUDA device is available (libggb_cuda has no CPU path)\n");
        return -1;
    }
    r->R = R;
    r->radius = radius < 0.75f ? 0.75f : radius;
    r->alpha = alpha;
    r->g = 1.0;
    r->buf = (float *)managed_alloc(sizeof(float) * 6 * (size_t)R * R * 4);
    int sh = 32;
    if (sh < (int)ceilf(r->radius) + 1) sh = (int)ceilf(r->radius) + 1;
    if (sh > R) sh = R;
    r->strip_h = sh;
    r->nstrips = (R + sh - 1) / sh;
    r->nbins = 6 * r->nstrips;
    RenderPriv *Pv = new RenderPriv();
    Pv->R = R;
    Pv->ntx = (R + kT - 1) / kT;
    Pv->ntiles = 6 * Pv->ntx * Pv->ntx;
    Pv->tile_count = (unsigned *)dev_alloc(sizeof(unsigned) * (Pv->ntiles + 1));
    Pv->tile_start = (unsigned *)dev_alloc(sizeof(unsigned) * (Pv->ntiles + 1));
    Pv->tile_fill = (unsigned *)dev_alloc(sizeof(unsigned) * Pv->ntiles);
    Pv->slow_tiles = (unsigned *)dev_alloc(sizeof(unsigned) * Pv->ntiles);
    Pv->slow_count = (unsigned *)dev_alloc(sizeof(unsigned));
    GGB_CHECK(cudaMallocHost(&Pv->total_host, sizeof(unsigned)));
    GGB_CHECK(cudaFuncSetAttribute(k_rd_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TileSmem)));
    GGB_CHECK(cudaFuncSetAttribute(k_rd_tiles_fast, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FastSmem)));
    r->tr = reinterpret_cast<ThreadRecs *>(Pv);
    sync();
    return 0;
}

GGB_EXPORT void render_free(Render *r) {
    if (r->tr) {
        RenderPriv *Pv = rpriv(r);
        sync();
        dev_free(Pv->tile_count);
        dev_free(Pv->tile_start);
        dev_free(Pv->tile_fill);
        dev_free(Pv->slow_tiles);
        dev_free(Pv->slow_count);
        dev_free(Pv->list);
        cudaFreeHost(Pv->total_host);
        if (Pv->mirror) cudaFreeHost(Pv->mirror);
        delete Pv;
    }
    managed_free(r->buf);
    memset(r, 0, sizeof(*r));
}

// upstream src/render.c:55-66; the buffer scale is deferred into the next deposit
GGB_EXPORT void render_fade(Render *r, double fade) {
    RenderPriv *Pv = rpriv(r);
    r->g *= (1.0 - fade);
    if (r->g < 1e-4) {
        if (Pv->pending) flush_pending(r, Pv);
        Pv->pending = true;
        Pv->pending_scale = (float)r->g;
        r->g = 1.0;
        Pv->dev_gen++;
    }
}

GGB_EXPORT void render_deposit(Render *r, const Particles *P) {
    render_deposit_launch(r, P, true);
    sync();
}

GGB_EXPORT void render_texel(const Render *r, int face, int x, int y, float out[4]) {
    RenderPriv *Pv = rpriv(r);
    refresh_mirror(r, Pv);
    const float *d = Pv->mirror + (((size_t)face * r->R + y) * r->R + x) * 4;
    float g = (float)r->g;
    if (Pv->pending) {
        for (int c = 0; c < 4; c++) out[c] = (d[c] * Pv->pending_scale) * g;
    } else {
        for (int c = 0; c < 4; c++) out[c] = d[c] * g;
    }
}

// upstream src/render.c:228-251
GGB_EXPORT void render_sample_dir(const Render *r, double dx, double dy, double dz, float out[4]) {
    vec3 d = v3(dx, dy, dz);
    int f = cs_face_of(d), R = r->R;
    double dc = v3_dot(d, cs_face_center[f]);
    double u = v3_dot(d, cs_face_right[f]) / dc;
    double v = v3_dot(d, cs_face_up[f]) / dc;
    double px = (u + 1.0) * 0.5 * R - 0.5, py = (1.0 - v) * 0.5 * R - 0.5;
    px = px < 0 ? 0 : (px > R - 1 ? R - 1 : px);
    py = py < 0 ? 0 : (py > R - 1 ? R - 1 : py);
    int x0 = (int)px, y0 = (int)py;
    int x1 = x0 + 1 < R ? x0 + 1 : x0, y1 = y0 + 1 < R ? y0 + 1 : y0;
    float fx = (float)(px - x0), fy = (float)(py - y0);
    float a[4], b[4], c[4], e[4];
    render_texel(r, f, x0, y0, a);
    render_texel(r, f, x1, y0, b);
    render_texel(r, f, x0, y1, c);
    render_texel(r, f, x1, y1, e);
    for (int k = 0; k < 4; k++) out[k] = (1 - fy) * ((1 - fx) * a[k] + fx * b[k]) + fy * ((1 - fx) * c[k] + fx * e[k]);
}

static unsigned char to8(float v) {
    if (v <= 0) return 0;
    if (v >= 1) return 255;
    return (unsigned char)(v * 255.0f + 0.5f);
}

// upstream src/render.c:253-279
GGB_EXPORT void render_pixel8(const float c[4], const float *bg, unsigned char *out) {
    float a = c[3];
    a = a > 1 ? 1 : (a < 0 ? 0 : a);
    if (!bg) {
        if (a > 1e-6f) {
            out[0] = to8(c[0] / a);
            out[1] = to8(c[1] / a);
            out[2] = to8(c[2] / a);
        } else {
            out[0] = out[1] = out[2] = 0;
        }
        out[3] = to8(a);
    } else {
        for (int k = 0; k < 3; k++) out[k] = to8(c[k] + bg[k] * (1 - a));
    }
}

// Additive: all texels (premultiplied RGBA times g) into out[6*R*R*4] (host or
// device memory) with one copy.
GGB_EXPORT void ggb_render_read(const Render *r, float *out) {
    RenderPriv *Pv = rpriv(r);
    refresh_mirror(r, Pv);
    size_t n = (size_t)6 * r->R * r->R * 4;
    float g = (float)r->g;
    float sc = Pv->pending ? Pv->pending_scale : 1.f;
    for (size_t i = 0; i < n; i++) out[i] = Pv->pending ? (Pv->mirror[i] * sc) * g : Pv->mirror[i] * g;
}

// Diagnostics: tiles of the last deposit (all tiles, and those that took the
// sorted fallback path) and the number of (particle, tile) list entries.
GGB_EXPORT void ggb_render_stats(const Render *r, unsigned *ntiles, unsigned *slow_tiles, unsigned *entries) {
    RenderPriv *Pv = rpriv(r);
    sync();
    unsigned sc = 0;
    GGB_CHECK(cudaMemcpy(&sc, Pv->slow_count, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (ntiles) *ntiles = (unsigned)Pv->ntiles;
    if (slow_tiles) *slow_tiles = sc;
    if (entries) *entries = *Pv->total_host;
}
