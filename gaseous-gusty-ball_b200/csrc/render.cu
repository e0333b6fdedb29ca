// render.cu — the render.h entry points of libggb_cuda.so: tent-filtered,
// "over"-blended, globally fading particle-trail splatting into the six
// cube-face images.
//
// Upstream: src/render.c.  Per texel the composite must apply the splat
// samples in ascending (particle index, sample k) order (upstream records are
// binned thread-major over contiguous particle ranges, src/render.c:156-218).
// This library reaches the same per-texel order without a global sort:
//   1. count:  every particle reserves, on each 16x16 texel tile its arc may
//              touch (FP32 conservative bound), one record slot per sample
//              (FP32 upper bound on the sample count) — atomics; from the
//              second deposit on, each tile reserves instead from the largest
//              count of the previous deposit around it (no counting pass);
//   2. scan:   tile offsets (one block);
//   3. fill:   every particle expands its samples exactly (FP64, as upstream)
//              once and writes one record (order key, px, py) per (sample,
//              tile) its footprint touches into that tile's slots;
//   4. tiles:  one block per tile bins its records per texel, sorts each
//              texel's few entries by order key and applies the blends in
//              that order to the tile held in shared memory.  A tile whose
//              records do not fit one shared-memory window is composited in
//              consecutive key-range windows (found by a key histogram), each
//              window complete before the next, which keeps the order.
// The pending renormalisation of render_fade is fused into step 4.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "ggb_internal.h"

namespace ggb {

constexpr int kT = 16;              // tile edge in texels
constexpr unsigned kTileSpare = 64;  // spare record slots of a tile whose reservation is estimated
constexpr int kMaxSamples = 4096;   // upstream cap on samples per arc

// One splat sample on one tile: its compositing order key (particle index
// << 13 | sample k) and its texel-space centre on the tile's face (16 bytes).
// The particle's colour is not copied: compositing reads it from the
// particles' colour array by the index in the key (an L2-resident gather),
// which halves the record bytes that the fill writes and compositing reads.
struct __align__(16) Rec {
    unsigned long long key;
    float px, py;
};
static_assert(sizeof(Rec) == 16, "a record is 16 bytes");

struct SplatCfg {
    int R, ntx, ntiles;
    float rad, invrad, invg, alpha;
    double spacing;
    double edge_lim;  // 1 + (2 rad + 2) / R: beyond |u| or |v| of that a face's footprint is empty
    int renorm;
    float scale;
};

struct RenderPriv {
    int R = 0, ntx = 0, ntiles = 0;
    unsigned *tile_count = nullptr, *tile_start = nullptr, *tile_fill = nullptr;
    unsigned *tile_est = nullptr;  // next deposit's estimate: neighbourhood maxima of the record counts
    Rec *recs = nullptr;
    size_t rec_cap = 0;
    unsigned *diag = nullptr;        // device: [0] windowed tiles of the last deposit, [1] tiles whose slots overflowed
    unsigned *total_host = nullptr;  // pinned: [0] reserved record slots, [1] slot overflow
    bool pending = false;
    float pending_scale = 1.f;
    SplatCfg queued{};             // configuration of the last queued deposit (for its repeat)
    bool queued_est = false;       // its slots were estimated from the previous deposit's fills
    bool have_prev = false;        // tile_fill holds the previous deposit's record counts
    unsigned long repeats = 0;     // times a deposit's fill and compositing ran again
    unsigned long grown = 0;       // of those, after the record buffer grew
    int exact_next = 0;            // deposits still to reserve exactly after an estimate overflowed
    int backoff = 1;               // exact deposits after the next overflow (doubles up to 64)
    float *mirror = nullptr;
    unsigned char *enc = nullptr;  // device scratch of the 8-bit encoders (host outputs)
    size_t enc_cap = 0;
    std::atomic<unsigned long> dev_gen{1}, mirror_gen{0};
    std::mutex mu;
};

static RenderPriv *rpriv(const Render *r) {
    if (!r->tr) fail_msg("Render %p was not initialised by this library's render_init", (const void *)r);
    return reinterpret_cast<RenderPriv *>(r->tr);
}


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

// arc_samples for FP32 endpoints, the same value with less work: the FP32
// quotient q = angle / spacing differs from the FP64 one by less than
// err = 2e-6 (1 / spacing + q) + 1e-4 (the FP32 cross and dot products of
// unit vectors are off by ~2e-7 absolute, atan2f by 2 ulp, the division by
// half an ulp; err is twice their sum).  When q is farther than err from every
// integer, ceil(q) is the FP64 ceiling; otherwise the FP64 path decides.
__device__ __forceinline__ int arc_samples_f(float ax, float ay, float az, float bx, float by, float bz,
                                             double spacing) {
    const float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    const float q = atan2f(sqrtf(cx * cx + cy * cy + cz * cz), ax * bx + ay * by + az * bz) / (float)spacing;
    if (q < (float)(kMaxSamples - 1)) {
        const float err = 2e-6f * (1.0f / (float)spacing + q) + 1e-4f;
        const float fl = floorf(q);
        if (q - fl > err && fl + 1.0f - q > err) return (int)fl + 1;
    }
    return arc_samples(d3(ax, ay, az), d3(bx, by, bz), spacing);
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

// Upper bound on arc_samples from FP32 arithmetic on the same inputs: the
// FP32 angle differs from the FP64 one by orders of magnitude less than one
// sample spacing, so ceil(angle / spacing) + 1 is never below the exact count.
__device__ __forceinline__ unsigned arc_samples_bound(D3 a, D3 b, double spacing) {
    const float ax = (float)a.x, ay = (float)a.y, az = (float)a.z, bx = (float)b.x, by = (float)b.y, bz = (float)b.z;
    const float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    const float ang = atan2f(sqrtf(cx * cx + cy * cy + cz * cz), ax * bx + ay * by + az * bz);
    const float q = ang / (float)spacing;
    if (!(q < (float)kMaxSamples)) return kMaxSamples;  // also NaN
    return (unsigned)min(max((int)ceilf(q) + 1, 1), kMaxSamples);
}

__global__ void __launch_bounds__(256, 4) k_rd_count(int n, SplatCfg C, const float *prev, const float *pos,
                                                     unsigned *tile_count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D3 a = load3(prev + 3 * (size_t)i), b = load3(pos + 3 * (size_t)i);
        const unsigned nsb = arc_samples_bound(a, b, C.spacing);
        arc_tiles_bound(C, a, b, [&](int t) { atomicAdd(tile_count + t, nsb); });
    }
}

// The face of the largest |component| of d (its d.c >= 1/sqrt(3) > 0.5, so
// upstream src/render.c:92-98 always draws the sample there) as dc, dr, du
// exactly as face_proj(f) gives them.
__device__ __forceinline__ int primary_face(D3 d, double &dc, double &dr, double &du) {
    const double ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
    if (az >= ax && az >= ay) {
        if (d.z >= 0) { dc = d.z; dr = d.x; du = d.y; return 0; }
        dc = -d.z; dr = -d.x; du = d.y; return 2;
    }
    if (ax >= ay) {
        if (d.x >= 0) { dc = d.x; dr = -d.z; du = d.y; return 1; }
        dc = -d.x; dr = d.z; du = d.y; return 3;
    }
    if (d.y >= 0) { dc = d.y; dr = d.x; du = -d.z; return 4; }
    dc = -d.y; dr = d.x; du = d.z; return 5;
}

// Appends record r to tile tl.  Lanes of the warp that append to the same
// tile share one atomic (the lowest such lane adds the group's count).
__device__ __forceinline__ void append_rec(int tl, bool active, const Rec &r, const unsigned *tile_start,
                                           unsigned *tile_fill, Rec *recs, unsigned *diag) {
    const unsigned act = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const unsigned grp = __match_any_sync(act, tl);
    const int lane = threadIdx.x & 31, leader = __ffs(grp) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(tile_fill + tl, (unsigned)__popc(grp));
    base = __shfl_sync(grp, base, leader);
    const unsigned slot = base + __popc(grp & ((1u << lane) - 1u));
    const unsigned s0 = __ldg(tile_start + tl);
    if (s0 + slot < __ldg(tile_start + tl + 1))
        recs[s0 + slot] = r;
    else
        atomicOr(diag + 1, 1u);
}

// Records of one (sample, face): one per tile its clamped footprint touches.
__device__ __forceinline__ void emit_face(const SplatCfg &C, int f, float px, float py, bool active,
                                          unsigned long long key, const unsigned *tile_start, unsigned *tile_fill,
                                          Rec *recs, unsigned *diag) {
    Box bx = footprint(px, py, C.rad, C.R);
    if (bx.xlo > bx.xhi || bx.ylo > bx.yhi) active = false;
    const int tx0 = bx.xlo / kT, ty0 = bx.ylo / kT;
    const int ntxs = active ? bx.xhi / kT - tx0 + 1 : 0, ntys = active ? bx.yhi / kT - ty0 + 1 : 0;
    int most = ntxs * ntys;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) most = max(most, __shfl_xor_sync(0xffffffffu, most, o));
    Rec r;
    r.key = key;
    r.px = px;
    r.py = py;
    for (int u = 0; u < most; u++) {
        const bool on = u < ntxs * ntys;
        // tile u of the footprint's ntxs x ntys tiles, row-major (a footprint
        // of radius <= 1 spans at most two tiles per axis: shifts, no division)
        int dy = 0, dx = 0;
        if (on) {
            if (ntxs == 1) {
                dy = u;
            } else if (ntxs == 2) {
                dy = u >> 1;
                dx = u & 1;
            } else {
                dy = u / ntxs;
                dx = u - dy * ntxs;
            }
        }
        const int tl = on ? (f * C.ntx + ty0 + dy) * C.ntx + tx0 + dx : 0;
        append_rec(tl, on, r, tile_start, tile_fill, recs, diag);
    }
}

// Samples of every arc (FP64, upstream src/render.c:87-131), one record per
// (sample, face, tile) whose clamped footprint touches the tile.  A warp takes
// 32 particles, computes their sample counts (one lane each), then spreads all
// their samples evenly over its lanes (a warp prefix sum of the counts; each
// lane finds the particle of its sample by a shuffle search), so particles with
// many samples do not leave the other lanes idle.  Every sample is drawn on
// its primary face in lock-step; the other faces with d.c >= 0.5 (near cube
// edges only) follow.  Six blocks per SM (40 registers, some spilled) ran
// 4 % faster than five (48 registers) and eight (32).
__global__ void __launch_bounds__(256, 6)
    k_rd_fill(int n, SplatCfg C, const float *prev, const float *pos, const unsigned *tile_start, unsigned *tile_fill,
              Rec *recs, size_t cap, unsigned *diag) {
    if (tile_start[C.ntiles] > cap) return;  // the host grows the record buffer and runs this again
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * 32; base < n; base += nwarps * 32) {
        const int i = base + lane;
        float p0 = 0.f, p1 = 0.f, p2 = 0.f, q0 = 0.f, q1 = 0.f, q2 = 0.f;
        int ns = 0;
        if (i < n) {
            p0 = prev[3 * (size_t)i];
            p1 = prev[3 * (size_t)i + 1];
            p2 = prev[3 * (size_t)i + 2];
            q0 = pos[3 * (size_t)i];
            q1 = pos[3 * (size_t)i + 1];
            q2 = pos[3 * (size_t)i + 2];
            ns = arc_samples_f(p0, p1, p2, q0, q1, q2, C.spacing);
        }
        int incl = ns;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - ns;
        const int total = __shfl_sync(0xffffffffu, incl, 31);
        for (int t0 = 0; t0 < total; t0 += 32) {
            const int t = t0 + lane;
            int j = 0;  // the last lane whose samples start at or before t
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int ex = __shfl_sync(0xffffffffu, excl, j + step);
                if (t >= ex) j += step;
            }
            const int k = t - __shfl_sync(0xffffffffu, excl, j) + 1;
            const int nsj = __shfl_sync(0xffffffffu, ns, j);
            const D3 a = d3(__shfl_sync(0xffffffffu, p0, j), __shfl_sync(0xffffffffu, p1, j),
                            __shfl_sync(0xffffffffu, p2, j));
            const D3 b = d3(__shfl_sync(0xffffffffu, q0, j), __shfl_sync(0xffffffffu, q1, j),
                            __shfl_sync(0xffffffffu, q2, j));
            const bool live = t < total;
            const D3 d = arc_point(a, b, live ? k : 1, live ? nsj : 1);
            const unsigned long long key = ((unsigned long long)(base + j) << 13) | (unsigned)k;
            double dc, dr, du;
            const int f0 = primary_face(d, dc, dr, du);
            {
                const double u = dr / dc, v = du / dc;
                const float px = (float)__fma_rn((u + 1.0) * 0.5, (double)C.R, -0.5);
                const float py = (float)__fma_rn((1.0 - v) * 0.5, (double)C.R, -0.5);
                emit_face(C, f0, px, py, live, key, tile_start, tile_fill, recs, diag);
            }
            // other faces with d.c >= 0.5 (cube edges and corners) whose texels
            // the sample reaches: its footprint on face f is empty unless
            // -rad <= px <= R - 1 + rad, i.e. |u|, |v| <= 1 + (2 rad + 1) / R;
            // edge_lim adds 1 / R for rounding and the test multiplies by
            // d.c instead of dividing.  Faces it skips make no records.
            unsigned reach = 0;
#pragma unroll
            for (int f = 0; f < 6; f++) {
                double ec, er, eu;
                face_proj(f, d, ec, er, eu);
                const double lim = C.edge_lim * ec;
                if (f != f0 && ec >= 0.5 && fabs(er) <= lim && fabs(eu) <= lim) reach |= 1u << f;
            }
            if (__any_sync(0xffffffffu, live && reach)) {
                for (int f = 0; f < 6; f++) {
                    float px = 0.f, py = 0.f;
                    const bool on = live && (reach >> f & 1u) && face_px(f, d, C.R, px, py);
                    if (__any_sync(0xffffffffu, on))
                        emit_face(C, f, px, py, on, key, tile_start, tile_fill, recs, diag);
                }
            }
        }
    }
}

// Exclusive scan of cnt[0..n) into start[0..n] and *total (one block of 1024
// threads).  Each warp owns a contiguous segment of the counts (a multiple of
// 128 long; cnt and start are 16-byte aligned) and walks it 128 counts at a
// time, a 16-byte load per lane (coalesced): a first pass sums the segment,
// the block scans the 32 warp sums, a second pass writes the prefixes (a warp
// scan per step, the running total carried from step to step); the second
// pass also zeroes clear[0..n) (the estimate array, which the following
// compositing fills for the next deposit; clear may be cnt).
// est: the counts are the previous deposit's estimates (for each tile the
// largest record count among the tile and its neighbours on the same face,
// left by k_rd_tiles), and each tile reserves that plus half of it plus
// kTileSpare (a particle moves up to one grid cell per step, which on a
// coarse grid under large faces is a whole tile, so a dense stream's records
// can move into a tile that held few of them; a tile that still overflows
// makes the deposit repeat with exact reservations).
__device__ __forceinline__ unsigned tile_reserve(unsigned x, int est) { return est ? x + x / 2 + kTileSpare : x; }

// Counts i..i+3 (zero past n), transformed by tile_reserve.
__device__ __forceinline__ uint4 tile_load4(const unsigned *cnt, int i, int n, int est) {
    uint4 v;
    if (i + 4 <= n) {
        v = reinterpret_cast<const uint4 *>(cnt)[i >> 2];
    } else {
        v.x = i < n ? cnt[i] : 0u;
        v.y = i + 1 < n ? cnt[i + 1] : 0u;
        v.z = i + 2 < n ? cnt[i + 2] : 0u;
        v.w = i + 3 < n ? cnt[i + 3] : 0u;
    }
    if (i < n) {
        v.x = tile_reserve(v.x, est);
        v.y = i + 1 < n ? tile_reserve(v.y, est) : 0u;
        v.z = i + 2 < n ? tile_reserve(v.z, est) : 0u;
        v.w = i + 3 < n ? tile_reserve(v.w, est) : 0u;
    }
    return v;
}

__global__ void __launch_bounds__(1024) k_tile_scan(int n, const unsigned *cnt, int est, unsigned *start,
                                                   unsigned *total, unsigned *clear) {
    __shared__ unsigned s_w[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = ((n + 31) / 32 + 127) & ~127;
    const int w0 = min(n, warp * seg), w1 = min(n, w0 + seg);
    unsigned sum = 0;
#pragma unroll 4
    for (int b = w0; b < w1; b += 128) {
        const uint4 v = tile_load4(cnt, b + 4 * lane, w1, est);
        sum += v.x + v.y + v.z + v.w;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) s_w[warp] = sum;
    __syncthreads();
    if (warp == 0) {
        const unsigned x = s_w[lane];
        unsigned incl = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        s_w[lane] = incl - x;  // exclusive: the counts before this warp's segment
        if (lane == 31) {
            start[n] = incl;
            *total = incl;
        }
    }
    __syncthreads();
    unsigned carry = s_w[warp];
    for (int b = w0; b < w1; b += 128) {
        const int i = b + 4 * lane;
        const uint4 v = tile_load4(cnt, i, w1, est);
        if (i + 4 <= w1) {  // clear may be cnt itself: these entries were read just above
            reinterpret_cast<uint4 *>(clear)[i >> 2] = make_uint4(0u, 0u, 0u, 0u);
        } else {
            for (int u = i; u < w1 && u < i + 4; u++) clear[u] = 0u;
        }
        const unsigned t = v.x + v.y + v.z + v.w;
        unsigned incl = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        uint4 o4;
        o4.x = carry + incl - t;
        o4.y = o4.x + v.x;
        o4.z = o4.y + v.y;
        o4.w = o4.z + v.z;
        if (i + 4 <= w1) {
            reinterpret_cast<uint4 *>(start)[i >> 2] = o4;
        } else {
            if (i < w1) start[i] = o4.x;
            if (i + 1 < w1) start[i + 1] = o4.y;
            if (i + 2 < w1) start[i + 2] = o4.z;
        }
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
}

// ---- tile compositing: one block per tile, one texel per thread ----------
constexpr int kTB = kT * kT;   // threads per tile block: one texel each
constexpr int kRec = 576;      // records of one window (shared memory)
constexpr int kEnt = 1728;     // (record, texel) entries of one window
constexpr int kHist = 1024;    // key buckets when a dense tile is cut into windows
constexpr int kBucket = 16;    // entry slots per texel of the one-pass path
constexpr int kBucketStride = 18;  // slots between texels: 9 words, so a warp's texels hit distinct banks

struct TileSmem {
    union {
        struct {
            unsigned long long key[kRec];
            float2 pos[kRec];
        } r;
        unsigned long long hist[kHist];  // window planning: entries << 32 | records per key bucket
    } u;
    float4 col[kRec];
    unsigned short box[kRec];
    union {
        unsigned short ent[kEnt];                 // entry lists packed by a count scan
        unsigned short bucket[kT * kT * kBucketStride];  // kBucket entry slots per texel (one-pass path)
    };
    int cnt[kT * kT];
    int start[kT * kT];
    unsigned long long scan_w[kTB / 32];
    int wsum[kTB / 32];
    int cut, tot, full;
};

struct TileGeo {
    int x0, y0, tw, th;
};

constexpr unsigned short kNoBox = 0xffff;  // no texel of the tile has positive weight

// The texels of the tile with positive tent weight for a sample at (px, py)
// (upstream src/render.c:135-151) form a box (the tent is positive on an
// interval per axis): x offset, y offset, width - 1, height - 1 in 4 bits each.
__device__ __forceinline__ unsigned short rec_box(const SplatCfg &C, const TileGeo &G, float px, float py) {
    const Box bx = footprint(px, py, C.rad, C.R);
    int xa = max(bx.xlo, G.x0), xb = min(bx.xhi, G.x0 + G.tw - 1);
    int ya = max(bx.ylo, G.y0), yb = min(bx.yhi, G.y0 + G.th - 1);
    while (xa <= xb && !(__fmaf_rn(-fabsf((float)xa - px), C.invrad, 1.0f) > 0)) xa++;
    while (xb >= xa && !(__fmaf_rn(-fabsf((float)xb - px), C.invrad, 1.0f) > 0)) xb--;
    while (ya <= yb && !(__fmaf_rn(-fabsf((float)ya - py), C.invrad, 1.0f) > 0)) ya++;
    while (yb >= ya && !(__fmaf_rn(-fabsf((float)yb - py), C.invrad, 1.0f) > 0)) yb--;
    if (xa > xb || ya > yb) return kNoBox;
    return (unsigned short)((xa - G.x0) | (ya - G.y0) << 4 | (xb - xa) << 8 | (yb - ya) << 12);
}
__device__ __forceinline__ int box_entries(unsigned short b) {
    return b == kNoBox ? 0 : ((b >> 8 & 15) + 1) * ((b >> 12) + 1);
}
// f(texel) for each texel of box b.  Boxes of at most 2 x 2 texels (every box
// when the splat radius is 1 or less: a positive weight needs |x - px| < r)
// take a straight-line path; the visiting order does not matter to callers.
template <class F>
__device__ __forceinline__ void box_texels(unsigned short b, F f) {
    if (b == kNoBox) return;
    const int x0 = b & 15, y0 = b >> 4 & 15, w = (b >> 8 & 15) + 1, h = (b >> 12) + 1;
    if (w <= 2 && h <= 2) {
        const int t = y0 * kT + x0;
        f(t);
        if (w == 2) f(t + 1);
        if (h == 2) {
            f(t + kT);
            if (w == 2) f(t + kT + 1);
        }
        return;
    }
    for (int y = y0; y < y0 + h; y++)
        for (int x = x0; x < x0 + w; x++) f(y * kT + x);
}

// Exclusive block scan of one value per thread (kTB threads); returns the total.
__device__ __forceinline__ unsigned long long block_excl_scan(unsigned long long v, unsigned long long &excl,
                                                              unsigned long long *s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = lane < kTB / 32 ? s_w[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kTB / 32) s_w[lane] = w;
    }
    __syncthreads();
    const unsigned long long before = warp ? s_w[warp - 1] : 0ull;
    const unsigned long long total = s_w[kTB / 32 - 1];
    excl = before + x - v;
    __syncthreads();
    return total;
}

// Record r with its box into slot s of the current window (its particle's
// colour: window_colours).
__device__ __forceinline__ void window_put(TileSmem &S, int s, const Rec &r, unsigned short box) {
    S.u.r.key[s] = r.key;
    S.u.r.pos[s] = make_float2(r.px, r.py);
    S.box[s] = box;
}

// The colours of the window's records 0..m-1, gathered by the particle index
// in each key after the records are binned, so that a thread's gathers are in
// flight together instead of one per record on the binning loop's path.
__device__ __forceinline__ void window_colours(TileSmem &S, int m, const float4 *col) {
    for (int s = threadIdx.x; s < m; s += blockDim.x) S.col[s] = __ldg(col + (S.u.r.key[s] >> 13));
}

// Blends the sorted entries e[0..m) of texel q into d (upstream
// src/render.c:135-151).
__device__ __forceinline__ void blend_texel(const TileSmem &S, unsigned short *e, int m, int q, const SplatCfg &C,
                                            const TileGeo &G, float4 &d) {
    for (int v0 = 1; v0 < m; v0++) {
        const unsigned short key = e[v0];
        const unsigned long long kk = S.u.r.key[key];
        int v = v0 - 1;
        while (v >= 0 && S.u.r.key[e[v]] > kk) {
            e[v + 1] = e[v];
            v--;
        }
        e[v + 1] = key;
    }
    const float invrad = C.invrad, invg = C.invg;
    const float xf = (float)(G.x0 + q % kT), yf = (float)(G.y0 + q / kT);
    for (int v = 0; v < m; v++) {
        const int s = e[v];
        const float2 pp = S.u.r.pos[s];
        const float4 c = S.col[s];
        const float w0 = C.alpha * c.w;
        const float wy = __fmaf_rn(-fabsf(yf - pp.y), invrad, 1.0f);
        const float wx = __fmaf_rn(-fabsf(xf - pp.x), invrad, 1.0f);
        const float w = __fmul_rn(__fmul_rn(w0, wx), wy);
        const float keep = 1.0f - w, add = __fmul_rn(w, invg);
        d.x = __fmaf_rn(d.x, keep, __fmul_rn(add, c.x));
        d.y = __fmaf_rn(d.y, keep, __fmul_rn(add, c.y));
        d.z = __fmaf_rn(d.z, keep, __fmul_rn(add, c.z));
        d.w = __fmaf_rn(d.w, keep, add);
    }
}

// Exclusive scan over the block of one count per thread with one barrier:
// a warp scan, the warp totals through shared memory, then each thread adds
// the totals of the warps before its own.
__device__ __forceinline__ int block_scan_1sync(int c, int *wsum) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; w++) before += wsum[w];
    return before + incl - c;
}

// Composites the window's records [0, nw) into this thread's texel d, per
// texel in ascending order key (every entry of the window fits: at most kEnt).
__device__ __forceinline__ void composite_window(TileSmem &S, int nw, const SplatCfg &C, const TileGeo &G,
                                                 float4 &d) {
    const int q = threadIdx.x;
    S.cnt[q] = 0;
    __syncthreads();
    for (int s = q; s < nw; s += kTB) box_texels(S.box[s], [&](int t) { atomicAdd(&S.cnt[t], 1); });
    __syncthreads();
    const int m = S.cnt[q];
    unsigned long long ex;
    block_excl_scan((unsigned long long)m, ex, S.scan_w);
    S.start[q] = (int)ex;
    S.cnt[q] = 0;
    __syncthreads();
    for (int s = q; s < nw; s += kTB)
        box_texels(S.box[s], [&](int t) {
            const int e = S.start[t] + atomicAdd(&S.cnt[t], 1);
            if (e < kEnt) S.ent[e] = (unsigned short)s;
        });
    __syncthreads();
    if (m) blend_texel(S, S.ent + (int)ex, m, q, C, G, d);
    __syncthreads();
}

// A tile whose records do not fit one window: consecutive key ranges [lo, hi),
// each holding at most kRec records and kEnt entries, composited in turn.  hi
// is the end of the longest run of key buckets (a histogram over [lo, top])
// within both limits; when the first bucket alone is over, the search narrows
// to that bucket.  One key is one record (a sample falls on a tile once), and
// a record has at most 256 entries (its box lies on the tile), so every window
// makes progress.
__device__ void composite_windowed(TileSmem &S, const Rec *R, const float4 *col, int m, const SplatCfg &C,
                                   const TileGeo &G, float4 &d) {
    const int tid = threadIdx.x, lane = tid & 31;
    unsigned long long kmin = ~0ull, kmax = 0;
    for (int s = tid; s < m; s += kTB) {
        const unsigned long long k = R[s].key;
        kmin = min(kmin, k);
        kmax = max(kmax, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
        kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
    }
    if (tid < 2) S.u.hist[tid] = tid ? 0ull : ~0ull;
    __syncthreads();
    if (lane == 0) {
        atomicMin(&S.u.hist[0], kmin);
        atomicMax(&S.u.hist[1], kmax);
    }
    __syncthreads();
    kmin = S.u.hist[0];
    kmax = S.u.hist[1];
    __syncthreads();
    unsigned long long lo = kmin;
    while (lo <= kmax) {
        unsigned long long top = kmax, hi;
        for (;;) {
            const unsigned long long span = top - lo + 1, bw = (span + kHist - 1) / kHist;
            for (int b = tid; b < kHist; b += kTB) S.u.hist[b] = 0;
            if (tid == 0) S.cut = kHist;
            __syncthreads();
            for (int s = tid; s < m; s += kTB) {
                const Rec r = R[s];
                if (r.key < lo || r.key > top) continue;
                const int e = box_entries(rec_box(C, G, r.px, r.py));
                if (e) atomicAdd(&S.u.hist[(r.key - lo) / bw], ((unsigned long long)e << 32) | 1ull);
            }
            __syncthreads();
            // first bucket at which the running totals pass a limit
            constexpr int per = kHist / kTB;
            unsigned long long mine = 0;
            for (int u = 0; u < per; u++) mine += S.u.hist[tid * per + u];
            unsigned long long run;
            block_excl_scan(mine, run, S.scan_w);
            for (int u = 0; u < per; u++) {
                run += S.u.hist[tid * per + u];
                if ((run >> 32) > (unsigned long long)kEnt || (run & 0xffffffffull) > (unsigned long long)kRec) {
                    atomicMin(&S.cut, tid * per + u);
                    break;
                }
            }
            __syncthreads();
            const int cut = S.cut;
            __syncthreads();
            if (cut > 0 || bw == 1) {
                hi = lo + (unsigned long long)max(cut, 1) * bw;
                if (hi > top + 1) hi = top + 1;
                break;
            }
            top = lo + bw - 1;
        }
        if (tid == 0) S.cut = 0;  // reused as the window's record count
        __syncthreads();
        for (int s = tid; s < m; s += kTB) {
            const Rec r = R[s];
            if (r.key < lo || r.key >= hi) continue;
            const unsigned short box = rec_box(C, G, r.px, r.py);
            if (box == kNoBox) continue;
            const int slot = atomicAdd(&S.cut, 1);
            if (slot < kRec) window_put(S, slot, r, box);
        }
        __syncthreads();
        const int nw = min(S.cut, kRec);
        window_colours(S, nw, col);
        __syncthreads();
        composite_window(S, nw, C, G, d);
        lo = hi;
    }
}

// One block per tile; see the file comment.  Seven blocks per SM (32
// registers, 30.2 KB of shared memory with a 576-record window) ran 6 % faster
// than six (40 registers, 768 records) and eight (448 records) did.
__global__ void __launch_bounds__(kTB, 7) k_rd_tiles(SplatCfg C, const unsigned *tile_start,
                                                  const unsigned *tile_fill, const Rec *recs, size_t cap,
                                                  const float4 *col, float *buf, unsigned *diag,
                                                  unsigned *est_next) {
    if (tile_start[C.ntiles] > cap) return;  // records not filled: see k_rd_fill
    if (diag[1]) return;                     // a tile's records overflowed: the deposit is repeated
    __shared__ TileSmem S;
    const int tile = blockIdx.x, q = threadIdx.x;
    const int R = C.R, ntx = C.ntx;
    const unsigned s0 = __ldg(tile_start + tile);
    const unsigned fl = __ldg(tile_fill + tile), s1 = __ldg(tile_start + tile + 1);
    const int f = tile / (ntx * ntx), rem = tile - f * ntx * ntx, ty = rem / ntx, tx = rem - ty * ntx;
    TileGeo G;
    G.x0 = tx * kT;
    G.y0 = ty * kT;
    G.tw = min(kT, R - G.x0);
    G.th = min(kT, R - G.y0);
    float4 *face = reinterpret_cast<float4 *>(buf) + (size_t)f * R * R;
    const int lx = q % kT, ly = q / kT;
    const bool inside = lx < G.tw && ly < G.th;
    // the texel is requested together with the tile's record count (before
    // knowing whether the tile has records), so that the two round trips
    // overlap; an empty tile then returns with the texel unused
    float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
    if (inside) d = face[(size_t)(G.y0 + ly) * R + G.x0 + lx];
    const int m = (int)min(fl, s1 - s0);
    if (m == 0 && !C.renorm) return;
    if (inside) {
        if (C.renorm) {
            d.x *= C.scale;
            d.y *= C.scale;
            d.z *= C.scale;
            d.w *= C.scale;
        }
    }
    if (m > 0) {
        const Rec *Rt = recs + s0;
        // one window: records, per-texel counts and, while no texel takes more
        // than kBucket entries, the entries themselves (each in the slot its
        // count gives it) in one pass
        S.cnt[q] = 0;
        if (q == 0) {
            S.tot = 0;
            S.full = 0;
        }
        __syncthreads();
        if (m <= kRec) {
            int e = 0;
            for (int s = q; s < m; s += kTB) {
                const Rec r = Rt[s];
                const unsigned short box = rec_box(C, G, r.px, r.py);
                window_put(S, s, r, box);
                box_texels(box, [&](int t) {
                    const int k = atomicAdd(&S.cnt[t], 1);
                    if (k < kBucket)
                        S.bucket[t * kBucketStride + k] = (unsigned short)s;
                    else
                        S.full = 1;
                });
                e += box_entries(box);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
            if ((q & 31) == 0 && e) atomicAdd(&S.tot, e);
            window_colours(S, m, col);  // each thread reads back the keys it stored itself
        }
        __syncthreads();
        if (m <= kRec && !S.full) {
            const int c = S.cnt[q];
            if (c) blend_texel(S, S.bucket + q * kBucketStride, c, q, C, G, d);
        } else if (m <= kRec && S.tot <= kEnt) {
            // a texel with more than kBucket entries: pack the lists by a count scan
            const int c = S.cnt[q];
            const int st = block_scan_1sync(c, S.wsum);
            S.start[q] = st;
            S.cnt[q] = 0;
            __syncthreads();
            for (int s = q; s < m; s += kTB)
                box_texels(S.box[s], [&](int t) {
                    const int e = S.start[t] + atomicAdd(&S.cnt[t], 1);
                    if (e < kEnt) S.ent[e] = (unsigned short)s;
                });
            __syncthreads();
            if (c) blend_texel(S, S.ent + st, c, q, C, G, d);
        } else {
            if (q == 0) atomicAdd(diag, 1u);
            __syncthreads();
            composite_windowed(S, Rt, col, m, C, G, d);
        }
    }
    if (inside) face[(size_t)(G.y0 + ly) * R + G.x0 + lx] = d;
    // the next deposit's estimate of this tile and its neighbours on the face
    // (nine threads, one neighbour each; the count is read again here so that
    // it need not stay in a register through the compositing)
    if (q < 9) {
        const int y = ty + q / 3 - 1, x = tx + q % 3 - 1;
        const unsigned mm = min(__ldg(tile_fill + tile), __ldg(tile_start + tile + 1) - s0);
        if (mm > 0 && y >= 0 && y < ntx && x >= 0 && x < ntx) atomicMax(est_next + (f * ntx + y) * ntx + x, mm);
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
    C.ntiles = Pv->ntiles;
    C.rad = r->radius;
    C.invrad = 1.0f / r->radius;
    C.invg = (float)(1.0 / r->g);
    C.alpha = r->alpha;
    C.spacing = 0.7 / r->R;
    C.edge_lim = 1.0 + (2.0 * (double)r->radius + 2.0) / r->R;
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

// Fill and composite (after the count and scan of the same deposit).  Both
// kernels do nothing when the reserved total exceeds the record buffer.
static void deposit_fill_tiles(Render *r, const Particles *P, RenderPriv *Pv, const SplatCfg &C) {
    cudaStream_t s = stream();
    const int n = P->n;
    const unsigned nb = (unsigned)std::max(1, std::min(n / 256 + 1, 148 * 16));
    stage_begin(ST_TILES);
    if (n > 0) {
        k_rd_fill<<<nb, 256, 0, s>>>(n, C, P->prev, P->pos, Pv->tile_start, Pv->tile_fill, Pv->recs,
                                     Pv->rec_cap, Pv->diag);
        GGB_LAUNCHED();
    }
    k_rd_tiles<<<Pv->ntiles, kTB, 0, s>>>(C, Pv->tile_start, Pv->tile_fill, Pv->recs, Pv->rec_cap,
                                          reinterpret_cast<const float4 *>(P->col), r->buf, Pv->diag, Pv->tile_est);
    GGB_LAUNCHED();
    stage_end(ST_TILES);
}

// The whole deposit without a host round trip: queues the slot reservation,
// scan, fill and compositing and the copies of the reserved total and the
// overflow count.  The reservation is exact (k_rd_count) for the first deposit
// and estimated from the neighbourhood maxima of the previous deposit's
// per-tile record counts afterwards (no counting pass), except for the b
// deposits after an estimate overflowed (b doubles with every overflow up to
// 64 and halves with every estimate that fits).  render_deposit_collect
// (after a synchronisation of the stream) checks the outcome.  Fill and compositing skip the whole deposit
// (the face buffer is untouched) when the record buffer was too small, and
// compositing skips it when an estimated tile overflowed.  The host then grows
// the buffer and runs them again on the same reservations, or repeats the
// deposit with exact reservations.
static void grow_records(RenderPriv *Pv, size_t need);

void render_deposit_queue(Render *r, const Particles *P) {
    RenderPriv *Pv = rpriv(r);
    cudaStream_t s = stream();
    SplatCfg C = splat_cfg(r, Pv);
    int n = P->n;
    // the first deposit's records are not known before its fill: size the
    // buffer for eight per particle (the default workload makes about 4.3, and
    // the next deposit's neighbourhood estimate reserves about 2.5 times its
    // records), so that neither fill has to run a second time on a grown buffer
    if (!Pv->have_prev) grow_records(Pv, (size_t)8 * n);
    // estimated reservations unless a recent estimate overflowed (a sparse
    // planet's tile counts can jump from one step to the next; each overflow
    // costs a repeated deposit, each exact reservation only the counting pass)
    const bool est = Pv->have_prev && Pv->exact_next == 0;
    if (Pv->have_prev && !est) Pv->exact_next--;
    stage_begin(ST_BIN);
    GGB_CHECK(cudaMemsetAsync(Pv->diag, 0, 2 * sizeof(unsigned), s));
    if (est) {
        k_tile_scan<<<1, 1024, 0, s>>>(Pv->ntiles, Pv->tile_est, 1, Pv->tile_start, Pv->tile_count + Pv->ntiles,
                                       Pv->tile_est);
        GGB_LAUNCHED();
    } else {
        GGB_CHECK(cudaMemsetAsync(Pv->tile_count, 0, sizeof(unsigned) * Pv->ntiles, s));
        unsigned nb = (unsigned)std::max(1, std::min(n / 256 + 1, 148 * 16));
        if (n > 0) {
            k_rd_count<<<nb, 256, 0, s>>>(n, C, P->prev, P->pos, Pv->tile_count);
            GGB_LAUNCHED();
        }
        k_tile_scan<<<1, 1024, 0, s>>>(Pv->ntiles, Pv->tile_count, 0, Pv->tile_start, Pv->tile_count + Pv->ntiles,
                                       Pv->tile_est);
        GGB_LAUNCHED();
    }
    GGB_CHECK(cudaMemsetAsync(Pv->tile_fill, 0, sizeof(unsigned) * Pv->ntiles, s));
    stage_end(ST_BIN);
    deposit_fill_tiles(r, P, Pv, C);
    GGB_CHECK(cudaMemcpyAsync(Pv->total_host, Pv->tile_count + Pv->ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    GGB_CHECK(cudaMemcpyAsync(Pv->total_host + 1, Pv->diag + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    Pv->queued = C;
    Pv->queued_est = est;
    Pv->pending = false;
    Pv->pending_scale = 1.f;
    Pv->dev_gen++;
}

// Grows the record buffer to hold need records, with room for the next
// deposit's estimated reservation (1.5 x the neighbourhood maxima of this
// deposit's counts plus kTileSpare per tile, about as much as this one's).
// Without that room a sparse planet, whose estimate is mostly the spare
// slots, would outgrow the buffer at every deposit.
static void grow_records(RenderPriv *Pv, size_t need) {
    if (need <= Pv->rec_cap) return;
    dev_free(Pv->recs);
    Pv->rec_cap = need + need / 2 + (size_t)kTileSpare * Pv->ntiles + 1024;
    Pv->recs = (Rec *)dev_alloc(sizeof(Rec) * Pv->rec_cap);
}

// Fill and compositing of the queued deposit again, with the reservations
// already in tile_start (synchronous; after the record buffer grew).  Returns
// the tile overflow flag.
static unsigned deposit_refill(Render *r, const Particles *P, RenderPriv *Pv) {
    cudaStream_t s = stream();
    Pv->repeats++;
    Pv->grown++;
    GGB_CHECK(cudaMemsetAsync(Pv->diag, 0, 2 * sizeof(unsigned), s));
    GGB_CHECK(cudaMemsetAsync(Pv->tile_fill, 0, sizeof(unsigned) * Pv->ntiles, s));
    deposit_fill_tiles(r, P, Pv, Pv->queued);
    GGB_CHECK(cudaMemcpyAsync(Pv->total_host + 1, Pv->diag + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    GGB_CHECK(cudaStreamSynchronize(s));
    Pv->dev_gen++;
    return Pv->total_host[1];
}

// The queued deposit again with exact reservations (synchronous).
static void deposit_exact(Render *r, const Particles *P, RenderPriv *Pv) {
    cudaStream_t s = stream();
    Pv->repeats++;
    const SplatCfg &C = Pv->queued;
    const int n = P->n;
    GGB_CHECK(cudaMemsetAsync(Pv->diag, 0, 2 * sizeof(unsigned), s));
    GGB_CHECK(cudaMemsetAsync(Pv->tile_count, 0, sizeof(unsigned) * Pv->ntiles, s));
    unsigned nb = (unsigned)std::max(1, std::min(n / 256 + 1, 148 * 16));
    if (n > 0) {
        k_rd_count<<<nb, 256, 0, s>>>(n, C, P->prev, P->pos, Pv->tile_count);
        GGB_LAUNCHED();
    }
    k_tile_scan<<<1, 1024, 0, s>>>(Pv->ntiles, Pv->tile_count, 0, Pv->tile_start, Pv->tile_count + Pv->ntiles,
                                   Pv->tile_est);
    GGB_LAUNCHED();
    GGB_CHECK(cudaMemcpyAsync(Pv->total_host, Pv->tile_count + Pv->ntiles, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    GGB_CHECK(cudaStreamSynchronize(s));
    grow_records(Pv, Pv->total_host[0]);
    GGB_CHECK(cudaMemsetAsync(Pv->tile_fill, 0, sizeof(unsigned) * Pv->ntiles, s));
    deposit_fill_tiles(r, P, Pv, C);
    GGB_CHECK(cudaMemcpyAsync(Pv->total_host + 1, Pv->diag + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    GGB_CHECK(cudaStreamSynchronize(s));
    if (Pv->total_host[1])
        fail_msg("render_deposit: a tile's sample records exceeded their exact reservation (internal error)");
    Pv->dev_gen++;
}

void render_deposit_collect(Render *r, const Particles *P) {
    RenderPriv *Pv = rpriv(r);
    const size_t need = Pv->total_host[0];
    unsigned over = Pv->total_host[1];
    if (need > Pv->rec_cap) {  // fill and compositing were skipped: grow the buffer, run them again
        grow_records(Pv, need);
        over = deposit_refill(r, P, Pv);
    }
    if (Pv->queued_est) {
        if (over) {  // a tile outgrew its estimate: exact reservations, for this and the next deposits
            Pv->exact_next = Pv->backoff;
            Pv->backoff = std::min(2 * Pv->backoff, 64);
            deposit_exact(r, P, Pv);
        } else {
            Pv->backoff = std::max(1, Pv->backoff / 2);
        }
    } else if (over) {
        fail_msg("render_deposit: a tile's sample records exceeded their exact reservation (internal error)");
    }
    Pv->have_prev = true;
}

void render_deposit_launch(Render *r, const Particles *P) {
    render_deposit_queue(r, P);
    GGB_CHECK(cudaStreamSynchronize(stream()));
    render_deposit_collect(r, P);
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

void render_pending_get(const Render *r, int *pending, float *scale) {
    const RenderPriv *Pv = rpriv(r);
    *pending = Pv->pending ? 1 : 0;
    *scale = Pv->pending_scale;
}

void render_pending_set(Render *r, int pending, float scale) {
    RenderPriv *Pv = rpriv(r);
    Pv->pending = pending != 0;
    Pv->pending_scale = pending ? scale : 1.f;
    Pv->dev_gen++;
}

// The particles were replaced (a checkpoint restore): the previous deposit's
// per-tile record counts describe other positions, so the next deposit
// reserves exactly instead of from them.
void render_particles_replaced(Render *r) {
    RenderPriv *Pv = rpriv(r);
    if (Pv->have_prev) Pv->exact_next = std::max(Pv->exact_next, 1);
}

// ---- 8-bit output encoding (upstream src/main.c:249-318) --------------------

struct EncCfg {
    int R, ch, has_bg, pending;
    float g, pscale, bg[3];
    int order[6];
};

// render_texel (upstream src/render.c:220-226), with a pending renormalisation
// of render_fade applied first, as render_texel of this library does.
__device__ __forceinline__ float4 enc_texel(const float4 *buf, const EncCfg &E, int f, int x, int y) {
    float4 d = buf[((size_t)f * E.R + y) * E.R + x];
    if (E.pending) {
        d.x = __fmul_rn(d.x, E.pscale);
        d.y = __fmul_rn(d.y, E.pscale);
        d.z = __fmul_rn(d.z, E.pscale);
        d.w = __fmul_rn(d.w, E.pscale);
    }
    return make_float4(__fmul_rn(d.x, E.g), __fmul_rn(d.y, E.g), __fmul_rn(d.z, E.g), __fmul_rn(d.w, E.g));
}

// to8 and render_pixel8 (upstream src/render.c:253-279), with the
// contractions of the upstream gcc build (v * 255 + 0.5, c + bg (1 - a)).
__device__ __forceinline__ unsigned char enc_u8(float v) {
    if (v <= 0.f) return 0;
    if (v >= 1.f) return 255;
    return (unsigned char)__fmaf_rn(v, 255.0f, 0.5f);
}
__device__ __forceinline__ void enc_pixel8(float4 c, const EncCfg &E, unsigned char out[4]) {
    float a = c.w;
    a = a > 1.f ? 1.f : (a < 0.f ? 0.f : a);
    if (!E.has_bg) {
        if (a > 1e-6f) {
            out[0] = enc_u8(__fdiv_rn(c.x, a));
            out[1] = enc_u8(__fdiv_rn(c.y, a));
            out[2] = enc_u8(__fdiv_rn(c.z, a));
        } else {
            out[0] = out[1] = out[2] = 0;
        }
        out[3] = enc_u8(a);
    } else {
        const float k = 1.0f - a;
        out[0] = enc_u8(__fmaf_rn(E.bg[0], k, c.x));
        out[1] = enc_u8(__fmaf_rn(E.bg[1], k, c.y));
        out[2] = enc_u8(__fmaf_rn(E.bg[2], k, c.z));
    }
}

__device__ __forceinline__ void enc_store(unsigned char *dst, const unsigned char px[4], int ch) {
    for (int k = 0; k < ch; k++) dst[k] = px[k];
}

// The six faces (in the order E.order) as R x R images of ch channels.
__global__ void k_enc_faces(EncCfg E, const float4 *buf, unsigned char *out) {
    const int k = blockIdx.y, f = E.order[k];
    const size_t np = (size_t)E.R * E.R;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / E.R), x = (int)(i - (size_t)y * E.R);
        unsigned char px[4] = {0, 0, 0, 255};
        enc_pixel8(enc_texel(buf, E, f, x, y), E, px);
        enc_store(out + ((size_t)k * np + i) * E.ch, px, E.ch);
    }
}

// The 4R x 3R cross net, RGBA (the caller clears it: cells without a face stay 0).
__global__ void k_enc_net(EncCfg E, const float4 *buf, unsigned char *out) {
    const int R = E.R, W = 4 * R;
    const size_t np = (size_t)6 * R * R;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
        const int fy = (int)(i / R), x = (int)(i - (size_t)fy * R);
        const int f = fy / R, y = fy - f * R;
        const int cx = f < 4 ? f : 0, cy = f < 4 ? 1 : (f == 4 ? 0 : 2);
        unsigned char px[4] = {0, 0, 0, 255};
        enc_pixel8(enc_texel(buf, E, f, x, y), E, px);
        enc_store(out + (((size_t)cy * R + y) * W + (size_t)cx * R + x) * 4, px, 4);
    }
}

// The 2R x R equirectangular preview of ch channels: render_sample_dir
// (upstream src/render.c:228-251) at the pixel centres' directions.
__global__ void k_enc_preview(EncCfg E, const float4 *buf, unsigned char *out) {
    const int R = E.R, W = 2 * R, H = R;
    const size_t np = (size_t)W * H;
    const double kPiD = 3.14159265358979323846;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i - (size_t)y * W);
        const double lat = __fma_rn(-((y + 0.5) / H), kPiD, kPiD / 2);
        const double lon = __fma_rn((x + 0.5) / W * 2, kPiD, -kPiD);
        const double cl = cos(lat);
        const D3 d = d3(cl * sin(lon), sin(lat), cl * cos(lon));
        const int f = face_of(d);
        double dc, dr, du;
        face_proj(f, d, dc, dr, du);
        const double u = dr / dc, v = du / dc;
        double px = __fma_rn((u + 1.0) * 0.5, (double)R, -0.5), py = __fma_rn((1.0 - v) * 0.5, (double)R, -0.5);
        px = px < 0 ? 0 : (px > R - 1 ? R - 1 : px);
        py = py < 0 ? 0 : (py > R - 1 ? R - 1 : py);
        const int x0 = (int)px, y0 = (int)py;
        const int x1 = x0 + 1 < R ? x0 + 1 : x0, y1 = y0 + 1 < R ? y0 + 1 : y0;
        const float fx = (float)(px - x0), fy = (float)(py - y0);
        const float4 a = enc_texel(buf, E, f, x0, y0), b = enc_texel(buf, E, f, x1, y0);
        const float4 c = enc_texel(buf, E, f, x0, y1), e = enc_texel(buf, E, f, x1, y1);
        const float gx = 1.0f - fx, gy = 1.0f - fy;
        auto lerp2 = [&](float t00, float t10, float t01, float t11) {
            const float lo = __fmaf_rn(gx, t00, __fmul_rn(fx, t10));
            const float hi = __fmaf_rn(gx, t01, __fmul_rn(fx, t11));
            return __fmaf_rn(gy, lo, __fmul_rn(fy, hi));
        };
        const float4 s = make_float4(lerp2(a.x, b.x, c.x, e.x), lerp2(a.y, b.y, c.y, e.y), lerp2(a.z, b.z, c.z, e.z),
                                     lerp2(a.w, b.w, c.w, e.w));
        unsigned char q[4] = {0, 0, 0, 255};
        enc_pixel8(s, E, q);
        enc_store(out + i * E.ch, q, E.ch);
    }
}

static EncCfg enc_cfg(const Render *r, const RenderPriv *Pv, const float *bg) {
    EncCfg E;
    E.R = r->R;
    E.has_bg = bg != nullptr;
    E.ch = bg ? 3 : 4;
    E.pending = Pv->pending ? 1 : 0;
    E.pscale = Pv->pending_scale;
    E.g = (float)r->g;
    for (int k = 0; k < 3; k++) E.bg[k] = bg ? bg[k] : 0.f;
    for (int k = 0; k < 6; k++) E.order[k] = k;
    return E;
}

// Device destination of an encoder: out itself when the GPU can write it,
// otherwise the cached scratch (copied to out by enc_finish).
static unsigned char *enc_target(RenderPriv *Pv, unsigned char *out, size_t bytes, bool &staged) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, out) == cudaSuccess &&
        (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged)) {
        staged = false;
        return out;
    }
    cudaGetLastError();
    staged = true;
    if (bytes > Pv->enc_cap) {
        dev_free(Pv->enc);
        Pv->enc = (unsigned char *)dev_alloc(bytes);
        Pv->enc_cap = bytes;
    }
    return Pv->enc;
}

static void enc_finish(RenderPriv *Pv, unsigned char *out, size_t bytes, bool staged) {
    if (staged) GGB_CHECK(cudaMemcpyAsync(out, Pv->enc, bytes, cudaMemcpyDeviceToHost, stream()));
    sync();
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
    r->buf = (float *)managed_try_alloc(sizeof(float) * 6 * (size_t)R * R * 4);
    if (!r->buf) {
        fprintf(stderr, "render: device memory allocation failed for 6 faces of %d x %d\n", R, R);
        memset(r, 0, sizeof(*r));
        return -1;
    }
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
    Pv->tile_est = (unsigned *)dev_alloc(sizeof(unsigned) * Pv->ntiles);  // zeroed
    Pv->diag = (unsigned *)dev_alloc(sizeof(unsigned) * 2);  // zeroed
    GGB_CHECK(cudaMallocHost(&Pv->total_host, sizeof(unsigned) * 2));
    Pv->total_host[0] = Pv->total_host[1] = 0;
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
        dev_free(Pv->tile_est);
        dev_free(Pv->diag);
        dev_free(Pv->recs);
        cudaFreeHost(Pv->total_host);
        if (Pv->mirror) cudaFreeHost(Pv->mirror);
        dev_free(Pv->enc);
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
    render_deposit_launch(r, P);
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

// Diagnostics of the last deposit: all tiles, the tiles composited in several
// key-range windows, and the record slots reserved for (sample, tile) records.
GGB_EXPORT void ggb_render_stats(const Render *r, unsigned *ntiles, unsigned *slow_tiles, unsigned *entries) {
    RenderPriv *Pv = rpriv(r);
    sync();
    unsigned sc = 0;
    GGB_CHECK(cudaMemcpy(&sc, Pv->diag, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (ntiles) *ntiles = (unsigned)Pv->ntiles;
    if (slow_tiles) *slow_tiles = sc;
    if (entries) *entries = Pv->total_host[0];
}

// Additive diagnostics: how many times the fill and compositing of this
// Render's deposits ran again (record buffer grown, or an estimated tile
// reservation overflowed).
GGB_EXPORT unsigned long ggb_render_repeats(const Render *r) { return rpriv(r)->repeats; }
GGB_EXPORT unsigned long ggb_render_repeats_grown(const Render *r) { return rpriv(r)->grown; }

// Additive: the application driver's 8-bit images, encoded on the GPU (upstream
// src/main.c:249-318).  bg == NULL: transparent (RGBA, un-premultiplied);
// otherwise RGB over bg[3].  out: host or device memory.
GGB_EXPORT int ggb_encode_faces(const Render *r, const float *bg, const int *face_order, unsigned char *out) {
    RenderPriv *Pv = rpriv(r);
    EncCfg E = enc_cfg(r, Pv, bg);
    if (face_order) {
        int seen = 0;
        for (int k = 0; k < 6; k++) {
            if (face_order[k] < 0 || face_order[k] > 5 || (seen >> face_order[k] & 1)) {
                fprintf(stderr, "ggb_encode_faces: face_order must be a permutation of 0..5\n");
                return -1;
            }
            seen |= 1 << face_order[k];
            E.order[k] = face_order[k];
        }
    }
    const size_t bytes = (size_t)6 * r->R * r->R * E.ch;
    bool staged;
    unsigned char *dst = enc_target(Pv, out, bytes, staged);
    dim3 grid((unsigned)std::min<size_t>(((size_t)r->R * r->R + 255) / 256, 148 * 4), 6);
    k_enc_faces<<<grid, 256, 0, stream()>>>(E, reinterpret_cast<const float4 *>(r->buf), dst);
    GGB_LAUNCHED();
    enc_finish(Pv, out, bytes, staged);
    return 0;
}

GGB_EXPORT int ggb_encode_net(const Render *r, const float *bg, unsigned char *out) {
    RenderPriv *Pv = rpriv(r);
    EncCfg E = enc_cfg(r, Pv, bg);
    const size_t bytes = (size_t)12 * r->R * r->R * 4;
    bool staged;
    unsigned char *dst = enc_target(Pv, out, bytes, staged);
    GGB_CHECK(cudaMemsetAsync(dst, 0, bytes, stream()));
    const unsigned nb = (unsigned)std::min<size_t>(((size_t)6 * r->R * r->R + 255) / 256, 148 * 8);
    k_enc_net<<<nb, 256, 0, stream()>>>(E, reinterpret_cast<const float4 *>(r->buf), dst);
    GGB_LAUNCHED();
    enc_finish(Pv, out, bytes, staged);
    return 0;
}

GGB_EXPORT int ggb_encode_preview(const Render *r, const float *bg, unsigned char *out) {
    RenderPriv *Pv = rpriv(r);
    EncCfg E = enc_cfg(r, Pv, bg);
    const size_t bytes = (size_t)2 * r->R * r->R * E.ch;
    bool staged;
    unsigned char *dst = enc_target(Pv, out, bytes, staged);
    const unsigned nb = (unsigned)std::min<size_t>(((size_t)2 * r->R * r->R + 255) / 256, 148 * 8);
    k_enc_preview<<<nb, 256, 0, stream()>>>(E, reinterpret_cast<const float4 *>(r->buf), dst);
    GGB_LAUNCHED();
    enc_finish(Pv, out, bytes, staged);
    return 0;
}
