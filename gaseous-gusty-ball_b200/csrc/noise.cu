// noise.cu — 3-D simplex noise with analytic gradient and multi-octave curl
// noise (the noise.h API, on the host), and the initial velocity field of the
// application driver as a GPU kernel (curl noise projected and scaled to a
// target RMS speed, plus zonal bands), used by the batched planet API.
//
// Upstream: src/noise.c (simplex / curl noise), src/main.c:321-360 (initial
// velocity).  The gradient table, the seeding generator and the octave
// offsets are the upstream constants: they define the noise field, so the
// same seed must give the same field.
#include <cstdio>
#include <cstring>

#include "ggb_internal.h"
#include "noise.h"

namespace ggb {

__host__ __device__ __forceinline__ double simplex3_impl(const unsigned char *perm, D3 pt, D3 *g) {
    // 12 edge-midpoint gradient directions of 3-D simplex noise
    const signed char grad[12][3] = {{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1},
                                     {1, 0, -1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1}};
    const double F3 = 1.0 / 3.0, G3 = 1.0 / 6.0;
    double x = pt.x, y = pt.y, z = pt.z;
    double s = (x + y + z) * F3;
    int i = (int)floor(x + s), j = (int)floor(y + s), k = (int)floor(z + s);
    double t = (i + j + k) * G3;
    double x0 = x - (i - t), y0 = y - (j - t), z0 = z - (k - t);
    int a1, b1, c1, a2, b2, c2;  // offsets of the second and third simplex corners
    if (x0 >= y0) {
        if (y0 >= z0) { a1 = 1; b1 = 0; c1 = 0; a2 = 1; b2 = 1; c2 = 0; }
        else if (x0 >= z0) { a1 = 1; b1 = 0; c1 = 0; a2 = 1; b2 = 0; c2 = 1; }
        else { a1 = 0; b1 = 0; c1 = 1; a2 = 1; b2 = 0; c2 = 1; }
    } else {
        if (y0 < z0) { a1 = 0; b1 = 0; c1 = 1; a2 = 0; b2 = 1; c2 = 1; }
        else if (x0 < z0) { a1 = 0; b1 = 1; c1 = 0; a2 = 0; b2 = 1; c2 = 1; }
        else { a1 = 0; b1 = 1; c1 = 0; a2 = 1; b2 = 1; c2 = 0; }
    }
    double xs[4] = {x0, x0 - a1 + G3, x0 - a2 + 2 * G3, x0 - 1 + 3 * G3};
    double ys[4] = {y0, y0 - b1 + G3, y0 - b2 + 2 * G3, y0 - 1 + 3 * G3};
    double zs[4] = {z0, z0 - c1 + G3, z0 - c2 + 2 * G3, z0 - 1 + 3 * G3};
    int ii = i & 255, jj = j & 255, kk = k & 255;
    int gi[4];
    gi[0] = perm[ii + perm[jj + perm[kk]]] % 12;
    gi[1] = perm[ii + a1 + perm[jj + b1 + perm[kk + c1]]] % 12;
    gi[2] = perm[ii + a2 + perm[jj + b2 + perm[kk + c2]]] % 12;
    gi[3] = perm[ii + 1 + perm[jj + 1 + perm[kk + 1]]] % 12;
    double n = 0, dx = 0, dy = 0, dz = 0;
    for (int c = 0; c < 4; c++) {
        double tt = 0.5 - xs[c] * xs[c] - ys[c] * ys[c] - zs[c] * zs[c];
        if (tt <= 0) continue;
        double gx = grad[gi[c]][0], gy = grad[gi[c]][1], gz = grad[gi[c]][2];
        double gd = gx * xs[c] + gy * ys[c] + gz * zs[c];
        double t2 = tt * tt, t4 = t2 * t2, t3 = t2 * tt;
        n += t4 * gd;
        dx += t4 * gx - 8.0 * t3 * gd * xs[c];
        dy += t4 * gy - 8.0 * t3 * gd * ys[c];
        dz += t4 * gz - 8.0 * t3 * gd * zs[c];
    }
    const double sc = 72.0;
    if (g) *g = d3(dx * sc, dy * sc, dz * sc);
    return n * sc;
}

__host__ __device__ __forceinline__ D3 curl_noise_impl(const unsigned char *perm, D3 p, double scale, double lac,
                                                       double gain, int octaves) {
    D3 c = d3(0, 0, 0);
    double f = scale, a = 1.0;
    for (int k = 0; k < octaves; k++) {
        D3 q = add(::ggb::scale(p, f), d3(17.13 * k, 5.31 * k, 11.71 * k));
        D3 gx, gy, gz;
        simplex3_impl(perm, add(q, d3(0.0, 0.0, 0.0)), &gx);
        simplex3_impl(perm, add(q, d3(31.416, -47.853, 12.793)), &gy);
        simplex3_impl(perm, add(q, d3(-93.11, 63.2, 109.7)), &gz);
        double m = a * f;
        c = add(c, ::ggb::scale(d3(gz.y - gy.z, gx.z - gz.x, gy.x - gx.y), m));
        f *= lac;
        a *= gain;
    }
    return c;
}

void perm_table(unsigned int seed, unsigned char out[512]) {
    unsigned char p[256];
    unsigned long long s = 0x9E3779B97F4A7C15ULL ^ ((unsigned long long)seed * 0xD1B54A32D192ED03ULL);
    for (int i = 0; i < 256; i++) p[i] = (unsigned char)i;
    for (int i = 255; i > 0; i--) {
        s ^= s >> 12;
        s ^= s << 25;
        s ^= s >> 27;
        unsigned long long r = s * 2685821657736338717ULL;
        int j = (int)((r >> 33) % (unsigned long long)(i + 1));
        unsigned char t = p[i];
        p[i] = p[j];
        p[j] = t;
    }
    for (int i = 0; i < 512; i++) out[i] = p[i & 255];
}

struct InitDev {
    double band_amp, noise_amp, scale, lac, gain;
    int bands, octaves;
};

// pass 1: projected curl noise and its per-block FP64 sum of A |v|^2
__global__ void k_init_noise(int n, const float *pos, const float *area, const unsigned char *perm_g, InitDev I,
                             float *vel, double *part) {
    __shared__ unsigned char perm[512];
    __shared__ double s_red[256 / 32 + 2];
    for (int t = threadIdx.x; t < 512; t += blockDim.x) perm[t] = perm_g[t];
    __syncthreads();
    double ss = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D3 p = load3(pos + 3 * i);
        D3 v = I.octaves > 0 ? tangent(curl_noise_impl(perm, p, I.scale, I.lac, I.gain, I.octaves), p) : d3(0, 0, 0);
        store3(vel + 3 * i, v);
        ss += dot(v, v) * area[i];
    }
    double t = block_sum<256>(ss, s_red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// pass 2: scale to the RMS speed and add the zonal bands
__global__ void k_init_bands(int n, const float *pos, const double *part, int nparts, double total_area, InitDev I,
                             float *vel, float *vband) {
    __shared__ double s_red[256 / 32 + 2];
    double ss = sum_partials<256>(part, nparts, s_red);
    double rms = sqrt(ss / total_area);
    double sc = rms > 0 ? I.noise_amp / rms : 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D3 p = load3(pos + 3 * i);
        double colat = acos(p.y > 1 ? 1 : (p.y < -1 ? -1 : p.y));
        double s = sin(colat);
        double mag = I.band_amp * sin(I.bands * colat);
        D3 east = cross(d3(0, 1, 0), p);
        D3 b = s > 1e-9 ? ::ggb::scale(east, mag / s) : d3(0, 0, 0);
        store3(vband + 3 * i, b);
        store3(vel + 3 * i, add(::ggb::scale(load3(vel + 3 * i), sc), b));
    }
}

}  // namespace ggb

using namespace ggb;

// ---- noise.h (host)

GGB_EXPORT void noise_init(Noise *nz, unsigned int seed) { perm_table(seed, nz->perm); }

GGB_EXPORT double simplex3(const Noise *nz, vec3 p, vec3 *g) {
    D3 gd;
    double v = simplex3_impl(nz->perm, d3(p.x, p.y, p.z), g ? &gd : nullptr);
    if (g) *g = v3(gd.x, gd.y, gd.z);
    return v;
}

GGB_EXPORT vec3 curl_noise(const Noise *nz, vec3 p, const CurlParams *cp) {
    D3 c = curl_noise_impl(nz->perm, d3(p.x, p.y, p.z), cp->scale, cp->lacunarity, cp->gain, cp->octaves);
    return v3(c.x, c.y, c.z);
}

// ---- additive: initial velocity on the GPU


// vel / vband: [ncells*3] (host or device memory).  Same field as the
// application driver's initial_velocity (upstream src/main.c:321-351).
GGB_EXPORT void ggb_initial_velocity(const CubeSphere *cs, const GGBInitParams *ip, float *vel, float *vband) {
    GridTables *t = grid_lookup(cs);
    cudaStream_t s = stream();
    unsigned char perm[512];
    perm_table(ip->seed, perm);
    unsigned char *perm_d = (unsigned char *)dev_alloc(512);
    GGB_CHECK(cudaMemcpyAsync(perm_d, perm, 512, cudaMemcpyHostToDevice, s));
    InitDev I;
    I.band_amp = ip->band_amp;
    I.noise_amp = ip->noise_amp;
    I.scale = ip->noise_scale;
    I.lac = ip->noise_lacunarity;
    I.gain = ip->noise_gain;
    I.bands = ip->bands;
    I.octaves = ip->noise_octaves;
    Staged ov, ob;
    stage_out(ov, vel, sizeof(float) * 3 * t->n);
    stage_out(ob, vband, sizeof(float) * 3 * t->n);
    unsigned nb = std::min(grid_for(t->n, 256), 1024u);
    double *part = (double *)dev_alloc(sizeof(double) * nb);
    k_init_noise<<<nb, 256, 0, s>>>(t->n, t->pos, t->area, perm_d, I, (float *)ov.dev, part);
    GGB_LAUNCHED();
    k_init_bands<<<nb, 256, 0, s>>>(t->n, t->pos, part, nb, t->total_area, I, (float *)ov.dev, (float *)ob.dev);
    GGB_LAUNCHED();
    stage_finish(ov);
    stage_finish(ob);
    dev_free(part);
    dev_free(perm_d);
}
