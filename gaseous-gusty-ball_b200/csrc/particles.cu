// particles.cu — the particles.h entry points of libggb_cuda.so: Fibonacci
// lattice initialisation, equirectangular colour lookup and RK2 (midpoint)
// advection along great circles, one thread per particle.
//
// Upstream: src/particles.c.  pos / prev / col are managed memory; every entry
// point synchronises before returning.
#include <cstdio>
#include <cstring>

#include "ggb_internal.h"

namespace ggb {

constexpr int kPB = 256;

static unsigned blocks_for(size_t n) { return (unsigned)std::max<size_t>(1, std::min<size_t>(grid_for(n, kPB), 148u * 32u)); }

// upstream src/particles.c:18-29
__global__ void k_fibonacci(int n, float *pos, float *prev, float *col) {
    const double golden = kPi * (3.0 - sqrt(5.0));
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double y = 1.0 - 2.0 * (i + 0.5) / n;
        double r = sqrt(1.0 - y * y);
        double phi = golden * i;
        D3 p = d3(r * cos(phi), y, r * sin(phi));
        store3(pos + 3 * (size_t)i, p);
        store3(prev + 3 * (size_t)i, p);
        float4 one = make_float4(1.f, 1.f, 1.f, 1.f);
        reinterpret_cast<float4 *>(col)[i] = one;
    }
}

// upstream src/particles.c:41-61
__global__ void k_colour(int n, const float *pos, const float *img, int w, int h, float *col) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        D3 d = load3(pos + 3 * (size_t)i);
        double lon = atan2(d.x, d.z);
        double yy = d.y > 1.0 ? 1.0 : (d.y < -1.0 ? -1.0 : d.y);
        double lat = asin(yy);
        double x = (lon + kPi) / (2 * kPi) * w - 0.5;
        double y = (kPi / 2 - lat) / kPi * h - 0.5;
        int x0 = (int)floor(x), y0 = (int)floor(y);
        double fx = x - x0, fy = y - y0;
        int xs0 = ((x0 % w) + w) % w, xs1 = (((x0 + 1) % w) + w) % w;
        int ys0 = clampi(y0, 0, h - 1), ys1 = clampi(y0 + 1, 0, h - 1);
        double wts[4] = {(1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy};
        const float *t00 = img + ((size_t)ys0 * w + xs0) * 4, *t01 = img + ((size_t)ys0 * w + xs1) * 4;
        const float *t10 = img + ((size_t)ys1 * w + xs0) * 4, *t11 = img + ((size_t)ys1 * w + xs1) * 4;
        for (int c = 0; c < 4; c++) {
            double v = 0;
            v += wts[0] * t00[c];
            v += wts[1] * t01[c];
            v += wts[2] * t10[c];
            v += wts[3] * t11[c];
            col[4 * (size_t)i + c] = (float)v;
        }
    }
}

// RK2 midpoint step; upstream src/particles.c:63-74.  Over blocks vb_ of vnb_.
__device__ __forceinline__ void advect_body(int n, const GridDev &g, const float *vel, double dt_in, const double *dtp,
                                            float *pos, float *prev, int vb_, int vnb_) {
    const double dt = dtp ? *dtp : dt_in;  // *dtp: a device-side CFL step
    for (int i = vb_ * blockDim.x + threadIdx.x; i < n; i += vnb_ * blockDim.x) {
        float *pp = pos + 3 * (size_t)i;
        float p0 = pp[0], p1 = pp[1], p2 = pp[2];
        float *qq = prev + 3 * (size_t)i;
        qq[0] = p0;
        qq[1] = p1;
        qq[2] = p2;
        D3 p = d3(p0, p1, p2);
        D3 u1 = sample_vec(g, vel, p);
        D3 pm = sphere_move(p, u1, 0.5 * dt);
        D3 u2 = tangent(sample_vec(g, vel, pm), p);
        store3(pp, sphere_move(p, u2, dt));
    }
}

__global__ void __launch_bounds__(kPB) k_advect(int n, GridDev g, const float *vel, double dt_in, const double *dtp,
                                                float *pos, float *prev) {
    advect_body(n, g, vel, dt_in, dtp, pos, prev, blockIdx.x, gridDim.x);
}

// Every planet's particles in one launch (block map over the planets' particles).
__global__ void __launch_bounds__(kPB) k_advect_batch(const PlanetStepDev *pl, const int4 *map) {
    const int4 m = map[blockIdx.x];
    const PlanetStepDev &P = pl[m.x];
    advect_body(P.np, P.g, P.vel, 0.0, P.dt, P.ppos, P.pprev, m.y, m.z);
}

unsigned batch_particle_blocks(int n) { return blocks_for((size_t)n); }

void particles_step_dev(Particles *P, PlanetStepDev *out) {
    out->np = P ? P->n : 0;
    out->ppos = P ? P->pos : nullptr;
    out->pprev = P ? P->prev : nullptr;
}

void batch_particles_launch(const PlanetStepDev *pl, const int4 *map, int nb) {
    if (nb <= 0) return;
    stage_begin(ST_PARTICLES);
    k_advect_batch<<<nb, kPB, 0, stream()>>>(pl, map);
    GGB_LAUNCHED();
    stage_end(ST_PARTICLES);
}

void particles_advect_launch(int n, const GridDev &g, const float *vel, double dt, const double *dtp, float *pos,
                             float *prev, cudaStream_t s) {
    stage_begin(ST_PARTICLES);
    k_advect<<<blocks_for(n), kPB, 0, s>>>(n, g, vel, dt, dtp, pos, prev);
    GGB_LAUNCHED();
    stage_end(ST_PARTICLES);
}

void particles_advect_queue(Particles *P, const CubeSphere *cs, const float *vel, const double *dt_dev) {
    if (P->n <= 0) return;
    GridTables *t = grid_lookup(cs);
    particles_advect_launch(P->n, t->dev(), vel, 0.0, dt_dev, P->pos, P->prev, stream());
}

}  // namespace ggb

using namespace ggb;

GGB_EXPORT int particles_init(Particles *P, int n) {
    memset(P, 0, sizeof(*P));
    if (n < 0) {
        fprintf(stderr, "particles: bad count %d\n", n);
        return -1;
    }
    if (!have_device()) {
        fprintf(stderr, "particles: no CUDA device is available (libggb_cuda has no CPU path)\n");
        return -1;
    }
    P->n = n;
    P->pos = (float *)managed_try_alloc(sizeof(float) * 3 * (size_t)n);
    P->prev = (float *)managed_try_alloc(sizeof(float) * 3 * (size_t)n);
    P->col = (float *)managed_try_alloc(sizeof(float) * 4 * (size_t)n);
    if (!P->pos || !P->prev || !P->col) {
        fprintf(stderr, "particles: device memory allocation failed for %d particles\n", n);
        managed_free(P->pos);
        managed_free(P->prev);
        managed_free(P->col);
        memset(P, 0, sizeof(*P));
        return -1;
    }
    if (n > 0) {
        k_fibonacci<<<blocks_for(n), kPB, 0, stream()>>>(n, P->pos, P->prev, P->col);
        GGB_LAUNCHED();
    }
    sync();
    return 0;
}

GGB_EXPORT void particles_free(Particles *P) {
    sync();
    managed_free(P->pos);
    managed_free(P->prev);
    managed_free(P->col);
    memset(P, 0, sizeof(*P));
}

GGB_EXPORT void particles_color_from_image(Particles *P, const float *img, int w, int h) {
    if (P->n <= 0) return;
    Staged in;
    stage_in(in, img, sizeof(float) * 4 * (size_t)w * h);
    k_colour<<<blocks_for(P->n), kPB, 0, stream()>>>(P->n, P->pos, (const float *)in.dev, w, h, P->col);
    GGB_LAUNCHED();
    sync();
}

GGB_EXPORT void particles_advect(Particles *P, const CubeSphere *cs, const float *vel, double dt) {
    if (P->n <= 0) return;
    GridTables *t = grid_lookup(cs);
    Staged in;
    stage_in(in, vel, sizeof(float) * 3 * t->n);
    particles_advect_launch(P->n, t->dev(), (const float *)in.dev, dt, nullptr, P->pos, P->prev, stream());
    sync();
}
