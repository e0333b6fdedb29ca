// checkpoint.cu — ggb_checkpoint_save / ggb_checkpoint_load: the state of a
// running planet (fluid, particles, face buffer) in one file, so that a long
// run can stop and resume with bit-identical results.
//
// What the next steps read is saved: omega, omega_band (forcing target), psi
// (the warm start of the next solve), vel, the last solve's iteration count
// and residual; the particles' pos, prev and col; the face buffer, its global
// fade factor g and a deferred renormalisation of render_fade.  Everything
// else (grid tables, multigrid hierarchy, scratch) is rebuilt by *_init from
// the sizes, which the header records and the loader checks.
//
// File layout (host byte order): a fixed header, then the arrays in the order
// omega, omega_band, psi, vel, pos, prev, col, buf as raw FP32.
#include <cstdio>
#include <cstring>
#include <vector>

#include "ggb_internal.h"

namespace ggb {

struct CkptHeader {
    char magic[8];  // "GGBCKPT" + version byte
    int N;
    long long ncells;
    FluidParams prm;
    int cg_iters;
    double cg_relres;
    int has_particles, nparticles;
    int has_render, R;
    double g;
    float radius, alpha;
    int pending;
    float pending_scale;
};

constexpr char kMagic[8] = {'G', 'G', 'B', 'C', 'K', 'P', 'T', 1};

static bool put(FILE *fp, const float *dev, size_t n, std::vector<float> &tmp) {
    tmp.resize(n);
    GGB_CHECK(cudaMemcpy(tmp.data(), dev, sizeof(float) * n, cudaMemcpyDefault));
    return fwrite(tmp.data(), sizeof(float), n, fp) == n;
}

static bool get(FILE *fp, float *dev, size_t n, std::vector<float> &tmp) {
    tmp.resize(n);
    if (fread(tmp.data(), sizeof(float), n, fp) != n) return false;
    GGB_CHECK(cudaMemcpy(dev, tmp.data(), sizeof(float) * n, cudaMemcpyDefault));
    return true;
}

}  // namespace ggb

using namespace ggb;

GGB_EXPORT int ggb_checkpoint_save(const char *path, const Fluid *F, const Particles *P, const Render *r) {
    if (!F || !F->cs) {
        fprintf(stderr, "ggb_checkpoint_save: a Fluid initialised by fluid_init is required\n");
        return -1;
    }
    sync();
    CkptHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, kMagic, 8);
    h.N = F->cs->N;
    h.ncells = F->cs->ncells;
    h.prm = F->prm;
    h.cg_iters = F->cg_iters;
    h.cg_relres = F->cg_relres;
    h.has_particles = P != nullptr;
    h.nparticles = P ? P->n : 0;
    h.has_render = r != nullptr;
    if (r) {
        h.R = r->R;
        h.g = r->g;
        h.radius = r->radius;
        h.alpha = r->alpha;
        render_pending_get(r, &h.pending, &h.pending_scale);
    }
    FILE *fp = fopen(path, "wb");
    if (!fp) {
        fprintf(stderr, "ggb_checkpoint_save: cannot open %s for writing\n", path);
        return -1;
    }
    std::vector<float> tmp;
    const size_t n = (size_t)h.ncells;
    bool ok = fwrite(&h, sizeof(h), 1, fp) == 1;
    ok = ok && put(fp, F->omega, n, tmp) && put(fp, F->omega_band, n, tmp) && put(fp, F->psi, n, tmp) &&
         put(fp, F->vel, 3 * n, tmp);
    if (P) ok = ok && put(fp, P->pos, 3 * (size_t)P->n, tmp) && put(fp, P->prev, 3 * (size_t)P->n, tmp) &&
                put(fp, P->col, 4 * (size_t)P->n, tmp);
    if (r) ok = ok && put(fp, r->buf, (size_t)6 * r->R * r->R * 4, tmp);
    ok = (fclose(fp) == 0) && ok;
    if (!ok) fprintf(stderr, "ggb_checkpoint_save: writing %s failed\n", path);
    return ok ? 0 : -1;
}

GGB_EXPORT int ggb_checkpoint_load(const char *path, Fluid *F, Particles *P, Render *r) {
    if (!F || !F->cs) {
        fprintf(stderr, "ggb_checkpoint_load: a Fluid initialised by fluid_init is required\n");
        return -1;
    }
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        fprintf(stderr, "ggb_checkpoint_load: cannot open %s\n", path);
        return -1;
    }
    CkptHeader h;
    auto fail = [&](const char *why) {
        fprintf(stderr, "ggb_checkpoint_load: %s: %s\n", path, why);
        fclose(fp);
        return -1;
    };
    if (fread(&h, sizeof(h), 1, fp) != 1 || memcmp(h.magic, kMagic, 8) != 0)
        return fail("not a checkpoint of this library version");
    if (h.N != F->cs->N || h.ncells != F->cs->ncells) return fail("grid size differs from the Fluid's");
    if (!!P != !!h.has_particles || (P && P->n != h.nparticles))
        return fail("particle count differs (or particles present in only one of file and call)");
    if (!!r != !!h.has_render || (r && r->R != h.R)) return fail("face resolution differs (or faces missing)");
    sync();
    std::vector<float> tmp;
    const size_t n = (size_t)h.ncells;
    bool ok = get(fp, F->omega, n, tmp) && get(fp, F->omega_band, n, tmp) && get(fp, F->psi, n, tmp) &&
              get(fp, F->vel, 3 * n, tmp);
    if (P) ok = ok && get(fp, P->pos, 3 * (size_t)P->n, tmp) && get(fp, P->prev, 3 * (size_t)P->n, tmp) &&
                get(fp, P->col, 4 * (size_t)P->n, tmp);
    if (r) ok = ok && get(fp, r->buf, (size_t)6 * r->R * r->R * 4, tmp);
    if (!ok) return fail("file is truncated");
    fclose(fp);
    F->cg_iters = h.cg_iters;
    F->cg_relres = h.cg_relres;
    if (r) {
        r->g = h.g;
        render_pending_set(r, h.pending, h.pending_scale);
        if (P) render_particles_replaced(r);
    }
    sync();
    return 0;
}
