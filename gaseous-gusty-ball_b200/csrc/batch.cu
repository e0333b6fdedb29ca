// batch.cu — many planets advanced together: ggb_batch_create / _step / _free.
//
// A planet is the usual set of objects (cs_init, fluid_init, particles_init,
// render_init; grids may be shared between planets of the same N).  One
// batched step is the application driver's step for every planet (upstream
// src/main.c:421-434: CFL dt from the maximum speed, particles_advect,
// fluid_step, render_fade, render_deposit), with these differences from
// calling those entry points planet after planet:
//   - the Poisson solves of all planets run in ONE persistent cooperative
//     launch: every planet gets a share of the resident blocks and runs its
//     solve on them with its own barrier, reductions and convergence test, so
//     a small planet's solve is not a whole-GPU launch that waits on its own
//     latency, and the planets' solves fill the GPU together;
//   - the shares are chosen by an autotuner that this file implements: each
//     solve reports its device time, from which a cost per cell and block is
//     estimated for every grid size (and precision); blocks are then given out
//     so that the estimated finishing times are equal (the largest finishing
//     time is minimised under the launch's capacity).  The estimates are kept
//     per grid size for the life of the process, so a later batch with the
//     same grid sizes starts from them;
//   - the per-cell and per-particle stages around the solve (maximum speed
//     and CFL dt, particle advection, departures + BFECC + limiter, velocity)
//     are one launch per stage for all planets: each block finds its planet
//     and its share of that planet's cells or particles in a block map, with
//     the per-planet kernels' arithmetic;
//   - fade and splat are queued on one stream per planet after the velocity,
//     so the deposits of different planets overlap;
//   - the CFL dt is computed on the device (same expression, same IEEE square
//     root and division as the driver, so the same dt), so nothing returns to
//     the host inside a step.
// The host synchronises once per batched step, then reads each solve's
// statistics and checks each deposit's record buffer (growing it and
// repeating that planet's compositing in the rare step where it was short).
// Planets of the two precisions are solved in separate batched launches, as
// are planets beyond what one launch can hold.
// Results equal the per-planet entry points' up to the order of the solve's
// FP64 block sums (another number of blocks) and the device's exp in the
// forcing's relaxation factor, 1 - exp(-forcing dt).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <vector>

#include "ggb_internal.h"
#include "ggb_solver.h"

using namespace ggb;

namespace {

// Tuned cost of a solve: device seconds per cell for one block, per (grid N,
// precision); shared by all batches of the process.
std::mutex g_tune_mu;
std::map<std::pair<int, int>, double> g_cost;

double cost_of(int N, int mixed) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_cost.find({N, mixed});
    return it == g_cost.end() ? 0.0 : it->second;
}

void cost_update(int N, int mixed, double c) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_cost.find({N, mixed});
    if (it == g_cost.end())
        g_cost[{N, mixed}] = c;
    else
        it->second = 0.5 * (it->second + c);  // smooth over steps
}

}  // namespace

struct GGBBatch {
    int n = 0;
    std::vector<Fluid *> F;
    std::vector<Particles *> P;
    std::vector<Render *> r;
    std::vector<double> cfl, fade;
    std::vector<cudaStream_t> st;
    double *dt_dev = nullptr;  // [n] device-side time steps
    // the batched per-cell and per-particle stages
    PlanetStepDev *steps_dev = nullptr;   // [n]
    unsigned int *vmax_dev = nullptr;     // [n]
    int4 *cell_map = nullptr, *part_map = nullptr;
    int cell_blocks = 0, part_blocks = 0;
    bool any_bfecc = false;
    cudaEvent_t ev_solve = nullptr;
    // the batched solve
    GridBarrier *bars = nullptr;          // [n] one barrier per planet (zeroed before each launch)
    SolveParams *prm_host = nullptr;      // [n] pinned
    SolveParams *prm_dev = nullptr;       // [n]
    std::vector<std::vector<int>> groups;  // planets of each launch
    std::vector<size_t> group_smem;        // dynamic shared memory of each launch
    std::vector<int> blocks;               // blocks of each planet's solve
    int4 *bmap_host = nullptr, *bmap_dev = nullptr;  // [sum of blocks] block -> (planet, block, blocks)
    int bmap_cap = 0;
    int tune_steps = 0;     // batched steps over which the cost estimates are refined
    int fixed_blocks = 0;   // > 0: every planet's solve gets this many blocks (no tuning)
    double enqueue_ms = 0, wait_ms = 0, collect_ms = 0;  // host time of the last step's three parts
    double solve_ms = 0;  // device time of the last step's slowest planet solve
};

static int n_cells(const GGBBatch *b, int i) { return b->F[i]->cs->ncells; }
static int grid_n(const GGBBatch *b, int i) { return b->F[i]->cs->N; }

// Blocks per planet of one launch: minimise the largest estimated finishing
// time  cost(N_i) * cells_i / blocks_i  with sum blocks_i <= cap, blocks_i >= 1
// (binary search on the finishing time).  Unknown costs count as the
// smallest known cost of that precision (or 1), which makes the first split
// proportional to the planets' cells.
static void allocate(GGBBatch *b, const std::vector<int> &grp, int cap) {
    const int mixed = fluid_solve_mixed(b->F[grp[0]]);
    std::vector<double> w(grp.size());
    double known = 0;
    for (size_t k = 0; k < grp.size(); k++) {
        double c = cost_of(grid_n(b, grp[k]), mixed);
        if (c > 0) known = known > 0 ? std::min(known, c) : c;
    }
    for (size_t k = 0; k < grp.size(); k++) {
        double c = cost_of(grid_n(b, grp[k]), mixed);
        w[k] = (c > 0 ? c : (known > 0 ? known : 1.0)) * n_cells(b, grp[k]);
    }
    auto need = [&](double T) {
        long s = 0;
        for (size_t k = 0; k < grp.size(); k++) s += std::max(1L, (long)std::ceil(w[k] / T));
        return s;
    };
    double lo = 0, hi = *std::max_element(w.begin(), w.end());  // at T = hi every planet needs 1 block
    for (int it = 0; it < 60; it++) {
        double mid = 0.5 * (lo + hi);
        if (need(mid) <= cap)
            hi = mid;
        else
            lo = mid;
    }
    long used = 0;
    for (size_t k = 0; k < grp.size(); k++) {
        b->blocks[grp[k]] = std::max(1, (int)std::ceil(w[k] / hi));
        used += b->blocks[grp[k]];
    }
    // blocks left over go to the planets with the largest time per block (a
    // planet never gets more than one block per 512 cells)
    while (used < cap) {
        long best = -1;
        double bt = -1;
        for (size_t k = 0; k < grp.size(); k++) {
            if ((long)b->blocks[grp[k]] * 512 >= n_cells(b, grp[k])) continue;
            const double t = w[k] / b->blocks[grp[k]];
            if (t > bt) {
                bt = t;
                best = (long)k;
            }
        }
        if (best < 0) break;
        b->blocks[grp[best]]++;
        used++;
    }
}

// Launch groups (planets of one precision, at most cap of them each), block
// shares and the block map.
static void plan(GGBBatch *b) {
    b->groups.clear();
    b->group_smem.clear();
    b->blocks.assign(b->n, 1);
    std::vector<int> order[2];
    for (int i = 0; i < b->n; i++) order[fluid_solve_mixed(b->F[i])].push_back(i);
    int total = 0;
    for (int m = 0; m < 2; m++) {
        if (order[m].empty()) continue;
        // the launch's shared memory: the largest of its planets' needs
        size_t smem = 0;
        for (int i : order[m]) smem = std::max(smem, pcg_launch_smem(b->prm_host[i]));
        const int cap = pcg_batch_capacity(smem, m == 1);
        if (b->fixed_blocks >= cap) {
            // every planet alone on the whole launch: one launch per planet,
            // the same blocks (and so the same arithmetic) as fluid_step's solve
            for (int i : order[m]) {
                b->blocks[i] = cap;
                total += cap;
                b->groups.push_back(std::vector<int>{i});
                b->group_smem.push_back(smem);
            }
            continue;
        }
        for (size_t k0 = 0; k0 < order[m].size(); k0 += cap) {
            std::vector<int> grp(order[m].begin() + k0,
                                 order[m].begin() + std::min(order[m].size(), k0 + (size_t)cap));
            if (b->fixed_blocks > 0) {
                // a fixed share, scaled down when the launch cannot hold it
                const int per = std::max(1, std::min(b->fixed_blocks, cap / (int)grp.size()));
                for (int i : grp) b->blocks[i] = per;
            } else {
                allocate(b, grp, cap);
            }
            for (int i : grp) total += b->blocks[i];
            b->groups.push_back(grp);
            b->group_smem.push_back(smem);
        }
    }
    if (total > b->bmap_cap) {
        cudaFreeHost(b->bmap_host);
        dev_free(b->bmap_dev);
        GGB_CHECK(cudaMallocHost(&b->bmap_host, sizeof(int4) * total));
        b->bmap_dev = (int4 *)dev_alloc(sizeof(int4) * total);
        b->bmap_cap = total;
    }
    int q = 0;
    for (auto &grp : b->groups)
        for (int i : grp)
            for (int k = 0; k < b->blocks[i]; k++) b->bmap_host[q++] = make_int4(i, k, b->blocks[i], 0);
    GGB_CHECK(cudaMemcpyAsync(b->bmap_dev, b->bmap_host, sizeof(int4) * total, cudaMemcpyHostToDevice, stream()));
}

// The planets' solve parameters (they hold the planets' buffers, which do not
// move, and the precision, which ggb_fluid_set_precision may change).
static void refresh_params(GGBBatch *b) {
    sync();  // the pinned parameter and block-map buffers may still be in use by queued copies
    for (int i = 0; i < b->n; i++) fluid_step_solve_params(b->F[i], b->bars + i, b->prm_host + i);
    GGB_CHECK(cudaMemcpyAsync(b->prm_dev, b->prm_host, sizeof(SolveParams) * b->n, cudaMemcpyHostToDevice,
                              stream()));
    plan(b);
}

// Cost estimates from the last step's solve times.
static void tune(GGBBatch *b) {
    std::map<std::pair<int, int>, std::pair<double, int>> acc;
    for (int i = 0; i < b->n; i++) {
        const double t = fluid_last_solve_seconds(b->F[i]);
        if (t <= 0) continue;
        auto &a = acc[{grid_n(b, i), fluid_solve_mixed(b->F[i])}];
        a.first += t * b->blocks[i] / n_cells(b, i);
        a.second++;
    }
    for (auto &kv : acc) cost_update(kv.first.first, kv.first.second, kv.second.first / kv.second.second);
}

GGB_EXPORT GGBBatch *ggb_batch_create(int n, Fluid *const *F, Particles *const *P, Render *const *r,
                                      const double *cfl, const double *fade) {
    if (n < 1 || !F || !cfl) {
        fprintf(stderr, "ggb_batch_create: need n >= 1 planets with fluids and CFL numbers\n");
        return nullptr;
    }
    for (int i = 0; i < n; i++) {
        if (!F[i] || !F[i]->cs || (P && P[i] && (!r || !r[i] || !fade))) {
            fprintf(stderr, "ggb_batch_create: planet %d: a fluid is required, and particles need faces and a fade\n",
                    i);
            return nullptr;
        }
    }
    GGBBatch *b = new GGBBatch();
    b->n = n;
    for (int i = 0; i < n; i++) {
        b->F.push_back(F[i]);
        b->P.push_back(P ? P[i] : nullptr);
        b->r.push_back(r ? r[i] : nullptr);
        b->cfl.push_back(cfl[i]);
        b->fade.push_back(fade ? fade[i] : 0.0);
        cudaStream_t s;
        GGB_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        b->st.push_back(s);
    }
    b->dt_dev = (double *)dev_alloc(sizeof(double) * n);
    b->vmax_dev = (unsigned int *)dev_alloc(sizeof(unsigned int) * n);
    // per-planet arguments and block maps of the batched stages (fixed for the batch)
    {
        std::vector<PlanetStepDev> st(n);
        std::vector<int4> cm, pm;
        for (int i = 0; i < n; i++) {
            fluid_step_dev(b->F[i], b->cfl[i], b->dt_dev + i, b->vmax_dev + i, &st[i]);
            particles_step_dev(b->P[i], &st[i]);
            b->any_bfecc |= st[i].bfecc != 0;
            const int cb = (int)batch_cell_blocks(b->F[i]->cs->ncells);
            for (int k = 0; k < cb; k++) cm.push_back(make_int4(i, k, cb, 0));
            if (st[i].np > 0) {
                const int pb = (int)batch_particle_blocks(st[i].np);
                for (int k = 0; k < pb; k++) pm.push_back(make_int4(i, k, pb, 0));
            }
        }
        b->cell_blocks = (int)cm.size();
        b->part_blocks = (int)pm.size();
        b->steps_dev = (PlanetStepDev *)dev_alloc(sizeof(PlanetStepDev) * n);
        b->cell_map = (int4 *)dev_alloc(sizeof(int4) * cm.size());
        b->part_map = (int4 *)dev_alloc(sizeof(int4) * std::max<size_t>(1, pm.size()));
        GGB_CHECK(cudaMemcpy(b->steps_dev, st.data(), sizeof(PlanetStepDev) * n, cudaMemcpyHostToDevice));
        GGB_CHECK(cudaMemcpy(b->cell_map, cm.data(), sizeof(int4) * cm.size(), cudaMemcpyHostToDevice));
        if (!pm.empty()) GGB_CHECK(cudaMemcpy(b->part_map, pm.data(), sizeof(int4) * pm.size(), cudaMemcpyHostToDevice));
    }
    b->bars = (GridBarrier *)dev_alloc(sizeof(GridBarrier) * n);
    GGB_CHECK(cudaMallocHost(&b->prm_host, sizeof(SolveParams) * n));
    b->prm_dev = (SolveParams *)dev_alloc(sizeof(SolveParams) * n);
    GGB_CHECK(cudaEventCreateWithFlags(&b->ev_solve, cudaEventDisableTiming));
    b->tune_steps = 4;
    sync();
    return b;
}

// Fixed blocks per planet solve (blocks > 0: that many for every planet,
// without tuning, and at or above the launch's capacity one launch per planet
// on all of it; 0: the autotuned shares; < 0: query).  Returns the setting.
GGB_EXPORT int ggb_batch_solve_blocks(GGBBatch *b, int blocks) {
    if (blocks >= 0) b->fixed_blocks = blocks;
    return b->fixed_blocks;
}

// The blocks each planet's solve ran on in the last step (host array of n).
GGB_EXPORT void ggb_batch_blocks(const GGBBatch *b, int *blocks) {
    for (int i = 0; i < b->n; i++) blocks[i] = (int)b->blocks.size() > i ? b->blocks[i] : 0;
}

// The time steps of the last batched step (host array of n).
GGB_EXPORT void ggb_batch_dt(const GGBBatch *b, double *dt) {
    GGB_CHECK(cudaMemcpy(dt, b->dt_dev, sizeof(double) * b->n, cudaMemcpyDeviceToHost));
}

GGB_EXPORT int ggb_batch_step(GGBBatch *b, int steps) {
    if (!b) return -1;
    const cudaStream_t base = stream();
    using clk = std::chrono::steady_clock;
    refresh_params(b);
    for (int k = 0; k < steps; k++) {
        const auto t0 = clk::now();
        // CFL dt, particles and advection of every planet: one launch per stage
        batch_cfl_launch(b->steps_dev, b->n, b->cell_map, b->cell_blocks, b->vmax_dev);
        batch_particles_launch(b->steps_dev, b->part_map, b->part_blocks);
        batch_advect_launch(b->steps_dev, b->cell_map, b->cell_blocks, b->any_bfecc);
        // the batched solves
        GGB_CHECK(cudaMemsetAsync(b->bars, 0, sizeof(GridBarrier) * b->n, base));
        int q = 0;
        for (size_t g = 0; g < b->groups.size(); g++) {
            const std::vector<int> &grp = b->groups[g];
            int nb = 0;
            for (int i : grp) nb += b->blocks[i];
            pcg_launch_batch(b->prm_dev, b->bmap_dev + q, nb, fluid_solve_mixed(b->F[grp[0]]) != 0, b->group_smem[g],
                             base);
            q += nb;
        }
        for (int i = 0; i < b->n; i++) fluid_result_queue(b->F[i]);
        batch_velocity_launch(b->steps_dev, b->cell_map, b->cell_blocks);
        GGB_CHECK(cudaEventRecord(b->ev_solve, base));
        // fade and splat per planet, each on its own stream
        for (int i = 0; i < b->n; i++) {
            if (!b->r[i]) continue;
            GGB_CHECK(cudaStreamWaitEvent(b->st[i], b->ev_solve, 0));
            set_stream(b->st[i]);
            render_fade(b->r[i], b->fade[i]);
            if (b->P[i]) render_deposit_queue(b->r[i], b->P[i]);
        }
        set_stream(nullptr);
        const auto t1 = clk::now();
        GGB_CHECK(cudaStreamSynchronize(base));
        for (int i = 0; i < b->n; i++) GGB_CHECK(cudaStreamSynchronize(b->st[i]));
        const auto t2 = clk::now();
        double smax = 0;
        for (int i = 0; i < b->n; i++) {
            set_stream(b->st[i]);
            fluid_step_collect(b->F[i]);
            smax = std::max(smax, fluid_last_solve_seconds(b->F[i]));
            if (b->r[i] && b->P[i]) render_deposit_collect(b->r[i], b->P[i]);
        }
        set_stream(nullptr);
        b->solve_ms = 1000 * smax;
        if (b->fixed_blocks <= 0 && b->tune_steps > 0) {
            tune(b);
            b->tune_steps--;
            plan(b);
        }
        const auto t3 = clk::now();
        b->enqueue_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
        b->wait_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
        b->collect_ms = std::chrono::duration<double, std::milli>(t3 - t2).count();
    }
    set_stream(nullptr);
    return 0;
}

// Diagnostics: host time (ms) of the last batched step's queueing, waiting
// for the GPU, and collecting; returns the queueing time.
GGB_EXPORT double ggb_batch_host_ms(const GGBBatch *b, double *wait_ms, double *collect_ms) {
    if (wait_ms) *wait_ms = b->wait_ms;
    if (collect_ms) *collect_ms = b->collect_ms;
    return b->enqueue_ms;
}

// Device time (ms) of the last step's batched solves (the slowest planet's).
GGB_EXPORT double ggb_batch_solve_ms(const GGBBatch *b) { return b->solve_ms; }

// The autotuner's current cost estimate for grid N (precision mixed): device
// seconds per cell for one block of the solve; 0 when not measured yet.
GGB_EXPORT double ggb_batch_cost(int N, int mixed) { return cost_of(N, mixed); }

GGB_EXPORT void ggb_batch_free(GGBBatch *b) {
    if (!b) return;
    for (cudaStream_t s : b->st) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    sync();
    dev_free(b->dt_dev);
    dev_free(b->vmax_dev);
    dev_free(b->steps_dev);
    dev_free(b->cell_map);
    dev_free(b->part_map);
    dev_free(b->bars);
    dev_free(b->prm_dev);
    dev_free(b->bmap_dev);
    cudaFreeHost(b->prm_host);
    cudaFreeHost(b->bmap_host);
    cudaEventDestroy(b->ev_solve);
    delete b;
}
