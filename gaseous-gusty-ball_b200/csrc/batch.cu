// batch.cu — many planets advanced together: ggb_batch_create / _step / _free.
//
// A planet is the usual set of objects (cs_init, fluid_init, particles_init,
// render_init; grids may be shared between planets of the same N).  One
// batched step is the application driver's step for every planet (upstream
// src/main.c:421-434: CFL dt from the maximum speed, particles_advect,
// fluid_step, render_fade, render_deposit), with three differences from
// calling those entry points planet after planet:
//   - each planet's work is queued on its own stream, so the kernels of
//     different planets overlap on the GPU;
//   - the CFL dt is computed on the device (same expression, same IEEE
//     square root and division as the driver, so the same dt), so nothing
//     returns to the host inside a step;
//   - a planet's solve runs on a grid proportional to its size (one block
//     per `cells_per_block` cells, at most one per SM), so small planets take
//     a share of the SMs and several solves run at once.
// The host synchronises once per batched step, then reads each solve's
// statistics and checks each deposit's record buffer (growing it and
// repeating that planet's compositing in the rare step where it was short).
// Results equal the per-planet entry points' up to the relaxation factor of
// the forcing, 1 - exp(-forcing dt), which the device computes with its own
// exp (last-bit differences).
#include <chrono>
#include <cstdio>
#include <vector>

#include "ggb_internal.h"

struct GGBBatch {
    int n = 0;
    std::vector<Fluid *> F;
    std::vector<Particles *> P;
    std::vector<Render *> r;
    std::vector<double> cfl, fade;
    std::vector<cudaStream_t> st;
    double *dt_dev = nullptr;  // [n] device-side time steps
    int cells_per_block = 2048;
    cudaEvent_t fork = nullptr;
    double enqueue_ms = 0, wait_ms = 0, collect_ms = 0;  // host time of the last step's three parts
};

using namespace ggb;

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
    GGB_CHECK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    sync();
    return b;
}

// Cells per block of the batched solves (default 2048); returns the value in use.
GGB_EXPORT int ggb_batch_cells_per_block(GGBBatch *b, int cells) {
    if (cells > 0) b->cells_per_block = cells;
    return b->cells_per_block;
}

// The time steps of the last batched step (host array of n).
GGB_EXPORT void ggb_batch_dt(const GGBBatch *b, double *dt) {
    GGB_CHECK(cudaMemcpy(dt, b->dt_dev, sizeof(double) * b->n, cudaMemcpyDeviceToHost));
}

GGB_EXPORT int ggb_batch_step(GGBBatch *b, int steps) {
    if (!b) return -1;
    const cudaStream_t base = stream();
    using clk = std::chrono::steady_clock;
    for (int k = 0; k < steps; k++) {
        const auto t0 = clk::now();
        // every planet's stream starts after the work already queued on the library stream
        GGB_CHECK(cudaEventRecord(b->fork, base));
        for (int i = 0; i < b->n; i++) {
            GGB_CHECK(cudaStreamWaitEvent(b->st[i], b->fork, 0));
            set_stream(b->st[i]);
            Fluid *F = b->F[i];
            const int blocks = (F->cs->ncells + b->cells_per_block - 1) / b->cells_per_block;
            fluid_cfl_dt_launch(F, b->cfl[i], b->dt_dev + i);
            if (b->P[i]) particles_advect_queue(b->P[i], F->cs, F->vel, b->dt_dev + i);
            fluid_step_queue(F, b->dt_dev + i, blocks);
            if (b->r[i]) {
                render_fade(b->r[i], b->fade[i]);
                if (b->P[i]) render_deposit_queue(b->r[i], b->P[i]);
            }
        }
        const auto t1 = clk::now();
        for (int i = 0; i < b->n; i++) GGB_CHECK(cudaStreamSynchronize(b->st[i]));
        const auto t2 = clk::now();
        for (int i = 0; i < b->n; i++) {
            set_stream(b->st[i]);
            fluid_step_collect(b->F[i]);
            if (b->r[i] && b->P[i]) render_deposit_collect(b->r[i], b->P[i]);
        }
        set_stream(nullptr);
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

GGB_EXPORT void ggb_batch_free(GGBBatch *b) {
    if (!b) return;
    for (cudaStream_t s : b->st) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    dev_free(b->dt_dev);
    cudaEventDestroy(b->fork);
    delete b;
}
