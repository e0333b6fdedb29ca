// ggb_internal.h — host-side internals of libggb_cuda.so: error handling, the
// library stream, allocation helpers, the launch counter and the private
// device-side tables attached to every CubeSphere / Fluid / Render.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "cubesphere.h"
#include "fluid.h"
#include "particles.h"
#include "render.h"
#include "ggb_ext.h"
#include "ggb_device.cuh"

#define GGB_EXPORT extern "C" __attribute__((visibility("default")))

namespace ggb {

[[noreturn]] void fail_cuda(const char *what, cudaError_t e, const char *file, int line);
[[noreturn]] void fail_msg(const char *fmt, ...);

#define GGB_CHECK(x)                                                         \
    do {                                                                     \
        cudaError_t e_ = (x);                                                \
        if (e_ != cudaSuccess) ::ggb::fail_cuda(#x, e_, __FILE__, __LINE__); \
    } while (0)

// Call after every kernel launch: counts it and surfaces launch errors.
#define GGB_LAUNCHED()                                                                 \
    do {                                                                               \
        ::ggb::note_launch(1);                                                         \
        cudaError_t e_ = cudaGetLastError();                                           \
        if (e_ != cudaSuccess) ::ggb::fail_cuda("kernel launch", e_, __FILE__, __LINE__); \
    } while (0)

void note_launch(long k);
long launch_count();

// The stream every entry point issues its work on; created on first use for
// the current device.  The batched API may redirect it while capturing.
cudaStream_t stream();
// The device the library's own stream was created on (-1 before the first stream()).
int stream_device();
void set_stream(cudaStream_t s);
void sync();
int device_sm_count();
// True when there is a usable CUDA device; entry points fail loudly otherwise.
bool have_device();

// Optional per-stage CUDA-event timing on the library stream (off by default).
enum Stage { ST_PARTICLES = 0, ST_ADVECT, ST_SOLVE, ST_VELOCITY, ST_MAXSPEED, ST_BIN, ST_TILES, ST_N };
void stage_begin(int s);
void stage_end(int s);
void stage_collect();  // after a stream sync: accumulate the recorded intervals

// Pieces of the batched step (batch.cu): every *_queue / *_launch call only
// queues work on stream(); the *_collect calls run after that stream has been
// synchronised.  dt_dev points at a device-side time step.
void fluid_cfl_dt_launch(const Fluid *F, double cfl, double *dt_dev);
void fluid_step_queue(Fluid *F, const double *dt_dev, int max_blocks);
void fluid_step_collect(Fluid *F);
// One planet's arguments of the batched per-cell and per-particle stages (one
// launch per stage for all planets; each block finds its planet, its block of
// that planet and the planet's block count in a block map of int4
// {planet, block, blocks, 0}).
struct PlanetStepDev {
    GridDev g;                 // the planet's grid
    const float *pos;          // [n*3] cell centres
    const unsigned char *nnb;  // [n]
    const int *nbr;            // [n*8]
    const float *gc;           // [n*24]
    float *vel, *omega, *omega_band, *psi, *q0, *q1, *q2, *dep_b, *dep_f;
    double two_omega, forcing, cfl;
    int bfecc;
    double *dt;                // device-side time step of the planet
    unsigned int *vmax;        // max |u|^2 as float bits
    int np;                    // particles (0: none)
    float *ppos, *pprev;
};
void fluid_step_dev(Fluid *F, double cfl, double *dt_dev, unsigned int *vmax_dev, PlanetStepDev *out);
void particles_step_dev(Particles *P, PlanetStepDev *out);
// The batched stages, queued on stream(): CFL dt (after zeroing the planets'
// vmax), particle advection, departures + BFECC + limiter, velocity.  map:
// block map of the planets' cells (nb blocks) or particles.
void batch_cfl_launch(const PlanetStepDev *pl, int n, const int4 *map, int nb, unsigned int *vmax_all);
void batch_particles_launch(const PlanetStepDev *pl, const int4 *map, int nb);
void batch_advect_launch(const PlanetStepDev *pl, const int4 *map, int nb, bool any_bfecc);
void batch_velocity_launch(const PlanetStepDev *pl, const int4 *map, int nb);
// blocks of the per-cell (per-particle) stages for a planet of n cells (particles)
unsigned batch_cell_blocks(int n);
unsigned batch_particle_blocks(int n);
// the result read-back of the last batched solve (fluid_result_velocity_queue without the velocity)
void fluid_result_queue(Fluid *F);

// The same step split around one batched solve launch (batch.cu): advection,
// the solve's parameters (with the barrier the batched launch assigns), and
// after the solve the result read-back and the velocity.
struct SolveParams;
void fluid_advect_queue(Fluid *F, const double *dt_dev);
void fluid_step_solve_params(Fluid *F, GridBarrier *bar, SolveParams *out);
int fluid_solve_mixed(const Fluid *F);
double fluid_last_solve_seconds(const Fluid *F);
void fluid_result_velocity_queue(Fluid *F);
size_t pcg_launch_smem(const SolveParams &p);
int pcg_batch_capacity(size_t smem, bool mixed);
void pcg_launch_batch(const SolveParams *dev_prm, const int4 *dev_bmap, int nblocks, bool mixed, size_t smem,
                      cudaStream_t s);
void render_deposit_queue(Render *r, const Particles *P);
void render_deposit_collect(Render *r, const Particles *P);
void particles_advect_queue(Particles *P, const CubeSphere *cs, const float *vel, const double *dt_dev);

// The deferred renormalisation of render_fade (private state of a Render).
void render_pending_get(const Render *r, int *pending, float *scale);
void render_pending_set(Render *r, int pending, float scale);
void render_particles_replaced(Render *r);

void *dev_alloc(size_t bytes);      // cudaMalloc, zero-filled; exits on failure
void dev_free(void *p);
void *managed_alloc(size_t bytes);  // cudaMallocManaged, zero-filled, resident on the device; exits on failure
// The same, returning nullptr when the allocation fails (for entry points
// that report failure with -1, as upstream's *_init do).
void *dev_try_alloc(size_t bytes);
void *managed_try_alloc(size_t bytes);
void managed_free(void *p);

inline unsigned grid_for(size_t n, int block) { return (unsigned)((n + block - 1) / block); }

// Face-tiled operator tables of one cubed-sphere grid (device memory).
//   wslot[s*n + c], s = 0..3: weight of the link from cell c to its on-face
//       neighbour at (+1,0) E, (0,+1) N, (+1,+1) NE, (-1,+1) NW (0 = no link).
//       The opposite directions of c are read from the neighbour's slots,
//       which hold the same (symmetric) weight.
//   ring_nb / ring_w [r*8 + k]: links of boundary-ring cell r that leave the
//       face (or the 3x3 box); -1 terminates.  Only ring cells have such links.
struct GridTables {
    int N = 0, n = 0, nring = 0;
    int device = -1;  // the CUDA device the tables live on
    double h = 0;
    bool managed = false;
    // upstream layout (managed memory for a public grid, device memory otherwise)
    float *pos = nullptr, *area = nullptr, *w = nullptr, *elen = nullptr, *gc = nullptr;
    unsigned char *nnb = nullptr;
    int *nbr = nullptr;
    // device-only
    int *ghost = nullptr;
    float *wslot = nullptr;
    double *wslot_d = nullptr;  // the same four slot weights in FP64 (staged solver phases)
    int *ring_nb = nullptr;
    float *ring_w = nullptr;
    float *dinv = nullptr;
    double total_area = 0;
    int asym_count = 0, open_cells = 0;

    GridDev dev() const {
        GridDev g;
        g.N = N;
        g.n = n;
        g.h = h;
        g.ghost = ghost;
        return g;
    }
};

inline int ring_count(int N) { return N == 1 ? 1 : 4 * N - 4; }

// Builds every table of an N grid on the GPU (FP64 geometry).  With
// managed = true the upstream-layout arrays are managed memory.  Returns 0, or
// -1 with a message on stderr.
int grid_build(GridTables *t, int N, bool managed);
void grid_release(GridTables *t);

// Registry: the private tables of a public CubeSphere, keyed by cs->pos.
GridTables *grid_lookup(const CubeSphere *cs);  // fails loudly when unknown
GridTables *grid_find(const CubeSphere *cs);    // nullptr when unknown

// Device copy of an argument that may live in pageable host memory: returns
// a device-accessible pointer to `bytes` bytes equal to `src` (staging it
// through `scratch` when needed).  copy_back() writes a staged buffer back.
struct Staged {
    void *dev = nullptr;
    void *host = nullptr;
    size_t bytes = 0;
    bool owned = false;
    ~Staged();
};
void stage_in(Staged &s, const void *src, size_t bytes);
void stage_out(Staged &s, void *dst, size_t bytes);  // for an output buffer
void stage_finish(Staged &s);                          // copies an output back to the host

}  // namespace ggb
