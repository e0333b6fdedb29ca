/* ggb_ext.h — entry points of libggb_cuda.so that have no upstream
 * counterpart: device selection, synchronisation, timing and diagnostics,
 * bulk read-back, batched point location, and the GPU version of the
 * application driver's initial condition.  All are additive; the upstream
 * API in cubesphere.h / fluid.h / particles.h / render.h / noise.h is
 * unchanged.
 */
#ifndef GGB_EXT_H
#define GGB_EXT_H

#include "cubesphere.h"
#include "fluid.h"
#include "particles.h"
#include "render.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- runtime ---------------------------------------------------------- */

/* Selects the CUDA device used by every later call (call first). 0 / -1. */
int ggb_set_device(int dev);
/* Waits until all work issued by the library has finished. */
void ggb_sync(void);
/* Number of kernels the library has launched so far in this process. */
long ggb_launch_count(void);

/* ---- timing and diagnostics ------------------------------------------- */

/* CUDA-event interval on the library stream: start, then stop -> milliseconds. */
void ggb_timer_start(void);
double ggb_timer_stop(void);
/* Per-stage CUDA-event timing (on = 1 resets the totals).  ggb_stage_times
 * writes up to n totals (ms) and interval counts in the order particles,
 * advect, solve, velocity, max_speed, render binning, render tiles, and
 * returns the number of stages. */
void ggb_stage_timing(int on);
int ggb_stage_times(double *ms, long *count, int n);
/* Mean cost of one grid-wide barrier of the solve kernel's launch shape (us),
 * measured over `rounds` barriers; -1 if a barrier timed out. */
double ggb_barrier_bench(int rounds);
/* Failure detection without a GPU fault: one cooperative launch in which one
 * block never arrives at the grid barrier; the other blocks give up after
 * limit_ms, raise the barrier's error flag and return.  Returns 1 when the
 * waits ran out as they should (0 if the barrier completed), with the
 * launch's duration in *elapsed_ms.  The device stays usable afterwards. */
int ggb_barrier_timeout_probe(double limit_ms, double *elapsed_ms);
/* Status bits of the last Poisson solve of F (fluid_solve_psi, fluid_step,
 * fluid_set_state, a batched step): GGB_SOLVE_* below, 0 when the solve
 * converged normally.  The upstream API reports none of these: upstream
 * src/fluid.c:329-330 ends CG silently on p.Ap <= 0 and a NaN ends it with
 * relres NaN; the solve here behaves the same and records why. */
#define GGB_SOLVE_TIMEOUT 1   /* a grid barrier timed out (the process exits, as upstream on OOM) */
#define GGB_SOLVE_NONFINITE 2 /* NaN or Inf in b.b, r.r, r.z or p.Ap */
#define GGB_SOLVE_BREAKDOWN 4 /* p.Ap <= 0 stopped CG */
#define GGB_SOLVE_MAXIT 8     /* cg_maxit iterations without reaching cg_tol */
int ggb_solve_flags(const Fluid *F);
/* Checks the public grid arrays for corruption: non-finite or non-positive
 * areas, link weights and edge lengths, neighbour counts above 8 and
 * neighbour indices out of range.  Returns the number of bad entries (0 for
 * an intact grid).  The solve reads the operator tables built at cs_init,
 * not these arrays; a caller that edits them can detect it here. */
long ggb_grid_validate(const CubeSphere *cs);
/* Host-side fault injection for tests: after `after` more successful device
 * or managed allocations, every allocation of the library fails as if device
 * memory were exhausted (no allocator call is made); after < 0 turns it off.
 * cs_init, particles_init and render_init then return -1 with a message and
 * release what they had allocated (upstream's convention for these three);
 * other entry points end the process, as upstream does on OOM. */
void ggb_inject_alloc_failure(long after);
/* The next solves record up to `cap` (mark, nanoseconds) pairs of their phase
 * schedule (cap = 0: off); ggb_solve_trace copies them out, returns the count. */
void ggb_solve_trace_enable(int cap);
int ggb_solve_trace(unsigned long long *out, int cap);

/* ---- data ------------------------------------------------------------- */

/* All texels of the faces (premultiplied RGBA times g, as render_texel gives
 * them) into out[6*R*R*4], host or device memory, with one device copy. */
void ggb_render_read(const Render *r, float *out);

/* Diagnostics of the last render_deposit: number of 16x16 texel tiles, tiles
 * composited in several key-range windows, and the record slots reserved for
 * (sample, tile) records. */
void ggb_render_stats(const Render *r, unsigned *ntiles, unsigned *slow_tiles, unsigned *entries);
/* Diagnostics: how many times the fill and compositing of this Render's
 * deposits ran again (the record buffer grew, or a tile outgrew its estimated
 * reservation). */
unsigned long ggb_render_repeats(const Render *r);
/* Of ggb_render_repeats, those that followed a growth of the record buffer
 * (the others followed a tile that outgrew its estimated reservation). */
unsigned long ggb_render_repeats_grown(const Render *r);

/* The application driver's 8-bit output images (its write_outputs), encoded
 * on the GPU from the face buffer: render_texel then render_pixel8 per texel.
 * bg == NULL: transparent RGBA (4 channels), else RGB over bg[3] (3 channels).
 * out is host or device memory; returns 0, or -1 with a message.
 *  ggb_encode_faces:   6 images of R x R x ch, image k is face face_order[k]
 *                      (NULL: 0..5; the driver's GL layout is {1,3,4,5,0,2});
 *  ggb_encode_net:     the 4R x 3R RGBA cross net (cells without a face are 0);
 *  ggb_encode_preview: the 2R x R x ch equirectangular preview (render_sample_dir
 *                      at each pixel centre's longitude and latitude). */
int ggb_encode_faces(const Render *r, const float *bg, const int *face_order, unsigned char *out);
int ggb_encode_net(const Render *r, const float *bg, unsigned char *out);
int ggb_encode_preview(const Render *r, const float *bg, unsigned char *out);

/* cs_cell_of / cs_taps for n directions (dirs: n*3 doubles) on the GPU;
 * out: n ints; idx: n*4 ints, wt: n*4 doubles (host or device memory). */
void ggb_cell_of_batch(const CubeSphere *cs, const double *dirs, int n, int *out);
void ggb_taps_batch(const CubeSphere *cs, const double *dirs, int n, int *idx, double *wt);

/* No counterpart in the upstream code.  fluid_remove_mean without any device
 * allocation, for callers that cannot allocate: processes whose device memory
 * is entirely reserved up front by another allocator, and steady-state loops
 * that must not call cudaMalloc / cudaFree (both synchronise the device).
 * Removes the area-weighted mean of f[ncells] in place; f must already be
 * device or managed memory.  Its scratch is one fixed 32 KB device array per
 * GPU (held until the process exits), which limits grids to 16,777,216 cells
 * (N <= 1672).  Returns 0 on success.  Returns -1 with a message, f unchanged,
 * when the grid is unknown or larger than that, f is a host buffer, the
 * current device is not the one of the grid and the library stream, or the
 * scratch address cannot be looked up; -1 with f undefined when a launch or
 * the final synchronisation fails.  The first call on a device looks up the
 * array's device address (once per device).  Every call synchronises the
 * library stream before it returns, so it must not be called while that
 * stream is being captured.  All calls share the array, so calls whose GPU
 * work overlaps (from several host threads) race. */
int ggb_remove_mean_noalloc(const CubeSphere *cs, float *f);

/* Precision of F's Poisson solve.  mixed = 0 (the default): FP32 vectors with
 * FP64 stencil accumulation and the upstream CG.  mixed = 1: the multigrid
 * V-cycle stores its level vectors and the coarse levels' slot weights in
 * FP16 and accumulates in FP32, inside a flexible (Polak-Ribiere) FP32 CG;
 * psi, omega and u stay FP32, and the CG dots, the residual norm and the
 * zero-mean projections stay FP64.  Returns 0, or -1 when F has no multigrid
 * preconditioner.  The FluidParams layout of the upstream header is kept, so
 * the choice is made here rather than there. */
int ggb_fluid_set_precision(Fluid *F, int mixed);

/* Checkpoint / resume of a running planet.  save writes the state the next
 * steps read (omega, omega_band, psi, vel and the last solve's statistics; the
 * particles' pos, prev, col; the face buffer, g and a deferred fade
 * renormalisation) to `path`; P and r may be NULL.  load restores it into
 * objects initialised by fluid_init / particles_init / render_init with the
 * same grid, particle count and face resolution (checked; the fluid
 * parameters of F are kept), after which stepping continues bit-identically.
 * Both return 0, or -1 with a message (and leave the objects' state undefined
 * when a load fails part-way). */
int ggb_checkpoint_save(const char *path, const Fluid *F, const Particles *P, const Render *r);
int ggb_checkpoint_load(const char *path, Fluid *F, Particles *P, Render *r);

/* Batched planets.  A planet is the usual objects (cs_init, fluid_init,
 * particles_init, render_init; planets of the same N may share a grid).
 * ggb_batch_step advances every planet by `steps` application-driver steps
 * (CFL dt from the maximum speed, particles_advect, fluid_step, render_fade,
 * render_deposit).  The Poisson solves of all planets run in one persistent
 * cooperative launch, each planet on its own share of the blocks with its
 * own barrier and convergence test; the shares come from an autotuner that
 * estimates, from the solves' measured device times, a cost per cell for
 * every grid size and precision, and equalises the planets' estimated
 * finishing times (it refines the estimates over the first steps of a batch
 * and keeps them for the process).  The other stages are queued on one
 * stream per planet, the CFL dt is computed on the device, and the host
 * synchronises once per step.  P[i] and r[i] may be NULL (fluid only);
 * fade[i] is render_fade's argument.  Results equal the per-planet entry
 * points' up to the order of the solve's FP64 block sums (another number of
 * blocks) and the device's exp in the forcing's relaxation factor.  create
 * returns NULL with a message on bad arguments; step returns 0. */
typedef struct GGBBatch GGBBatch;
GGBBatch *ggb_batch_create(int n, Fluid *const *F, Particles *const *P, Render *const *r, const double *cfl,
                           const double *fade);
int ggb_batch_step(GGBBatch *b, int steps);
/* blocks > 0: every planet's solve gets that many blocks (no tuning; at or
 * above the launch's capacity, every planet is solved alone on all of it,
 * which reproduces fluid_step's arithmetic exactly); 0: the autotuned shares
 * (the default); < 0: query.  Returns the setting. */
int ggb_batch_solve_blocks(GGBBatch *b, int blocks);
void ggb_batch_blocks(const GGBBatch *b, int *blocks); /* each planet's blocks in the last step */
void ggb_batch_dt(const GGBBatch *b, double *dt);      /* the last step's dt per planet */
/* host time (ms) of the last step's queueing (returned), GPU wait and collection */
double ggb_batch_host_ms(const GGBBatch *b, double *wait_ms, double *collect_ms);
/* device time (ms) of the last step's batched solves (the slowest planet's) */
double ggb_batch_solve_ms(const GGBBatch *b);
/* the autotuner's estimate for grid N in the given precision: device seconds
 * per cell for one block of a solve (0: not measured yet) */
double ggb_batch_cost(int N, int mixed);
void ggb_batch_free(GGBBatch *b);

/* Initial-condition parameters of the application driver (bands and curl noise). */
typedef struct {
	int bands;
	double band_amp;
	double noise_amp, noise_scale, noise_lacunarity, noise_gain;
	int noise_octaves;
	unsigned int seed;
} GGBInitParams;

/* The application driver's initial velocity (projected curl noise scaled to
 * noise_amp RMS plus zonal bands; vband gets the bands alone), computed on the
 * GPU.  vel, vband: [ncells*3], host or device memory. */
void ggb_initial_velocity(const CubeSphere *cs, const GGBInitParams *ip, float *vel, float *vband);

#ifdef __cplusplus
}
#endif

#endif
