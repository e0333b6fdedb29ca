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
/* The next solves record up to `cap` (mark, nanoseconds) pairs of their phase
 * schedule (cap = 0: off); ggb_solve_trace copies them out, returns the count. */
void ggb_solve_trace_enable(int cap);
int ggb_solve_trace(unsigned long long *out, int cap);

/* ---- data ------------------------------------------------------------- */

/* All texels of the faces (premultiplied RGBA times g, as render_texel gives
 * them) into out[6*R*R*4], host or device memory, with one device copy. */
void ggb_render_read(const Render *r, float *out);

/* Diagnostics of the last render_deposit: number of texel tiles, tiles that
 * took the sorted fallback path, and (particle, tile) list entries. */
void ggb_render_stats(const Render *r, unsigned *ntiles, unsigned *slow_tiles, unsigned *entries);

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
 * (N <= 1672); larger grids, host buffers or a failed set-up return -1 with a
 * message and leave f unchanged, success returns 0.  The first call on a
 * device looks up the array's device address (once per device); make that
 * first call before any stream capture.  All calls share the array, so calls
 * whose GPU work overlaps (from several host threads) race. */
int ggb_remove_mean_noalloc(const CubeSphere *cs, float *f);

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
