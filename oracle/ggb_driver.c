/* ggb_driver.c — run driver for the CPU checkers (test infrastructure only).
 *
 * Compiled twice: against the include/ headers with the restatement (ggb_oracle.c),
 * and against the upstream headers with the upstream sources (oracle/_ref).
 * It only calls the public grid / fluid / particle / render / noise API, so
 * the same code drives both CPU implementations:
 *   drv_initial_velocity — the initial condition of the application driver
 *                          (restates upstream src/main.c:321-360);
 *   drv_run              — the per-step loop of the application driver
 *                          without image output (upstream src/main.c:419-449),
 *                          timed with omp_get_wtime per phase.
 */
#include <math.h>
#include <omp.h>
#include <stdio.h>

#include "cubesphere.h"
#include "fluid.h"
#include "noise.h"
#include "particles.h"
#include "render.h"

typedef struct {
	int bands;
	double band_amp;
	double noise_amp, noise_scale, noise_lacunarity, noise_gain;
	int noise_octaves;
	unsigned int seed;
} DrvInit;

/* Curl noise projected to the sphere and scaled to RMS speed noise_amp,
 * plus zonal bands u_east = band_amp * sin(bands * colatitude).
 * vel and vband are [ncells*3].  Restates upstream src/main.c:321-351. */
void drv_initial_velocity(const CubeSphere *cs, const DrvInit *o, float *vel, float *vband)
{
	int n = cs->ncells;
	Noise nz;
	noise_init(&nz, o->seed);
	CurlParams cp = {o->noise_scale, o->noise_lacunarity, o->noise_gain, o->noise_octaves};
	double ss = 0;
#pragma omp parallel for schedule(static) reduction(+ : ss)
	for (int i = 0; i < n; i++) {
		vec3 p = cs_pos(cs, i);
		vec3 v = o->noise_octaves > 0 ? v3_tangent(curl_noise(&nz, p, &cp), p) : v3(0, 0, 0);
		v3_store(vel + 3 * i, v);
		ss += v3_dot(v, v) * cs->area[i];
	}
	double rms = sqrt(ss / cs->total_area);
	double sc = rms > 0 ? o->noise_amp / rms : 0;
#pragma omp parallel for schedule(static)
	for (int i = 0; i < n; i++) {
		vec3 p = cs_pos(cs, i);
		double colat = acos(p.y > 1 ? 1 : (p.y < -1 ? -1 : p.y));
		double s = sin(colat);
		double mag = o->band_amp * sin(o->bands * colat);
		vec3 east = v3_cross(v3(0, 1, 0), p);
		vec3 b = s > 1e-9 ? v3_scale(east, mag / s) : v3(0, 0, 0);
		v3_store(vband + 3 * i, b);
		v3_store(vel + 3 * i, v3_add(v3_scale(v3_load(vel + 3 * i), sc), b));
	}
}

/* `steps` iterations of: dt from the CFL number (or fixed_dt > 0),
 * particles_advect, fluid_step, render_fade, render_deposit.  Per step the dt
 * and CG iteration count are written when the arrays are non-NULL; phase
 * seconds (particles, fluid, render) accumulate into t_phase[3].
 * Returns the summed CG iterations.  Restates upstream src/main.c:421-438. */
long drv_run(const CubeSphere *cs, Fluid *F, Particles *P, Render *R, int steps, double cfl,
             double fixed_dt, double fade, double *dt_out, int *cg_out, double *t_phase)
{
	long cgsum = 0;
	for (int s = 0; s < steps; s++) {
		double dt = fixed_dt;
		if (dt <= 0) {
			double vmax = fluid_max_speed(F);
			dt = cfl * cs->h / (vmax > 1e-6 ? vmax : 1e-6);
		}
		double a = omp_get_wtime();
		particles_advect(P, cs, F->vel, dt);
		double b = omp_get_wtime();
		fluid_step(F, dt);
		double c = omp_get_wtime();
		render_fade(R, fade);
		render_deposit(R, P);
		double d = omp_get_wtime();
		cgsum += F->cg_iters;
		if (dt_out)
			dt_out[s] = dt;
		if (cg_out)
			cg_out[s] = F->cg_iters;
		if (t_phase) {
			t_phase[0] += b - a;
			t_phase[1] += c - b;
			t_phase[2] += d - c;
		}
	}
	return cgsum;
}

int drv_max_threads(void) { return omp_get_max_threads(); }
void drv_set_threads(int n) { omp_set_num_threads(n); }
