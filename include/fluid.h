/* fluid.h — barotropic vorticity / stream-function solver on the cubed sphere:
 *
 *   d(omega)/dt + u . grad(omega) = forcing,   Laplacian(psi) = omega,
 *   u = r_hat x grad(psi).
 *
 * Drop-in for upstream gaseous-gusty-ball src/fluid.h (same struct layouts and
 * signatures).  In libggb_cuda.so every array field of Fluid is CUDA managed
 * memory that the GPU updates in place; each entry point below returns only
 * after its GPU work has finished, so callers may read or write the fields
 * between calls exactly as with the upstream CPU code.
 */
#ifndef GGB_FLUID_H
#define GGB_FLUID_H

#include "cubesphere.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Upstream src/fluid.h:12-19. */
typedef struct {
	double forcing;  /* relaxation rate toward the band vorticity (0 = off) */
	double rotation; /* planetary rotation rate for the Coriolis term (0 = off) */
	int bfecc;       /* BFECC (back-and-forth error compensated) advection */
	double cg_tol;   /* PCG relative residual tolerance */
	int cg_maxit;    /* PCG iteration cap */
	int multigrid;   /* multigrid V-cycle preconditioner (else Jacobi) */
} FluidParams;

/* One multigrid level.  Upstream src/fluid.h:21-31.  libggb_cuda.so fills
 * `cs` with the level's grid size fields only and keeps the level's arrays
 * (device-resident, face-tiled) privately; the pointer fields are NULL. */
typedef struct {
	CubeSphere cs;
	float *x, *b, *r, *dinv;
	int *ptap;
	float *pw;
	int *rstart;
	int *ridx;
	float *rw;
} MGLevel;

/* Upstream src/fluid.h:33-47.  `lev` points into library-owned storage. */
typedef struct {
	const CubeSphere *cs;
	FluidParams prm;
	int nlev;
	MGLevel *lev;
	float *omega;      /* relative vorticity */
	float *omega_band; /* forcing target (zeros when unused) */
	float *psi;        /* stream function */
	float *vel;        /* [ncells*3] tangent velocity */
	float *q0, *q1, *q2;
	float *dep_b, *dep_f;          /* [ncells*3] backward / forward departure points */
	float *r, *p, *Ap, *z, *dinv;  /* PCG work vectors and inverse diagonal */
	int cg_iters;      /* iterations of the last solve */
	double cg_relres;  /* relative residual at the end of the last solve */
} Fluid;

/* Upstream src/fluid.h:49-64. */
int fluid_init(Fluid *F, const CubeSphere *cs, const FluidParams *prm);
void fluid_free(Fluid *F);

/* Discrete operators on [ncells] / [ncells*3] arrays (host or device pointers). */
void fluid_curl(const CubeSphere *cs, const float *vel, float *omega);
void fluid_divergence(const CubeSphere *cs, const float *vel, float *div);
void fluid_laplacian(const CubeSphere *cs, const float *x, float *y);
void fluid_remove_mean(const CubeSphere *cs, float *f);

/* Initial state from a velocity field (vel_band may be NULL). */
void fluid_set_state(Fluid *F, const float *vel_initial, const float *vel_band);
/* Warm-started PCG for Laplacian(psi) = omega; returns the iteration count. */
int fluid_solve_psi(Fluid *F);
void fluid_compute_velocity(Fluid *F);
void fluid_step(Fluid *F, double dt);
double fluid_max_speed(const Fluid *F);

#ifdef __cplusplus
}
#endif

#endif
