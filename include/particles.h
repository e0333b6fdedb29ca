/* particles.h — passive coloured tracer particles on the unit sphere.
 *
 * Drop-in for upstream gaseous-gusty-ball src/particles.h (same layout and
 * signatures).  In libggb_cuda.so pos / prev / col are CUDA managed memory
 * updated in place by GPU kernels; entry points return after the GPU is done.
 */
#ifndef GGB_PARTICLES_H
#define GGB_PARTICLES_H

#include "cubesphere.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Upstream src/particles.h:7-12. */
typedef struct {
	int n;
	float *pos;  /* [n*3] current positions */
	float *prev; /* [n*3] positions before the last advection step */
	float *col;  /* [n*4] RGBA colours */
} Particles;

/* Fibonacci-lattice positions, colour 1.  Upstream src/particles.c:8-31. */
int particles_init(Particles *P, int n);
void particles_free(Particles *P);
/* Bilinear equirectangular colour lookup (x wraps in longitude, row 0 = north).
 * `img` is w*h RGBA floats (host or device pointer).  Upstream src/particles.c:41-61. */
void particles_color_from_image(Particles *P, const float *img, int w, int h);
/* RK2 midpoint advection along great circles; saves prev.  Upstream src/particles.c:63-74. */
void particles_advect(Particles *P, const CubeSphere *cs, const float *vel, double dt);

#ifdef __cplusplus
}
#endif

#endif
