/* noise.h — 3-D simplex noise with analytic gradient and multi-octave curl
 * noise, used to build initial velocity fields.
 *
 * Drop-in for upstream gaseous-gusty-ball src/noise.h (same layouts and
 * signatures); libggb_cuda.so implements these on the host, and a device
 * version of the same arithmetic builds per-planet initial conditions for the
 * batched API (ggb_batch.h).
 */
#ifndef GGB_NOISE_H
#define GGB_NOISE_H

#include "vec3.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Upstream src/noise.h:7-9. */
typedef struct {
	unsigned char perm[512];
} Noise;

/* Upstream src/noise.h:11-16. */
typedef struct {
	double scale;      /* base frequency on the unit sphere */
	double lacunarity; /* frequency ratio between octaves */
	double gain;       /* amplitude ratio between octaves */
	int octaves;
} CurlParams;

/* Seeded permutation table.  Upstream src/noise.c:12-31. */
void noise_init(Noise *nz, unsigned int seed);
/* Noise value at p; writes the analytic gradient to g when g != NULL.  Upstream src/noise.c:33-79. */
double simplex3(const Noise *nz, vec3 p, vec3 *g);
/* Divergence-free 3-D curl noise (not projected).  Upstream src/noise.c:81-103. */
vec3 curl_noise(const Noise *nz, vec3 p, const CurlParams *cp);

#ifdef __cplusplus
}
#endif

#endif
