/* render.h — fading, "over"-blended particle-trail splatting into the six
 * cube-face images (gnomonic projection, face basis of cubesphere.h; pixel
 * row 0 is the top of a face image).
 *
 * Drop-in for upstream gaseous-gusty-ball src/render.h (same layouts and
 * signatures).  `buf` holds premultiplied RGBA divided by the global decay
 * factor g, so fading costs O(1) per step (upstream src/render.h:1-8).
 *
 * In libggb_cuda.so `buf` is CUDA managed memory written by GPU kernels,
 * `tr` points to library-private device state, and sorted / sorted_cap /
 * bin_start / maxthreads are unused (zero).  render_texel and
 * render_sample_dir may be called concurrently from many host threads: the
 * first call after a deposit copies the face buffer to a host mirror once,
 * under a lock, and later calls read the mirror.
 */
#ifndef GGB_RENDER_H
#define GGB_RENDER_H

#include <stddef.h>
#include <stdint.h>

#include "particles.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Upstream src/render.h:17-21 (kept for layout compatibility). */
typedef struct {
	float px, py;
	uint32_t pidx;
	uint32_t bin;
} SplatRec;

/* Upstream src/render.h:23-28 (kept for layout compatibility). */
typedef struct {
	SplatRec *v;
	size_t n, cap;
	size_t *hist;
	size_t *cursor;
} ThreadRecs;

/* Upstream src/render.h:30-42. */
typedef struct {
	int R;          /* face resolution */
	float *buf;     /* [6*R*R*4] premultiplied RGBA / g, face-major, row-major */
	double g;       /* global decay factor */
	float radius;   /* splat radius in texels (>= 0.75) */
	float alpha;    /* per-splat opacity */
	int strip_h, nstrips, nbins;
	int maxthreads;
	ThreadRecs *tr;
	SplatRec *sorted;
	size_t sorted_cap;
	size_t *bin_start;
} Render;

/* Upstream src/render.h:44-54. */
int render_init(Render *r, int R, float radius, float alpha);
void render_free(Render *r);
void render_fade(Render *r, double fade);
void render_deposit(Render *r, const Particles *P);
/* Premultiplied RGBA of one texel. */
void render_texel(const Render *r, int face, int x, int y, float out[4]);
/* Bilinear sample in direction (dx, dy, dz), premultiplied RGBA. */
void render_sample_dir(const Render *r, double dx, double dy, double dz, float out[4]);
/* Premultiplied RGBA to 8 bit: bg == NULL gives un-premultiplied RGBA, else
 * RGB composited over bg. */
void render_pixel8(const float c[4], const float *bg, unsigned char *out);

#ifdef __cplusplus
}
#endif

#endif
