/* cubesphere.h — equiangular cubed-sphere grid: cell geometry, spherical-Voronoi
 * operator tables and point location / bilinear sampling.
 *
 * Drop-in for upstream gaseous-gusty-ball src/cubesphere.h.  The struct layout,
 * field meaning and function signatures are identical (callers allocate
 * CubeSphere themselves and read its fields), so the upstream driver and tests
 * compile against this header and link against libggb_cuda.so unchanged.
 *
 * Face numbering / basis (upstream src/cubesphere.c:8-10): face 0 = +Z,
 * 1 = +X, 2 = -Z, 3 = -X, 4 = +Y (north), 5 = -Y (south).  On face f, cell
 * (i, j) has i growing along cs_face_right[f] and j along cs_face_up[f];
 * its flat index is (f*N + j)*N + i.
 *
 * In libggb_cuda.so the table arrays below live in CUDA managed memory: the
 * GPU kernels read them in place and host code may dereference them after
 * cs_init returns.  The library additionally keeps private, face-tiled copies
 * of the operator tables on the device (looked up through the `pos` pointer).
 */
#ifndef GGB_CUBESPHERE_H
#define GGB_CUBESPHERE_H

#include "vec3.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Face basis: centre, right and up unit vectors.  Upstream src/cubesphere.h:29-31. */
extern const vec3 cs_face_center[6];
extern const vec3 cs_face_right[6];
extern const vec3 cs_face_up[6];

/* Maximum Voronoi neighbours kept per cell.  Upstream src/cubesphere.h:33. */
#define CS_MAXNB 8

/* Upstream src/cubesphere.h:35-50 (same field order and types). */
typedef struct {
	int N;              /* cells along a face edge */
	int ncells;         /* 6*N*N */
	double h;           /* angular cell width, (pi/2)/N */
	float *pos;         /* [ncells*3] unit cell centres */
	float *area;        /* [ncells] spherical Voronoi cell area */
	unsigned char *nnb; /* [ncells] Voronoi neighbour count (<= CS_MAXNB) */
	int *nbr;           /* [ncells*CS_MAXNB] neighbour cell indices */
	float *w;           /* [ncells*CS_MAXNB] Laplacian weights edge length / centre distance */
	float *elen;        /* [ncells*CS_MAXNB] Voronoi edge length (radians) */
	float *gc;          /* [ncells*CS_MAXNB*3] least-squares gradient coefficients:
	                     * grad f(i) ~ sum_k gc_k * (f(nbr_k) - f(i)) */
	double total_area;  /* sum of cell areas (should be 4*pi) */
	int asym_count;     /* non-reciprocal Voronoi links dropped (should be 0) */
	int open_cells;     /* cells not closed by their candidates (should be 0) */
} CubeSphere;

/* Build the grid for N cells per face edge.  Returns 0, or -1 with a message
 * on stderr.  Upstream src/cubesphere.h:52, src/cubesphere.c:233-359. */
int cs_init(CubeSphere *cs, int N);
/* Release everything cs_init allocated and zero the struct.  Upstream src/cubesphere.c:361-371. */
void cs_free(CubeSphere *cs);

/* Face whose axis has the largest |component| of d.  Upstream src/cubesphere.c:12-20. */
int cs_face_of(vec3 d);
/* Unit direction for equiangular face angles (a, b).  Upstream src/cubesphere.c:22-27. */
vec3 cs_face_ab_to_dir(int f, double a, double b);
/* Continuous cell coordinates of d (cell centres at integers).  Upstream src/cubesphere.c:29-38. */
void cs_locate(const CubeSphere *cs, vec3 d, int *f, double *x, double *y);
/* Index of the cell containing d.  Upstream src/cubesphere.c:40-51. */
int cs_cell_of(const CubeSphere *cs, vec3 d);
/* Bilinear taps at p (4 cell indices, 4 weights).  Upstream src/cubesphere.c:68-92. */
void cs_taps(const CubeSphere *cs, vec3 p, int idx[4], double wt[4]);
/* Bilinear sample of a scalar field.  Upstream src/cubesphere.c:94-100. */
double cs_sample_scalar(const CubeSphere *cs, const float *fld, vec3 p);
/* Bilinear sample of a [ncells*3] vector field, projected to the tangent
 * plane at p.  Upstream src/cubesphere.c:102-111. */
vec3 cs_sample_vec(const CubeSphere *cs, const float *fld3, vec3 p);

/* Upstream src/cubesphere.h:68-73. */
static inline int cs_index(const CubeSphere *cs, int f, int i, int j)
{
	return (f * cs->N + j) * cs->N + i;
}

static inline vec3 cs_pos(const CubeSphere *cs, int c) { return v3_load(cs->pos + 3 * c); }

#ifdef __cplusplus
}
#endif

#endif
