/* ggb_oracle.c — CPU restatement of the gaseous-gusty-ball per-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker of the parity tests: it
 * is built into oracle/_build/liboracle{32,64}.so and loaded only by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg.  The product
 * (gaseous-gusty-ball_b200/libggb_cuda.so) never links or calls it.
 *
 * It implements the API declared in include/{cubesphere,fluid,particles,
 * render,noise}.h, serially, in plain C, following the upstream algorithm
 * step by step (each function cites the upstream file:line it restates).
 * Floating-point expressions are written in the upstream evaluation order so
 * that, compiled with the same gcc flags, the one-pass outputs (grid tables,
 * operator applications, a render deposit) agree bit for bit with the
 * upstream build; reductions are summed serially in index order, so results
 * that pass through a reduction agree to rounding only.
 *
 * Built with -Dfloat=double it becomes the FP64 oracle (every stored array,
 * cast and sizeof switches to double), like the upstream all-double build.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "cubesphere.h"
#include "fluid.h"
#include "noise.h"
#include "particles.h"
#include "render.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ grid */

/* Face basis; upstream src/cubesphere.c:8-10 (this numbering is the file
 * format of the cube-face outputs, so it must be identical). */
const vec3 cs_face_center[6] = {{0, 0, 1}, {1, 0, 0}, {0, 0, -1}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
const vec3 cs_face_right[6] = {{1, 0, 0}, {0, 0, -1}, {-1, 0, 0}, {0, 0, 1}, {1, 0, 0}, {1, 0, 0}};
const vec3 cs_face_up[6] = {{0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

/* upstream src/cubesphere.c:12-20 — ties go to x, then y, then z. */
int cs_face_of(vec3 d)
{
	double ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
	if (ax >= ay && ax >= az)
		return d.x > 0 ? 1 : 3;
	if (ay >= az)
		return d.y > 0 ? 4 : 5;
	return d.z > 0 ? 0 : 2;
}

/* upstream src/cubesphere.c:22-27 */
vec3 cs_face_ab_to_dir(int f, double a, double b)
{
	vec3 off = v3_add(v3_scale(cs_face_right[f], tan(a)), v3_scale(cs_face_up[f], tan(b)));
	return v3_normalize(v3_add(cs_face_center[f], off));
}

/* upstream src/cubesphere.c:29-38 */
void cs_locate(const CubeSphere *cs, vec3 d, int *f, double *x, double *y)
{
	int face = cs_face_of(d);
	double dc = v3_dot(d, cs_face_center[face]);
	double u = v3_dot(d, cs_face_right[face]) / dc;
	double v = v3_dot(d, cs_face_up[face]) / dc;
	*f = face;
	*x = (atan(u) + M_PI / 4) / cs->h - 0.5;
	*y = (atan(v) + M_PI / 4) / cs->h - 0.5;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* upstream src/cubesphere.c:40-51 */
int cs_cell_of(const CubeSphere *cs, vec3 d)
{
	int f;
	double x, y;
	cs_locate(cs, d, &f, &x, &y);
	int i = clampi((int) floor(x + 0.5), 0, cs->N - 1);
	int j = clampi((int) floor(y + 0.5), 0, cs->N - 1);
	return cs_index(cs, f, i, j);
}

/* Centre direction of (possibly off-face) cell (i, j) of face f; upstream src/cubesphere.c:53-56. */
static vec3 centre_dir(const CubeSphere *cs, int f, int i, int j)
{
	return cs_face_ab_to_dir(f, -M_PI / 4 + (i + 0.5) * cs->h, -M_PI / 4 + (j + 0.5) * cs->h);
}

/* Cell (i, j) of face f; an off-face (ghost) cell is the real cell containing
 * its extended centre direction.  upstream src/cubesphere.c:61-66 */
static int ghost_index(const CubeSphere *cs, int f, int i, int j)
{
	int N = cs->N;
	if (i >= 0 && j >= 0 && i < N && j < N)
		return cs_index(cs, f, i, j);
	return cs_cell_of(cs, centre_dir(cs, f, i, j));
}

/* upstream src/cubesphere.c:68-92 */
void cs_taps(const CubeSphere *cs, vec3 p, int idx[4], double wt[4])
{
	int f, N = cs->N;
	double x, y;
	cs_locate(cs, p, &f, &x, &y);
	int i0 = (int) floor(x), j0 = (int) floor(y);
	double fx = x - i0, fy = y - j0;
	if (i0 >= 0 && j0 >= 0 && i0 + 1 < N && j0 + 1 < N) {
		int base = cs_index(cs, f, i0, j0);
		idx[0] = base;
		idx[1] = base + 1;
		idx[2] = base + N;
		idx[3] = base + N + 1;
	} else {
		for (int k = 0; k < 4; k++)
			idx[k] = ghost_index(cs, f, i0 + (k & 1), j0 + (k >> 1));
	}
	wt[0] = (1 - fx) * (1 - fy);
	wt[1] = fx * (1 - fy);
	wt[2] = (1 - fx) * fy;
	wt[3] = fx * fy;
}

/* upstream src/cubesphere.c:94-100 */
double cs_sample_scalar(const CubeSphere *cs, const float *fld, vec3 p)
{
	int idx[4];
	double wt[4];
	cs_taps(cs, p, idx, wt);
	return wt[0] * fld[idx[0]] + wt[1] * fld[idx[1]] + wt[2] * fld[idx[2]] + wt[3] * fld[idx[3]];
}

/* upstream src/cubesphere.c:102-111 */
vec3 cs_sample_vec(const CubeSphere *cs, const float *fld3, vec3 p)
{
	int idx[4];
	double wt[4];
	cs_taps(cs, p, idx, wt);
	vec3 acc = v3(0, 0, 0);
	for (int k = 0; k < 4; k++)
		acc = v3_add(acc, v3_scale(v3_load(fld3 + 3 * idx[k]), wt[k]));
	return v3_tangent(acc, p);
}

/* Spherical triangle area of unit vectors; upstream src/cubesphere.c:114-119. */
static double tri_area(vec3 a, vec3 b, vec3 c)
{
	double num = fabs(v3_dot(a, v3_cross(b, c)));
	double den = 1.0 + v3_dot(a, b) + v3_dot(b, c) + v3_dot(c, a);
	return 2.0 * atan2(num, den);
}

/* Voronoi construction in the gnomonic plane of the cell (bisectors of
 * sphere points are straight lines there).  upstream src/cubesphere.c:121-225 */
#define ORC_MAXPV 64
typedef struct {
	double a, b;
	int label; /* neighbour whose bisector starts at this vertex (-1: box) */
} OVert;

/* Keep the part of polygon `in` where A*a + B*b + C >= 0; upstream src/cubesphere.c:130-152. */
static int half_plane_clip(const OVert *in, int n, OVert *out, double A, double B, double C, int label)
{
	int m = 0;
	for (int k = 0; k < n; k++) {
		const OVert *v0 = &in[k], *v1 = &in[(k + 1) % n];
		double f0 = A * v0->a + B * v0->b + C;
		double f1 = A * v1->a + B * v1->b + C;
		int keep0 = f0 >= 0, keep1 = f1 >= 0;
		if (keep0 && m < ORC_MAXPV)
			out[m++] = *v0;
		if (keep0 != keep1) {
			double t = f0 / (f0 - f1);
			OVert cut;
			cut.a = v0->a + t * (v1->a - v0->a);
			cut.b = v0->b + t * (v1->b - v0->b);
			cut.label = keep0 ? label : v0->label;
			if (m < ORC_MAXPV)
				out[m++] = cut;
		}
	}
	return m;
}

typedef struct {
	int nb;
	double len;
} OLink;

static int voronoi_links(const CubeSphere *cs, int c, OLink *links, double *area, int *open)
{
	int N = cs->N;
	int f = c / (N * N), i = (c % (N * N)) % N, j = (c % (N * N)) / N;
	vec3 p = cs_pos(cs, c);
	vec3 e1 = v3_normalize(v3_tangent(cs_face_right[f], p));
	vec3 e2 = v3_cross(p, e1);

	/* candidates: the 5x5 window, row by row, deduplicated (upstream :166-180) */
	int cand[24], nc = 0;
	for (int dj = -2; dj <= 2; dj++)
		for (int di = -2; di <= 2; di++) {
			if (di == 0 && dj == 0)
				continue;
			int q = ghost_index(cs, f, i + di, j + dj);
			int seen = q == c;
			for (int k = 0; k < nc && !seen; k++)
				seen = cand[k] == q;
			if (!seen)
				cand[nc++] = q;
		}

	OVert A[ORC_MAXPV], B[ORC_MAXPV];
	OVert *poly = A, *spare = B;
	double S = 4 * cs->h;
	int n = 4;
	poly[0] = (OVert){-S, -S, -1};
	poly[1] = (OVert){S, -S, -1};
	poly[2] = (OVert){S, S, -1};
	poly[3] = (OVert){-S, S, -1};
	for (int k = 0; k < nc; k++) {
		vec3 m = v3_sub(p, cs_pos(cs, cand[k]));
		n = half_plane_clip(poly, n, spare, v3_dot(e1, m), v3_dot(e2, m), v3_dot(p, m), cand[k]);
		OVert *t = poly;
		poly = spare;
		spare = t;
	}

	int nl = 0;
	double ar = 0;
	*open = 0;
	for (int k = 0; k < n; k++) {
		const OVert *v0 = &poly[k], *v1 = &poly[(k + 1) % n];
		vec3 P0 = v3_normalize(v3_add(p, v3_add(v3_scale(e1, v0->a), v3_scale(e2, v0->b))));
		vec3 P1 = v3_normalize(v3_add(p, v3_add(v3_scale(e1, v1->a), v3_scale(e2, v1->b))));
		ar += tri_area(p, P0, P1);
		if (v0->label < 0) {
			*open = 1;
			continue;
		}
		double len = v3_angle(P0, P1);
		int l = 0;
		while (l < nl && links[l].nb != v0->label)
			l++;
		if (l < nl)
			links[l].len += len;
		else if (nl < 24) {
			links[nl].nb = v0->label;
			links[nl].len = len;
			nl++;
		}
	}
	*area = ar;
	return nl;
}

/* Descending by length with the C library qsort, as upstream does
 * (src/cubesphere.c:227-231, 273): qsort's order of equal lengths is part of
 * the upstream result (it fixes the link order, hence FP summation orders). */
static int link_longer_first(const void *pa, const void *pb)
{
	double la = ((const OLink *) pa)->len, lb = ((const OLink *) pb)->len;
	return la < lb ? 1 : (la > lb ? -1 : 0);
}

static void sort_links_desc(OLink *v, int n) { qsort(v, n, sizeof(OLink), link_longer_first); }

static void *xalloc(size_t bytes)
{
	void *p = calloc(1, bytes ? bytes : 1);
	if (!p) {
		fprintf(stderr, "oracle: out of memory\n");
		exit(1);
	}
	return p;
}

/* upstream src/cubesphere.c:233-359 */
int cs_init(CubeSphere *cs, int N)
{
	memset(cs, 0, sizeof(*cs));
	if (N < 1) {
		fprintf(stderr, "cs_init: bad N %d\n", N);
		return -1;
	}
	int n = 6 * N * N;
	cs->N = N;
	cs->ncells = n;
	cs->h = (M_PI / 2) / N;
	cs->pos = xalloc(sizeof(float) * 3 * n);
	cs->area = xalloc(sizeof(float) * n);
	cs->nnb = xalloc(n);
	cs->nbr = xalloc(sizeof(int) * CS_MAXNB * n);
	cs->w = xalloc(sizeof(float) * CS_MAXNB * n);
	cs->elen = xalloc(sizeof(float) * CS_MAXNB * n);
	cs->gc = xalloc(sizeof(float) * 3 * CS_MAXNB * n);
	float *raw_len = xalloc(sizeof(float) * CS_MAXNB * n);
	float *sym_len = xalloc(sizeof(float) * CS_MAXNB * n);
	double h = cs->h;

	for (int c = 0; c < n; c++) {
		int f = c / (N * N), rem = c % (N * N);
		v3_store(cs->pos + 3 * c, centre_dir(cs, f, rem % N, rem / N));
	}

	/* Voronoi links, longest first, at most CS_MAXNB, slivers < 1e-4 h dropped */
	double minlen = 1e-4 * h, total = 0;
	for (int c = 0; c < n; c++) {
		OLink links[24];
		double ar;
		int op;
		int nl = voronoi_links(cs, c, links, &ar, &op);
		cs->open_cells += op;
		total += ar;
		cs->area[c] = (float) ar;
		sort_links_desc(links, nl);
		int m = 0;
		while (m < nl && m < CS_MAXNB && links[m].len >= minlen) {
			cs->nbr[CS_MAXNB * c + m] = links[m].nb;
			raw_len[CS_MAXNB * c + m] = (float) links[m].len;
			m++;
		}
		cs->nnb[c] = (unsigned char) m;
	}
	cs->total_area = total;

	/* reciprocal links only, averaged lengths (upstream :287-308) */
	for (int c = 0; c < n; c++)
		for (int k = 0; k < cs->nnb[c]; k++) {
			int o = cs->nbr[CS_MAXNB * c + k], back = -1;
			for (int kk = 0; kk < cs->nnb[o]; kk++)
				if (cs->nbr[CS_MAXNB * o + kk] == c)
					back = kk;
			double l = raw_len[CS_MAXNB * c + k];
			if (back < 0) {
				if (l > 1e-2 * h)
					cs->asym_count++;
				sym_len[CS_MAXNB * c + k] = -1.0f;
			} else {
				sym_len[CS_MAXNB * c + k] = (float) (0.5 * (l + raw_len[CS_MAXNB * o + back]));
			}
		}

	/* Laplacian weights and least-squares gradient coefficients (upstream :310-351) */
	for (int c = 0; c < n; c++) {
		vec3 p = cs_pos(cs, c);
		int nb[CS_MAXNB], m = 0;
		double ln[CS_MAXNB];
		for (int k = 0; k < cs->nnb[c]; k++)
			if (sym_len[CS_MAXNB * c + k] >= 0) {
				nb[m] = cs->nbr[CS_MAXNB * c + k];
				ln[m] = sym_len[CS_MAXNB * c + k];
				m++;
			}
		cs->nnb[c] = (unsigned char) m;
		int f = c / (N * N);
		vec3 e1 = v3_normalize(v3_tangent(cs_face_right[f], p));
		vec3 e2 = v3_cross(p, e1);
		double M00 = 0, M01 = 0, M11 = 0, tx[CS_MAXNB], ty[CS_MAXNB], wk[CS_MAXNB];
		for (int k = 0; k < m; k++) {
			vec3 q = cs_pos(cs, nb[k]);
			double d = v3_angle(p, q);
			cs->nbr[CS_MAXNB * c + k] = nb[k];
			cs->w[CS_MAXNB * c + k] = (float) (ln[k] / d);
			cs->elen[CS_MAXNB * c + k] = (float) ln[k];
			vec3 t = v3_tangent(v3_sub(q, p), p);
			tx[k] = v3_dot(t, e1);
			ty[k] = v3_dot(t, e2);
			wk[k] = ln[k] / (d * d * d);
			M00 += wk[k] * tx[k] * tx[k];
			M01 += wk[k] * tx[k] * ty[k];
			M11 += wk[k] * ty[k] * ty[k];
		}
		double det = M00 * M11 - M01 * M01;
		double i00 = M11 / det, i01 = -M01 / det, i11 = M00 / det;
		for (int k = 0; k < m; k++) {
			double c1 = wk[k] * (i00 * tx[k] + i01 * ty[k]);
			double c2 = wk[k] * (i01 * tx[k] + i11 * ty[k]);
			v3_store(cs->gc + 3 * (CS_MAXNB * c + k), v3_add(v3_scale(e1, c1), v3_scale(e2, c2)));
		}
	}
	free(raw_len);
	free(sym_len);
	return 0;
}

void cs_free(CubeSphere *cs)
{
	free(cs->pos);
	free(cs->area);
	free(cs->nnb);
	free(cs->nbr);
	free(cs->w);
	free(cs->elen);
	free(cs->gc);
	memset(cs, 0, sizeof(*cs));
}

/* ------------------------------------------------------------- operators */

/* K x at cell i = sum_k w_ik (x_i - x_k); upstream src/fluid.c:278-286. */
static double apply_k(const CubeSphere *cs, const float *x, int i)
{
	const int *nb = cs->nbr + CS_MAXNB * i;
	const float *w = cs->w + CS_MAXNB * i;
	double xi = x[i], s = 0;
	for (int k = 0; k < cs->nnb[i]; k++)
		s += w[k] * (xi - x[nb[k]]);
	return s;
}

/* upstream src/fluid.c:214-230 */
void fluid_divergence(const CubeSphere *cs, const float *vel, float *div)
{
	for (int i = 0; i < cs->ncells; i++) {
		vec3 p = cs_pos(cs, i), ui = v3_load(vel + 3 * i);
		double s = 0;
		for (int k = 0; k < cs->nnb[i]; k++) {
			int j = cs->nbr[CS_MAXNB * i + k];
			vec3 nrm = v3_normalize(v3_sub(cs_pos(cs, j), p));
			vec3 um = v3_add(ui, v3_load(vel + 3 * j));
			s += cs->elen[CS_MAXNB * i + k] * 0.5 * v3_dot(um, nrm);
		}
		div[i] = (float) (s / cs->area[i]);
	}
}

/* upstream src/fluid.c:233-250 */
void fluid_curl(const CubeSphere *cs, const float *vel, float *omega)
{
	for (int i = 0; i < cs->ncells; i++) {
		vec3 p = cs_pos(cs, i);
		vec3 wi = v3_cross(v3_load(vel + 3 * i), p);
		double s = 0;
		for (int k = 0; k < cs->nnb[i]; k++) {
			int j = cs->nbr[CS_MAXNB * i + k];
			vec3 pj = cs_pos(cs, j);
			vec3 wj = v3_cross(v3_load(vel + 3 * j), pj);
			vec3 nrm = v3_normalize(v3_sub(pj, p));
			s += cs->elen[CS_MAXNB * i + k] * 0.5 * v3_dot(v3_add(wi, wj), nrm);
		}
		omega[i] = (float) (s / cs->area[i]);
	}
}

/* upstream src/fluid.c:252-262 */
void fluid_laplacian(const CubeSphere *cs, const float *x, float *y)
{
	for (int i = 0; i < cs->ncells; i++) {
		double s = 0, xi = x[i];
		for (int k = 0; k < cs->nnb[i]; k++)
			s += cs->w[CS_MAXNB * i + k] * (x[cs->nbr[CS_MAXNB * i + k]] - xi);
		y[i] = (float) (s / cs->area[i]);
	}
}

/* upstream src/fluid.c:264-275 */
void fluid_remove_mean(const CubeSphere *cs, float *f)
{
	double s = 0;
	for (int i = 0; i < cs->ncells; i++)
		s += (double) cs->area[i] * f[i];
	float m = (float) (s / cs->total_area);
	for (int i = 0; i < cs->ncells; i++)
		f[i] -= m;
}

/* ------------------------------------------------------------ multigrid */

/* upstream src/fluid.c:26-37 */
#define ORC_MG_SWEEPS 1
#define ORC_MG_OMEGA 0.8
#define ORC_MG_COARSE_SWEEPS 60
#define ORC_MG_CORR_SCALE 1.0

static float *falloc(size_t n) { return xalloc(sizeof(float) * n); }

static float *inverse_diagonal(const CubeSphere *cs)
{
	float *d = falloc(cs->ncells);
	for (int i = 0; i < cs->ncells; i++) {
		double s = 0;
		for (int k = 0; k < cs->nnb[i]; k++)
			s += cs->w[CS_MAXNB * i + k];
		d[i] = (float) (1.0 / s);
	}
	return d;
}

/* Levels N, N/2, ... (>= 4, only while the finer size is even); bilinear P
 * from the coarse grid's taps at each fine centre, R = P^T in CSR form
 * (fine indices ascending per coarse row).  upstream src/fluid.c:41-98 */
static void mg_build(Fluid *F)
{
	int N = F->cs->N, nlev = 1;
	while ((N >> nlev) >= 4 && ((N >> (nlev - 1)) % 2) == 0)
		nlev++;
	F->nlev = nlev;
	F->lev = xalloc(sizeof(MGLevel) * nlev);
	F->lev[0].dinv = F->dinv;
	for (int l = 1; l < nlev; l++) {
		MGLevel *C = &F->lev[l], *Fl = &F->lev[l - 1];
		cs_init(&C->cs, N >> l);
		int nc = C->cs.ncells;
		C->x = falloc(nc);
		C->b = falloc(nc);
		C->r = falloc(nc);
		C->dinv = inverse_diagonal(&C->cs);
		const CubeSphere *fine = l == 1 ? F->cs : &F->lev[l - 1].cs;
		int nf = fine->ncells;
		Fl->ptap = xalloc(sizeof(int) * 4 * nf);
		Fl->pw = falloc(4 * (size_t) nf);
		for (int i = 0; i < nf; i++) {
			int idx[4];
			double wt[4];
			cs_taps(&C->cs, cs_pos(fine, i), idx, wt);
			for (int k = 0; k < 4; k++) {
				Fl->ptap[4 * i + k] = idx[k];
				Fl->pw[4 * i + k] = (float) wt[k];
			}
		}
		Fl->rstart = xalloc(sizeof(int) * (nc + 1));
		for (int t = 0; t < 4 * nf; t++)
			Fl->rstart[Fl->ptap[t] + 1]++;
		for (int c = 0; c < nc; c++)
			Fl->rstart[c + 1] += Fl->rstart[c];
		Fl->ridx = xalloc(sizeof(int) * 4 * nf);
		Fl->rw = falloc(4 * (size_t) nf);
		int *fill = xalloc(sizeof(int) * nc);
		memcpy(fill, Fl->rstart, sizeof(int) * nc);
		for (int i = 0; i < nf; i++)
			for (int k = 0; k < 4; k++) {
				int c = Fl->ptap[4 * i + k];
				Fl->ridx[fill[c]] = i;
				Fl->rw[fill[c]] = Fl->pw[4 * i + k];
				fill[c]++;
			}
		free(fill);
	}
}

/* Damped Jacobi; upstream src/fluid.c:100-111. */
static void jacobi(const CubeSphere *cs, const float *dinv, const float *b, float *x, float *r, int sweeps)
{
	int n = cs->ncells;
	for (int s = 0; s < sweeps; s++) {
		for (int i = 0; i < n; i++)
			r[i] = (float) (b[i] - apply_k(cs, x, i));
		for (int i = 0; i < n; i++)
			x[i] += (float) (ORC_MG_OMEGA * dinv[i] * r[i]);
	}
}

/* x = V(b) on level l; upstream src/fluid.c:114-146. */
static void vcycle(Fluid *F, int l, const float *b, float *x, float *r)
{
	const CubeSphere *cs = l == 0 ? F->cs : &F->lev[l].cs;
	const float *dinv = F->lev[l].dinv;
	int n = cs->ncells;
	memset(x, 0, sizeof(float) * n);
	if (l == F->nlev - 1) {
		jacobi(cs, dinv, b, x, r, ORC_MG_COARSE_SWEEPS);
		return;
	}
	jacobi(cs, dinv, b, x, r, ORC_MG_SWEEPS);
	for (int i = 0; i < n; i++)
		r[i] = (float) (b[i] - apply_k(cs, x, i));
	MGLevel *C = &F->lev[l + 1];
	const MGLevel *L = &F->lev[l];
	for (int c = 0; c < C->cs.ncells; c++) {
		double acc = 0;
		for (int k = L->rstart[c]; k < L->rstart[c + 1]; k++)
			acc += L->rw[k] * r[L->ridx[k]];
		C->b[c] = (float) acc;
	}
	vcycle(F, l + 1, C->b, C->x, C->r);
	for (int i = 0; i < n; i++) {
		const int *t = L->ptap + 4 * i;
		const float *w = L->pw + 4 * i;
		x[i] += (float) (ORC_MG_CORR_SCALE *
		                 (w[0] * C->x[t[0]] + w[1] * C->x[t[1]] + w[2] * C->x[t[2]] + w[3] * C->x[t[3]]));
	}
	jacobi(cs, dinv, b, x, r, ORC_MG_SWEEPS);
}

/* z = M^-1 r; upstream src/fluid.c:149-160. */
static void precondition(Fluid *F, const float *r, float *z)
{
	if (F->nlev > 0) {
		vcycle(F, 0, r, z, F->Ap);
		return;
	}
	for (int i = 0; i < F->cs->ncells; i++)
		z[i] = F->dinv[i] * r[i];
}

/* ----------------------------------------------------------------- fluid */

/* upstream src/fluid.c:162-190 */
int fluid_init(Fluid *F, const CubeSphere *cs, const FluidParams *prm)
{
	memset(F, 0, sizeof(*F));
	F->cs = cs;
	F->prm = *prm;
	size_t n = cs->ncells;
	F->omega = falloc(n);
	F->omega_band = falloc(n);
	F->psi = falloc(n);
	F->vel = falloc(3 * n);
	F->q0 = falloc(n);
	F->q1 = falloc(n);
	F->q2 = falloc(n);
	F->dep_b = falloc(3 * n);
	F->dep_f = falloc(3 * n);
	F->r = falloc(n);
	F->p = falloc(n);
	F->Ap = falloc(n);
	F->z = falloc(n);
	F->dinv = inverse_diagonal(cs);
	if (prm->multigrid)
		mg_build(F);
	return 0;
}

/* upstream src/fluid.c:192-209 */
void fluid_free(Fluid *F)
{
	float *arrays[] = {F->omega, F->omega_band, F->psi, F->vel, F->q0, F->q1, F->q2,
	                   F->dep_b, F->dep_f, F->r, F->p, F->Ap, F->z, F->dinv};
	for (size_t k = 0; k < sizeof(arrays) / sizeof(arrays[0]); k++)
		free(arrays[k]);
	for (int l = 0; l < F->nlev; l++) {
		MGLevel *L = &F->lev[l];
		if (l > 0) {
			cs_free(&L->cs);
			free(L->x);
			free(L->b);
			free(L->r);
			free(L->dinv);
		}
		free(L->ptap);
		free(L->pw);
		free(L->rstart);
		free(L->ridx);
		free(L->rw);
	}
	free(F->lev);
	memset(F, 0, sizeof(*F));
}

/* Warm-started PCG on K psi = -A omega; upstream src/fluid.c:290-358. */
int fluid_solve_psi(Fluid *F)
{
	const CubeSphere *cs = F->cs;
	int n = cs->ncells;
	float *psi = F->psi, *r = F->r, *p = F->p, *Ap = F->Ap, *z = F->z;
	double bb = 0, rr = 0, rz = 0;
	for (int i = 0; i < n; i++) {
		double b = -(double) cs->area[i] * F->omega[i];
		double ri = b - apply_k(cs, psi, i);
		r[i] = (float) ri;
		bb += b * b;
		rr += ri * ri;
	}
	F->cg_iters = 0;
	if (bb == 0.0) {
		memset(psi, 0, sizeof(float) * n);
		F->cg_relres = 0;
		return 0;
	}
	double tol2 = F->prm.cg_tol * F->prm.cg_tol * bb;
	int it = 0;
	if (rr > tol2) {
		precondition(F, r, z);
		for (int i = 0; i < n; i++) {
			p[i] = z[i];
			rz += (double) r[i] * z[i];
		}
	}
	while (rr > tol2 && it < F->prm.cg_maxit) {
		double pAp = 0;
		for (int i = 0; i < n; i++) {
			double a = apply_k(cs, p, i);
			Ap[i] = (float) a;
			pAp += a * p[i];
		}
		if (pAp <= 0)
			break;
		double alpha = rz / pAp;
		rr = 0;
		for (int i = 0; i < n; i++) {
			psi[i] += (float) (alpha * p[i]);
			double ri = r[i] - alpha * Ap[i];
			r[i] = (float) ri;
			rr += ri * ri;
		}
		it++;
		if (rr <= tol2)
			break;
		precondition(F, r, z);
		double rznew = 0;
		for (int i = 0; i < n; i++)
			rznew += (double) r[i] * z[i];
		double beta = rznew / rz;
		rz = rznew;
		for (int i = 0; i < n; i++)
			p[i] = (float) (z[i] + beta * p[i]);
	}
	fluid_remove_mean(cs, psi);
	F->cg_iters = it;
	F->cg_relres = sqrt(rr / bb);
	return it;
}

/* u = p x grad(psi); upstream src/fluid.c:361-376. */
void fluid_compute_velocity(Fluid *F)
{
	const CubeSphere *cs = F->cs;
	for (int i = 0; i < cs->ncells; i++) {
		vec3 p = cs_pos(cs, i), g = v3(0, 0, 0);
		double pi = F->psi[i];
		for (int k = 0; k < cs->nnb[i]; k++) {
			int j = cs->nbr[CS_MAXNB * i + k];
			g = v3_add(g, v3_scale(v3_load(cs->gc + 3 * (CS_MAXNB * i + k)), F->psi[j] - pi));
		}
		v3_store(F->vel + 3 * i, v3_cross(p, g));
	}
}

/* upstream src/fluid.c:378-395 */
void fluid_set_state(Fluid *F, const float *vel_initial, const float *vel_band)
{
	const CubeSphere *cs = F->cs;
	fluid_curl(cs, vel_initial, F->omega);
	fluid_remove_mean(cs, F->omega);
	if (vel_band) {
		fluid_curl(cs, vel_band, F->omega_band);
		fluid_remove_mean(cs, F->omega_band);
	} else {
		memset(F->omega_band, 0, sizeof(float) * cs->ncells);
	}
	memset(F->psi, 0, sizeof(float) * cs->ncells);
	int keep = F->prm.cg_maxit;
	F->prm.cg_maxit = keep * 20 > 20000 ? keep * 20 : 20000;
	fluid_solve_psi(F);
	F->prm.cg_maxit = keep;
	fluid_compute_velocity(F);
}

/* Midpoint backtraces along great circles; upstream src/fluid.c:397-414. */
static void departures(Fluid *F, double dt, int forward_too)
{
	const CubeSphere *cs = F->cs;
	for (int i = 0; i < cs->ncells; i++) {
		vec3 p = cs_pos(cs, i), u = v3_load(F->vel + 3 * i);
		vec3 mid = sphere_move(p, u, -0.5 * dt);
		vec3 um = v3_tangent(cs_sample_vec(cs, F->vel, mid), p);
		v3_store(F->dep_b + 3 * i, sphere_move(p, um, -dt));
		if (forward_too) {
			mid = sphere_move(p, u, 0.5 * dt);
			um = v3_tangent(cs_sample_vec(cs, F->vel, mid), p);
			v3_store(F->dep_f + 3 * i, sphere_move(p, um, dt));
		}
	}
}

static void resample(const CubeSphere *cs, const float *src, const float *dep, float *dst)
{
	for (int i = 0; i < cs->ncells; i++)
		dst[i] = (float) cs_sample_scalar(cs, src, v3_load(dep + 3 * i));
}

/* BFECC semi-Lagrangian step of absolute vorticity; upstream src/fluid.c:424-478. */
void fluid_step(Fluid *F, double dt)
{
	const CubeSphere *cs = F->cs;
	int n = cs->ncells;
	double two_omega = 2.0 * F->prm.rotation;
	departures(F, dt, F->prm.bfecc);
	float *q = F->q0, *qn = F->q1;
	for (int i = 0; i < n; i++)
		q[i] = (float) (F->omega[i] + two_omega * cs->pos[3 * i + 1]);
	if (!F->prm.bfecc) {
		resample(cs, q, F->dep_b, qn);
	} else {
		float *q1 = F->q1, *q2 = F->q2;
		resample(cs, q, F->dep_b, q1);
		resample(cs, q1, F->dep_f, q2);
		for (int i = 0; i < n; i++)
			q2[i] = q[i] + 0.5f * (q[i] - q2[i]);
		for (int i = 0; i < n; i++) {
			int idx[4];
			double wt[4];
			cs_taps(cs, v3_load(F->dep_b + 3 * i), idx, wt);
			double v = 0, lo = 1e30, hi = -1e30;
			for (int k = 0; k < 4; k++) {
				v += wt[k] * q2[idx[k]];
				double o = q[idx[k]];
				if (o < lo)
					lo = o;
				if (o > hi)
					hi = o;
			}
			if (v < lo)
				v = lo;
			if (v > hi)
				v = hi;
			q1[i] = (float) v;
		}
	}
	double relax = F->prm.forcing > 0 ? 1.0 - exp(-F->prm.forcing * dt) : 0.0;
	for (int i = 0; i < n; i++) {
		double w = qn[i] - two_omega * cs->pos[3 * i + 1];
		w += relax * (F->omega_band[i] - w);
		F->omega[i] = (float) w;
	}
	fluid_remove_mean(cs, F->omega);
	fluid_solve_psi(F);
	fluid_compute_velocity(F);
}

/* upstream src/fluid.c:480-491 (the squared speed is formed in storage precision) */
double fluid_max_speed(const Fluid *F)
{
	double m = 0;
	for (int i = 0; i < F->cs->ncells; i++) {
		const float *v = F->vel + 3 * i;
		double s = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
		if (s > m)
			m = s;
	}
	return sqrt(m);
}

/* ------------------------------------------------------------- particles */

/* upstream src/particles.c:8-31 */
int particles_init(Particles *P, int n)
{
	P->n = n;
	P->pos = falloc(3 * (size_t) n);
	P->prev = falloc(3 * (size_t) n);
	P->col = falloc(4 * (size_t) n);
	const double golden = M_PI * (3.0 - sqrt(5.0));
	for (int i = 0; i < n; i++) {
		double y = 1.0 - 2.0 * (i + 0.5) / n;
		double r = sqrt(1.0 - y * y);
		double phi = golden * i;
		vec3 p = v3(r * cos(phi), y, r * sin(phi));
		v3_store(P->pos + 3 * i, p);
		v3_store(P->prev + 3 * i, p);
	}
	for (size_t i = 0; i < 4 * (size_t) n; i++)
		P->col[i] = 1.0f;
	return 0;
}

void particles_free(Particles *P)
{
	free(P->pos);
	free(P->prev);
	free(P->col);
	memset(P, 0, sizeof(*P));
}

/* upstream src/particles.c:41-61 */
void particles_color_from_image(Particles *P, const float *img, int w, int h)
{
	for (int i = 0; i < P->n; i++) {
		double lon, lat;
		dir_to_lonlat(v3_load(P->pos + 3 * i), &lon, &lat);
		double x = (lon + M_PI) / (2 * M_PI) * w - 0.5;
		double y = (M_PI / 2 - lat) / M_PI * h - 0.5;
		int x0 = (int) floor(x), y0 = (int) floor(y);
		double fx = x - x0, fy = y - y0;
		int xs[2] = {((x0 % w) + w) % w, (((x0 + 1) % w) + w) % w};
		int ys[2] = {clampi(y0, 0, h - 1), clampi(y0 + 1, 0, h - 1)};
		double wts[4] = {(1 - fx) * (1 - fy), fx * (1 - fy), (1 - fx) * fy, fx * fy};
		for (int c = 0; c < 4; c++) {
			double v = 0;
			for (int k = 0; k < 4; k++)
				v += wts[k] * img[((size_t) ys[k >> 1] * w + xs[k & 1]) * 4 + c];
			P->col[4 * i + c] = (float) v;
		}
	}
}

/* upstream src/particles.c:63-74 */
void particles_advect(Particles *P, const CubeSphere *cs, const float *vel, double dt)
{
	for (int i = 0; i < P->n; i++) {
		vec3 p = v3_load(P->pos + 3 * i);
		v3_store(P->prev + 3 * i, p);
		vec3 u1 = cs_sample_vec(cs, vel, p);
		vec3 mid = sphere_move(p, u1, 0.5 * dt);
		vec3 u2 = v3_tangent(cs_sample_vec(cs, vel, mid), p);
		v3_store(P->pos + 3 * i, sphere_move(p, u2, dt));
	}
}

/* ---------------------------------------------------------------- render */

/* upstream src/render.c:11-39 */
int render_init(Render *r, int R, float radius, float alpha)
{
	memset(r, 0, sizeof(*r));
	r->R = R;
	r->radius = radius < 0.75f ? 0.75f : radius;
	r->alpha = alpha;
	r->g = 1.0;
	r->buf = falloc((size_t) 6 * R * R * 4);
	int sh = 32;
	if (sh < (int) ceilf(r->radius) + 1)
		sh = (int) ceilf(r->radius) + 1;
	if (sh > R)
		sh = R;
	r->strip_h = sh;
	r->nstrips = (R + sh - 1) / sh;
	r->nbins = 6 * r->nstrips;
	return 0;
}

void render_free(Render *r)
{
	free(r->buf);
	memset(r, 0, sizeof(*r));
}

/* upstream src/render.c:55-66 */
void render_fade(Render *r, double fade)
{
	r->g *= (1.0 - fade);
	if (r->g < 1e-4) {
		size_t n = (size_t) 6 * r->R * r->R * 4;
		float g = (float) r->g;
		for (size_t i = 0; i < n; i++)
			r->buf[i] *= g;
		r->g = 1.0;
	}
}

/* One tent splat of sample (px, py) with colour col on face f; the texel
 * arithmetic of upstream src/render.c:121-152. */
static void splat(Render *r, int f, float px, float py, const float *col)
{
	int R = r->R;
	float rad = r->radius, invrad = 1.0f / rad;
	float invg = (float) (1.0 / r->g);
	float w0 = r->alpha * col[3];
	int xlo = (int) ceilf(px - rad), xhi = (int) floorf(px + rad);
	int ylo = (int) ceilf(py - rad), yhi = (int) floorf(py + rad);
	xlo = xlo < 0 ? 0 : xlo;
	ylo = ylo < 0 ? 0 : ylo;
	xhi = xhi > R - 1 ? R - 1 : xhi;
	yhi = yhi > R - 1 ? R - 1 : yhi;
	float *face = r->buf + (size_t) f * R * R * 4;
	for (int y = ylo; y <= yhi; y++) {
		float wy = 1.0f - fabsf(y - py) * invrad;
		if (wy <= 0)
			continue;
		for (int x = xlo; x <= xhi; x++) {
			float wx = 1.0f - fabsf(x - px) * invrad;
			if (wx <= 0)
				continue;
			float w = w0 * wx * wy;
			float keep = 1.0f - w, add = w * invg;
			float *d = face + ((size_t) y * R + x) * 4;
			d[0] = d[0] * keep + add * col[0];
			d[1] = d[1] * keep + add * col[1];
			d[2] = d[2] * keep + add * col[2];
			d[3] = d[3] * keep + add;
		}
	}
}

/* Serial deposit: particle by particle, sample k = 1..ns, faces 0..5.  Per
 * texel this is the compositing order of upstream src/render.c:156-218
 * (ascending particle index, then ascending k). */
void render_deposit(Render *r, const Particles *P)
{
	int R = r->R;
	double spacing = 0.7 / R;
	float rad = r->radius;
	for (int i = 0; i < P->n; i++) {
		vec3 a = v3_load(P->prev + 3 * i), b = v3_load(P->pos + 3 * i);
		int ns = (int) ceil(v3_angle(a, b) / spacing);
		ns = clampi(ns, 1, 4096);
		for (int k = 1; k <= ns; k++) {
			double tt = (double) k / ns;
			vec3 d = v3_normalize(v3_add(v3_scale(a, 1 - tt), v3_scale(b, tt)));
			for (int f = 0; f < 6; f++) {
				double dc = v3_dot(d, cs_face_center[f]);
				if (dc < 0.5)
					continue;
				double u = v3_dot(d, cs_face_right[f]) / dc;
				double v = v3_dot(d, cs_face_up[f]) / dc;
				float px = (float) ((u + 1.0) * 0.5 * R - 0.5);
				float py = (float) ((1.0 - v) * 0.5 * R - 0.5);
				int xlo = (int) ceilf(px - rad), xhi = (int) floorf(px + rad);
				int ylo = (int) ceilf(py - rad), yhi = (int) floorf(py + rad);
				if (xlo < 0)
					xlo = 0;
				if (xhi > R - 1)
					xhi = R - 1;
				if (ylo < 0)
					ylo = 0;
				if (yhi > R - 1)
					yhi = R - 1;
				if (xlo > xhi || ylo > yhi)
					continue;
				splat(r, f, px, py, P->col + 4 * (size_t) i);
			}
		}
	}
}

/* upstream src/render.c:220-226 */
void render_texel(const Render *r, int face, int x, int y, float out[4])
{
	const float *d = r->buf + (((size_t) face * r->R + y) * r->R + x) * 4;
	float g = (float) r->g;
	for (int c = 0; c < 4; c++)
		out[c] = d[c] * g;
}

/* upstream src/render.c:228-251 */
void render_sample_dir(const Render *r, double dx, double dy, double dz, float out[4])
{
	vec3 d = v3(dx, dy, dz);
	int f = cs_face_of(d), R = r->R;
	double dc = v3_dot(d, cs_face_center[f]);
	double u = v3_dot(d, cs_face_right[f]) / dc;
	double v = v3_dot(d, cs_face_up[f]) / dc;
	double px = (u + 1.0) * 0.5 * R - 0.5, py = (1.0 - v) * 0.5 * R - 0.5;
	if (px < 0)
		px = 0;
	if (py < 0)
		py = 0;
	if (px > R - 1)
		px = R - 1;
	if (py > R - 1)
		py = R - 1;
	int x0 = (int) px, y0 = (int) py;
	int x1 = x0 + 1 < R ? x0 + 1 : x0, y1 = y0 + 1 < R ? y0 + 1 : y0;
	float fx = (float) (px - x0), fy = (float) (py - y0);
	float t00[4], t10[4], t01[4], t11[4];
	render_texel(r, f, x0, y0, t00);
	render_texel(r, f, x1, y0, t10);
	render_texel(r, f, x0, y1, t01);
	render_texel(r, f, x1, y1, t11);
	for (int k = 0; k < 4; k++)
		out[k] = (1 - fy) * ((1 - fx) * t00[k] + fx * t10[k]) + fy * ((1 - fx) * t01[k] + fx * t11[k]);
}

static unsigned char to_u8(float v)
{
	if (v <= 0)
		return 0;
	if (v >= 1)
		return 255;
	return (unsigned char) (v * 255.0f + 0.5f);
}

/* upstream src/render.c:253-279 */
void render_pixel8(const float c[4], const float *bg, unsigned char *out)
{
	float a = c[3];
	a = a > 1 ? 1 : (a < 0 ? 0 : a);
	if (!bg) {
		if (a > 1e-6f) {
			out[0] = to_u8(c[0] / a);
			out[1] = to_u8(c[1] / a);
			out[2] = to_u8(c[2] / a);
		} else {
			out[0] = out[1] = out[2] = 0;
		}
		out[3] = to_u8(a);
	} else {
		for (int k = 0; k < 3; k++)
			out[k] = to_u8(c[k] + bg[k] * (1 - a));
	}
}

/* ----------------------------------------------------------------- noise */

/* The 12 edge-midpoint gradients of 3-D simplex noise; upstream src/noise.c:6-10. */
static const double orc_grad[12][3] = {
	{1, 1, 0}, {-1, 1, 0}, {1, -1, 0}, {-1, -1, 0}, {1, 0, 1}, {-1, 0, 1},
	{1, 0, -1}, {-1, 0, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1}, {0, -1, -1},
};

/* Fisher-Yates with xorshift64*; upstream src/noise.c:12-31. */
void noise_init(Noise *nz, unsigned int seed)
{
	unsigned char p[256];
	unsigned long long s = 0x9E3779B97F4A7C15ULL ^ ((unsigned long long) seed * 0xD1B54A32D192ED03ULL);
	for (int i = 0; i < 256; i++)
		p[i] = (unsigned char) i;
	for (int i = 255; i > 0; i--) {
		s ^= s >> 12;
		s ^= s << 25;
		s ^= s >> 27;
		unsigned long long r = s * 2685821657736338717ULL;
		int j = (int) ((r >> 33) % (unsigned long long) (i + 1));
		unsigned char t = p[i];
		p[i] = p[j];
		p[j] = t;
	}
	for (int i = 0; i < 512; i++)
		nz->perm[i] = p[i & 255];
}

/* upstream src/noise.c:33-79 */
double simplex3(const Noise *nz, vec3 pt, vec3 *g)
{
	const double F3 = 1.0 / 3.0, G3 = 1.0 / 6.0;
	const unsigned char *perm = nz->perm;
	double x = pt.x, y = pt.y, z = pt.z;
	double s = (x + y + z) * F3;
	int i = (int) floor(x + s), j = (int) floor(y + s), k = (int) floor(z + s);
	double t = (i + j + k) * G3;
	double x0 = x - (i - t), y0 = y - (j - t), z0 = z - (k - t);
	int o1[3], o2[3];
	if (x0 >= y0) {
		if (y0 >= z0) {
			o1[0] = 1; o1[1] = 0; o1[2] = 0; o2[0] = 1; o2[1] = 1; o2[2] = 0;
		} else if (x0 >= z0) {
			o1[0] = 1; o1[1] = 0; o1[2] = 0; o2[0] = 1; o2[1] = 0; o2[2] = 1;
		} else {
			o1[0] = 0; o1[1] = 0; o1[2] = 1; o2[0] = 1; o2[1] = 0; o2[2] = 1;
		}
	} else {
		if (y0 < z0) {
			o1[0] = 0; o1[1] = 0; o1[2] = 1; o2[0] = 0; o2[1] = 1; o2[2] = 1;
		} else if (x0 < z0) {
			o1[0] = 0; o1[1] = 1; o1[2] = 0; o2[0] = 0; o2[1] = 1; o2[2] = 1;
		} else {
			o1[0] = 0; o1[1] = 1; o1[2] = 0; o2[0] = 1; o2[1] = 1; o2[2] = 0;
		}
	}
	double xs[4] = {x0, x0 - o1[0] + G3, x0 - o2[0] + 2 * G3, x0 - 1 + 3 * G3};
	double ys[4] = {y0, y0 - o1[1] + G3, y0 - o2[1] + 2 * G3, y0 - 1 + 3 * G3};
	double zs[4] = {z0, z0 - o1[2] + G3, z0 - o2[2] + 2 * G3, z0 - 1 + 3 * G3};
	int ii = i & 255, jj = j & 255, kk = k & 255;
	int gi[4];
	gi[0] = perm[ii + perm[jj + perm[kk]]] % 12;
	gi[1] = perm[ii + o1[0] + perm[jj + o1[1] + perm[kk + o1[2]]]] % 12;
	gi[2] = perm[ii + o2[0] + perm[jj + o2[1] + perm[kk + o2[2]]]] % 12;
	gi[3] = perm[ii + 1 + perm[jj + 1 + perm[kk + 1]]] % 12;
	double n = 0, dx = 0, dy = 0, dz = 0;
	for (int c = 0; c < 4; c++) {
		double tt = 0.5 - xs[c] * xs[c] - ys[c] * ys[c] - zs[c] * zs[c];
		if (tt <= 0)
			continue;
		const double *gr = orc_grad[gi[c]];
		double gd = gr[0] * xs[c] + gr[1] * ys[c] + gr[2] * zs[c];
		double t2 = tt * tt, t4 = t2 * t2, t3 = t2 * tt;
		n += t4 * gd;
		dx += t4 * gr[0] - 8.0 * t3 * gd * xs[c];
		dy += t4 * gr[1] - 8.0 * t3 * gd * ys[c];
		dz += t4 * gr[2] - 8.0 * t3 * gd * zs[c];
	}
	const double scale = 72.0;
	if (g)
		*g = v3(dx * scale, dy * scale, dz * scale);
	return n * scale;
}

/* upstream src/noise.c:81-103 */
vec3 curl_noise(const Noise *nz, vec3 p, const CurlParams *cp)
{
	static const vec3 potential_off[3] = {
		{0.0, 0.0, 0.0}, {31.416, -47.853, 12.793}, {-93.11, 63.2, 109.7},
	};
	vec3 c = v3(0, 0, 0);
	double f = cp->scale, a = 1.0;
	for (int k = 0; k < cp->octaves; k++) {
		vec3 q = v3_add(v3_scale(p, f), v3(17.13 * k, 5.31 * k, 11.71 * k));
		vec3 gx, gy, gz;
		simplex3(nz, v3_add(q, potential_off[0]), &gx);
		simplex3(nz, v3_add(q, potential_off[1]), &gy);
		simplex3(nz, v3_add(q, potential_off[2]), &gz);
		double m = a * f;
		c = v3_add(c, v3_scale(v3(gz.y - gy.z, gx.z - gz.x, gy.x - gx.y), m));
		f *= cp->lacunarity;
		a *= cp->gain;
	}
	return c;
}
