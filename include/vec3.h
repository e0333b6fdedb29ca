/* vec3.h — double-precision 3-vector helpers used by callers of the library.
 *
 * Callers of the grid / fluid / particle / render API (the application driver
 * and its tests) use these inline helpers on the host.  The names, argument
 * order and floating-point expression order are the ones of the upstream
 * helper header (src/vec3.h:7-58 of gaseous-gusty-ball), because callers
 * compiled against either header must compute identical bits; the bodies
 * are written for this library.  Device code uses its own double3 helpers
 * (gaseous-gusty-ball_b200/csrc/ggb_device.cuh) with the same expression order.
 */
#ifndef GGB_VEC3_H
#define GGB_VEC3_H

#include <math.h>

typedef struct {
	double x, y, z;
} vec3; /* upstream src/vec3.h:7 */

static inline vec3 v3(double x, double y, double z)
{
	vec3 out;
	out.x = x;
	out.y = y;
	out.z = z;
	return out;
}

static inline vec3 v3_add(vec3 a, vec3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline vec3 v3_sub(vec3 a, vec3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline vec3 v3_scale(vec3 a, double k) { return v3(a.x * k, a.y * k, a.z * k); }
static inline double v3_dot(vec3 a, vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

static inline vec3 v3_cross(vec3 a, vec3 b)
{
	return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

static inline double v3_len(vec3 a) { return sqrt(v3_dot(a, a)); }

/* Unit vector along a; the zero vector is returned unchanged. */
static inline vec3 v3_normalize(vec3 a)
{
	double len = v3_len(a);
	if (len > 0.0)
		return v3_scale(a, 1.0 / len);
	return a;
}

/* Component of v orthogonal to the unit normal n. */
static inline vec3 v3_tangent(vec3 v, vec3 n) { return v3_sub(v, v3_scale(n, v3_dot(v, n))); }

/* Angle between a and b, accurate for small angles (atan2 of |a x b| and a.b). */
static inline double v3_angle(vec3 a, vec3 b) { return atan2(v3_len(v3_cross(a, b)), v3_dot(a, b)); }

static inline vec3 v3_load(const float *src) { return v3(src[0], src[1], src[2]); }

static inline void v3_store(float *dst, vec3 a)
{
	dst[0] = (float) a.x;
	dst[1] = (float) a.y;
	dst[2] = (float) a.z;
}

/* Great-circle motion of the unit vector p for time s with velocity v
 * (only the part of v tangent at p is used; s may be negative).
 * Upstream: src/vec3.h:33-42. */
static inline vec3 sphere_move(vec3 p, vec3 v, double s)
{
	vec3 t = v3_tangent(v, p);
	double speed = v3_len(t);
	if (speed < 1e-300)
		return p;
	double theta = speed * s;
	return v3_normalize(v3_add(v3_scale(p, cos(theta)), v3_scale(t, sin(theta) / speed)));
}

/* +Y is north; longitude 0 at +Z, increasing toward +X.  Upstream: src/vec3.h:46-58. */
static inline void dir_to_lonlat(vec3 d, double *lon, double *lat)
{
	*lon = atan2(d.x, d.z);
	double y = d.y;
	if (y > 1.0)
		y = 1.0;
	if (y < -1.0)
		y = -1.0;
	*lat = asin(y);
}

static inline vec3 lonlat_to_dir(double lon, double lat)
{
	return v3(cos(lat) * sin(lon), sin(lat), cos(lat) * cos(lon));
}

#endif
