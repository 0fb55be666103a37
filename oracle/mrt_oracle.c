/*
 * mrt_oracle.c — TEST INFRASTRUCTURE: FP64 CPU restatement of miniRT's
 * path-tracing hot path. See mrt_oracle.h. Never linked into the product.
 *
 * Every function states the reference function it restates. Arithmetic is
 * written in the same order and with the same float/double conversions as
 * the reference so that, with the reference's RNG stream, results are
 * bit-identical (build without -ffast-math and without FMA contraction).
 */
#include "mrt_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define PI_D 3.1415926535897          /* minirt.h:21 */
#define IT_MIN 0.001                  /* minirt.h:43-44 */
#define IT_MAX 1000
#define SHINE 64.0                    /* material.h:18-19 */
#define SPEC_STRENGTH 1.0
#define MAX_PHOTONS_PER_LEAF 1000     /* minirt.h:57 */

typedef struct { double x, y, z; } v3;
typedef struct { double r, g, b; } fc;
typedef struct { v3 orig, dir; } ray_t;

/* ------------------------------------------------------------- vec3 ops
 * src/math/vector: dot and cross are left-to-right sums, unit() returns
 * 0 for a zero vector, divide_scalar returns 0 for t == 0. */
static inline v3 vadd(v3 u, v3 v) { return (v3){u.x + v.x, u.y + v.y, u.z + v.z}; }
static inline v3 vsub(v3 u, v3 v) { return (v3){u.x - v.x, u.y - v.y, u.z - v.z}; }
static inline v3 vmul(v3 u, v3 v) { return (v3){u.x * v.x, u.y * v.y, u.z * v.z}; }
static inline v3 vscale(v3 v, double t) { return (v3){v.x * t, v.y * t, v.z * t}; }
static inline v3 vdiv(v3 v, double t)
{
	if (t != 0.0)
		return (v3){v.x / t, v.y / t, v.z / t};
	return (v3){0.0, 0.0, 0.0};
}
static inline double vdot(v3 u, v3 v) { return u.x * v.x + u.y * v.y + u.z * v.z; }
static inline v3 vcross(v3 u, v3 v)
{
	return (v3){u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x};
}
static inline double vlen2(v3 v) { return v.x * v.x + v.y * v.y + v.z * v.z; }
static inline double vlen(v3 v) { return sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }
static inline v3 vneg(v3 v) { return (v3){-v.x, -v.y, -v.z}; }
static inline v3 vunit(v3 v)
{
	double l = vlen(v);

	if (l > 0.0)
		return vdiv(v, l);
	return (v3){0.0, 0.0, 0.0};
}
static inline double dmin_(double a, double b) { return a < b ? a : b; }   /* ft_dmin.c:16 */
static inline double dmax_(double a, double b) { return a > b ? a : b; }
static inline v3 vmin(v3 a, v3 b) { return (v3){dmin_(a.x, b.x), dmin_(a.y, b.y), dmin_(a.z, b.z)}; }
static inline v3 vmax(v3 a, v3 b) { return (v3){dmax_(a.x, b.x), dmax_(a.y, b.y), dmax_(a.z, b.z)}; }
static inline v3 ray_at(ray_t r, double t)                                 /* ray.c:16 */
{
	return (v3){r.orig.x + t * r.dir.x, r.orig.y + t * r.dir.y, r.orig.z + t * r.dir.z};
}
static inline fc fadd(fc a, fc b) { return (fc){a.r + b.r, a.g + b.g, a.b + b.b}; }
static inline fc fsub(fc a, fc b) { return (fc){a.r - b.r, a.g - b.g, a.b - b.b}; }
static inline fc fmul(fc a, fc b) { return (fc){a.r * b.r, a.g * b.g, a.b * b.b}; }
static inline fc fscale(fc a, double c) { return (fc){a.r * c, a.g * c, a.b * c}; }
static inline fc c2f(const uint8_t *c) { return (fc){c[0] / 255.0, c[1] / 255.0, c[2] / 255.0}; }
static inline double clamp01(double v) { return v < 0 ? 0 : (v > 1 ? 1 : v); } /* clamp_int.c:39 */
static inline int mat_or_none(int32_t m, int n) { return (m >= 0 && m < n) ? m : -1; }
static inline double clampv(double v, double lo, double hi)               /* clamp_double.c:15 */
{
	if (v <= lo)
		return lo;
	else if (v >= hi)
		return hi;
	return v;
}

/* ------------------------------------------------------------------ RNG */

static uint64_t	g_ref_rng = 42;

void		ro_set_reference_rng(uint64_t state) { g_ref_rng = state ? state : 42; }
uint64_t	ro_get_reference_rng(void) { return g_ref_rng; }

static inline uint64_t splitmix64(uint64_t z)
{
	z += 0x9E3779B97F4A7C15ULL;
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
	return z ^ (z >> 31);
}

/* Per-path stream: a PCG32 state derived from (seed, pixel, sample). */
uint64_t	ro_path_seed(uint64_t seed, uint32_t pixel, uint32_t sample)
{
	return splitmix64(seed ^ splitmix64(((uint64_t)sample << 32) | pixel));
}

/* PCG32 XSH-RR (O'Neill 2014), 24-bit float in [0,1). */
float	ro_pcg_float(uint64_t *s)
{
	uint64_t	old = *s;
	uint32_t	xs;
	uint32_t	rot;
	uint32_t	out;

	*s = old * 6364136223846793005ULL + 1442695040888963407ULL;
	xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
	rot = (uint32_t)(old >> 59u);
	out = (xs >> rot) | (xs << ((32u - rot) & 31u));
	return (float)(out >> 8) * (1.0f / 16777216.0f);
}

typedef struct
{
	int			mode;
	uint64_t	state;
}	rng_t;

/* random_double (random.c:25-30) in reference mode. */
static inline double rnd(rng_t *r)
{
	if (r->mode == RO_RNG_REFERENCE)
	{
		g_ref_rng ^= g_ref_rng << 13;
		g_ref_rng ^= g_ref_rng >> 7;
		g_ref_rng ^= g_ref_rng << 17;
		return (g_ref_rng >> 11) / 9007199254740992.0;
	}
	return (double)ro_pcg_float(&r->state);
}

/* random_in_unit_sphere (random.c:42-50). */
static v3 rnd_in_unit_sphere(rng_t *r)
{
	v3	p;

	p.x = rnd(r) * 2 - 1.0;
	p.y = rnd(r) * 2 - 1.0;
	p.z = rnd(r) * 2 - 1.0;
	if (vlen2(p) >= 1.0)
		p = vscale(vunit(p), pow(rnd(r), 1.0 / 3.0));
	return p;
}

/* vec3_random_unit (vec3_random.c:33-44). */
static v3 rnd_unit(rng_t *r)
{
	v3		p;
	double	l2;

	while (1)
	{
		p.x = -1 + rnd(r) * (1 - -1);
		p.y = -1 + rnd(r) * (1 - -1);
		p.z = -1 + rnd(r) * (1 - -1);
		l2 = vlen2(p);
		if (1e-160 < l2 && l2 <= 1.0)
			return vdiv(p, sqrt(l2));
	}
}

/* ---------------------------------------------------------------- scene */

enum { TX_COLOR = 0, TX_METALLIC, TX_ROUGHNESS, TX_TRANSMISSION, TX_AO, TX_EMIS_STRENGTH,
	TX_EMIS_COLOR, TX_NORMAL, TX_SLOTS };

typedef struct
{
	uint8_t	c8[3];
	double	metallic, roughness, ior, transmission, ao, emission_strength, scale;
	fc		emission_color;
	int		tex[TX_SLOTS];     /* 1 + texture index, 0 none */
	double	normal_intensity;
	int		textured;          /* any tex[] set */
}	mat_t;

/* t_tex (scene_structs.h:61-82) */
typedef struct
{
	int			type;
	uint32_t	w, h;
	uint8_t		*rgba;
	double		scale;
	uint8_t		c1[3], c2[3];
}	tex_t;

enum { PT_SPHERE = 0, PT_TRI = 1, PT_CYL = 2, PT_CONE = 3, PT_HYP = 4 };

typedef struct
{
	int		type;
	int		flat;
	int		mat;
	uint8_t	color[3];
	v3		center;            /* sphere centre, triangle centroid, quadric position */
	double	radius, r2;
	v3		ori;               /* quadric orientation as given */
	double	diam, height;      /* cylinder, cone */
	double	qa, qb, qc, shape; /* hyperboloid (height in `height`) */
	int		mat_top, mat_bot;  /* cylinder / cone cap materials, -1 none */
	v3		p[3], n[3];
	double	uv[3][2];
}	prim_t;

typedef struct
{
	v3		point, normal;
	int		mat;
	uint8_t	color[3];
	int		flat;
}	plane_t;

typedef struct
{
	int		type;
	v3		pos;
	double	brightness;
	uint8_t	color[3];
	int		shadow_sample;
	float	radius;
}	light_t;

typedef struct
{
	v3			bmin, bmax;
	uint32_t	left, right, first, count;
	int			leaf;
}	node_t;

typedef struct { v3 pos; fc power; } photon_t;

typedef struct kd_t
{
	v3			bmin, bmax;
	int			axis;
	struct kd_t	*left, *right;
	float		split;
	int			start, count;
}	kd_t;

struct ro_scene
{
	int			W, H, max_bounces, one_sided;
	double		ior_all;
	mat_t		*mats;
	int			n_mats;
	tex_t		*texs;
	int			n_texs;
	rng_t		*rg;                /* the path's random stream (alpha test) */
	int			is_light;           /* tracing a shadow ray (apply_all_map's is_light) */
	prim_t		*prims;             /* bvh_make_lst order */
	int			n_prims;
	uint32_t	*prim_idx;          /* prim_indices after the median build */
	node_t		*nodes;
	uint32_t	n_nodes;
	plane_t		*planes;
	int			n_planes;
	light_t		*lights;
	int			n_lights;
	/* camera / viewport (viewport.c) */
	v3			cam_pos, cam_dir;
	double		focus_dist, defocus_angle;
	v3			pixel00, pdu, pdv, defocus_u, defocus_v;
	/* ambient / sky */
	double		amb_ratio;
	uint8_t		amb_color[3];
	int			hw, hh;
	const uint8_t	*rgbe;
	uint8_t		*rgbe_own;
	float		hdr_exposure, hdr_gamma;
	float		*pdf_joint, *cdf_m_inv, *cdf_c_inv;
	double		column_average;
	/* caustics */
	int			caustic_enable;
	double		caustic_radius, norm_factor;
	photon_t	*photons;
	size_t		n_photons;
	kd_t		*kd_nodes;
	size_t		kd_count;
	kd_t		*kd_root;
	ro_counters	cnt;
	int			render_mode;
	int			apply_mesh_transform;
	/* differentiable-parameter overrides (ro_set_params) */
	double		*albedo_d;          /* M*3, replaces color_value / 255 */
	double		*sky_d;             /* W*H*3 linear radiance, replaces the RGBE sky */
	double		*pdf_joint_d;       /* pdf_joint before its float store */
	int			exact;              /* FP64 throughout (no float intermediates) */
};

static int	g_apply_mesh_transform = 1;

/* 1 (default): mesh vertices go through the reference's load-time
 * re-transform; 0: they are used as given (already canonical). */
void	ro_set_mesh_transform(int on)
{
	g_apply_mesh_transform = on;
}

/* -------------------------------------------- median-split BVH build
 * bvh_build.c:16-127 and qshort_axis.c:16-102: median split of the node's
 * prim range on the longest axis of the node bounds, by the object position
 * compared as float (bvh_math.c:35-49), leaves of one primitive. */

static v3 obj_pos(ro_scene *s, uint32_t i)               /* bvh_utils.c:86 */
{
	return s->prims[i].center;
}

static float axis_of(v3 p, int a)                         /* bvh_utils.c:103 */
{
	if (a == 0)
		return (float)p.x;
	else if (a == 1)
		return (float)p.y;
	return (float)p.z;
}

static int cmp_axis(ro_scene *s, uint32_t a, uint32_t b, int axis)
{
	float	va = axis_of(obj_pos(s, a), axis);
	float	vb = axis_of(obj_pos(s, b), axis);

	if (va < vb)
		return -1;
	else if (va > vb)
		return 1;
	return 0;
}

static void swap_u32(uint32_t *a, uint32_t *b) { uint32_t t = *a; *a = *b; *b = t; }

static void isort(uint32_t *arr, double lo, double hi, ro_scene *s, int axis)
{
	for (int i = (int)lo + 1; i <= hi; i++)
	{
		uint32_t	key = arr[i];
		int			j = i - 1;

		while (j >= lo && cmp_axis(s, arr[j], key, axis) > 0)
		{
			arr[j + 1] = arr[j];
			j--;
		}
		arr[j + 1] = key;
	}
}

static uint32_t med3(uint32_t *arr, double lo, double hi, ro_scene *s, int axis)
{
	int	mid = lo + (hi - lo) / 2;

	if (cmp_axis(s, arr[(int)lo], arr[mid], axis) > 0)
		swap_u32(&arr[(int)lo], &arr[mid]);
	if (cmp_axis(s, arr[(int)lo], arr[(int)hi], axis) > 0)
		swap_u32(&arr[(int)lo], &arr[(int)hi]);
	if (cmp_axis(s, arr[mid], arr[(int)hi], axis) > 0)
		swap_u32(&arr[mid], &arr[(int)hi]);
	swap_u32(&arr[mid], &arr[(int)hi - 1]);
	return arr[(int)hi - 1];
}

static int partition_(uint32_t *arr, double lo, double hi, ro_scene *s, int axis)
{
	uint32_t	pivot = med3(arr, lo, hi, s, axis);
	int			i = lo;
	int			j = hi - 1;

	while (1)
	{
		while (cmp_axis(s, arr[++i], pivot, axis) < 0)
			;
		while (cmp_axis(s, arr[--j], pivot, axis) > 0)
			;
		if (i >= j)
			break ;
		swap_u32(&arr[i], &arr[j]);
	}
	swap_u32(&arr[i], &arr[(int)hi - 1]);
	return i;
}

static void qsort_axis_(uint32_t *arr, double lo, double hi, ro_scene *s, int axis)
{
	int	p;

	while (lo < hi)
	{
		if (hi - lo < 16)
		{
			isort(arr, lo, hi, s, axis);
			return ;
		}
		p = partition_(arr, lo, hi, s, axis);
		if (p - lo < hi - p)
		{
			qsort_axis_(arr, lo, p - 1, s, axis);
			lo = p + 1;
		}
		else
		{
			qsort_axis_(arr, p + 1, hi, s, axis);
			hi = p - 1;
		}
	}
}

/* extents of a disc of radius r with unit normal a, added to [p0, p1]
 * (compute_cylinder_bounds, bvh_obj_bounds.c:41-60) */
static void disc_bounds(v3 p0, v3 p1, v3 a, double r, v3 *mn, v3 *mx)
{
	v3	e = {r * sqrt(1.0 - a.x * a.x), r * sqrt(1.0 - a.y * a.y), r * sqrt(1.0 - a.z * a.z)};

	*mn = vsub(vmin(p0, p1), e);
	*mx = vadd(vmax(p0, p1), e);
}

static void prim_bounds(prim_t *p, v3 *mn, v3 *mx)     /* bvh_obj_bounds.c:16-96 */
{
	if (p->type == PT_SPHERE)
	{
		v3 r = {p->radius, p->radius, p->radius};
		*mn = vsub(p->center, r);
		*mx = vadd(p->center, r);
		return ;
	}
	if (p->type == PT_CYL)
	{
		v3	a = vunit(p->ori);
		v3	half = vscale(a, p->height * 0.5);

		disc_bounds(vsub(p->center, half), vadd(p->center, half), a, p->diam * 0.5, mn, mx);
		return ;
	}
	if (p->type == PT_CONE)
	{
		v3	a = vunit(p->ori);

		disc_bounds(p->center, vadd(p->center, vscale(a, p->height)), a, p->diam * 0.5, mn, mx);
		return ;
	}
	if (p->type == PT_HYP)
	{
		v3		a = vunit(p->ori);
		v3		half = vscale(a, p->height * 0.5);
		double	rmax = fmax(p->qa, p->qb) * sqrt(p->shape
				+ ((p->height * 0.5) * (p->height * 0.5)) / (p->qc * p->qc));

		disc_bounds(vsub(p->center, half), vadd(p->center, half), a, rmax, mn, mx);
		return ;
	}
	*mn = vmin(p->p[0], vmin(p->p[1], p->p[2]));
	*mx = vmax(p->p[0], vmax(p->p[1], p->p[2]));
}

static node_t init_node(ro_scene *s, uint32_t start, uint32_t count)   /* bvh_build.c:16 */
{
	node_t	nd;
	v3		mn, mx, bmn, bmx;

	prim_bounds(&s->prims[s->prim_idx[start]], &mn, &mx);
	for (uint32_t i = 0; i < count; i++)
	{
		prim_bounds(&s->prims[s->prim_idx[start + i]], &bmn, &bmx);
		mn = (v3){dmin_(mn.x, bmn.x), dmin_(mn.y, bmn.y), dmin_(mn.z, bmn.z)};
		mx = (v3){dmax_(mx.x, bmx.x), dmax_(mx.y, bmx.y), dmax_(mx.z, bmx.z)};
	}
	nd.bmin = mn;
	nd.bmax = mx;
	nd.first = start;
	nd.count = count;
	nd.leaf = count <= 1;
	nd.left = 0;
	nd.right = 0;
	return nd;
}

static int choose_axis(v3 e)                              /* bvh_build.c:44 */
{
	if (e.x > e.y && e.x > e.z)
		return 0;
	else if (e.y > e.z)
		return 1;
	return 2;
}

typedef struct { uint32_t start, count, parent; char is_left; } btask_t;

static void build_bvh(ro_scene *s)                        /* bvh_build.c:104-127 */
{
	btask_t		*stack;
	size_t		top = 0, cap = 64;
	uint32_t	n = s->n_prims;

	s->prim_idx = malloc(sizeof(uint32_t) * (n ? n : 1));
	s->nodes = malloc(sizeof(node_t) * (2 * (size_t)n + 1));
	for (uint32_t i = 0; i < n; i++)
		s->prim_idx[i] = i;
	s->n_nodes = 0;
	if (n == 0)
		return ;
	stack = malloc(sizeof(btask_t) * cap);
#define PUSH(T) do { if (top == cap) { cap *= 2; stack = realloc(stack, sizeof(btask_t) * cap); } stack[top++] = (T); } while (0)
#define SPLIT(IDX, TASK, ND) do { \
		v3 ext_ = vsub((ND).bmax, (ND).bmin); \
		uint32_t mid_ = (TASK).start + (TASK).count / 2; \
		int ax_ = choose_axis(ext_); \
		qsort_axis_(s->prim_idx + (TASK).start, 0, (TASK).count - 1, s, ax_); \
		if (mid_ - (TASK).start > 0) PUSH(((btask_t){(TASK).start, mid_ - (TASK).start, (IDX), 1})); \
		if ((TASK).start + (TASK).count - mid_ > 0) PUSH(((btask_t){mid_, (TASK).start + (TASK).count - mid_, (IDX), 0})); \
	} while (0)
	{
		uint32_t	idx = s->n_nodes++;
		node_t		nd = init_node(s, 0, n);
		btask_t		t = {0, n, UINT32_MAX, 0};

		s->nodes[idx] = nd;
		if (!nd.leaf)
			SPLIT(idx, t, nd);
	}
	while (top > 0)
	{
		btask_t		t = stack[--top];
		uint32_t	idx = s->n_nodes++;
		node_t		nd = init_node(s, t.start, t.count);

		s->nodes[idx] = nd;
		if (t.is_left)
			s->nodes[t.parent].left = idx;
		else
			s->nodes[t.parent].right = idx;
		if (!nd.leaf)
			SPLIT(idx, t, nd);
	}
#undef PUSH
#undef SPLIT
	free(stack);
}

/* ---------------------------------------------------------- intersection */

typedef struct
{
	int		hit;
	int		prim;       /* index into s->prims, or -1 - plane index */
	double	t;
	v3		point, normal;
	int		front_face;
	double	u, v;
	int		mat;
	const uint8_t	*objcolor;
	fc		color;
	int		has_hm;     /* hm holds this hit's textured material values */
	mat_t	hm;
}	hrec_t;

/* The material values at a hit: the material, or its copy with this hit's
 * texels (apply_all_map writes them into the shared t_mat before every use,
 * apply_map.c:60-85, which for one path at a time is the same thing). */
static inline const mat_t *hmat(ro_scene *s, const hrec_t *h)
{
	return (h->has_hm ? &h->hm : &s->mats[h->mat]);
}

/* intersect_aabb (bvh_utils.c:38-59); also returns the entry distance. */
static int isect_aabb(const ray_t *r, v3 mn, v3 mx, double *tentry)
{
	double	t1, tmax, tmin;

	t1 = fmin((mn.x - r->orig.x) / r->dir.x, (mx.x - r->orig.x) / r->dir.x);
	tmin = fmax(t1, fmin((mn.y - r->orig.y) / r->dir.y, (mx.y - r->orig.y) / r->dir.y));
	t1 = fmin((mn.z - r->orig.z) / r->dir.z, (mx.z - r->orig.z) / r->dir.z);
	tmin = fmax(tmin, t1);
	t1 = fmax((mn.x - r->orig.x) / r->dir.x, (mx.x - r->orig.x) / r->dir.x);
	tmax = fmin(t1, fmax((mn.y - r->orig.y) / r->dir.y, (mx.y - r->orig.y) / r->dir.y));
	t1 = fmax((mn.z - r->orig.z) / r->dir.z, (mx.z - r->orig.z) / r->dir.z);
	tmax = fmin(tmax, t1);
	*tentry = tmin;
	return (tmax >= fmax(tmin, 0.0) && tmin < 1000.0);
}

/* hit_sphere (hit_sphere.c:31) with init_sphere_quadratic / solve_quadratic
 * (quadratique.c:17,32), valid_t (valid_t.c:16), set_normal_face
 * (normal.c:16) and get_sphere_uv (hit_sphere.c:15). */
static int hit_sphere(ro_scene *s, prim_t *sp, const ray_t *r, hrec_t *rec)
{
	v3		oc = vsub(r->orig, sp->center);
	double	a = vdot(r->dir, r->dir);
	double	b = 2.0 * vdot(r->dir, oc);
	double	c = vdot(oc, oc) - sp->r2;
	double	disc, sq, den, t0, t1, th;
	v3		outward;

	s->cnt.sphere_tests++;
	disc = b * b - 4.0 * a * c;
	if (disc < 0.0)
		return 0;
	den = 2.0 * a;
	sq = sqrt(disc);
	t0 = (-b - sq) / den;
	t1 = (-b + sq) / den;
	th = t0;
	if (th < IT_MIN || th > IT_MAX)
	{
		th = t1;
		if (th < IT_MIN || th > IT_MAX)
			return 0;
	}
	rec->t = th;
	rec->point = ray_at(*r, th);
	outward = vdiv(vsub(rec->point, sp->center), sp->radius);
	if (vdot(r->dir, outward) < 0)
	{
		rec->front_face = 1;
		rec->normal = outward;
	}
	else
	{
		rec->front_face = 0;
		rec->normal = vneg(outward);
	}
	rec->u = clamp01((atan2((-rec->point.z + sp->center.z) / sp->radius,
					(rec->point.x - sp->center.x) / sp->radius) + PI_D) / (2 * PI_D));
	rec->v = clamp01(acos((-rec->point.y + sp->center.y) / sp->radius) / PI_D);
	if (sp->mat >= 0 && s->mats[sp->mat].scale != 1)
	{
		double	ip;

		rec->u *= s->mats[sp->mat].scale;
		rec->v *= s->mats[sp->mat].scale;
		rec->u = modf(rec->u, &ip);
		rec->v = modf(rec->v, &ip);
	}
	return 1;
}

/* hit_triangle (hit_triangle.c:68-93): Moller-Trumbore with the reference's
 * float intermediates (t_moller f/u/v/t are float, structs.h:99-110). */
static int hit_triangle_exact(ro_scene *s, prim_t *tr, const ray_t *r, hrec_t *rec);

static int hit_triangle(ro_scene *s, prim_t *tr, const ray_t *r, hrec_t *rec)
{
	v3		e1, e2, h, sv, q, n;
	float	a, f, u, v, t, w;

	if (s->exact)
		return hit_triangle_exact(s, tr, r, rec);
	s->cnt.tri_tests++;
	e1 = vsub(tr->p[1], tr->p[0]);
	e2 = vsub(tr->p[2], tr->p[0]);
	h = vcross(r->dir, e2);
	a = vdot(e1, h);
	if (s->one_sided == 1)
	{
		if (a < 1e-6)
			return 0;
	}
	else if (fabsf(a) < 1e-6)
		return 0;
	f = 1.0f / a;
	sv = vsub(r->orig, tr->p[0]);
	u = f * vdot(sv, h);
	if (u < 0.0f || u > 1.0f)
		return 0;
	q = vcross(sv, e1);
	v = f * vdot(r->dir, q);
	if (v < 0.0f || u + v > 1.0f)
		return 0;
	t = f * vdot(e2, q);
	if (t < IT_MIN || t > IT_MAX)
		return 0;
	rec->t = t;
	rec->point = ray_at(*r, t);
	w = 1.0f - u - v;
	n.x = w * tr->n[0].x + u * tr->n[1].x + v * tr->n[2].x;
	n.y = w * tr->n[0].y + u * tr->n[1].y + v * tr->n[2].y;
	n.z = w * tr->n[0].z + u * tr->n[1].z + v * tr->n[2].z;
	rec->normal = vunit(n);
	if (!s->one_sided && vdot(r->dir, rec->normal) > 0.0f)
	{
		rec->front_face = 0;
		rec->normal = vscale(rec->normal, -1.0f);
	}
	else
		rec->front_face = 1;
	rec->u = (1.0f - u - v) * tr->uv[0][0] + u * tr->uv[1][0] + v * tr->uv[2][0];
	rec->v = (1.0f - u - v) * tr->uv[0][1] + u * tr->uv[1][1] + v * tr->uv[2][1];
	return 1;
}

/* The same test with every intermediate in double (exact mode). */
static int hit_triangle_exact(ro_scene *s, prim_t *tr, const ray_t *r, hrec_t *rec)
{
	v3		e1, e2, h, sv, q, n;
	double	a, f, u, v, t, w;

	s->cnt.tri_tests++;
	e1 = vsub(tr->p[1], tr->p[0]);
	e2 = vsub(tr->p[2], tr->p[0]);
	h = vcross(r->dir, e2);
	a = vdot(e1, h);
	if (s->one_sided == 1 ? a < 1e-6 : fabs(a) < 1e-6)
		return 0;
	f = 1.0 / a;
	sv = vsub(r->orig, tr->p[0]);
	u = f * vdot(sv, h);
	if (u < 0.0 || u > 1.0)
		return 0;
	q = vcross(sv, e1);
	v = f * vdot(r->dir, q);
	if (v < 0.0 || u + v > 1.0)
		return 0;
	t = f * vdot(e2, q);
	if (t < IT_MIN || t > IT_MAX)
		return 0;
	rec->t = t;
	rec->point = ray_at(*r, t);
	w = 1.0 - u - v;
	n.x = w * tr->n[0].x + u * tr->n[1].x + v * tr->n[2].x;
	n.y = w * tr->n[0].y + u * tr->n[1].y + v * tr->n[2].y;
	n.z = w * tr->n[0].z + u * tr->n[1].z + v * tr->n[2].z;
	rec->normal = vunit(n);
	if (!s->one_sided && vdot(r->dir, rec->normal) > 0.0)
	{
		rec->front_face = 0;
		rec->normal = vscale(rec->normal, -1.0);
	}
	else
		rec->front_face = 1;
	rec->u = w * tr->uv[0][0] + u * tr->uv[1][0] + v * tr->uv[2][0];
	rec->v = w * tr->uv[0][1] + u * tr->uv[1][1] + v * tr->uv[2][1];
	return 1;
}

/* ------------------------------------------------------------ quadrics */

/* solve_quadratic (quadratique.c:17) */
static int solve_q(double a, double b, double c, double *t0, double *t1)
{
	double	disc = b * b - 4.0 * a * c;
	double	sq, den;

	if (disc < 0.0)
		return (0);
	den = 2.0 * a;
	sq = sqrt(disc);
	*t0 = (-b - sq) / den;
	*t1 = (-b + sq) / den;
	return (1);
}

/* valid_t (valid_t.c:16) */
static int valid_root(double t0, double t1, double *th)
{
	*th = t0;
	if (*th < IT_MIN || *th > IT_MAX)
	{
		*th = t1;
		if (*th < IT_MIN || *th > IT_MAX)
			return (0);
	}
	return (1);
}

/* set_normal_face (normal.c:16) */
static v3 face(const ray_t *r, v3 n, hrec_t *rec)
{
	if (vdot(r->dir, n) < 0)
	{
		rec->front_face = 1;
		return (n);
	}
	rec->front_face = 0;
	return (vneg(n));
}

/* texture coordinates of the quadrics (cylinder_uv.c:16-58,
 * hit_cone.c:14-52, hit_hyperboloid.c:14-34): the material's scale tiles
 * them as for spheres */
static void uv_tile(ro_scene *s, int mat, hrec_t *rec)
{
	double	ip;

	if (mat >= 0 && s->mats[mat].scale != 1)
	{
		rec->u *= s->mats[mat].scale;
		rec->v *= s->mats[mat].scale;
		rec->u = modf(rec->u, &ip);
		rec->v = modf(rec->v, &ip);
	}
}

static v3 uv_right(v3 ori)
{
	if (fabs(ori.y) < 0.99)
		return (vunit(vcross((v3){0, 1, 0}, ori)));
	return (vunit(vcross((v3){1, 0, 0}, ori)));
}

static double uv_angle(v3 rel, v3 ori)
{
	v3	right = uv_right(ori);

	return (clamp01((atan2(vdot(rel, vcross(ori, right)), vdot(rel, right)) + PI_D) / (2.0 * PI_D)));
}

static void uv_cap(hrec_t *rec, v3 centre, v3 ori, double diam)
{
	v3	right = uv_right(ori);
	v3	rel = vsub(rec->point, centre);

	rec->u = clamp01((vdot(rel, right) / diam) + 0.5);
	rec->v = clamp01((vdot(rel, vcross(ori, right)) / diam) + 0.5);
}

/* one cap of hit_cylinder (hit_cylinder.c:39-99); normal n as given */
static int cyl_cap(const ray_t *r, v3 c, v3 ori, double rad, v3 n, hrec_t *rec)
{
	double	den = vdot(r->dir, ori);
	double	t;
	v3		hp;

	if (fabs(den) < 1e-6)
		return (0);
	t = -vdot(vsub(r->orig, c), ori) / den;
	if (t < IT_MIN || t > IT_MAX)
		return (0);
	hp = ray_at(*r, t);
	if (vlen(vsub(hp, c)) > rad)
		return (0);
	rec->t = t;
	rec->point = hp;
	rec->normal = n;
	rec->front_face = (vdot(r->dir, rec->normal) < 0);
	return (1);
}

/* hit_cylinder (hit_cylinder.c:110-134) with handle_cylinder_hit (:15-37)
 * and the cap materials of update_hit_cylinder (hit_obj.c:16-32) */
static int hit_cylinder(ro_scene *s, prim_t *p, const ray_t *r, hrec_t *rec)
{
	v3		ori = p->ori;
	v3		axis, oc, pt, base;
	double	dd, oo, t0, t1, th, proj, rad = p->diam * 0.5;
	int		hit_any = 0;
	hrec_t	tmp;

	if (ori.x == 0 && ori.y == 0 && ori.z == 0)
		ori.y = 1;
	axis = vunit(ori);
	oc = vsub(r->orig, p->center);
	dd = vdot(r->dir, ori);
	oo = vdot(oc, ori);
	if (solve_q(vdot(r->dir, r->dir) - dd * dd, 2.0 * (vdot(r->dir, oc) - dd * oo),
			vdot(oc, oc) - oo * oo - rad * rad, &t0, &t1) && valid_root(t0, t1, &th))
	{
		pt = ray_at(*r, th);
		base = vsub(p->center, vscale(axis, p->height * 0.5));
		proj = vdot(vsub(pt, base), axis);
		if (!(proj < 0.0 || proj > p->height))
		{
			v3	out = vunit(vsub(vsub(pt, base), vscale(axis, proj)));

			rec->t = th;
			rec->point = pt;
			rec->normal = face(r, out, rec);
			rec->mat = p->mat;
			rec->u = uv_angle(vsub(pt, p->center), ori);
			rec->v = clamp01((vdot(vsub(pt, p->center), ori) / p->height) + 0.5);
			uv_tile(s, rec->mat, rec);
			hit_any = 1;
		}
	}
	memset(&tmp, 0, sizeof(tmp));
	if (cyl_cap(r, vsub(p->center, vscale(axis, p->height * 0.5)), ori, rad, vneg(ori), &tmp)
		&& (!hit_any || tmp.t < rec->t))
	{
		tmp.mat = p->mat_bot >= 0 ? p->mat_bot : p->mat;
		uv_cap(&tmp, vadd(p->center, vscale(ori, p->height * 0.5 * -1)), ori, p->diam);
		uv_tile(s, tmp.mat, &tmp);
		*rec = tmp;
		hit_any = 1;
	}
	memset(&tmp, 0, sizeof(tmp));
	if (cyl_cap(r, vadd(p->center, vscale(axis, p->height * 0.5)), ori, rad, ori, &tmp)
		&& (!hit_any || tmp.t < rec->t))
	{
		tmp.mat = p->mat_top >= 0 ? p->mat_top : p->mat;
		uv_cap(&tmp, vadd(p->center, vscale(ori, p->height * 0.5 * 1)), ori, p->diam);
		uv_tile(s, tmp.mat, &tmp);
		*rec = tmp;
		hit_any = 1;
	}
	if (!hit_any)
		return (0);
	rec->front_face = (vdot(r->dir, rec->normal) < 0);
	rec->normal = face(r, rec->normal, rec);
	return (1);
}

/* hit_cone (hit_cone.c:108-129) with handle_cone_hit (:54-75), cone_cap
 * (:77-106) and update_hit_cone (hit_obj.c:34-47) */
static int hit_cone(ro_scene *s, prim_t *p, const ray_t *r, hrec_t *rec)
{
	v3		ori = p->ori;
	v3		axis, oc, pt, n, cap;
	double	k, dd, oo, t0, t1, th, proj, den, t, q;

	if (ori.x == 0 && ori.y == 0 && ori.z == 0)
		ori.y = 1;
	k = pow((p->diam * 0.5) / p->height, 2);
	oc = vsub(r->orig, p->center);
	dd = vdot(r->dir, ori);
	oo = vdot(oc, ori);
	if (!solve_q(vdot(r->dir, r->dir) - (1.0 + k) * dd * dd, 2.0 * (vdot(r->dir, oc) - (1.0 + k) * dd * oo),
			vdot(oc, oc) - (1.0 + k) * oo * oo, &t0, &t1) || !valid_root(t0, t1, &th))
		return (0);
	axis = vunit(ori);
	pt = ray_at(*r, th);
	proj = vdot(vsub(pt, p->center), axis);
	if (!(proj < 0.0 || proj > p->height))
	{
		q = p->diam * 0.5 / p->height;
		n = vunit(vsub(vsub(pt, p->center), vscale(axis, (1.0 + q * q) * proj)));
		rec->t = th;
		rec->point = pt;
		rec->normal = face(r, n, rec);
		rec->mat = p->mat;
		rec->u = uv_angle(vsub(pt, p->center), ori);
		rec->v = clamp01((vdot(vsub(pt, p->center), ori) / (p->height)));
		uv_tile(s, rec->mat, rec);
		return (1);
	}
	cap = vadd(p->center, vscale(axis, p->height));
	den = vdot(r->dir, axis);
	if (fabs(den) < 1e-6)
		return (0);
	t = vdot(vsub(cap, r->orig), axis) / den;
	if (t < IT_MIN || t > IT_MAX)
		return (0);
	pt = ray_at(*r, t);
	if (vlen(vsub(pt, cap)) > p->diam * 0.5)
		return (0);
	rec->t = t;
	rec->point = pt;
	rec->normal = axis;
	rec->mat = p->mat_top >= 0 ? p->mat_top : p->mat;
	uv_cap(rec, vadd(p->center, vscale(ori, p->height * 0.5)), ori, p->diam);
	uv_tile(s, rec->mat, rec);
	rec->front_face = (vdot(r->dir, rec->normal) < 0);
	rec->normal = face(r, rec->normal, rec);
	return (1);
}

/* hit_hyperboloid (hit_hyperboloid.c:80-104), init_hyperboloid_quadratic
 * (quadratique_hyperboloid.c:15-63), compute_normal (hit_hyperboloid.c:36-52) */
static int hyp_side(ro_scene *s, prim_t *p, const ray_t *r, double t, hrec_t *rec)
{
	v3		axis = vunit(p->ori);
	v3		pt = ray_at(*r, t);
	v3		to_p = vsub(pt, p->center);
	v3		tmp, u, v, n;

	if (!(fabs(vdot(to_p, axis)) <= p->height * 0.5))
		return (0);
	tmp = fabs(axis.y) < 0.99 ? (v3){0, 1, 0} : (v3){1, 0, 0};
	u = vunit(vcross(tmp, axis));
	v = vcross(axis, u);
	n = vunit(vadd(vadd(vscale(u, 2.0 * vdot(to_p, u) / (p->qa * p->qa)),
					vscale(v, 2.0 * vdot(to_p, v) / (p->qb * p->qb))),
				vscale(axis, -2.0 * vdot(to_p, axis) / (p->qc * p->qc))));
	rec->t = t;
	rec->point = pt;
	rec->normal = face(r, n, rec);
	rec->front_face = vdot(r->dir, n) < 0;
	rec->mat = p->mat;
	rec->u = uv_angle(to_p, p->ori);
	rec->v = clamp01((vdot(vsub(pt, p->center), p->ori) / (p->height * 0.5)) * 0.5 + 0.5);
	uv_tile(s, p->mat, rec);
	return (1);
}

static int hit_hyperboloid(ro_scene *s, prim_t *p, const ray_t *r, hrec_t *rec)
{
	v3		x, y, z, tmp, rel, ld, lo;
	double	aa = p->qa * p->qa, bb = p->qb * p->qb, cc = p->qc * p->qc, t0, t1, imax = IT_MAX;
	int		hit = 0;
	prim_t	q = *p;

	if (vlen2(q.ori) < 1e-6)
		q.ori = (v3){0, 0, 1};
	z = vunit(q.ori);
	tmp = fabs(z.x) > 0.9 ? (v3){0, 1, 0} : (v3){1, 0, 0};
	x = vunit(vcross(tmp, z));
	y = vcross(z, x);
	rel = vsub(r->orig, q.center);
	ld = (v3){vdot(r->dir, x), vdot(r->dir, y), vdot(r->dir, z)};
	lo = (v3){vdot(rel, x), vdot(rel, y), vdot(rel, z)};
	if (!solve_q((ld.x * ld.x) / aa + (ld.y * ld.y) / bb - (ld.z * ld.z) / cc,
			2.0 * ((ld.x * lo.x) / aa + (ld.y * lo.y) / bb - (ld.z * lo.z) / cc),
			(lo.x * lo.x) / aa + (lo.y * lo.y) / bb - (lo.z * lo.z) / cc - q.shape, &t0, &t1))
		return (0);
	if (t0 > IT_MIN && t0 < imax && hyp_side(s, &q, r, t0, rec))
	{
		hit = 1;
		imax = t0;
	}
	if (t1 > IT_MIN && t1 < imax && hyp_side(s, &q, r, t1, rec))
		hit = 1;
	return (hit);
}

static int hit_prim(ro_scene *s, prim_t *p, const ray_t *r, hrec_t *rec)
{
	if (p->type == PT_SPHERE)
		return (hit_sphere(s, p, r, rec));
	if (p->type == PT_TRI)
		return (hit_triangle(s, p, r, rec));
	if (p->type == PT_CYL)
		return (hit_cylinder(s, p, r, rec));
	if (p->type == PT_CONE)
		return (hit_cone(s, p, r, rec));
	return (hit_hyperboloid(s, p, r, rec));
}

/* hit_plane + get_uv_plane (hit_plane.c:18-71). */
static int hit_plane(ro_scene *s, plane_t *p, const ray_t *r, hrec_t *rec)
{
	double	denom = p->normal.x * r->dir.x + p->normal.y * r->dir.y + p->normal.z * r->dir.z;
	double	t = ((p->point.x - r->orig.x) * p->normal.x + (p->point.y - r->orig.y) * p->normal.y
			+ (p->point.z - r->orig.z) * p->normal.z) / denom;
	v3		up, tg, loc;
	double	u, v;

	s->cnt.plane_tests++;
	if (fabs(denom) < 1e-8)
		return 0;
	if (t < IT_MIN || t > IT_MAX)
		return 0;
	rec->t = t;
	rec->point.x = r->orig.x + t * r->dir.x;
	rec->point.y = r->orig.y + t * r->dir.y;
	rec->point.z = r->orig.z + t * r->dir.z;
	rec->front_face = ((r->dir.x * p->normal.x + r->dir.y * p->normal.y
				+ r->dir.z * p->normal.z) < 0);
	rec->normal = rec->front_face ? p->normal : (v3){-p->normal.x, -p->normal.y, -p->normal.z};
	up = fabs(p->normal.y) < 0.99 ? (v3){0, 1, 0} : (v3){1, 0, 0};
	tg = vunit(vcross(up, p->normal));
	loc = vsub(rec->point, p->point);
	u = vdot(loc, tg);
	v = vdot(loc, vcross(p->normal, tg));
	if (p->mat >= 0)
	{
		u *= s->mats[p->mat].scale * 0.1;
		v *= s->mats[p->mat].scale * 0.1;
	}
	rec->u = u - floor(u);
	rec->v = v - floor(v);
	return 1;
}

/* Closest BVH hit. The reference (hit_bvh, bvh_hit.c:16-43) recurses into
 * both children of every node whose box the ray enters and keeps the smaller
 * t, the left result on ties. With one primitive per leaf and leaves laid out
 * left-to-right in prim_indices order, that is: minimum t, ties to the lowest
 * leaf position. This traversal visits near children first and skips boxes
 * entered beyond the best t (strictly), which gives the same answer. */
/* ------------------------------------------------------------ textures */

/* get_solid_texture_default / get_solid_texture (get_solid_texture.c:15-43) */
static fc solid_checker(v3 p, double scale, const uint8_t *c1, const uint8_t *c2)
{
	int	a, b, c;

	p = vscale(p, scale);
	a = floor(p.x);
	b = floor(p.y + 0.5);
	c = floor(p.z);
	if ((a + b + c) % 2 == 0)
		return (c2f(c1));
	return (c2f(c2));
}

/* get_tex_color (get_tex_color.c:27-48); k is 1 + the texture index */
static fc tex_color(ro_scene *s, int k, double u, double v, v3 point)
{
	static const uint8_t	black[3] = {0, 0, 0}, magenta[3] = {243, 0, 243};
	tex_t					*t = &s->texs[k - 1];
	int						a, b;

	if (t->type == MRT_TEX_IMAGE)
	{
		const uint8_t	*px;

		if (!t->rgba || !t->w || !t->h)
			return (solid_checker(point, 2, black, magenta));
		px = t->rgba + 4 * ((size_t)t->w * (int)(v * (t->h - 1)) + (int)(u * (t->w - 1)));
		return ((fc){px[0] / 255.0, px[1] / 255.0, px[2] / 255.0});
	}
	if (t->type == MRT_TEX_CHECKER_LOCAL)
	{
		a = floor(u * t->scale);
		b = floor(v * t->scale);
		if ((a + b) % 2 == 0)
			return (c2f(t->c1));
		return (c2f(t->c2));
	}
	if (t->type == MRT_TEX_CHECKER_GLOBAL)
		return (solid_checker(point, t->scale, t->c1, t->c2));
	return ((fc){0.0, 0.0, 0.0});
}

/* get_tex_transparency (get_tex_color.c:51-62) */
static double tex_transparency(ro_scene *s, int k, double u, double v)
{
	tex_t	*t = &s->texs[k - 1];

	if (t->type != MRT_TEX_IMAGE || !t->rgba || !t->w || !t->h)
		return (0.0);
	return (1 - t->rgba[4 * ((size_t)t->w * (int)(v * (t->h - 1)) + (int)(u * (t->w - 1))) + 3] / 255.0);
}

/* Uniform of the partial-transparency test in counter mode: a hash of the
 * path's stream state at the traversal and the object's flat id, the same
 * function as the kernels' alpha_uniform. The reference draws
 * random_double() here (hit_register.c:66-71), in the order of its
 * exhaustive leaf recursion, which no culled traversal reproduces. */
static double alpha_uniform(uint64_t key, uint32_t flat)
{
	uint64_t	z = key ^ ((uint64_t)(flat + 1) * 0x9E3779B97F4A7C15ULL);

	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
	z ^= z >> 31;
	return (double)(float)((float)(z >> 40) * (1.0f / 16777216.0f));
}

/* The leaf's alpha test (hit_register_bvh, hit_register.c:62-72): 1 when
 * the candidate hit is dropped. */
static int alpha_drops(ro_scene *s, const hrec_t *h, uint32_t flat)
{
	double	tr;
	rng_t	ref = {RO_RNG_REFERENCE, 0};

	if (h->mat < 0 || !s->mats[h->mat].tex[TX_COLOR])
		return (0);
	tr = tex_transparency(s, s->mats[h->mat].tex[TX_COLOR], h->u, h->v);
	if (tr == 1)
		return (1);
	if (tr == 0)
		return (0);
	if (s->rg && s->rg->mode == RO_RNG_COUNTER)
		return (alpha_uniform(s->rg->state, flat) < tr);
	return (rnd(s->rg ? s->rg : &ref) < tr);
}

static void bvh_closest(ro_scene *s, const ray_t *r, hrec_t *best, int *best_pos)
{
	uint32_t	stack[128];
	int			sp = 0;
	double		te;
	hrec_t		tmp;

	if (!s->n_nodes)
		return ;
	stack[sp++] = 0;
	while (sp > 0)
	{
		node_t	*nd = &s->nodes[stack[--sp]];

		s->cnt.node_visits++;
		if (!isect_aabb(r, nd->bmin, nd->bmax, &te))
			continue ;
		if (best->hit && te > best->t)
			continue ;
		if (nd->leaf)
		{
			prim_t	*p = &s->prims[s->prim_idx[nd->first]];
			int		ok;

			s->cnt.prim_tests++;
			memset(&tmp, 0, sizeof(tmp));
			ok = hit_prim(s, p, r, &tmp);
			if (!ok || tmp.t >= 1000)
				continue ;
			if (p->type == PT_SPHERE || p->type == PT_TRI)
				tmp.mat = p->mat;
			if (s->n_texs && alpha_drops(s, &tmp, p->flat))
				continue ;
			if (!best->hit || tmp.t < best->t || (tmp.t == best->t && (int)nd->first < *best_pos))
			{
				tmp.hit = 1;
				tmp.prim = s->prim_idx[nd->first];
				if (p->type == PT_SPHERE || p->type == PT_TRI)
					tmp.mat = p->mat;
				tmp.objcolor = p->color;
				*best = tmp;
				*best_pos = nd->first;
			}
			continue ;
		}
		{
			node_t	*L = &s->nodes[nd->left], *R = &s->nodes[nd->right];
			double	tl, tr;
			int		hl = isect_aabb(r, L->bmin, L->bmax, &tl);
			int		hr = isect_aabb(r, R->bmin, R->bmax, &tr);

			if (sp + 2 > 128)
				abort();
			if (hl && hr && tr < tl)
			{
				stack[sp++] = nd->left;
				stack[sp++] = nd->right;
			}
			else
			{
				stack[sp++] = nd->right;
				stack[sp++] = nd->left;
			}
		}
	}
}

/* Node-visit count of the reference's exhaustive recursion (the BVH heat
 * map, bvh_hit.c:25: one count per hit_bvh call). */
static int bvh_depth_count(ro_scene *s, const ray_t *r, uint32_t idx)
{
	node_t	*nd = &s->nodes[idx];
	double	te;
	int		c = 1;

	if (!isect_aabb(r, nd->bmin, nd->bmax, &te))
		return c;
	if (nd->leaf)
		return c;
	c += bvh_depth_count(s, r, nd->left);
	c += bvh_depth_count(s, r, nd->right);
	return c;
}

/* apply_normal_map + init_tbn (apply_map.c:15-58): the texel in [-1, 1]
 * (float arithmetic, as map.r / 127.5f - 1.0f) in the frame tangent =
 * unit(n x (0,-1,0)) (or n x (0,0,1)), bitangent = unit(n x tangent), n. */
static void normal_map(ro_scene *s, hrec_t *h, const mat_t *m)
{
	tex_t			*t = &s->texs[m->tex[TX_NORMAL] - 1];
	const uint8_t	*px;
	v3				mp, tg, bt, n = h->normal, res;

	if (!t->rgba)
		return ;
	px = t->rgba + 4 * ((size_t)t->w * (int)(h->v * (t->h - 1)) + (int)(h->u * (t->w - 1)));
	mp = (v3){(px[0] / 127.5f) - 1.0f, (px[1] / 127.5f) - 1.0f, (px[2] / 127.5f) - 1.0f};
	tg = vcross(n, (v3){0, -1, 0});
	if (vlen(tg) == 0)
		tg = vcross(n, (v3){0, 0, 1});
	tg = vunit(tg);
	bt = vunit(vcross(n, tg));
	res.x = mp.x * tg.x + mp.y * bt.x + mp.z * n.x;
	res.y = mp.x * tg.y + mp.y * bt.y + mp.z * n.y;
	res.z = mp.x * tg.z + mp.y * bt.z + mp.z * n.z;
	if (m->normal_intensity == 1.0)
		h->normal = vunit(res);
	else
	{
		double	w = m->normal_intensity;
		v3		b = vunit(res);

		h->normal = vunit((v3){(1 - w) * n.x + w * b.x, (1 - w) * n.y + w * b.y, (1 - w) * n.z + w * b.z});
	}
}

/* apply_all_map (apply_map.c:60-85) into the hit's own copy of the
 * material: normal map, transmission, then (not for shadow rays) roughness,
 * metallic, ao, emission strength and colour, each the texel's .r (the
 * colour for emission colour). */
static void apply_maps(ro_scene *s, hrec_t *h)
{
	const mat_t	*m;

	if (h->mat < 0 || !s->mats[h->mat].textured)
		return ;
	m = &s->mats[h->mat];
	h->hm = *m;
	h->has_hm = 1;
	if (m->tex[TX_NORMAL])
		normal_map(s, h, m);
	if (m->tex[TX_TRANSMISSION])
		h->hm.transmission = tex_color(s, m->tex[TX_TRANSMISSION], h->u, h->v, h->point).r;
	if (s->is_light)
		return ;
	if (m->tex[TX_ROUGHNESS])
		h->hm.roughness = tex_color(s, m->tex[TX_ROUGHNESS], h->u, h->v, h->point).r;
	if (m->tex[TX_METALLIC])
		h->hm.metallic = tex_color(s, m->tex[TX_METALLIC], h->u, h->v, h->point).r;
	if (m->tex[TX_AO])
		h->hm.ao = tex_color(s, m->tex[TX_AO], h->u, h->v, h->point).r;
	if (m->tex[TX_EMIS_STRENGTH])
		h->hm.emission_strength = tex_color(s, m->tex[TX_EMIS_STRENGTH], h->u, h->v, h->point).r;
	if (m->tex[TX_EMIS_COLOR])
		h->hm.emission_color = tex_color(s, m->tex[TX_EMIS_COLOR], h->u, h->v, h->point);
}

/* get_hit_register_color (get_hit_color.c:17-36). */
static fc hit_color(ro_scene *s, hrec_t *h)
{
	if (s->render_mode == 2)
		return (fc){(h->normal.x + 1) * 0.5, (h->normal.z + 1) * 0.5, (h->normal.y + 1) * 0.5};
	if (h->mat >= 0 && s->mats[h->mat].tex[TX_COLOR])
		return tex_color(s, s->mats[h->mat].tex[TX_COLOR], h->u, h->v, h->point);
	if (h->mat >= 0 && s->albedo_d)
		return (fc){s->albedo_d[3 * h->mat], s->albedo_d[3 * h->mat + 1], s->albedo_d[3 * h->mat + 2]};
	if (h->mat >= 0)
		return c2f(s->mats[h->mat].c8);
	return c2f(h->objcolor);
}

/* hit_register_all (hit_register.c:79-120): BVH primitives, then every
 * plane (a plane wins only with a strictly smaller t). */
static int hit_register_all_(ro_scene *s, const ray_t *r, hrec_t *out, int *bvh_hit)
{
	hrec_t	best;
	hrec_t	tmp;
	int		pos = 0x7fffffff;

	memset(&best, 0, sizeof(best));
	bvh_closest(s, r, &best, &pos);
	if (bvh_hit)
		*bvh_hit = best.hit;
	if (best.hit)
	{
		apply_maps(s, &best);
		best.color = hit_color(s, &best);
	}
	for (int i = 0; i < s->n_planes; i++)
	{
		memset(&tmp, 0, sizeof(tmp));
		if (hit_plane(s, &s->planes[i], r, &tmp))
		{
			if (!best.hit || tmp.t < best.t)
			{
				tmp.hit = 1;
				tmp.prim = -1 - i;
				tmp.mat = s->planes[i].mat;
				tmp.objcolor = s->planes[i].color;
				apply_maps(s, &tmp);
				tmp.color = hit_color(s, &tmp);
				best = tmp;
			}
		}
	}
	if (best.hit)
		*out = best;
	return best.hit;
}

static int hit_register_all(ro_scene *s, const ray_t *r, hrec_t *out)
{
	return hit_register_all_(s, r, out, NULL);
}

static int flat_of(ro_scene *s, int prim)
{
	if (prim >= 0)
		return s->prims[prim].flat;
	return s->planes[-1 - prim].flat;
}

static int flat_of_prim(ro_scene *s, int prim)
{
	return flat_of(s, prim);
}

/* ------------------------------------------------------------------ sky */

/* get_hdr_pixel_skybox (get_hdr_value.c:43-68). */
static fc hdr_pixel_sky(ro_scene *s, int x, int y)
{
	const uint8_t	*px = s->rgbe + 4 * ((size_t)y * s->hw + x);
	double			exposure = s->hdr_exposure + s->amb_ratio - 1;
	double			scale, g;

	if (s->sky_d)
	{
		const double	*t = s->sky_d + 3 * ((size_t)y * s->hw + x);

		return (fc){t[0], t[1], t[2]};
	}
	if (exposure == 0)
		scale = ldexp(1.0, px[3] - 128);
	else
		scale = ldexp(1.0, px[3] - 128) * powf(2.0, exposure);
	if (s->hdr_gamma == 1.0)
		return (fc){px[0] * scale / 255.0, px[1] * scale / 255.0, px[2] * scale / 255.0};
	g = 1.0 / s->hdr_gamma;
	return (fc){pow(px[0] * scale / 255.0, g), pow(px[1] * scale / 255.0, g),
		pow(px[2] * scale / 255.0, g)};
}

/* get_background_color[_clamp] (background.c:15-84) for HDR or no sky. */
static fc background(ro_scene *s, ray_t r, int clamp)
{
	double	u, v;
	fc		c;

	if (!s->rgbe)
		return fscale(c2f(s->amb_color), s->amb_ratio);
	r.dir = vunit(r.dir);
	v = 0.5 + asin(r.dir.y) / PI_D;
	u = 0.5 - atan2(r.dir.z, r.dir.x) / (2.0 * PI_D);
	c = hdr_pixel_sky(s, (int)(u * (s->hw - 1)), (int)(v * (s->hh - 1)));
	if (clamp)
		c = (fc){clampv(c.r, 0, 16), clampv(c.g, 0, 16), clampv(c.b, 0, 16)};
	return c;
}

/* ------------------------------------------------------ HDRI tables
 * importance_sampling_manager.c:41-62, calc_pdf.c:16-115, calc_cdf.c:16-129. */

static double grey_value(ro_scene *s, size_t i)          /* calc_pdf.c:16 */
{
	const uint8_t	*p = s->rgbe + 4 * i;
	double			scale;

	if (s->sky_d)   /* linear sky: grey of the 0..255-scaled radiance */
		return 0.2126 * (s->sky_d[3 * i] * 255.0) + 0.7152 * (s->sky_d[3 * i + 1] * 255.0)
			+ 0.0722 * (s->sky_d[3 * i + 2] * 255.0);
	if (s->hdr_exposure == 0)
		scale = ldexp(1.0, p[3] - 128);
	else
		scale = ldexp(1.0, p[3] - 128) * powf(2.0, s->hdr_exposure);
	return 0.2126 * (p[0] * scale) + 0.7152 * (p[1] * scale) + 0.0722 * (p[2] * scale);
}

static void build_env_tables(ro_scene *s)
{
	int		W = s->hw, H = s->hh;
	double	*gray = calloc((size_t)W * H, sizeof(double));
	double	*raw = calloc(H, sizeof(double));
	double	*pm = calloc(H, sizeof(double));
	double	*pc = calloc((size_t)W * H, sizeof(double));
	double	*ch = calloc(H, sizeof(double));
	double	*cw = calloc(W, sizeof(double));
	double	sum;

	free(s->pdf_joint);
	free(s->pdf_joint_d);
	free(s->cdf_m_inv);
	free(s->cdf_c_inv);
	s->pdf_joint = calloc((size_t)W * H, sizeof(float));
	s->pdf_joint_d = calloc((size_t)W * H, sizeof(double));
	s->cdf_m_inv = calloc(H, sizeof(float));
	s->cdf_c_inv = calloc((size_t)W * H, sizeof(float));
	for (size_t i = 0; i < (size_t)W * H; i++)
		gray[i] = grey_value(s, i);
	for (int i = 0; i < H; i++)
	{
		sum = 0;
		for (int j = 0; j < W; j++)
			sum += gray[i * W + j];
		raw[i] = sum / W;
	}
	sum = 0;
	for (int i = 0; i < H; i++)
		sum += raw[i];
	s->column_average = sum / H;
	for (int i = 0; i < H * W; i++)
	{
		s->pdf_joint[i] = gray[i] / (s->column_average);
		s->pdf_joint_d[i] = gray[i] / (s->column_average);
	}
	for (int i = 0; i < H; i++)
		pm[i] = raw[i] / (s->column_average / 255);
	for (int i = 0; i < H; i++)
		for (int j = 0; j < W; j++)
			pc[i * W + j] = gray[i * W + j] / (raw[i] / 255);
	/* marginal (calc_cdf.c:16-58) */
	sum = 0.0;
	for (int i = 0; i < H; i++)
	{
		sum += pm[i];
		ch[i] = sum;
	}
	if (sum > 0.0)
		for (int i = 0; i < H; i++)
			ch[i] /= sum;
	for (int i = 0; i < H; i++)
	{
		double u = (double)i / (H - 1);
		for (int y = 0; y < H; y++)
			if (ch[y] >= u)
			{
				s->cdf_m_inv[i] = (double)y / (H - 1);
				break ;
			}
	}
	/* conditional rows (calc_cdf.c:60-129) */
	for (int y = 0; y < H; y++)
	{
		sum = 0.0;
		for (int x = 0; x < W; x++)
		{
			sum += pc[y * W + x];
			cw[x] = sum;
		}
		if (sum > 0.0)
			for (int x = 0; x < W; x++)
				cw[x] /= sum;
		for (int i = 0; i < W; i++)
		{
			double u = (double)i / (double)(W - 1);
			for (int x = 0; x < W; x++)
				if (cw[x] >= u)
				{
					s->cdf_c_inv[y * W + i] = (double)x / (double)(W - 1);
					break ;
				}
		}
	}
	free(gray);
	free(raw);
	free(pm);
	free(pc);
	free(ch);
	free(cw);
}

/* ------------------------------------------------------------- caustics */

static int kd_partition(photon_t *p, int l, int r, int a)        /* kd_tree_build_utils.c:32 */
{
	float	pivot = (float)(a == 0 ? p[r].pos.x : a == 1 ? p[r].pos.y : p[r].pos.z);
	int		i = l - 1, j = r;
	photon_t	t;

#define POS_A(P) ((float)((a) == 0 ? (P).pos.x : (a) == 1 ? (P).pos.y : (P).pos.z))
	while (1)
	{
		while (POS_A(p[++i]) < pivot)
			;
		while (j > l && POS_A(p[--j]) > pivot)
			;
		if (i >= j)
			break ;
		t = p[i]; p[i] = p[j]; p[j] = t;
	}
	t = p[i]; p[i] = p[r]; p[r] = t;
#undef POS_A
	return i;
}

static void kd_median(photon_t *p, int start, int end, int med, int a)  /* :57 */
{
	while (start < end)
	{
		int i = kd_partition(p, start, end, a);

		if (i == med)
			return ;
		else if (i < med)
			start = i + 1;
		else
			end = i - 1;
	}
}

typedef struct { int start, end, depth; kd_t **link; v3 mn, mx; } kdtask_t;

/* kd_tree_build (kd_tree_build.c:17-105) + process_task (kd_tree_task.c:16-96):
 * axis = depth % 3, quickselect median, leaves of <= 1000 photons; the median
 * photon of an internal node belongs to neither child. */
static void kd_build(ro_scene *s)
{
	size_t		n = s->n_photons;
	kdtask_t	*st = malloc(sizeof(kdtask_t) * (n + 1));
	int			top = 0;
	size_t		cur = 0;

	s->kd_nodes = malloc(sizeof(kd_t) * (n + 1));
	s->kd_root = NULL;
	st[0].start = 0;
	st[0].end = (int)n - 1;
	st[0].depth = 0;
	st[0].link = &s->kd_root;
	st[0].mn = s->photons[0].pos;
	st[0].mx = s->photons[0].pos;
	for (size_t i = 0; i < n; i++)
	{
		st[0].mn.x = fmin(st[0].mn.x, s->photons[i].pos.x);
		st[0].mn.y = fmin(st[0].mn.y, s->photons[i].pos.y);
		st[0].mn.z = fmin(st[0].mn.z, s->photons[i].pos.z);
		st[0].mx.x = fmax(st[0].mx.x, s->photons[i].pos.x);
		st[0].mx.y = fmax(st[0].mx.y, s->photons[i].pos.y);
		st[0].mx.z = fmax(st[0].mx.z, s->photons[i].pos.z);
	}
	top = 1;
	while (top > 0)
	{
		kdtask_t	t = st[--top];
		kd_t		*nd;

		if (t.start > t.end)
		{
			*t.link = NULL;
			continue ;
		}
		nd = &s->kd_nodes[cur++];
		*t.link = nd;
		nd->bmin = t.mn;
		nd->bmax = t.mx;
		if (t.end - t.start + 1 <= MAX_PHOTONS_PER_LEAF)
		{
			nd->axis = -1;
			nd->start = t.start;
			nd->count = t.end - t.start + 1;
			continue ;
		}
		{
			int		axis = t.depth % 3;
			int		mi = t.start + (t.end - t.start) / 2;
			float	sp;

			kd_median(s->photons, t.start, t.end, mi, axis);
			sp = (float)(axis == 0 ? s->photons[mi].pos.x : axis == 1
					? s->photons[mi].pos.y : s->photons[mi].pos.z);
			nd->axis = axis;
			nd->split = sp;
			st[top] = (kdtask_t){mi + 1, t.end, t.depth + 1, &nd->right, t.mn, t.mx};
			if (axis == 0) st[top].mn.x = sp; else if (axis == 1) st[top].mn.y = sp; else st[top].mn.z = sp;
			top++;
			st[top] = (kdtask_t){t.start, mi - 1, t.depth + 1, &nd->left, t.mn, t.mx};
			if (axis == 0) st[top].mx.x = sp; else if (axis == 1) st[top].mx.y = sp; else st[top].mx.z = sp;
			top++;
		}
	}
	s->kd_count = cur;
	free(st);
}

typedef struct { photon_t *ph; double d2; } knn_r;
typedef struct { knn_r *res; size_t k, count, far; } knn_s;

static void knn_update(knn_s *q)                          /* kd_tree_find_near.c:16 */
{
	q->far = 0;
	for (size_t i = 1; i < q->count; i++)
		if (q->res[i].d2 > q->res[q->far].d2)
			q->far = i;
}

static void knn_set(photon_t *p, knn_s *q, double d2)     /* :30 */
{
	if (q->count < q->k)
	{
		q->res[q->count].ph = p;
		q->res[q->count].d2 = d2;
		q->count++;
		if (q->count == q->k)
			knn_update(q);
	}
	else if (d2 < q->res[q->far].d2)
	{
		q->res[q->far].ph = p;
		q->res[q->far].d2 = d2;
		knn_update(q);
	}
}

static int sphere_box(v3 p, double r2, v3 mn, v3 mx)     /* :48 */
{
	double	d = 0.0;

	if (p.x < mn.x) d += (mn.x - p.x) * (mn.x - p.x);
	else if (p.x > mx.x) d += (p.x - mx.x) * (p.x - mx.x);
	if (p.y < mn.y) d += (mn.y - p.y) * (mn.y - p.y);
	else if (p.y > mx.y) d += (p.y - mx.y) * (p.y - mx.y);
	if (p.z < mn.z) d += (mn.z - p.z) * (mn.z - p.z);
	else if (p.z > mx.z) d += (p.z - mx.z) * (p.z - mx.z);
	return d <= r2;
}

static void knn_rec(ro_scene *s, kd_t *n, knn_s *q, v3 p)   /* :93 */
{
	kd_t	*nb, *ob;
	double	dp;

	if (n == NULL || (q->count == q->k && !sphere_box(p, q->res[q->far].d2, n->bmin, n->bmax)))
		return ;
	if (n->axis == -1)
	{
		for (int i = 0; i < n->count; i++)
		{
			photon_t	*ph = &s->photons[n->start + i];
			double		d2 = (ph->pos.x - p.x) * (ph->pos.x - p.x)
				+ (ph->pos.y - p.y) * (ph->pos.y - p.y) + (ph->pos.z - p.z) * (ph->pos.z - p.z);

			knn_set(ph, q, d2);
		}
		return ;
	}
	{
		float	df = axis_of(p, n->axis) - n->split;   /* float - float, then widened */

		dp = df;
	}
	if (dp < 0)
	{
		nb = n->left;
		ob = n->right;
	}
	else
	{
		nb = n->right;
		ob = n->left;
	}
	knn_rec(s, nb, q, p);
	if (q->count < q->k || (dp * dp) < q->res[q->far].d2)
		knn_rec(s, ob, q, p);
}

/* estimate_caustics_physically_based + calculate_caustic_radiance
 * (get_caustic.c:37-88). */
static fc caustic_estimate(ro_scene *s, v3 p, int k)
{
	knn_s	q;
	knn_r	res[64];
	fc		sum = {0, 0, 0};
	double	r2, area;

	if (!s->kd_root || k <= 0 || k > 64)
		return sum;
	q.res = res;
	q.k = k;
	q.count = 0;
	q.far = 0;
	for (int i = 0; i < k; i++)
		res[i].d2 = DBL_MAX;
	s->cnt.caustic_gathers++;
	knn_rec(s, s->kd_root, &q, p);
	if (q.count < (size_t)k)
		return sum;
	r2 = q.res[q.far].d2;
	if (r2 > s->caustic_radius)
		return sum;
	area = M_PI * r2;
	if (area < 1e-9)
		return sum;
	for (size_t i = 0; i < q.count; i++)
	{
		sum.r += q.res[i].ph->power.r;
		sum.g += q.res[i].ph->power.g;
		sum.b += q.res[i].ph->power.b;
	}
	sum.r = (sum.r / area) / s->norm_factor;
	sum.g = (sum.g / area) / s->norm_factor;
	sum.b = (sum.b / area) / s->norm_factor;
	return sum;
}

/* -------------------------------------------------------------- BSDFs */

/* ggx_sample_hemisphere (material/utils.c:39-62). */
static v3 ggx_sample(rng_t *rg, v3 n, double rough)
{
	double	u2 = rnd(rg);
	double	phi = 2.0 * PI_D * rnd(rg);
	double	ct = sqrt((1.0 - u2) / (1.0 + ((rough * rough) * (rough * rough) - 1.0) * u2));
	double	st = sqrt(1.0 - ct * ct);
	v3		tg = vunit(vcross(n, (v3){1.0, 0.0, 0.0}));

	if (vlen2(tg) < 0.0001)
		tg = vunit(vcross(n, (v3){0.0, 1.0, 0.0}));
	return vadd(vscale(n, ct), vadd(vscale(tg, cos(phi) * st),
				vscale(vunit(vcross(n, tg)), sin(phi) * st)));
}

static inline double cos_theta_in(v3 d, v3 n) { return -vdot(vunit(d), n); }  /* utils.c:16 */

/* fresnel_schlick_color / _f (fresnel_schlick.c:19,35): powf on floats. */
static fc fresnel_color(double ct, fc f0)
{
	return fadd(f0, fscale(fsub((fc){1.0, 1.0, 1.0}, f0), powf(1 - ct, 5)));
}

static double fresnel_f(double ct, double f0) { return f0 + ((1 - f0) * powf(1 - ct, 5)); }

/* metallic_color (metallic.c:25-46). */
static void metallic(rng_t *rg, ro_scene *s, ray_t *r, hrec_t *h, fc *power)
{
	double	ct = cos_theta_in(r->dir, h->normal);
	v3		m = hmat(s, h)->roughness > 0.0 ? ggx_sample(rg, h->normal, hmat(s, h)->roughness)
		: h->normal;

	r->dir = vunit(vsub(r->dir, vscale(m, 2 * vdot(r->dir, m))));
	if (s->exact)
		*power = fmul(*power, fadd(h->color, fscale(fsub((fc){1.0, 1.0, 1.0}, h->color), pow(1 - ct, 5))));
	else
		*power = fmul(*power, fresnel_color(ct, h->color));
}

/* reflected_dielectric_color (dielectric.c:15-33). */
static void dielectric_reflect(rng_t *rg, ro_scene *s, ray_t *r, hrec_t *h)
{
	v3	m = hmat(s, h)->roughness > 0.0 ? ggx_sample(rg, h->normal, hmat(s, h)->roughness)
		: h->normal;

	r->dir = vunit(vsub(r->dir, vscale(m, 2 * vdot(r->dir, m))));
}

/* refracted_ray + refracted_value + refracted_v (refraction.c:15-78). */
static void refract_ray(rng_t *rg, ro_scene *s, ray_t *r, hrec_t *h, fc *power)
{
	const mat_t	*m = hmat(s, h);
	double	eta = h->front_face ? s->ior_all / m->ior : m->ior / s->ior_all;
	double	ct, st;
	v3		perp, d;

	r->dir = vunit(r->dir);
	ct = fmin(-vdot(r->dir, h->normal), 1.0);
	st = sqrt(1.0 - ct * ct);
	if (eta * st > 1.0)
	{
		metallic(rg, s, r, h, power);
		return ;
	}
	perp = vscale(vadd(r->dir, vscale(h->normal, fmin(vdot(vneg(r->dir), h->normal), 1.0))), eta);
	d = vadd(vscale(h->normal, -sqrt(fabs(1.0 - vlen2(perp)))), perp);
	d = vunit(d);
	if (m->roughness > 0.0)
		d = ggx_sample(rg, d, m->roughness);
	r->dir = d;
	*power = fmul(*power, h->color);
}

/* cos_weighted_sample_hemishphere (material_default.c:20-38). */
static v3 cos_hemisphere(rng_t *rg, v3 *n)
{
	double	r1 = rnd(rg);
	double	r2 = rnd(rg);
	double	phi = 2 * PI_D * r1;
	v3		l = {cos(phi) * sqrt(r2), sqrt(1 - r2), sin(phi) * sqrt(r2)};
	v3		u;

	*n = vunit(*n);
	if (fabs(n->y) < 0.999)
		u = vunit(vcross((v3){0, 1, 0}, *n));
	else
		u = vunit(vcross((v3){1, 0, 0}, *n));
	return vunit(vadd(vadd(vscale(u, l.x), vscale(*n, l.y)), vscale(vcross(*n, u), l.z)));
}

/* ------------------------------------------------------------ lighting */

static int shadow_any(ro_scene *s, const ray_t *r, hrec_t *h)
{
	int	hit;

	s->cnt.shadow_rays++;
	s->is_light = 1;
	hit = hit_register_all(s, r, h);
	s->is_light = 0;
	return hit;
}

/* compute_light_v2 (light_manager.c:59-71) with add_all_light_contribution
 * (:32-57), try_to_add_plight (:16-30), check_plight_hit / compute_shadow_factor
 * / add_plight (p_light.c:19-89), check_dlight_hit_dir / add_dlight
 * (d_light.c:19-55). The accumulator is t_lcolor: uint64 channels, so every
 * addition truncates toward zero (structs.h t_lcolor). */
static fc compute_light(rng_t *rg, ro_scene *s, hrec_t *h)
{
	uint64_t	lc[3] = {0, 0, 0};
	v3			view = vunit(vsub(s->cam_pos, h->point));

	for (int i = 0; i < s->n_lights; i++)
	{
		light_t	*L = &s->lights[i];

		if (L->type == MRT_LIGHT_POINT)
		{
			double	sf;
			int		vis;

			if (L->radius == 0 || L->shadow_sample <= 1)
			{
				ray_t	sr;
				hrec_t	th;
				double	dist;

				sf = 1;
				sr.orig = h->point;
				sr.dir = vunit(vsub(L->pos, h->point));
				dist = vlen(vsub(L->pos, h->point));
				vis = !(shadow_any(s, &sr, &th) && th.t < dist);
			}
			else
			{
				int		hits = 0;
				ray_t	sr;
				hrec_t	th;

				sr.orig = h->point;
				for (int k = 0; k < L->shadow_sample; k++)
				{
					v3 tgt = vadd(L->pos, vscale(rnd_in_unit_sphere(rg), L->radius));

					sr.dir = vunit(vsub(tgt, h->point));
					if (shadow_any(s, &sr, &th) == 0 || th.t >= vlen(vsub(tgt, h->point)))
						hits++;
				}
				sf = (double)hits / (double)L->shadow_sample;
				vis = sf > 0.0;
			}
			if (vis)
			{
				v3		ld = vunit(vsub(L->pos, h->point));
				double	ndl = vdot(h->normal, ld);

				if (ndl > 0.0)
				{
					double	di = L->brightness * ndl * sf;
					double	rdv, spec;

					lc[0] += L->color[0] * di;
					lc[1] += L->color[1] * di;
					lc[2] += L->color[2] * di;
					rdv = vdot(vsub(vneg(ld), vscale(h->normal, 2 * vdot(vneg(ld), h->normal))), view);
					if (rdv < 0.0)
						rdv = 0.0;
					spec = pow(rdv, SHINE) * SPEC_STRENGTH * sf;
					lc[0] += L->color[0] * L->brightness * spec;
					lc[1] += L->color[1] * L->brightness * spec;
					lc[2] += L->color[2] * L->brightness * spec;
				}
			}
		}
		else
		{
			ray_t	sr;
			hrec_t	th;

			sr.orig = h->point;
			sr.dir = vunit(vneg(L->pos));
			if (shadow_any(s, &sr, &th) == 0)
			{
				v3		ld = vneg(L->pos);
				double	ndl = vdot(h->normal, ld);

				if (ndl > 0.0)
				{
					double	rdv, spec;

					lc[0] += L->color[0] * L->brightness * ndl;
					lc[1] += L->color[1] * L->brightness * ndl;
					lc[2] += L->color[2] * L->brightness * ndl;
					rdv = vdot(vsub(vneg(ld), vscale(h->normal, 2 * vdot(vneg(ld), h->normal))), view);
					if (rdv < 0.0)
						rdv = 0.0;
					spec = pow(rdv, SHINE);
					lc[0] += L->color[0] * L->brightness * SPEC_STRENGTH * spec;
					lc[1] += L->color[1] * L->brightness * SPEC_STRENGTH * spec;
					lc[2] += L->color[2] * L->brightness * SPEC_STRENGTH * spec;
				}
			}
		}
	}
	return (fc){lc[0] / 255.0, lc[1] / 255.0, lc[2] / 255.0};
}

/* importance_sampling (material_default.c:41-69) with
 * calc_inverse_transform_sampling_uv/dir (get_dir.c:15-41). */
static void env_nee(rng_t *rg, ro_scene *s, ray_t *r, hrec_t *h, fc *power, fc *acc)
{
	double	rx = rnd(rg);
	double	ry = rnd(rg);
	double	vy = s->cdf_m_inv[(int)(rx * (s->hh - 1))];
	double	vx = s->cdf_c_inv[(int)(vy * (s->hh - 1) * s->hw + ry * (s->hw - 1))];
	float	theta = (vy - 0.5) * PI_D;
	float	phi = (0.5 - vx) * 2 * PI_D;
	hrec_t	th;
	float	ct, pdf;
	fc		rad;

	s->cnt.env_nee++;
	r->dir = (v3){cos(theta) * cos(phi), sin(theta), cos(theta) * sin(phi)};
	if (shadow_any(s, r, &th))
		return ;
	if (s->exact)
	{
		double	ctd = vdot(h->normal, r->dir);
		double	pdfd = s->pdf_joint_d[(int)(vy * (s->hh - 1) * s->hw + vx * (s->hw - 1))];

		if (pdfd <= 0)
			return ;
		rad = background(s, *r, 0);
		if (h->mat >= 0)
			rad = fscale(rad, hmat(s, h)->ao);
		rad = fscale(fmul(rad, *power), ctd / pdfd);
		*acc = fadd(*acc, rad);
		*power = fscale(*power, 1 - ctd);
		return ;
	}
	ct = vdot(h->normal, r->dir);
	pdf = s->pdf_joint[(int)(vy * (s->hh - 1) * s->hw + vx * (s->hw - 1))];
	if (pdf <= 0)
		return ;
	rad = background(s, *r, 0);
	if (h->mat >= 0)
		rad = fscale(rad, hmat(s, h)->ao);
	rad = fmul(rad, *power);
	rad = fscale(rad, ct / (pdf));
	*acc = fadd(*acc, rad);
	*power = fscale(*power, 1 - ct);
}

/* default_mat (material_default.c:71-92). */
static void default_mat(rng_t *rg, ro_scene *s, ray_t *r, hrec_t *h, fc *power, fc *acc)
{
	fc	direct = compute_light(rg, s, h);
	fc	caus = s->kd_root ? caustic_estimate(s, h->point, 15) : (fc){0.0, 0.0, 0.0};
	fc	total = fadd(direct, caus);

	*acc = fadd(*acc, fmul(fmul(h->color, *power), total));
	*power = fmul(*power, h->color);
	if (s->pdf_joint)
		env_nee(rg, s, r, h, power, acc);
	r->dir = cos_hemisphere(rg, &h->normal);
}

/* dielectric_mat (dielectric.c:37-64). */
static void dielectric_mat(rng_t *rg, ro_scene *s, ray_t *r, hrec_t *h, fc *power, fc *acc)
{
	const mat_t	*m = hmat(s, h);

	if (m->ior > 0)
	{
		double	refl = fresnel_f(cos_theta_in(r->dir, h->normal),
				powf((m->ior - 1) / (m->ior + 1), 2));

		if (refl >= rnd(rg) && m->ior != 1.0)
			dielectric_reflect(rg, s, r, h);
		else if (m->transmission == 1.0)
			refract_ray(rg, s, r, h, power);
		else if (m->transmission == 0.0)
			default_mat(rg, s, r, h, power, acc);
		else if (m->transmission < rnd(rg))
			default_mat(rg, s, r, h, power, acc);
		else
			refract_ray(rg, s, r, h, power);
	}
	else
		default_mat(rg, s, r, h, power, acc);
}

/* material_manager_v3 (path_trace.c:15-35). */
static void material_manager(rng_t *rg, ro_scene *s, ray_t *r, hrec_t *h, fc *power, fc *acc)
{
	const mat_t	*m;

	if (h->mat < 0)
	{
		default_mat(rg, s, r, h, power, acc);
		return ;
	}
	m = hmat(s, h);
	if (m->emission_strength > 0)
		*acc = fadd(*acc, fmul(fscale(m->emission_color, m->emission_strength), *power));
	if (m->metallic == 1.0)
		metallic(rg, s, r, h, power);
	else if (m->metallic == 0.0)
		dielectric_mat(rg, s, r, h, power, acc);
	else if (m->metallic > rnd(rg))
		metallic(rg, s, r, h, power);
	else
		dielectric_mat(rg, s, r, h, power, acc);
}

/* Per-bounce event records for the debug probe (20 doubles per bounce:
 * flat prim or -1 for the final miss, t, point, normal, then direction,
 * power and radiance after shading, material). */
static double	*g_events = NULL;

static void put_event(int k, ro_scene *s, hrec_t *h, int hit, ray_t *r, fc power, fc acc)
{
	double	*e;

	if (!g_events || k >= 16)
		return ;
	e = g_events + 20 * k;
	e[0] = hit ? flat_of_prim(s, h->prim) : -1;
	e[1] = hit ? h->t : 0;
	e[2] = hit ? h->point.x : 0; e[3] = hit ? h->point.y : 0; e[4] = hit ? h->point.z : 0;
	e[5] = hit ? h->normal.x : 0; e[6] = hit ? h->normal.y : 0; e[7] = hit ? h->normal.z : 0;
	e[8] = r->dir.x; e[9] = r->dir.y; e[10] = r->dir.z;
	e[11] = power.r; e[12] = power.g; e[13] = power.b;
	e[14] = acc.r; e[15] = acc.g; e[16] = acc.b;
	e[17] = hit ? h->mat : -1;
}

/* path_trace + add_skybox (path_trace.c:37-76). On a miss the sky is scaled
 * by the ao of the last material hit (the hit record persists). */
static fc path_trace(rng_t *rg, ro_scene *s, ray_t r, int depth)
{
	fc		acc = {0.0, 0.0, 0.0};
	fc		power = {1.0, 1.0, 1.0};
	hrec_t	h;
	int		k = 0;

	memset(&h, 0, sizeof(h));
	h.mat = -1;
	s->cnt.paths++;
	while (--depth >= 0)
	{
		s->cnt.segments++;
		if (hit_register_all(s, &r, &h) == 1)
		{
			s->cnt.hits++;
			r.orig = h.point;
			material_manager(rg, s, &r, &h, &power, &acc);
			put_event(k++, s, &h, 1, &r, power, acc);
		}
		else
		{
			fc	bg = background(s, r, 1);

			if (h.mat >= 0)
				acc = fadd(acc, fmul(fscale(bg, hmat(s, &h)->ao), power));
			else
				acc = fadd(acc, fmul(bg, power));
			put_event(k, s, &h, 0, &r, power, acc);
			break ;
		}
	}
	return acc;
}

/* defocus_disk_sample (focus.c:16-42). */
static v3 defocus_origin(rng_t *rg, ro_scene *s)
{
	v3	p = {0, 0, 0};

	while (1)
	{
		p.x = -1 + rnd(rg) * (1 - -1);
		p.y = -1 + rnd(rg) * (1 - -1);
		if (vlen2(p) < 1)
			break ;
	}
	return vadd(s->cam_pos, vadd(vscale(s->defocus_u, p.x), vscale(s->defocus_v, p.y)));
}

/* calc_one_sample_task (calc_sample.c:44-71), render_mode 0 and 2. */
static fc sample_pixel_(rng_t *rg, ro_scene *s, uint32_t i, double ox, double oy);

/* One camera path; its stream keys the alpha test of its traversals. */
static fc sample_pixel(rng_t *rg, ro_scene *s, uint32_t i, double ox, double oy)
{
	fc	c;

	s->rg = rg;
	c = sample_pixel_(rg, s, i, ox, oy);
	s->rg = NULL;
	return c;
}

static fc sample_pixel_(rng_t *rg, ro_scene *s, uint32_t i, double ox, double oy)
{
	ray_t	r;
	hrec_t	h;

	if (s->defocus_angle <= 0)
		r.orig = s->cam_pos;
	else
		r.orig = defocus_origin(rg, s);
	r.dir = vsub(vadd(vadd(s->pixel00, vscale(s->pdu, (i % s->W) + ox)),
				vscale(s->pdv, (i / s->W) + oy)), r.orig);
	if (s->render_mode == 2)
		return hit_register_all(s, &r, &h) == 1 ? h.color : (fc){0, 0, 0};
	return path_trace(rg, s, r, s->max_bounces);
}

/* ------------------------------------------------------------ photons */

/* trace_single_photon_path + material_manager_v3_phothon
 * (trace_photon_path.c:18-72), dielectric_mat_photon (dielectric.c:66-91). */
static int trace_photon_(rng_t *rg, ro_scene *s, v3 lp, fc p0, photon_t *out);

/* Photon paths trace with is_light set (init_single_photon_path,
 * trace_photon_path.c:42): only normal and transmission maps apply. */
static int trace_photon(rng_t *rg, ro_scene *s, v3 lp, fc p0, photon_t *out)
{
	int	stored;

	s->rg = rg;
	s->is_light = 1;
	stored = trace_photon_(rg, s, lp, p0, out);
	s->is_light = 0;
	s->rg = NULL;
	return stored;
}

static int trace_photon_(rng_t *rg, ro_scene *s, v3 lp, fc p0, photon_t *out)
{
	ray_t	r;
	fc		pw = p0;
	hrec_t	h;

	r.dir = rnd_unit(rg);
	r.orig = lp;
	for (int depth = 0; depth < 10; depth++)
	{
		int	stored = 0;

		if (hit_register_all(s, &r, &h) != 1)
			return 0;
		r.orig = h.point;
		if (h.mat < 0)
		{
			pw = fmul(pw, h.color);
			stored = 1;
		}
		else
		{
			const mat_t	*m = hmat(s, &h);
			int		as_metal;

			if (m->metallic == 1.0)
				as_metal = 1;
			else if (m->metallic == 0.0)
				as_metal = 0;
			else
				as_metal = m->metallic > rnd(rg);
			if (as_metal)
				metallic(rg, s, &r, &h, &pw);
			else if (m->ior > 0)
			{
				double	refl = fresnel_f(cos_theta_in(r.dir, h.normal),
						powf((m->ior - 1) / (m->ior + 1), 2));

				if (refl >= rnd(rg) && m->ior != 1.0)
					dielectric_reflect(rg, s, &r, &h);
				else if (m->transmission == 1.0)
					refract_ray(rg, s, &r, &h, &pw);
				else if (m->transmission == 0.0)
				{
					pw = fmul(pw, h.color);
					stored = 1;
				}
				else if (m->transmission < rnd(rg))
				{
					pw = fmul(pw, h.color);
					stored = 1;
				}
				else
					refract_ray(rg, s, &r, &h, &pw);
			}
			else
			{
				pw = fmul(pw, h.color);
				stored = 1;
			}
		}
		if (stored)
		{
			out->pos = h.point;
			out->power = pw;
			return depth != 0;
		}
	}
	return 0;
}

/* caustic_manager / init_photon_map / emit_photon_from_one_light
 * (caustic_manager.c:16-105). The light list holds point and directional
 * lights; directional lights are read through the t_light layout there, so
 * only point lights are emitted here (the reference's directional entries
 * would emit from a garbage position). */
static void build_photon_map(ro_scene *s, uint64_t per_light)
{
	size_t	cap = 1024;
	rng_t	rg = {RO_RNG_REFERENCE, 0};

	s->photons = malloc(sizeof(photon_t) * cap);
	s->n_photons = 0;
	for (int i = 0; i < s->n_lights; i++)
	{
		light_t	*L = &s->lights[i];

		if (L->type != MRT_LIGHT_POINT)
			continue ;
		for (uint64_t j = 0; j < per_light; j++)
		{
			photon_t	ph;
			fc			p0 = {L->color[0] * L->brightness / per_light,
				L->color[1] * L->brightness / per_light, L->color[2] * L->brightness / per_light};

			if (trace_photon(&rg, s, L->pos, p0, &ph))
			{
				if (s->n_photons == cap)
				{
					cap *= 2;
					s->photons = realloc(s->photons, sizeof(photon_t) * cap);
				}
				s->photons[s->n_photons++] = ph;
			}
		}
	}
	if (s->n_photons)
		kd_build(s);
}

/* ------------------------------------------------------------- creation */

/* rotate_around_axis (obj_parser_utils.c:15-23): cos/sin of a float angle
 * stored as float. */
static v3 rotate_axis(v3 v, v3 axis, float angle)
{
	const float	ct = cos(angle);
	const float	st = sin(angle);

	return vadd(vadd(vscale(v, ct), vscale(vcross(axis, v), st)),
		vscale(axis, vdot(axis, v) * (1 - ct)));
}

/* ft_update_obj_position / update_position_scale (obj_parser_utils.c:25-66)
 * for a custom object at the origin, orientation (0,1,0), scale 1, applied by
 * init_bvh -> bvh_make_lst to every mesh vertex (bvh_make_lst.c:34). */
static v3 mesh_transform(v3 p)
{
	const v3	axis = {0, 1, 0};

	p = vsub(p, (v3){0, 0, 0});
	p = rotate_axis(p, axis, -1.0f);
	p = vmul(p, (v3){1.0, 1.0, 1.0});
	p = rotate_axis(p, axis, 1.0f);
	return vadd(p, (v3){0, 0, 0});
}

static v3 a3(const double *p) { return (v3){p[0], p[1], p[2]}; }

/* init_viewport_values / init_viewport_vectors (viewport.c:38-87). */
static void init_viewport(ro_scene *s, const mrt_camera *c)
{
	float	vw, vh;
	v3		up, u, vu, vv;

	s->cam_pos = a3(c->position);
	s->cam_dir = vunit(a3(c->orientation));
	s->focus_dist = c->focus_dist == 0 ? 1 : c->focus_dist;
	s->defocus_angle = c->defocus_angle;
	vw = 2.0 * tan(c->fov * (PI_D / 180.0) / 2.0) * s->focus_dist;
	vh = vw / ((double)s->W / (double)s->H);
	up = (v3){0, 1, 0};
	if (fabs(s->cam_dir.y) > 0.999)
		up = (v3){1, 0, 0};
	u = vunit(vcross(up, vneg(s->cam_dir)));
	vu = vscale(u, vw);
	vv = vscale(vcross(s->cam_dir, u), vh);
	s->pdu = vdiv(vu, s->W);
	s->pdv = vdiv(vv, s->H);
	s->pixel00 = vadd(vsub(vsub(vadd(s->cam_pos, vscale(s->cam_dir, s->focus_dist)),
					vdiv(vu, 2)), vdiv(vv, 2)), vscale(vadd(s->pdu, s->pdv), 0.5));
	{
		double	rad = s->focus_dist * tan(s->defocus_angle * PI_D / 360);

		s->defocus_u = vscale(u, rad);
		s->defocus_v = vscale(vcross(s->cam_dir, u), rad);
	}
}

ro_scene	*ro_create(const mrt_scene_desc *d)
{
	ro_scene	*s;
	int			np = 0;

	if (!d || d->abi_version != MRT_ABI_VERSION || d->render_width <= 0 || d->render_height <= 0)
		return NULL;
	s = calloc(1, sizeof(*s));
	s->apply_mesh_transform = g_apply_mesh_transform;
	s->W = d->render_width;
	s->H = d->render_height;
	s->max_bounces = d->max_bounces;
	s->one_sided = d->triangle_one_sided;
	s->ior_all = d->ior_all;
	s->n_texs = (d->n_textures > 0 && d->textures) ? d->n_textures : 0;
	s->texs = calloc(s->n_texs + 1, sizeof(tex_t));
	for (int i = 0; i < s->n_texs; i++)
	{
		const mrt_texture	*t = &d->textures[i];
		tex_t				*o = &s->texs[i];

		o->type = t->type;
		o->scale = t->checker_scale;
		memcpy(o->c1, t->c1, 3);
		memcpy(o->c2, t->c2, 3);
		if (t->rgba && t->width && t->height)
		{
			o->w = t->width;
			o->h = t->height;
			o->rgba = malloc(4 * (size_t)t->width * t->height);
			memcpy(o->rgba, t->rgba, 4 * (size_t)t->width * t->height);
		}
	}
	s->n_mats = d->n_materials;
	s->mats = calloc(d->n_materials + 1, sizeof(mat_t));
	for (int i = 0; i < d->n_materials; i++)
	{
		const mrt_material	*m = &d->materials[i];
		mat_t				*o = &s->mats[i];

		memcpy(o->c8, m->color, 3);
		o->metallic = clamp01(m->metallic);
		o->roughness = clamp01(m->roughness);
		o->ior = m->ior;
		o->transmission = m->transmission;
		o->ao = m->ao;
		o->emission_strength = m->emission_strength;
		o->scale = m->scale;
		o->emission_color = c2f(m->emission_color);
		{
			const int32_t	*tx = &m->color_tex;   /* color_tex .. normal_tex, in TX_ order */

			for (int k = 0; k < TX_SLOTS; k++)
			{
				o->tex[k] = (tx[k] > 0 && tx[k] <= s->n_texs) ? tx[k] : 0;
				o->textured |= o->tex[k] != 0;
			}
			o->normal_intensity = m->normal_intensity;
		}
	}
	/* primitive order of bvh_make_lst (bvh_make_lst.c:46-65) over the object
	 * list spheres, cylinders, cones, hyperboloids, then one custom object
	 * per (mesh, material) in order of first appearance. */
	{
		size_t	total = d->n_spheres + (size_t)d->n_cylinders + d->n_cones + d->n_hyperboloids;

		for (int i = 0; i < d->n_meshes; i++)
			total += d->meshes[i].n_triangles;
		s->prims = calloc(total + 1, sizeof(prim_t));
	}
	for (int i = 0; i < d->n_spheres; i++)
	{
		prim_t	*p = &s->prims[np++];

		p->type = PT_SPHERE;
		p->flat = i;
		p->mat = d->spheres[i].material < d->n_materials ? d->spheres[i].material : -1;
		memcpy(p->color, d->spheres[i].color, 3);
		p->center = a3(d->spheres[i].center);
		p->radius = (d->spheres[i].radius * 2.0) * 0.5;
		p->r2 = p->radius * p->radius;
	}
	for (int i = 0; i < d->n_cylinders; i++)
	{
		const mrt_cylinder	*c = &d->cylinders[i];
		prim_t				*p = &s->prims[np++];

		p->type = PT_CYL;
		p->flat = d->n_spheres + i;
		p->mat = mat_or_none(c->material, d->n_materials);
		p->mat_top = mat_or_none(c->material_top, d->n_materials);
		p->mat_bot = mat_or_none(c->material_bot, d->n_materials);
		memcpy(p->color, c->color, 3);
		p->center = a3(c->position);
		p->ori = a3(c->orientation);
		p->diam = c->diameter;
		p->height = c->height;
	}
	for (int i = 0; i < d->n_cones; i++)
	{
		const mrt_cone	*c = &d->cones[i];
		prim_t			*p = &s->prims[np++];

		p->type = PT_CONE;
		p->flat = d->n_spheres + d->n_cylinders + i;
		p->mat = mat_or_none(c->material, d->n_materials);
		p->mat_top = mat_or_none(c->material_top, d->n_materials);
		p->mat_bot = -1;
		memcpy(p->color, c->color, 3);
		p->center = a3(c->position);
		p->ori = a3(c->orientation);
		p->diam = c->diameter;
		p->height = c->height;
	}
	for (int i = 0; i < d->n_hyperboloids; i++)
	{
		const mrt_hyperboloid	*c = &d->hyperboloids[i];
		prim_t					*p = &s->prims[np++];

		p->type = PT_HYP;
		p->flat = d->n_spheres + d->n_cylinders + d->n_cones + i;
		p->mat = mat_or_none(c->material, d->n_materials);
		p->mat_top = p->mat_bot = -1;
		memcpy(p->color, c->color, 3);
		p->center = a3(c->position);
		p->ori = a3(c->orientation);
		p->qa = c->a;
		p->qb = c->b;
		p->qc = c->c;
		p->shape = c->shape;
		p->height = c->height;
	}
	{
		uint32_t	flat = d->n_spheres + d->n_cylinders + d->n_cones + d->n_hyperboloids;

		for (int mi = 0; mi < d->n_meshes; mi++)
		{
			const mrt_mesh	*me = &d->meshes[mi];
			char			*done = calloc(me->n_triangles + 1, 1);

			for (uint32_t t = 0; t < me->n_triangles; t++)
			{
				int32_t	mat;

				if (done[t])
					continue ;
				mat = me->tri_material ? me->tri_material[t] : me->material;
				for (uint32_t k = t; k < me->n_triangles; k++)
				{
					int32_t		mk = me->tri_material ? me->tri_material[k] : me->material;
					prim_t		*p;
					uint32_t	ix[3];

					if (done[k] || mk != mat)
						continue ;
					done[k] = 1;
					p = &s->prims[np++];
					p->type = PT_TRI;
					p->flat = flat + k;
					p->mat = (mat >= 0 && mat < d->n_materials) ? mat : -1;
					memcpy(p->color, me->color, 3);
					for (int c = 0; c < 3; c++)
					{
						ix[c] = me->indices ? me->indices[3 * (size_t)k + c] : 3 * k + c;
						p->p[c] = a3(me->positions + 3 * (size_t)ix[c]);
						p->n[c] = a3(me->normals + 3 * (size_t)ix[c]);
						p->uv[c][0] = me->uvs ? me->uvs[2 * (size_t)ix[c]] : 0;
						p->uv[c][1] = me->uvs ? me->uvs[2 * (size_t)ix[c] + 1] : 0;
					}
					/* the sort key is the centre of the loaded vertices; the
					 * re-transform moves the vertices only */
					p->center = vdiv(vadd(vadd(p->p[0], p->p[1]), p->p[2]), 3.0);
					if (s->apply_mesh_transform)
						for (int c = 0; c < 3; c++)
							p->p[c] = mesh_transform(p->p[c]);
				}
			}
			free(done);
			flat += me->n_triangles;
		}
		s->n_prims = np;
		s->n_planes = d->n_planes;
		s->planes = calloc(d->n_planes + 1, sizeof(plane_t));
		for (int i = 0; i < d->n_planes; i++)
		{
			s->planes[i].point = a3(d->planes[i].point);
			s->planes[i].normal = vunit(a3(d->planes[i].normal));
			s->planes[i].mat = d->planes[i].material < d->n_materials ? d->planes[i].material : -1;
			memcpy(s->planes[i].color, d->planes[i].color, 3);
			s->planes[i].flat = flat + i;
		}
	}
	s->n_lights = d->n_lights;
	s->lights = calloc(d->n_lights + 1, sizeof(light_t));
	for (int i = 0; i < d->n_lights; i++)
	{
		light_t	*L = &s->lights[i];

		L->type = d->lights[i].type;
		L->pos = d->lights[i].type == MRT_LIGHT_DIRECTIONAL ? vunit(a3(d->lights[i].position))
			: a3(d->lights[i].position);
		L->brightness = d->lights[i].brightness;
		if (L->type == MRT_LIGHT_POINT && L->brightness < 0)
			L->brightness = 0;
		memcpy(L->color, d->lights[i].color, 3);
		L->shadow_sample = d->lights[i].shadow_sample;
		L->radius = d->lights[i].radius;
	}
	s->amb_ratio = d->ambient.ratio;
	memcpy(s->amb_color, d->ambient.color, 3);
	if (d->ambient.hdr_rgbe && d->ambient.hdr_width > 0 && d->ambient.hdr_height > 0)
	{
		size_t	n = (size_t)d->ambient.hdr_width * d->ambient.hdr_height * 4;

		s->rgbe_own = malloc(n);
		memcpy(s->rgbe_own, d->ambient.hdr_rgbe, n);
		s->rgbe = s->rgbe_own;
		s->hw = d->ambient.hdr_width;
		s->hh = d->ambient.hdr_height;
		s->hdr_exposure = d->ambient.hdr_exposure;
		s->hdr_gamma = d->ambient.hdr_gamma;
		build_env_tables(s);
	}
	init_viewport(s, &d->camera);
	build_bvh(s);
	if (d->caustic.enable)
	{
		s->caustic_enable = 1;
		s->caustic_radius = d->caustic.radius;
		s->norm_factor = d->caustic.norm_factor;
		build_photon_map(s, d->caustic.photons_per_light);
	}
	memset(&s->cnt, 0, sizeof(s->cnt));
	return s;
}

void	ro_destroy(ro_scene *s)
{
	if (!s)
		return ;
	for (int i = 0; i < s->n_texs; i++)
		free(s->texs[i].rgba);
	free(s->texs);
	free(s->mats);
	free(s->prims);
	free(s->prim_idx);
	free(s->nodes);
	free(s->planes);
	free(s->lights);
	free(s->rgbe_own);
	free(s->albedo_d);
	free(s->sky_d);
	free(s->pdf_joint_d);
	free(s->pdf_joint);
	free(s->cdf_m_inv);
	free(s->cdf_c_inv);
	free(s->photons);
	free(s->kd_nodes);
	free(s);
}

/* ------------------------------------------------------------- queries */

int	ro_first_hit(ro_scene *s, const mrt_ray *rays, int64_t n, ro_hit *out)
{
	for (int64_t i = 0; i < n; i++)
	{
		ray_t	r = {a3(rays[i].orig), a3(rays[i].dir)};
		hrec_t	h;

		int		bh = 0;
		int		any;

		memset(&out[i], 0, sizeof(out[i]));
		any = hit_register_all_(s, &r, &h, &bh);
		/* hit_register_all resets the counter when the BVH part missed
		 * (hit_register.c:116-117) */
		out[i].depth = (s->n_nodes && bh) ? bvh_depth_count(s, &r, 0) : 0;
		if (any)
		{
			out[i].prim = flat_of(s, h.prim);
			out[i].front_face = h.front_face;
			out[i].material = h.mat;
			out[i].t = h.t;
			out[i].u = h.u;
			out[i].v = h.v;
			out[i].point[0] = h.point.x;
			out[i].point[1] = h.point.y;
			out[i].point[2] = h.point.z;
			out[i].normal[0] = h.normal.x;
			out[i].normal[1] = h.normal.y;
			out[i].normal[2] = h.normal.z;
			out[i].color[0] = h.color.r;
			out[i].color[1] = h.color.g;
			out[i].color[2] = h.color.b;
		}
		else
			out[i].prim = -1;
	}
	return 0;
}

/* render_cpu/draw_pixels/calc_one_sample (render.c:28-36, calc_sample.c:73-101):
 * offset = vec3_random() (three draws, x and y used), then every pixel. */
int	ro_render_reference(ro_scene *s, int spp, double *accum)
{
	rng_t	rg = {RO_RNG_REFERENCE, 0};

	for (int k = 0; k < spp; k++)
	{
		double	ox = rnd(&rg), oy = rnd(&rg);

		(void)rnd(&rg);
		for (uint32_t i = 0; i < (uint32_t)(s->W * s->H); i++)
		{
			fc	c = sample_pixel(&rg, s, i, ox, oy);

			accum[3 * i] += c.r;
			accum[3 * i + 1] += c.g;
			accum[3 * i + 2] += c.b;
		}
	}
	return 0;
}

/* Shared jitter of sample `sample`: two draws of its own stream. */
static void shared_offset(uint64_t seed, uint32_t sample, double *ox, double *oy)
{
	uint64_t	st = ro_path_seed(seed, 0xFFFFFFFFu, sample);

	*ox = ro_pcg_float(&st);
	*oy = ro_pcg_float(&st);
}

int	ro_trace_path_counter(ro_scene *s, uint64_t seed, int32_t pixel, int32_t sample,
	int jitter, double *rgb)
{
	rng_t	rg = {RO_RNG_COUNTER, ro_path_seed(seed, (uint32_t)pixel, (uint32_t)sample)};
	double	ox, oy;
	fc		c;

	if (jitter == MRT_JITTER_SHARED)
		shared_offset(seed, (uint32_t)sample, &ox, &oy);
	else
	{
		ox = rnd(&rg);
		oy = rnd(&rg);
	}
	c = sample_pixel(&rg, s, (uint32_t)pixel, ox, oy);
	rgb[0] = c.r;
	rgb[1] = c.g;
	rgb[2] = c.b;
	return 0;
}

int	ro_render_counter(ro_scene *s, uint64_t seed, int sample_base, int spp, int jitter,
	const int32_t *pix, int64_t n, double *accum, ro_counters *cnt)
{
	int64_t	count = pix ? n : (int64_t)s->W * s->H;
	double	rgb[3];

	memset(&s->cnt, 0, sizeof(s->cnt));
	for (int k = 0; k < spp; k++)
		for (int64_t i = 0; i < count; i++)
		{
			int32_t	p = pix ? pix[i] : (int32_t)i;

			ro_trace_path_counter(s, seed, p, sample_base + k, jitter, rgb);
			accum[3 * i] += rgb[0];
			accum[3 * i + 1] += rgb[1];
			accum[3 * i + 2] += rgb[2];
		}
	if (cnt)
		*cnt = s->cnt;
	return 0;
}

int	ro_counters_read(ro_scene *s, ro_counters *out)
{
	*out = s->cnt;
	return 0;
}

int	ro_env_tables(ro_scene *s, float *pdf, float *cm, float *cc, double *avg)
{
	size_t	n;

	if (!s->pdf_joint)
		return 0;
	n = (size_t)s->hw * s->hh;
	if (pdf)
		memcpy(pdf, s->pdf_joint, n * sizeof(float));
	if (cm)
		memcpy(cm, s->cdf_m_inv, s->hh * sizeof(float));
	if (cc)
		memcpy(cc, s->cdf_c_inv, n * sizeof(float));
	if (avg)
		*avg = s->column_average;
	return 1;
}

/* Distribution induced by the two-step lookup of get_dir.c:15-27 with
 * continuous r1, r2 in [0,1): row iy = floor(r1 (H-1)) uniform over
 * [0, H-2]; then j = floor(A + r2 (W-1)) with A = v (H-1) W,
 * v = cdf_marginal_inverse[iy]. P(j) is the length of the r2-interval that
 * lands on j, divided by (W-1)... expressed here per unit r2. Outcome slots
 * are iy * (W + 1) + (j - floor(A)). */
int64_t	ro_env_outcome_probs(ro_scene *s, double *prob, int32_t *cond_index)
{
	int		W = s->hw, H = s->hh;
	int64_t	k = 0;

	if (!s->pdf_joint)
		return 0;
	for (int iy = 0; iy < H - 1; iy++)
	{
		double	v = s->cdf_m_inv[iy];
		double	A = v * (H - 1) * W;
		double	j0 = floor(A);

		for (int d = 0; d <= W; d++, k++)
		{
			double	lo = (j0 + d - A) / (W - 1);
			double	hi = (j0 + d + 1 - A) / (W - 1);

			lo = lo < 0 ? 0 : lo;
			hi = hi > 1 ? 1 : hi;
			prob[k] = hi > lo ? (hi - lo) / (H - 1) : 0.0;
			cond_index[k] = (int32_t)(j0 + d);
		}
	}
	return k;
}

int64_t	ro_photon_count(ro_scene *s)
{
	return (int64_t)s->n_photons;
}

int	ro_photons(ro_scene *s, double *pos3, double *pow3, int32_t *in_leaf)
{
	for (size_t i = 0; i < s->n_photons; i++)
	{
		pos3[3 * i] = s->photons[i].pos.x;
		pos3[3 * i + 1] = s->photons[i].pos.y;
		pos3[3 * i + 2] = s->photons[i].pos.z;
		pow3[3 * i] = s->photons[i].power.r;
		pow3[3 * i + 1] = s->photons[i].power.g;
		pow3[3 * i + 2] = s->photons[i].power.b;
	}
	if (in_leaf)
	{
		memset(in_leaf, 0, sizeof(int32_t) * s->n_photons);
		for (size_t n = 0; n < s->kd_count; n++)
			if (s->kd_nodes[n].axis == -1)
				for (int j = 0; j < s->kd_nodes[n].count; j++)
					in_leaf[s->kd_nodes[n].start + j] = 1;
	}
	return 0;
}

int	ro_caustic_query(ro_scene *s, const double *pts, int64_t n, int k, double *rgb)
{
	for (int64_t i = 0; i < n; i++)
	{
		fc	c = caustic_estimate(s, a3(pts + 3 * i), k);

		rgb[3 * i] = c.r;
		rgb[3 * i + 1] = c.g;
		rgb[3 * i + 2] = c.b;
	}
	return 0;
}

/* Triangle positions as intersected (after the load-time re-transform),
 * 9 doubles per flat triangle. */
int	ro_triangle_positions(ro_scene *s, double *out)
{
	int	base = -1;
	int	n = 0;

	for (int i = 0; i < s->n_prims; i++)
		if (s->prims[i].type == PT_TRI && (base < 0 || s->prims[i].flat < base))
			base = s->prims[i].flat;
	for (int i = 0; i < s->n_prims; i++)
	{
		prim_t	*p = &s->prims[i];

		if (p->type != PT_TRI)
			continue ;
		for (int c = 0; c < 3; c++)
		{
			out[9 * (size_t)(p->flat - base) + 3 * c] = p->p[c].x;
			out[9 * (size_t)(p->flat - base) + 3 * c + 1] = p->p[c].y;
			out[9 * (size_t)(p->flat - base) + 3 * c + 2] = p->p[c].z;
		}
		n++;
	}
	return n;
}

/* One counter-RNG path with its per-bounce events (16 x 20 doubles). */
int	ro_trace_path_events(ro_scene *s, uint64_t seed, int32_t pixel, int32_t sample,
	int jitter, double *events, double *rgb)
{
	int	rc;

	for (int k = 0; k < 16 * 20; k++)
		events[k] = 0;
	for (int k = 0; k < 16; k++)
		events[20 * k] = -2;
	g_events = events;
	rc = ro_trace_path_counter(s, seed, pixel, sample, jitter, rgb);
	g_events = NULL;
	return rc;
}

/* ------------------------------------------ differentiable parameters */

int64_t	ro_param_count(ro_scene *s)
{
	int64_t	sky = s->rgbe ? (int64_t)s->hw * s->hh * 3 : 0;

	return (int64_t)s->n_mats * 5 + sky;
}

int	ro_set_params(ro_scene *s, const double *theta, int64_t n, int exact)
{
	int	m, M = s->n_mats;

	if (n != ro_param_count(s))
		return -1;
	free(s->albedo_d);
	s->albedo_d = malloc(sizeof(double) * 3 * (M ? M : 1));
	for (m = 0; m < M; m++)
	{
		s->albedo_d[3 * m] = theta[3 * m];
		s->albedo_d[3 * m + 1] = theta[3 * m + 1];
		s->albedo_d[3 * m + 2] = theta[3 * m + 2];
		s->mats[m].roughness = theta[3 * M + m];
		s->mats[m].emission_strength = theta[4 * M + m];
	}
	if (s->rgbe)
	{
		size_t	t = (size_t)s->hw * s->hh * 3;

		free(s->sky_d);
		s->sky_d = malloc(sizeof(double) * t);
		memcpy(s->sky_d, theta + 5 * M, sizeof(double) * t);
		if (s->pdf_joint && s->hw >= 2 && s->hh >= 2)
			build_env_tables(s);
	}
	s->exact = exact;
	return 0;
}
