/*
 * mrt_oracle.h — TEST INFRASTRUCTURE: FP64 CPU restatement of miniRT's
 * path-tracing hot path (the oracle). Only tests, the smoke check and the
 * benchmark's CPU-baseline leg use it; the product never links it.
 *
 * The restatement follows the reference's C code function by function (each
 * function cites the file:line it restates) and reproduces its floating-point
 * operation order, so that with the reference's own RNG stream
 * (RO_RNG_REFERENCE: global xorshift64 13/7/17, src/math/random.c:17-30) it
 * renders bit-identical images. With RO_RNG_COUNTER it draws from the
 * per-path counter-based generator that the CUDA kernels use, so single paths
 * can be compared between CPU (FP64) and GPU (FP32).
 */
#ifndef MRT_ORACLE_H
# define MRT_ORACLE_H

# include <stdint.h>
# include "mrt.h"

# ifdef __cplusplus
extern "C" {
# endif

typedef struct ro_scene	ro_scene;

enum { RO_RNG_REFERENCE = 0, RO_RNG_COUNTER = 1 };

typedef struct ro_hit
{
	int32_t	prim;        /* flat id, -1 miss */
	int32_t	front_face;
	int32_t	depth;       /* nodes visited by the reference's exhaustive DFS */
	int32_t	material;
	double	t;
	double	u;
	double	v;
	double	point[3];
	double	normal[3];
	double	color[3];
}	ro_hit;

typedef struct ro_counters
{
	uint64_t	paths;
	uint64_t	segments;      /* closest-hit queries on extension rays */
	uint64_t	shadow_rays;   /* any/closest-hit queries for lights and env NEE */
	uint64_t	node_visits;   /* near-first, t-culled traversal over the median BVH */
	uint64_t	prim_tests;
	uint64_t	sphere_tests;
	uint64_t	tri_tests;
	uint64_t	plane_tests;
	uint64_t	hits;          /* shading events */
	uint64_t	env_nee;
	uint64_t	caustic_gathers;
}	ro_counters;

ro_scene	*ro_create(const mrt_scene_desc *d);
void		ro_destroy(ro_scene *s);

void		ro_set_reference_rng(uint64_t state);
uint64_t	ro_get_reference_rng(void);

/* Closest hit per ray (hit_register_all, hit_register.c:109). */
int			ro_first_hit(ro_scene *s, const mrt_ray *rays, int64_t n, ro_hit *out);

/* Full-frame samples exactly like render_cpu/draw_pixels/calc_one_sample
 * with the reference RNG; accum is W*H*3 doubles (t_fcolor layout). */
int			ro_render_reference(ro_scene *s, int spp, double *accum);

/* Counter-RNG render of a pixel subset (or all pixels if pix == NULL):
 * sample indices [sample_base, sample_base+spp), jitter 0 = shared per
 * sample, 1 = per pixel. accum is n*3 doubles (or W*H*3). */
int			ro_render_counter(ro_scene *s, uint64_t seed, int sample_base, int spp,
				int jitter, const int32_t *pix, int64_t n, double *accum,
				ro_counters *cnt);

/* One path with the counter RNG for (seed, pixel, sample). */
int			ro_trace_path_counter(ro_scene *s, uint64_t seed, int32_t pixel,
				int32_t sample, int jitter, double *rgb);

/* The same path with its per-bounce event records (16 x 20 doubles, the
 * layout of mrt_trace_paths). */
int			ro_trace_path_events(ro_scene *s, uint64_t seed, int32_t pixel,
				int32_t sample, int jitter, double *events, double *rgb);

/* HDRI tables (importance_sampling_manager.c:41). Returns 0 if no sky. */
int			ro_env_tables(ro_scene *s, float *pdf_joint, float *cdf_m_inv,
				float *cdf_c_inv, double *column_average);
/* Exact probability of each (row index, conditional index) outcome of the
 * reference's two-step inverse-CDF sampler (get_dir.c:15-27), for
 * outcome k = iy * (W + 1) + (j - j_lo(iy)). Returns the number of entries. */
int64_t		ro_env_outcome_probs(ro_scene *s, double *prob, int32_t *cond_index);

/* Photon map with the reference RNG (caustic_manager.c:83). */
int64_t		ro_photon_count(ro_scene *s);
int			ro_photons(ro_scene *s, double *pos3, double *pow3, int32_t *in_leaf);
int			ro_caustic_query(ro_scene *s, const double *pts3, int64_t n, int k,
				double *rgb);

/* Canonical per-path work counters used for the algorithmic-bytes figure. */
int			ro_counters_read(ro_scene *s, ro_counters *out);

/* Mesh vertices: 1 = apply the reference's load-time re-transform
 * (default), 0 = use them as given. Affects scenes created afterwards. */
void		ro_set_mesh_transform(int on);
/* Triangle corner positions as intersected, 9 doubles per flat triangle. */
int			ro_triangle_positions(ro_scene *s, double *out);

/* Differentiable parameters, the layout of mrt_forward's theta:
 * [albedo M*3 | roughness M | emission M | sky W*H*3]. ro_set_params
 * replaces the scene's values (colours by the doubles given, the RGBE sky by
 * linear radiance, HDRI tables rebuilt from it); exact = 1 also keeps every
 * intermediate in double (triangle t/u/v, NEE cosine and pdf, Fresnel), so
 * that central differences with a tiny step give the FP64 reference
 * gradient. Returns -1 if n does not match ro_param_count. */
int64_t		ro_param_count(ro_scene *s);
int			ro_set_params(ro_scene *s, const double *theta, int64_t n, int exact);

/* Counter-based RNG shared with the CUDA kernels (PCG32, XSH-RR output). */
uint64_t	ro_path_seed(uint64_t seed, uint32_t pixel, uint32_t sample);
float		ro_pcg_float(uint64_t *state);

# ifdef __cplusplus
}
# endif

#endif
