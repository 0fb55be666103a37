/*
 * mrt.h — C-ABI of the B200 path-tracing library (libmrt.so).
 *
 * This is the boundary that replaces miniRT's OpenGL compute path
 * (the src/gpu C files and the src/shaders GLSL tree) and its serial CPU sample loop
 * (src/ray_tracing/calc_sample.c). Everything crossing it is a plain C type:
 * pointers, sizes and fixed-layout structs; no CUDA or PyTorch type appears.
 *
 * Two layers use it:
 *  - the reference-named entry points (init_shader, convert_scene_build,
 *    convert_scene, compute_frame_gpu, clean_shaders, clean_scene,
 *    calc_one_sample) in libmrt_minirt.so, compiled against miniRT's own
 *    headers; they walk t_scene and call the functions below;
 *  - any other host (tests, benchmarks, ctypes) that describes a scene with
 *    the flat structs below.
 *
 * Scene values keep the reference's types and units (doubles for geometry,
 * 8-bit t_color colours, RGBE sky texels) so that the reference and this
 * library read identical numbers; the library repacks them to float32
 * device layouts itself.
 *
 * Error convention (reference: int 0 / -1 plus an "[Error]" line on stderr):
 * every int-returning call returns MRT_OK (0) or a negative mrt_status and
 * stores a message retrievable with mrt_last_error() (thread-local).
 * Threading: one context per host thread; calls on a context are serialised
 * by the caller (the reference calls its GPU path from the mlx loop thread
 * only, main_shader_utils.c:20-38).
 */
#ifndef MRT_H
# define MRT_H

# include <stddef.h>
# include <stdint.h>

# ifdef __cplusplus
extern "C" {
# endif

# define MRT_ABI_VERSION 4

# if defined(__GNUC__)
#  define MRT_API __attribute__((visibility("default")))
# else
#  define MRT_API
# endif

typedef enum mrt_status
{
	MRT_OK = 0,
	MRT_ERR_INVALID = -1,        /* bad argument or malformed scene */
	MRT_ERR_CUDA = -2,           /* CUDA runtime error */
	MRT_ERR_OOM = -3,            /* device or host allocation failed */
	MRT_ERR_QUEUE_OVERFLOW = -4, /* a wavefront queue overflowed (device status word) */
	MRT_ERR_BUDGET = -5,         /* a bounded device loop ran out of iterations */
	MRT_ERR_ABORTED = -6,        /* host watchdog raised the abort flag */
	MRT_ERR_NO_DEVICE = -7,      /* no CUDA device / extension not loadable */
	MRT_ERR_STACK = -8           /* traversal stack overflow (restart also failed) */
}	mrt_status;

/* ------------------------------------------------------------------ scene */

/* t_tex (scene_structs.h:61-82), t_tex_type order (scene_structs.h:20-27). */
typedef enum mrt_tex_type
{
	MRT_TEX_IMAGE = 0,          /* nearest texel of rgba (get_tex_color.c:31-37) */
	MRT_TEX_HDR = 1,            /* the reference returns black for it (get_tex_color.c:46) */
	MRT_TEX_COLOR = 2,          /* black, as the reference */
	MRT_TEX_CHECKER_LOCAL = 3,  /* uv checker (get_tex_color.c:38-44) */
	MRT_TEX_CHECKER_GLOBAL = 4  /* 3-D checker of the hit point (get_solid_texture.c:31) */
}	mrt_tex_type;

typedef struct mrt_texture
{
	int32_t			type;          /* mrt_tex_type */
	uint32_t		width;         /* IMAGE */
	uint32_t		height;
	int32_t			pad_;
	const uint8_t	*rgba;         /* IMAGE: 4 * width * height bytes, row-major, or NULL
	                                * (a NULL or empty image reads the reference's
	                                * magenta/black fallback checker) */
	double			checker_scale; /* CHECKER_* */
	uint8_t			c1[3];
	uint8_t			c2[3];
	uint8_t			pad2_[2];
}	mrt_texture;

/* t_mat (scene_structs.h:84-106). Colours are the 8-bit values the
 * reference stores; emission_color is emission_color_tmp, which
 * set_values_mat turns into emission_color = c / 255
 * (set_dependant_values_objs2.c:34). The *_tex fields name a texture as
 * 1 + its index in mrt_scene_desc.textures, 0 for none (so a zeroed struct
 * is untextured); a texture replaces the value at each hit with its texel
 * (the .r channel for scalars), as apply_all_map does (apply_map.c:60-85). */
typedef struct mrt_material
{
	uint8_t	color[3];
	uint8_t	emission_color[3];
	uint8_t	pad_[2];
	double	metallic;          /* clamped to [0,1] like set_values_mat */
	double	roughness;         /* clamped to [0,1] */
	double	ior;               /* <= 0 means "diffuse only" (dielectric.c:42) */
	double	transmission;
	double	ao;                /* ambient occlusion factor, default 1 */
	double	emission_strength;
	double	scale;             /* uv scale, default 1 */
	int32_t	color_tex;         /* texture colour and, for IMAGE, alpha: a texel of
	                            * alpha a hides the object with probability
	                            * 1 - a/255 (hit_register.c:62-72) */
	int32_t	metallic_tex;
	int32_t	roughness_tex;
	int32_t	transmission_tex;  /* also read at shadow-ray hits (is_light) */
	int32_t	ao_tex;
	int32_t	emission_strength_tex;
	int32_t	emission_color_tex;
	int32_t	normal_tex;        /* tangent-space normal map (apply_map.c:38-58) */
	double	normal_intensity;  /* lerp weight of the mapped normal; the reference's
	                            * default is 1 */
}	mrt_material;

/* t_sphere (scene_structs.h:167-175); material < 0 means no material
 * (the object's own colour is used, like "sp ... 255,0,0"). */
typedef struct mrt_sphere
{
	double	center[3];
	double	radius;
	int32_t	material;
	uint8_t	color[3];
	uint8_t	pad_;
}	mrt_sphere;

/* t_plane (scene_structs.h:177-183); normal must be unit length. */
typedef struct mrt_plane
{
	double	point[3];
	double	normal[3];
	int32_t	material;
	uint8_t	color[3];
	uint8_t	pad_;
}	mrt_plane;

/* t_cylinder (scene_structs.h:196-206): centred on position, axis along
 * orientation (unit, as parse_elements.c:28 leaves it), caps at
 * position +- height/2 * orientation. */
typedef struct mrt_cylinder
{
	double	position[3];
	double	orientation[3];
	double	diameter;
	double	height;
	int32_t	material;          /* < 0: none (the object's colour) */
	int32_t	material_top;      /* < 0: material */
	int32_t	material_bot;      /* < 0: material */
	uint8_t	color[3];
	uint8_t	pad_;
}	mrt_cylinder;

/* t_cone (scene_structs.h:185-194): position is the apex, the cap of the
 * given diameter lies at apex + height * orientation. */
typedef struct mrt_cone
{
	double	position[3];
	double	orientation[3];
	double	diameter;
	double	height;
	int32_t	material;
	int32_t	material_top;      /* < 0: material */
	uint8_t	color[3];
	uint8_t	pad_[5];
}	mrt_cone;

/* t_hyperboloid (scene_structs.h:154-165): x^2/a^2 + y^2/b^2 - z^2/c^2 =
 * shape in the frame of its orientation, clipped to |z| <= height / 2. */
typedef struct mrt_hyperboloid
{
	double	position[3];
	double	orientation[3];
	double	a;
	double	b;
	double	c;
	double	shape;
	double	height;
	int32_t	material;
	uint8_t	color[3];
	uint8_t	pad_;
}	mrt_hyperboloid;

/* Triangle mesh (t_custom_object + t_triangle/t_vertex, scene_structs.h:208-252).
 * Indexed: positions/normals per vertex, 3 indices per triangle. indices may
 * be NULL (triangle t uses vertices 3t..3t+2). uvs may be NULL (all zero).
 * tri_material may be NULL (every triangle uses `material`). Positions must
 * be the final world-space values (the reference re-transforms custom
 * objects in ft_update_obj_position; the miniRT adapter reads the vertices
 * after that step). */
typedef struct mrt_mesh
{
	uint32_t		n_vertices;
	uint32_t		n_triangles;
	const double	*positions;     /* 3 * n_vertices */
	const double	*normals;       /* 3 * n_vertices */
	const double	*uvs;           /* 2 * n_vertices or NULL */
	const uint32_t	*indices;       /* 3 * n_triangles or NULL */
	const int32_t	*tri_material;  /* n_triangles or NULL */
	int32_t			material;
	uint8_t			color[3];
	uint8_t			pad_;
}	mrt_mesh;

typedef enum mrt_light_type
{
	MRT_LIGHT_POINT = 0,       /* t_light (scene_structs.h:137-145) */
	MRT_LIGHT_DIRECTIONAL = 1  /* t_dlight (scene_structs.h:147-152) */
}	mrt_light_type;

typedef struct mrt_light
{
	int32_t	type;
	int32_t	shadow_sample;     /* soft-shadow samples (default 5 when radius given) */
	double	position[3];       /* point: position; directional: orientation (unit) */
	double	brightness;
	float	radius;            /* point light radius (0 = hard shadow) */
	uint8_t	color[3];
	uint8_t	pad_;
}	mrt_light;

/* t_camera (scene_structs.h:128-135). fov is the HORIZONTAL field of view in
 * integer degrees, as in the reference (viewport.c:57). */
typedef struct mrt_camera
{
	double	position[3];
	double	orientation[3];
	double	focus_dist;        /* 0 -> 1, as the reference UI does */
	double	defocus_angle;
	uint8_t	fov;
	uint8_t	pad_[7];
}	mrt_camera;

/* t_amb_light (scene_structs.h:108-126) with an optional Radiance RGBE sky
 * (t_hdr, hdr_parsing.h:18-35). hdr_rgbe == NULL means a uniform sky of
 * colour color * ratio / 255. */
typedef struct mrt_ambient
{
	double			ratio;
	const uint8_t	*hdr_rgbe;     /* 4 * hdr_width * hdr_height (r,g,b,e) */
	int32_t			hdr_width;
	int32_t			hdr_height;
	float			hdr_exposure;
	float			hdr_gamma;     /* 1 = linear */
	uint8_t			color[3];
	uint8_t			pad_[5];
}	mrt_ambient;

/* --caustic=N;radius;norm (option_caustic.c:63) plus the progressive
 * extension (fixed radius, shrinking by `shrink` per pass). */
typedef struct mrt_caustic
{
	int32_t		enable;
	int32_t		passes;          /* 1 = the reference's single kNN pass */
	uint64_t	photons_per_light;
	double		radius;          /* compared against r^2 (get_caustic.c:45) */
	double		norm_factor;
	double		shrink;          /* progressive mode radius factor per pass */
	int32_t		knn;             /* k nearest (reference: 15, material_default.c:81) */
	int32_t		mode;            /* 0 = kNN parity mode, 1 = fixed-radius progressive */
	int32_t		spp_per_pass;    /* progressive mode (mode 1, passes > 1): sample s uses
	                              * photon pass min(s / spp_per_pass, passes - 1), emitted
	                              * from its own streams, gathered within radius
	                              * radius * shrink^(2 pass) (radius is compared against
	                              * squared distances); 0 = one pass */
	int32_t		pad_;
}	mrt_caustic;

typedef struct mrt_scene_desc
{
	uint32_t			abi_version;    /* MRT_ABI_VERSION */
	int32_t				render_width;
	int32_t				render_height;
	int32_t				max_bounces;
	int32_t				triangle_one_sided;
	int32_t				pad_;
	double				ior_all;        /* scene ior, default 1 (parse_scene.c:122) */
	mrt_camera			camera;
	mrt_ambient			ambient;
	mrt_caustic			caustic;
	const mrt_material	*materials;
	int32_t				n_materials;
	int32_t				n_spheres;
	const mrt_sphere	*spheres;
	const mrt_plane		*planes;
	int32_t				n_planes;
	int32_t				n_meshes;
	const mrt_mesh		*meshes;
	const mrt_light		*lights;
	int32_t				n_lights;
	int32_t				pad2_;
	/* Objects of the BVH are numbered (flat prim ids) spheres, cylinders,
	 * cones, hyperboloids, then mesh triangles, then planes. */
	const mrt_cylinder		*cylinders;
	const mrt_cone			*cones;
	const mrt_hyperboloid	*hyperboloids;
	int32_t				n_cylinders;
	int32_t				n_cones;
	int32_t				n_hyperboloids;
	int32_t				n_textures;
	const mrt_texture	*textures;
}	mrt_scene_desc;

/* ------------------------------------------------------------- rendering */

typedef enum mrt_form
{
	MRT_FORM_MEGAKERNEL = 0,       /* persistent megakernel, lanes regenerate paths */
	MRT_FORM_WAVEFRONT = 1,        /* per-bounce queues, material-sorted shading */
	MRT_FORM_AUTO = 2,             /* autotuned choice for this scene */
	MRT_FORM_MEGAKERNEL_PLAIN = 3  /* one thread = one path, all bounces (baseline form) */
}	mrt_form;

typedef enum mrt_jitter
{
	MRT_JITTER_SHARED = 0,     /* one sub-pixel offset per sample for all pixels (render.c:33) */
	MRT_JITTER_PIXEL = 1       /* independent offset per pixel and sample */
}	mrt_jitter;

typedef struct mrt_render_params
{
	int32_t		spp;            /* samples per pixel this call */
	int32_t		sample_base;    /* index of the first sample (RNG counter) */
	uint64_t	seed;
	int32_t		max_bounces;    /* <= 0: the scene's value */
	int32_t		form;           /* mrt_form */
	int32_t		jitter;         /* mrt_jitter */
	int32_t		render_mode;    /* 0 path trace, 1 BVH heat map, 2 normals (minirt->render_mode) */
	int32_t		block_size;     /* threads per block, multiple of 32, <= 256; 0 = tuned default */
	int32_t		queue_capacity; /* wavefront paths in flight, 0 = tuned default */
	int32_t		sort_threshold; /* wavefront: sort shading queue above this many paths */
	int32_t		use_graph;      /* capture the spp loop in a CUDA graph */
	int32_t		env_sampler;    /* HDRI sampler: 0 alias table, 1 the reference's two-step
	                             * inverse-CDF lookup (get_dir.c:15-27), same distribution */
	const double *offset;       /* optional explicit shared jitter (x,y) for spp == 1 */
}	mrt_render_params;

typedef struct mrt_render_stats
{
	double		ms;             /* device time of the call (CUDA events) */
	uint64_t	paths;          /* camera paths traced */
	uint64_t	segments;       /* extension rays traced */
	uint64_t	shadow_rays;    /* shadow / NEE rays traced */
	uint32_t	kernel_launches;
	int32_t		status;         /* device status word (mrt_status) */
}	mrt_render_stats;

typedef struct mrt_ctx	mrt_ctx;

MRT_API const char	*mrt_last_error(void);
MRT_API int			mrt_version(void);
MRT_API int			mrt_device_count(void);

/* init_shader (init_shader.c:133): context + W*H accumulation buffer. */
MRT_API mrt_ctx		*mrt_create(int device, int width, int height);
MRT_API void		mrt_destroy(mrt_ctx *ctx);

/* convert_scene_build (gpu_scene.c:104): repack, build the BVH, upload,
 * build HDRI sampling tables on the device, emit photons if enabled. */
MRT_API int			mrt_scene_build(mrt_ctx *ctx, const mrt_scene_desc *scene);
/* convert_scene (gpu_scene.c:62): camera / ambient ratio / ior only. */
MRT_API int			mrt_set_camera(mrt_ctx *ctx, const mrt_camera *camera,
				double ior_all, double ambient_ratio);

/* Render params->spp samples per pixel into the device accumulator. */
MRT_API int			mrt_render(mrt_ctx *ctx, const mrt_render_params *params,
				mrt_render_stats *stats);
/* Multi-scene batch: renders params[i] on ctx[i] for all i in one call (all
 * contexts on the same device, each with a built scene, no context twice).
 * Each scene takes params[i].form (MRT_FORM_AUTO: its mrt_tune choice;
 * textured scenes always a megakernel). Megakernel scenes share one
 * persistent launch per view type (spheres / triangles, + quadrics,
 * + textures), their paths in one work queue, longest scene first by
 * predicted cost (paths x depth x log2 primitives); wavefront scenes each
 * run their own wavefront. These jobs run on four streams forked from and
 * joined back into ctx[0]'s stream, longest first onto the least-loaded
 * stream, so small scenes overlap large ones. params[0].block_size applies
 * to the megakernel launches; offset must be NULL. stats (may be NULL)
 * receives the call's device time, paths and kernel launches. */
MRT_API int			mrt_render_batch(mrt_ctx **ctx, const mrt_render_params *params,
				int32_t n, mrt_render_stats *stats);

/* BVH build options, applied by the next mrt_scene_build.
 * MRT_BVH_SAH (default): this library's binned-SAH binary tree, up to 8
 * primitives per leaf, traversed nearer child first. MRT_BVH_WIDE: the same
 * SAH tree built with leaves of up to 4 primitives and collapsed to an
 * 8-wide tree with 8-bit quantised child boxes (80-byte nodes, SAH-optimal
 * slot distribution), children visited in the ray's octant order; for
 * scenes of spheres, triangles and planes without textures (others get the
 * binary tree), and the binary tree when a scene's wide tree would be too
 * deep for its stack. MRT_BVH_REFERENCE: the reference's
 * own tree (bvh_build.c:16-127: one primitive per leaf, split at the median
 * of the object positions on the longest axis of the node bounds, in the
 * reference's sort order), traversed left child first, with the reference's
 * node-visit count for render_mode 1 (hit_bvh, bvh_hit.c:16). Use it for
 * parity runs: exact-t ties and heat-map counts then come out as the
 * reference's. order (may be NULL) lists the flat primitive ids (spheres,
 * cylinders, cones, hyperboloids, then mesh triangles, as mrt_scene_desc
 * holds them) in the order of the reference's object list (bvh_make_lst.c);
 * positions (may be NULL) gives, per flat id, the point the split sorts by
 * (get_obj_position, bvh_utils.c:88; default: the centre of a sphere or
 * quadric, the vertex mean of a triangle). Both arrays have n_prims entries
 * (3 doubles each for positions) and are copied by the call. */
typedef enum mrt_bvh_mode
{
	MRT_BVH_SAH = 0,
	MRT_BVH_REFERENCE = 1,
	MRT_BVH_WIDE = 2
}	mrt_bvh_mode;

typedef struct mrt_bvh_options
{
	int32_t			mode;
	int32_t			pad_;
	int64_t			n_prims;
	const int32_t	*order;
	const double	*positions;
}	mrt_bvh_options;

MRT_API int			mrt_set_bvh_options(mrt_ctx *ctx, const mrt_bvh_options *options);
/* Parity probe of the tree: the flat primitive id in each leaf slot of the
 * last build, in leaf order (up to cap entries); returns the slot count.
 * With MRT_BVH_REFERENCE this is the reference's sorted prim_indices order
 * (one primitive per leaf). */
MRT_API int64_t		mrt_read_bvh_leaves(mrt_ctx *ctx, int32_t *flat, int64_t cap);
/* Host-only diagnostic (no device needed): builds the MRT_BVH_SAH (binary)
 * or MRT_BVH_WIDE tree over n boxes (6 doubles each: min xyz, max xyz)
 * and, for the wide tree, checks its structure: every node reached once,
 * leaves inside the primitive array, each primitive in one leaf, and every
 * quantised slot box containing the boxes below it. stats (may be NULL)
 * receives 4 values: nodes, depth, leaves, 1 if the wide tree was built. */
MRT_API int			mrt_bvh_build_check(const double *boxes, int64_t n, int32_t mode, int64_t *stats);

/* Zero the device accumulator. */
MRT_API int			mrt_clear(mrt_ctx *ctx);
/* Copy the device accumulator (sum over samples, W*H*3 floats, row-major,
 * pixel i = y*W + x) to host memory. Returns the accumulated spp in *spp. */
MRT_API int			mrt_read_accum(mrt_ctx *ctx, float *rgb, int32_t *spp);
/* Add the device accumulator into a caller-owned double buffer laid out
 * like t_fcolor[W*H] (the reference's screen.float_render) and clear it. */
MRT_API int			mrt_accumulate_double(mrt_ctx *ctx, double *float_render);
/* BVH heat map (render_mode 1): per-pixel node-visit count of the last call. */
MRT_API int			mrt_read_depth(mrt_ctx *ctx, int32_t *depth);

/* Checkpoint of a progressive render in the reference's render_state.rts
 * format (export_render_state.c:15-33): int32 width, int32 height, int32
 * sample count, then width*height t_fcolor (3 doubles: the per-pixel sums),
 * little-endian. save writes the device accumulator and its sample count;
 * load replaces them (init_float_render, :35-51, accepts the file only when
 * its size and dimensions match; so does load, returning MRT_ERR_INVALID
 * otherwise), so that rendering continues from sample_base = that count.
 * The miniRT drop-in accumulates into the host float_render, which the
 * reference's own export_render_state / init_float_render handle. */
MRT_API int			mrt_render_state_save(mrt_ctx *ctx, const char *path);
MRT_API int			mrt_render_state_load(mrt_ctx *ctx, const char *path);

/* --------------------------------------------------- multi-GPU sharding
 * Replaces the render farm (src/network/handle_client.c:67-75: clients
 * render samples, the server adds their float_render buffers) with one
 * process per GPU over NCCL (NVLink / NVSwitch). Every rank builds the same
 * scene, renders its own contiguous sample range (mrt_shard_samples) with
 * render params sample_base = first, spp = count and the same seed, then
 * mrt_reduce_frame sums the accumulators: the root's frame equals a
 * single-GPU render of all samples up to summation order. libnccl.so.2 is
 * loaded on the first call; without it these calls return MRT_ERR_CUDA. */
# define MRT_COMM_ID_BYTES 128
/* A new communicator id (ncclGetUniqueId) on one rank; the caller sends its
 * MRT_COMM_ID_BYTES bytes to the other ranks by its own means. */
MRT_API int			mrt_comm_unique_id(unsigned char *id);
/* Joins ctx to the communicator `id` as `rank` of `world` (collective: every
 * rank calls it). One communicator per context, released by
 * mrt_comm_destroy or mrt_destroy. */
MRT_API int			mrt_comm_init(mrt_ctx *ctx, const unsigned char *id,
				int32_t rank, int32_t world);
/* Collective: sums every rank's device accumulator into root's (in place)
 * and every rank's accumulated sample count into root's, on the context's
 * stream; the other ranks' accumulators are left as they were. */
MRT_API int			mrt_reduce_frame(mrt_ctx *ctx, int32_t root);
MRT_API int			mrt_comm_destroy(mrt_ctx *ctx);
/* Contiguous shard of `total` samples for `rank` of `world`, balanced to
 * within one sample: [*first, *first + *count). */
MRT_API void		mrt_shard_samples(int64_t total, int32_t world, int32_t rank,
				int64_t *first, int64_t *count);

/* ------------------------------------------------------------ autotuner */

# define MRT_TUNE_MAX 32

/* One timed candidate of mrt_tune. */
typedef struct mrt_tune_entry
{
	int32_t	form;            /* MRT_FORM_MEGAKERNEL or MRT_FORM_WAVEFRONT */
	int32_t	block_size;
	int32_t	queue_capacity;
	int32_t	sort_threshold;
	double	mpaths_s;        /* measured throughput, 0 if the candidate failed */
}	mrt_tune_entry;

typedef struct mrt_tune_result
{
	int32_t			n;       /* candidates timed */
	int32_t			best;    /* index of the fastest */
	mrt_tune_entry	entry[MRT_TUNE_MAX];
}	mrt_tune_result;

/* Times the render forms and their launch shapes (block size, queue
 * capacity, material-sort threshold) on the current scene with `spp`
 * samples per candidate, keeps the fastest as the context's choice for
 * MRT_FORM_AUTO and zero-valued launch parameters, and reports all of them.
 * Leaves the accumulator cleared. */
MRT_API int			mrt_tune(mrt_ctx *ctx, int32_t spp, uint64_t seed, mrt_tune_result *out);

/* ------------------------------------------------------- parity probes */

/* A ray in the reference's double layout (t_ray, structs.h:63-67). */
typedef struct mrt_ray
{
	double	orig[3];
	double	dir[3];
}	mrt_ray;

/* Closest hit (hit_register_all, hit_register.c:109).
 * prim: flat primitive id — spheres, cylinders, cones, hyperboloids,
 * triangles in mesh order, then planes — or -1 for a miss. u, v: a
 * triangle's barycentrics; for a quadric u is the part hit (0 lateral
 * surface, 1 top cap, 2 bottom cap). */
typedef struct mrt_hit
{
	int32_t	prim;
	int32_t	front_face;
	float	t;
	float	u;
	float	v;
	float	normal[3];
	float	point[3];
	int32_t	visits;         /* BVH nodes visited (heat-map counter) */
}	mrt_hit;

MRT_API int			mrt_trace_first_hit(mrt_ctx *ctx, const mrt_ray *rays, int64_t n,
				mrt_hit *hits);

/* Debug probe: traces single paths (pixel[i], sample[i]) with the render
 * seed / jitter / env_sampler of params and records each bounce as 20
 * floats (flat prim id or -1 for the final miss, t, point.xyz, normal.xyz,
 * then direction.xyz, power.rgb and radiance.rgb after shading, material),
 * up to 16 bounces per path (unused records start with -2). rgb receives
 * each path's radiance. */
MRT_API int			mrt_trace_paths(mrt_ctx *ctx, const mrt_render_params *params,
				const int32_t *pixel, const int32_t *sample, int32_t n,
				float *events, float *rgb);

/* HDRI tables (importance_sampling_manager.c:41) as built on the device:
 * pdf_joint W*H f32, cdf_marginal_inverse H f32, cdf_conditional_inverse W*H f32.
 * Any pointer may be NULL. */
MRT_API int			mrt_read_env_tables(mrt_ctx *ctx, float *pdf_joint,
				float *cdf_marginal_inverse, float *cdf_conditional_inverse);

/* Draw n HDRI importance samples on the device (seed, sampler as in
 * mrt_render_params.env_sampler): outcome[i] is the sampled outcome of the
 * reference's two-step lookup (row * W + column offset), out4 holds n float4
 * (dir.x, dir.y, dir.z, pdf). */
MRT_API int			mrt_env_sample(mrt_ctx *ctx, int64_t n, uint64_t seed, int32_t sampler,
				int32_t *outcome, float *out4);

/* Photon map (caustic_manager.c:83): number of stored photons, and their
 * positions / powers as float4 (x,y,z,_) pairs if the pointers are non-NULL. */
MRT_API int64_t		mrt_photon_count(mrt_ctx *ctx);
MRT_API int			mrt_read_photons(mrt_ctx *ctx, float *pos4, float *power4, int64_t cap);
/* Upload an explicit photon set (replacing the emitted one) and rebuild the grid. */
MRT_API int			mrt_set_photons(mrt_ctx *ctx, const double *pos3, const double *power3,
				int64_t n);
/* Caustic radiance at query points (estimate_caustics_physically_based,
 * get_caustic.c:67), k nearest photons, as RGB doubles. */
MRT_API int			mrt_caustic_query(mrt_ctx *ctx, const double *points3, int64_t n,
				int32_t k, double *rgb_out);

/* ------------------------------------- table build without allocation
 * No counterpart in the reference. The HDRI importance-sampling tables that
 * mrt_scene_build makes (importance_sampling_manager.c:41; read them back with
 * mrt_read_env_tables), built into buffers the caller owns, for hosts that
 * cannot allocate GPU memory when they need the tables: a host whose device
 * memory all comes from its own pre-sized arena or pool, or a loop that must
 * never reach the allocator. This call allocates nothing: no cudaMalloc, no
 * cudaFree, no allocating library routine.
 *
 * rgbe: width*height texels of 4 bytes (r, g, b, e), device memory,
 * 4-byte aligned;
 * hdr_exposure as in mrt_ambient; outputs as for mrt_read_env_tables
 * (pdf_joint W*H, cdf_marginal_inverse H, cdf_conditional_inverse W*H
 * floats), device memory. stream is a cudaStream_t (NULL: the legacy default
 * stream); the call returns once the tables are written. Runs on `device`,
 * restoring the caller's current device afterwards.
 *
 * Limits: 2 <= width, 2 <= height <= MRT_ENV_NOALLOC_MAX_ROWS and
 * width*height <= MRT_ENV_NOALLOC_MAX_TEXELS (512x512 or 1024x256);
 * larger skies get MRT_ERR_INVALID with the limit in mrt_last_error(). The
 * build's scratch (about 4 MiB of doubles) is a fixed array in the library
 * that each GPU holds, once loaded, until the process exits.
 *
 * First call per device: with CUDA's lazy module loading (the default), the
 * modules that hold the array and the table kernels load on first use, and
 * the first call also looks up the array's device address (set-up done once
 * per device). That first call therefore does take device memory (the
 * modules and the 4 MiB array) through the driver: make it once at start-up,
 * before the host fixes its arena; later calls allocate nothing.
 * The call synchronises `stream` before it returns, so it must not be made on
 * a stream that is being captured into a CUDA graph.
 * The cached device address is not refreshed after cudaDeviceReset: a host
 * that resets a device must not call this entry point on it afterwards.
 * All calls on a device share the array, so calls that overlap on the GPU
 * (from several host threads or streams at once) race and must be serialised
 * by the caller. Every scratch value a call reads it has written itself, so
 * what an earlier call left there does not matter. */
# define MRT_ENV_NOALLOC_MAX_TEXELS 262144
# define MRT_ENV_NOALLOC_MAX_ROWS 4096
MRT_API int			mrt_env_tables_noalloc(int device, const uint8_t *rgbe, int32_t width,
				int32_t height, float hdr_exposure, float *pdf_joint,
				float *cdf_marginal_inverse, float *cdf_conditional_inverse, void *stream);

/* ------------------------------------------------ differentiable rendering
 * (no counterpart in the reference, which renders only; the parameters are
 * float shadows of its fields.)
 *
 * theta, M materials and a W x H sky, as one float array:
 *   [albedo M*3 (t_mat.color_value / 255) | roughness M (roughness_value) |
 *    emission strength M (emission_strength) |
 *    sky radiance H*W*3 (what get_hdr_pixel_skybox returns, get_hdr_value.c:43)]
 * The sky block is empty without an HDR sky; a differentiable sky must be
 * linear (hdr gamma 1).
 *
 * The pair follows the torch.autograd.Function contract: mrt_forward(theta)
 * returns the image (W*H*3 floats, the mean over params->spp samples);
 * mrt_backward(theta, dL/dimage) returns dL/dtheta for the same theta and
 * the same params (seed, sample_base, spp, max_bounces, jitter: the
 * backward replays exactly the forward's paths). Fields of params other
 * than those five are ignored; max_bounces must be <= 16. Array
 * arguments may be host memory or device memory of the context's GPU.
 * The forward is the production renderer (persistent megakernel) over
 * materials, sky and HDRI sampling tables rebuilt from theta; the backward
 * is the path-replay adjoint: the derivative for fixed random numbers,
 * which central differences with common random numbers converge to as the
 * step shrinks. Discrete choices (hit primitive, branch, visibility,
 * inverse-CDF and nearest-texel lookups) carry no gradient. */

/* counts[0..3] = albedo, roughness, emission and sky entries; returns the
 * total (>= 0) or a negative mrt_status. */
MRT_API int64_t		mrt_diff_layout(mrt_ctx *ctx, int64_t counts[4]);
/* theta of the scene as built (colours / 255, roughness, emission, sky). */
MRT_API int			mrt_diff_get_params(mrt_ctx *ctx, float *theta);
MRT_API int			mrt_forward(mrt_ctx *ctx, const float *theta,
				const mrt_render_params *params, float *image, mrt_render_stats *stats);
MRT_API int			mrt_backward(mrt_ctx *ctx, const float *theta,
				const mrt_render_params *params, const float *grad_image,
				float *grad_theta, mrt_render_stats *stats);

# ifdef __cplusplus
}
# endif

#endif
