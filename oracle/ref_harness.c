/*
 * ref_harness.c — TEST INFRASTRUCTURE (oracle). Never part of the product.
 *
 * Builds the reference's own t_minirt/t_scene (includes/structs.h:419-431,
 * includes/scene_structs.h:362-383) from a flat mrt_scene_desc and exposes
 * the reference's CPU path through a small C API for the parity tests, the
 * CPU baseline and the fixture generators:
 *   refh_first_hit   -> hit_register_all        (src/ray_tracing/hit_register/hit_register.c:109)
 *   refh_render      -> calc_one_sample          (src/ray_tracing/calc_sample.c:73), offsets from
 *                       vec3_random() like draw_pixels (src/ray_tracing/render.c:28-33)
 *   refh_render_pixels -> calc_one_sample_task   (calc_sample.c:44) on a pixel subset
 *   refh_env_tables  -> make_importance_sampling_map (importance_sampling_manager.c:41)
 *   refh_photons / refh_caustic_query -> caustic_manager / estimate_caustics_physically_based
 *                       (src/caustic/caustic_manager.c:83, get_caustic.c:67)
 * Scene preparation runs the reference's own init_viewport (viewport.c:90),
 * which builds the median-split BVH (bvh_manager.c:17), the HDRI tables and
 * the photon map exactly as the reference application does.
 */
#include "minirt.h"
#include "bvh.h"
#include "caustic.h"
#include "importance_sampling.h"
#include "mrt.h"
#include <string.h>

extern uint64_t	oracle_ref_rng_state;
extern int		oracle_quiet;

void	calc_one_sample_task(t_minirt *minirt, t_vec3 offset, t_uint i,
			int max_bounces);

typedef struct s_refh_mesh_group
{
	t_custom_object	*obj;
	uint32_t		*flat_tri;      /* local triangle -> flat triangle id */
}	t_refh_mesh_group;

typedef struct s_refh
{
	t_minirt			*m;
	int					n_spheres;
	int					n_tris;
	int					tri_base;     /* flat id of the first triangle */
	int					n_planes;
	int					*elem_flat;    /* element index -> flat prim id (spheres/planes) */
	int					n_groups;
	t_refh_mesh_group	*groups;
	t_tex				sky;
	t_rgbe				*sky_pixels;
	int					max_bounces;
}	t_refh;

void	refh_set_quiet(int quiet)
{
	oracle_quiet = quiet;
}

void	refh_set_seed(uint64_t seed)
{
	oracle_ref_rng_state = seed ? seed : 42;
}

uint64_t	refh_get_seed(void)
{
	return (oracle_ref_rng_state);
}

double	refh_random_double(void)
{
	return (random_double());
}

static t_color	c3(const uint8_t *c)
{
	return ((t_color){c[0], c[1], c[2]});
}

static t_vec3	v3(const double *p)
{
	return ((t_vec3){p[0], p[1], p[2]});
}

/* texture k (1-based, 0 none) of the scene's t_tex array */
static t_tex	*tex_ptr(t_scene *sc, int32_t k)
{
	if (k <= 0 || k > sc->tex_amount)
		return (NULL);
	return (&sc->textures[k - 1]);
}

/* t_tex from an mrt_texture (scene_structs.h:61-82); the image copied */
static void	fill_texture(t_tex *o, const mrt_texture *t, int i)
{
	snprintf(o->name, sizeof(o->name), "t%d", i);
	o->type = (t_tex_type)t->type;
	o->checker.scale = t->checker_scale;
	o->checker.c1 = c3(t->c1);
	o->checker.c2 = c3(t->c2);
	if (t->rgba && t->width && t->height)
	{
		o->img.width = t->width;
		o->img.height = t->height;
		o->img.rgba = malloc(sizeof(t_rgba) * (size_t)t->width * t->height);
		memcpy(o->img.rgba, t->rgba, 4 * (size_t)t->width * t->height);
	}
}

static void	fill_material_tex(t_scene *sc, t_mat *m, const mrt_material *s)
{
	m->color_tex = tex_ptr(sc, s->color_tex);
	m->metallic_tex = tex_ptr(sc, s->metallic_tex);
	m->roughness_tex = tex_ptr(sc, s->roughness_tex);
	m->transmission_tex = tex_ptr(sc, s->transmission_tex);
	m->ao_tex = tex_ptr(sc, s->ao_tex);
	m->emission_strength_tex = tex_ptr(sc, s->emission_strength_tex);
	m->emission_color_tex = tex_ptr(sc, s->emission_color_tex);
	m->normal = tex_ptr(sc, s->normal_tex);
	m->normal_intensity = s->normal_intensity;
}

static void	fill_material(t_mat *m, const mrt_material *s, int i)
{
	snprintf(m->name, sizeof(m->name), "m%d", i);
	m->color_value = c3(s->color);
	m->metallic_value = s->metallic;
	m->roughness_value = s->roughness;
	m->ior = s->ior;
	m->transmission_value = s->transmission;
	m->ao_value = s->ao;
	m->emission_strength = s->emission_strength;
	m->emission_color_tmp = c3(s->emission_color);
	m->scale = s->scale;
	m->normal_intensity = 1;
	/* set_values_mat (set_dependant_values_objs2.c:32-37) */
	m->emission_color = color_to_fcolor(m->emission_color_tmp);
	m->metallic_value = clamp_double(m->metallic_value);
	m->roughness_value = clamp_double(m->roughness_value);
}

static t_mat	*mat_ptr(t_scene *sc, int32_t id)
{
	if (id < 0 || id >= sc->mat_amount)
		return (NULL);
	return (&sc->materials[id]);
}

static int	count_groups(const mrt_mesh *me)
{
	int		n;
	uint32_t	t;
	int32_t	*seen;
	int32_t	k;

	if (!me->tri_material)
		return (1);
	n = 0;
	seen = malloc(sizeof(int32_t) * (me->n_triangles + 1));
	for (t = 0; t < me->n_triangles; t++)
	{
		for (k = 0; k < n; k++)
			if (seen[k] == me->tri_material[t])
				break ;
		if (k == n)
			seen[n++] = me->tri_material[t];
	}
	free(seen);
	return (n);
}

static void	set_vertex(t_vertex *v, const mrt_mesh *me, uint32_t idx)
{
	v->pos = v3(me->positions + 3 * (size_t)idx);
	v->normal = v3(me->normals + 3 * (size_t)idx);
	v->u = me->uvs ? me->uvs[2 * (size_t)idx] : 0;
	v->v = me->uvs ? me->uvs[2 * (size_t)idx + 1] : 0;
}

/* One t_custom_object per (mesh, material): bvh_make_lst overwrites each
 * triangle's material with its object's (bvh_make_lst.c:16-27). */
static int	add_mesh_groups(t_refh *h, const mrt_mesh *me, uint32_t flat_base,
	int *el)
{
	t_scene		*sc;
	int32_t		mat;
	uint32_t	t;
	uint32_t	cnt;
	int			g;
	char		*done;

	sc = &h->m->scene;
	done = calloc(me->n_triangles + 1, 1);
	for (t = 0; t < me->n_triangles; t++)
	{
		if (done[t])
			continue ;
		mat = me->tri_material ? me->tri_material[t] : me->material;
		cnt = 0;
		for (uint32_t s = t; s < me->n_triangles; s++)
			if (!done[s] && (me->tri_material ? me->tri_material[s] : me->material) == mat)
				cnt++;
		g = h->n_groups++;
		h->groups[g].obj = calloc(1, sizeof(t_custom_object));
		h->groups[g].flat_tri = malloc(sizeof(uint32_t) * cnt);
		t_custom_object *o = h->groups[g].obj;
		o->name = "mesh";
		o->triangles = calloc(cnt, sizeof(t_triangle));
		o->obj_list = calloc(cnt, sizeof(t_object));
		o->triangle_count = cnt;
		o->orientation = (t_vec3){0, 1, 0};
		o->prev_orientation = (t_vec3){0, 1, 0};
		o->scale = (t_vec3){1, 1, 1};
		o->prev_scale = (t_vec3){1, 1, 1};
		o->material = mat_ptr(sc, mat);
		o->color = c3(me->color);
		o->index = g;
		cnt = 0;
		for (uint32_t s = t; s < me->n_triangles; s++)
		{
			if (done[s] || (me->tri_material ? me->tri_material[s] : me->material) != mat)
				continue ;
			done[s] = 1;
			t_triangle *tr = &o->triangles[cnt];
			uint32_t i0 = me->indices ? me->indices[3 * (size_t)s] : 3 * s;
			uint32_t i1 = me->indices ? me->indices[3 * (size_t)s + 1] : 3 * s + 1;
			uint32_t i2 = me->indices ? me->indices[3 * (size_t)s + 2] : 3 * s + 2;
			set_vertex(&tr->v0, me, i0);
			set_vertex(&tr->v1, me, i1);
			set_vertex(&tr->v2, me, i2);
			tr->center = vec3_divide_scalar(vec3_add(vec3_add(tr->v0.pos,
					tr->v1.pos), tr->v2.pos), 3.0);
			tr->material = o->material;
			tr->color = o->color;
			tr->obj = o;
			o->obj_list[cnt].object = tr;
			o->obj_list[cnt].type = TRIANGLE;
			h->groups[g].flat_tri[cnt] = flat_base + s;
			cnt++;
		}
		sc->elements[*el].object = o;
		sc->elements[*el].type = CUSTOM;
		h->elem_flat[*el] = -1;
		(*el)++;
	}
	free(done);
	return (0);
}

static void	setup_sky(t_refh *h, const mrt_ambient *a)
{
	t_scene	*sc;
	size_t	n;

	sc = &h->m->scene;
	sc->amb_light.ratio = a->ratio;
	sc->amb_light.skybox_c = c3(a->color);
	if (!a->hdr_rgbe || a->hdr_width <= 0 || a->hdr_height <= 0)
		return ;
	n = (size_t)a->hdr_width * a->hdr_height;
	h->sky_pixels = malloc(n * sizeof(t_rgbe));
	memcpy(h->sky_pixels, a->hdr_rgbe, n * 4);
	memset(&h->sky, 0, sizeof(h->sky));
	strcpy(h->sky.name, "sky");
	h->sky.type = HDR;
	h->sky.hdr.width = a->hdr_width;
	h->sky.hdr.height = a->hdr_height;
	h->sky.hdr.exposure = a->hdr_exposure;
	h->sky.hdr.gamma = a->hdr_gamma;
	h->sky.hdr.pixels = h->sky_pixels;
	sc->amb_light.skybox_t = &h->sky;
}

/* Build the reference scene and run its init_viewport (BVH build, HDRI
 * tables, photon map). Returns NULL on malformed input. */
void	*refh_create(const mrt_scene_desc *d)
{
	t_refh		*h;
	t_minirt	*m;
	t_scene		*sc;
	int			el;
	int			ngroups;
	int			nquad;
	uint32_t	flat_base;

	if (!d || d->abi_version != MRT_ABI_VERSION || d->render_width <= 0
		|| d->render_height <= 0)
		return (NULL);
	h = calloc(1, sizeof(t_refh));
	m = calloc(1, sizeof(t_minirt));
	h->m = m;
	sc = &m->scene;
	strcpy(sc->name, "flat");
	sc->mat_amount = d->n_materials;
	sc->materials = calloc(d->n_materials + 1, sizeof(t_mat));
	sc->tex_amount = (d->n_textures > 0 && d->textures) ? d->n_textures : 0;
	sc->textures = calloc(sc->tex_amount + 1, sizeof(t_tex));
	for (int i = 0; i < sc->tex_amount; i++)
		fill_texture(&sc->textures[i], &d->textures[i], i);
	for (int i = 0; i < d->n_materials; i++)
	{
		fill_material(&sc->materials[i], &d->materials[i], i);
		fill_material_tex(sc, &sc->materials[i], &d->materials[i]);
	}
	ngroups = 0;
	for (int i = 0; i < d->n_meshes; i++)
		ngroups += count_groups(&d->meshes[i]);
	h->groups = calloc(ngroups + 1, sizeof(t_refh_mesh_group));
	nquad = d->n_cylinders + d->n_cones + d->n_hyperboloids;
	sc->elements = calloc(d->n_spheres + nquad + ngroups + d->n_planes + d->n_lights + 1,
			sizeof(t_object));
	h->elem_flat = calloc(d->n_spheres + nquad + ngroups + d->n_planes + d->n_lights + 1,
			sizeof(int));
	el = 0;
	for (int i = 0; i < d->n_spheres; i++)
	{
		t_sphere *s = calloc(1, sizeof(t_sphere));
		s->position = v3(d->spheres[i].center);
		s->diameter = d->spheres[i].radius * 2.0;
		s->radius = s->diameter * 0.5;
		s->sqrt_radius = s->radius * s->radius;
		s->material = mat_ptr(sc, d->spheres[i].material);
		s->color = c3(d->spheres[i].color);
		sc->elements[el].object = s;
		sc->elements[el].type = SPHERE;
		h->elem_flat[el++] = i;
	}
	h->n_spheres = d->n_spheres;
	/* the element list is spheres, cylinders, cones, hyperboloids, meshes,
	 * planes, lights: bvh_make_lst keeps that order for the BVH objects */
	for (int i = 0; i < d->n_cylinders; i++)
	{
		const mrt_cylinder *c = &d->cylinders[i];
		t_cylinder *o = calloc(1, sizeof(t_cylinder));
		o->position = v3(c->position);
		o->orientation = v3(c->orientation);
		o->diameter = c->diameter;
		o->height = c->height;
		o->material = mat_ptr(sc, c->material);
		o->material_top = mat_ptr(sc, c->material_top);
		o->material_bot = mat_ptr(sc, c->material_bot);
		o->color = c3(c->color);
		sc->elements[el].object = o;
		sc->elements[el].type = CYLINDER;
		h->elem_flat[el++] = d->n_spheres + i;
	}
	for (int i = 0; i < d->n_cones; i++)
	{
		const mrt_cone *c = &d->cones[i];
		t_cone *o = calloc(1, sizeof(t_cone));
		o->position = v3(c->position);
		o->orientation = v3(c->orientation);
		o->diameter = c->diameter;
		o->height = c->height;
		o->material = mat_ptr(sc, c->material);
		o->material_top = mat_ptr(sc, c->material_top);
		o->color = c3(c->color);
		sc->elements[el].object = o;
		sc->elements[el].type = CONE;
		h->elem_flat[el++] = d->n_spheres + d->n_cylinders + i;
	}
	for (int i = 0; i < d->n_hyperboloids; i++)
	{
		const mrt_hyperboloid *c = &d->hyperboloids[i];
		t_hyperboloid *o = calloc(1, sizeof(t_hyperboloid));
		o->position = v3(c->position);
		o->orientation = v3(c->orientation);
		o->a = c->a;
		o->b = c->b;
		o->c = c->c;
		o->shape = c->shape;
		o->height = c->height;
		o->material = mat_ptr(sc, c->material);
		o->color = c3(c->color);
		sc->elements[el].object = o;
		sc->elements[el].type = HYPERBOLOID;
		h->elem_flat[el++] = d->n_spheres + d->n_cylinders + d->n_cones + i;
	}
	flat_base = d->n_spheres + nquad;
	for (int i = 0; i < d->n_meshes; i++)
	{
		add_mesh_groups(h, &d->meshes[i], flat_base, &el);
		flat_base += d->meshes[i].n_triangles;
	}
	h->tri_base = d->n_spheres + nquad;
	h->n_tris = flat_base - h->tri_base;
	for (int i = 0; i < d->n_planes; i++)
	{
		t_plane *p = calloc(1, sizeof(t_plane));
		p->position = v3(d->planes[i].point);
		p->normal = vec3_unit(v3(d->planes[i].normal));
		p->material = mat_ptr(sc, d->planes[i].material);
		p->color = c3(d->planes[i].color);
		sc->elements[el].object = p;
		sc->elements[el].type = PLANE;
		h->elem_flat[el++] = flat_base + i;
	}
	h->n_planes = d->n_planes;
	for (int i = 0; i < d->n_lights; i++)
	{
		const mrt_light *L = &d->lights[i];
		if (L->type == MRT_LIGHT_DIRECTIONAL)
		{
			t_dlight *dl = calloc(1, sizeof(t_dlight));
			dl->orientation = vec3_unit(v3(L->position));
			dl->brightness = L->brightness;
			dl->color = c3(L->color);
			sc->elements[el].object = dl;
			sc->elements[el].type = DIRECTIONAL_LIGHT;
		}
		else
		{
			t_light *pl = calloc(1, sizeof(t_light));
			pl->position = v3(L->position);
			pl->brightness = L->brightness < 0 ? 0 : L->brightness;
			pl->color = c3(L->color);
			pl->radius = L->radius;
			pl->shadow_sample = L->shadow_sample;
			sc->elements[el].object = pl;
			sc->elements[el].type = LIGHT;
		}
		h->elem_flat[el++] = -1;
	}
	sc->el_amount = el;
	sc->camera.position = v3(d->camera.position);
	sc->camera.orientation = vec3_unit(v3(d->camera.orientation));
	sc->camera.fov = d->camera.fov;
	sc->camera.focus_dist = d->camera.focus_dist == 0 ? 1 : d->camera.focus_dist;
	sc->camera.defocus_angle = d->camera.defocus_angle;
	m->controls.values.fov = d->camera.fov;
	sc->ior_all = d->ior_all;
	sc->render_width = d->render_width;
	sc->render_height = d->render_height;
	sc->win_width = d->render_width;
	sc->win_height = d->render_height;
	sc->build_bvh = 1;
	setup_sky(h, &d->ambient);
	m->options.triangle_one_sided = d->triangle_one_sided;
	m->options.no_display = 1;
	if (d->caustic.enable)
	{
		m->options.caustic.caustic_enable = 1;
		m->options.caustic.nb_photon = d->caustic.photons_per_light;
		m->options.caustic.caustic_radius = d->caustic.radius;
		m->options.caustic.norm_factor = d->caustic.norm_factor;
	}
	m->controls.max_bounces = d->max_bounces;
	h->max_bounces = d->max_bounces;
	m->render_mode = 0;
	m->screen.float_render = calloc((size_t)d->render_width * d->render_height,
			sizeof(t_fcolor));
	m->viewport = init_viewport(m);
	return (h);
}

/* A .rt file through the reference's own parser (parse_scene,
 * parse_scene.c:99) and the object set-up of set_dependant_values
 * (set_dependant_values.c:47-73, without its UI parts), then the same
 * render set-up as refh_create. The render size and depth are the caller's
 * (the reference takes them from its UI controls). */
extern int	oracle_ref_parse_mat_index;
extern int	oracle_ref_parse_tex_index;

void	*refh_create_from_rt(const char *path, int width, int height, int max_bounces)
{
	t_refh		*h;
	t_minirt	*m;
	t_scene		*sc;

	if (!path || width <= 0 || height <= 0)
		return (NULL);
	oracle_ref_parse_mat_index = 0;
	oracle_ref_parse_tex_index = 0;
	h = calloc(1, sizeof(t_refh));
	m = calloc(1, sizeof(t_minirt));
	h->m = m;
	if (parse_scene(m, (char *)path) == 0)
		return (NULL);
	sc = &m->scene;
	sc->camera.orientation = vec3_unit(sc->camera.orientation);
	for (int i = 0; i < sc->el_amount; i++)
	{
		void	*o = sc->elements[i].object;

		if (sc->elements[i].type == SPHERE)
			set_values_sphere(o);
		else if (sc->elements[i].type == CYLINDER)
			set_values_cylinder(o);
		else if (sc->elements[i].type == PLANE)
			set_values_plane(o);
		else if (sc->elements[i].type == LIGHT)
			set_values_light(o);
		else if (sc->elements[i].type == CONE)
			set_values_cone(o);
		else if (sc->elements[i].type == HYPERBOLOID)
			set_values_hyperboloid(o);
		else if (sc->elements[i].type == CUSTOM)
			set_values_custom(o);
		else if (sc->elements[i].type == DIRECTIONAL_LIGHT)
			set_values_directional_light(o);
	}
	for (int i = 0; i < sc->mat_amount; i++)
		set_values_mat(&sc->materials[i]);
	if ((!sc->amb_light.skybox_t || sc->amb_light.skybox_t->type != HDR)
		&& sc->amb_light.ratio < 0)
		sc->amb_light.ratio = 0;
	if (sc->camera.focus_dist == 0)
		sc->camera.focus_dist = 1;
	m->controls.values.fov = sc->camera.fov;
	sc->render_width = width;
	sc->render_height = height;
	sc->win_width = width;
	sc->win_height = height;
	sc->build_bvh = 1;
	m->options.no_display = 1;
	m->controls.max_bounces = max_bounces;
	h->max_bounces = max_bounces;
	m->render_mode = 0;
	m->screen.float_render = calloc((size_t)width * height, sizeof(t_fcolor));
	m->viewport = init_viewport(m);
	return (h);
}

void	refh_destroy(void *hv)
{
	t_refh	*h;

	h = hv;
	if (!h)
		return ;
	/* The oracle is short-lived test infrastructure: the scene graph is
	 * released with the process; only the large buffers are freed here. */
	free(h->m->screen.float_render);
	free(h->m->viewport.depth_buffer);
	for (int g = 0; g < h->n_groups; g++)
	{
		free(h->groups[g].obj->triangles);
		free(h->groups[g].obj->obj_list);
		free(h->groups[g].flat_tri);
		free(h->groups[g].obj);
	}
	free(h->groups);
	free(h->sky_pixels);
	free(h->elem_flat);
	free(h->m->scene.bvh.obj_list);
	free(h->m->scene.bvh.bvh_nodes);
	free(h->m->scene.bvh.prim_indices);
	free(h->m);
	free(h);
}

static int	flat_prim_of(t_refh *h, t_object *obj)
{
	t_scene	*sc;

	if (!obj)
		return (-1);
	sc = &h->m->scene;
	if (obj >= sc->elements && obj < sc->elements + sc->el_amount)
		return (h->elem_flat[obj - sc->elements]);
	for (int g = 0; g < h->n_groups; g++)
	{
		t_custom_object *o = h->groups[g].obj;
		if (obj >= o->obj_list && obj < o->obj_list + o->triangle_count)
			return (h->groups[g].flat_tri[obj - o->obj_list]);
	}
	return (-2);
}

typedef struct s_refh_hit
{
	int32_t	prim;
	int32_t	front_face;
	int32_t	depth;
	int32_t	pad_;
	double	t;
	double	u;
	double	v;
	double	point[3];
	double	normal[3];
	double	color[3];
}	t_refh_hit;

/* hit_register_all on each ray (hit_register.c:109). */
int	refh_first_hit(void *hv, const mrt_ray *rays, int64_t n, t_refh_hit *out)
{
	t_refh				*h;
	t_hit_register_data	data;
	t_ray				ray;

	h = hv;
	for (int64_t i = 0; i < n; i++)
	{
		ft_bzero(&data, sizeof(data));
		ray.orig = v3(rays[i].orig);
		ray.dir = v3(rays[i].dir);
		data.ray = &ray;
		memset(&out[i], 0, sizeof(out[i]));
		if (hit_register_all(h->m, &data) == 1)
		{
			out[i].prim = flat_prim_of(h, data.hit_record.obj);
			out[i].front_face = data.hit_record.front_face;
			out[i].t = data.hit_record.t;
			out[i].u = data.hit_record.u;
			out[i].v = data.hit_record.v;
			out[i].point[0] = data.hit_record.point.x;
			out[i].point[1] = data.hit_record.point.y;
			out[i].point[2] = data.hit_record.point.z;
			out[i].normal[0] = data.hit_record.normal.x;
			out[i].normal[1] = data.hit_record.normal.y;
			out[i].normal[2] = data.hit_record.normal.z;
			out[i].color[0] = data.hit_record.color.r;
			out[i].color[1] = data.hit_record.color.g;
			out[i].color[2] = data.hit_record.color.b;
		}
		else
			out[i].prim = -1;
		out[i].depth = data.depth;
	}
	return (0);
}

/* One ray through path_trace (path_trace.c:50) with the current RNG state. */
int	refh_path_trace(void *hv, const mrt_ray *ray, int max_depth, double *rgb)
{
	t_refh		*h;
	t_ray		r;
	t_fcolor	c;

	h = hv;
	r.orig = v3(ray->orig);
	r.dir = v3(ray->dir);
	c = path_trace(h->m, r, max_depth);
	rgb[0] = c.r;
	rgb[1] = c.g;
	rgb[2] = c.b;
	return (0);
}

/* spp samples of the full frame like render_cpu/draw_pixels
 * (render.c:28-36,86-102): offset = vec3_random() per sample, then
 * calc_one_sample. Accumulates into the harness's float_render. If offsets is
 * non-NULL the offsets used are written there (3 doubles per sample). */
int	refh_render(void *hv, int spp, double *offsets)
{
	t_refh	*h;
	t_vec3	off;

	h = hv;
	for (int s = 0; s < spp; s++)
	{
		off = vec3_random();
		if (offsets)
		{
			offsets[3 * s] = off.x;
			offsets[3 * s + 1] = off.y;
			offsets[3 * s + 2] = off.z;
		}
		calc_one_sample(h->m, off, h->max_bounces);
		h->m->screen.sample++;
	}
	return (0);
}

/* Pixel-subset render: for each sample one shared offset, then
 * calc_one_sample_task (calc_sample.c:44) on each listed pixel. */
int	refh_render_pixels(void *hv, const int32_t *pix, int64_t n, int spp)
{
	t_refh	*h;
	t_vec3	off;

	h = hv;
	for (int s = 0; s < spp; s++)
	{
		off = vec3_random();
		for (int64_t i = 0; i < n; i++)
			calc_one_sample_task(h->m, off, (t_uint)pix[i], h->max_bounces);
	}
	return (0);
}

int	refh_set_render_mode(void *hv, int mode)
{
	((t_refh *)hv)->m->render_mode = (char)mode;
	return (0);
}

double	*refh_float_render(void *hv)
{
	return ((double *)((t_refh *)hv)->m->screen.float_render);
}

int	*refh_depth_buffer(void *hv)
{
	return (((t_refh *)hv)->m->viewport.depth_buffer);
}

void	refh_clear(void *hv)
{
	t_refh	*h;

	h = hv;
	memset(h->m->screen.float_render, 0, sizeof(t_fcolor)
		* (size_t)h->m->viewport.render_w * h->m->viewport.render_h);
	h->m->screen.sample = 0;
}

/* Viewport as computed by init_viewport (viewport.c:38-87): 3 doubles each of
 * pixel00_loc, pixel_delta_u, pixel_delta_v, camera position. */
void	refh_viewport(void *hv, double *out)
{
	t_viewport	*vp;
	t_vec3		*cam;

	vp = &((t_refh *)hv)->m->viewport;
	cam = &((t_refh *)hv)->m->scene.camera.position;
	out[0] = vp->pixel00_loc.x;
	out[1] = vp->pixel00_loc.y;
	out[2] = vp->pixel00_loc.z;
	out[3] = vp->pixel_delta_u.x;
	out[4] = vp->pixel_delta_u.y;
	out[5] = vp->pixel_delta_u.z;
	out[6] = vp->pixel_delta_v.x;
	out[7] = vp->pixel_delta_v.y;
	out[8] = vp->pixel_delta_v.z;
	out[9] = cam->x;
	out[10] = cam->y;
	out[11] = cam->z;
}

/* Triangle vertex positions after init_bvh's ft_update_obj_position
 * (obj_parser_utils.c:48): 9 doubles per flat triangle. */
int	refh_triangle_positions(void *hv, double *out)
{
	t_refh	*h;

	h = hv;
	for (int g = 0; g < h->n_groups; g++)
	{
		t_custom_object *o = h->groups[g].obj;
		for (size_t k = 0; k < o->triangle_count; k++)
		{
			double *p = out + 9 * (size_t)(h->groups[g].flat_tri[k] - h->tri_base);
			t_triangle *t = &o->triangles[k];
			p[0] = t->v0.pos.x; p[1] = t->v0.pos.y; p[2] = t->v0.pos.z;
			p[3] = t->v1.pos.x; p[4] = t->v1.pos.y; p[5] = t->v1.pos.z;
			p[6] = t->v2.pos.x; p[7] = t->v2.pos.y; p[8] = t->v2.pos.z;
		}
	}
	return (h->n_tris);
}

/* BVH as built by the reference (bvh_build.c:104): node count, then per node
 * 6 doubles of bounds and 5 uint32 (left, right, first_prim, prim_count,
 * is_leaf), and the prim_indices permutation mapped to flat prim ids. */
int	refh_bvh(void *hv, double *bounds, uint32_t *info, int32_t *prim_flat)
{
	t_refh	*h;
	t_bvh	*b;

	h = hv;
	b = &h->m->scene.bvh;
	if (!b->valid)
		return (0);
	for (uint32_t i = 0; bounds && i < b->bvh_nodes_used; i++)
	{
		t_bvh_node *nd = &b->bvh_nodes[i];
		bounds[6 * i] = nd->node_bounds.min.x;
		bounds[6 * i + 1] = nd->node_bounds.min.y;
		bounds[6 * i + 2] = nd->node_bounds.min.z;
		bounds[6 * i + 3] = nd->node_bounds.max.x;
		bounds[6 * i + 4] = nd->node_bounds.max.y;
		bounds[6 * i + 5] = nd->node_bounds.max.z;
		info[5 * i] = nd->left_child;
		info[5 * i + 1] = nd->right_child;
		info[5 * i + 2] = nd->first_prim;
		info[5 * i + 3] = nd->prim_count;
		info[5 * i + 4] = nd->is_leaf;
	}
	for (uint32_t i = 0; prim_flat && i < b->size; i++)
		prim_flat[i] = flat_prim_of(h, b->obj_list[b->prim_indices[i]]);
	return ((int)b->bvh_nodes_used);
}

/* The BVH's object list before the build sorts it (bvh_make_lst.c:52): per
 * entry i, the flat id of its primitive and the position the median split
 * sorts by (get_obj_position, bvh_utils.c:88). Returns the entry count. */
int	refh_object_list(void *hv, int32_t *flat, double *pos)
{
	t_refh	*h;
	t_bvh	*b;

	h = hv;
	b = &h->m->scene.bvh;
	if (!b->valid)
		return (0);
	for (uint32_t i = 0; i < b->size; i++)
	{
		t_vec3	p = get_obj_position(i, b);

		flat[i] = flat_prim_of(h, b->obj_list[i]);
		pos[3 * i] = p.x;
		pos[3 * i + 1] = p.y;
		pos[3 * i + 2] = p.z;
	}
	return ((int)b->size);
}

/* HDRI tables (t_amb_light fields). Returns 0 if the scene has none. */
int	refh_env_tables(void *hv, float *pdf_joint, float *cdf_m_inv,
	float *cdf_c_inv, double *column_average)
{
	t_amb_light	*a;
	size_t		w;
	size_t		hh;

	a = &((t_refh *)hv)->m->scene.amb_light;
	if (!a->pdf_joint || !a->skybox_t)
		return (0);
	w = a->skybox_t->hdr.width;
	hh = a->skybox_t->hdr.height;
	if (pdf_joint)
		memcpy(pdf_joint, a->pdf_joint, w * hh * sizeof(float));
	if (cdf_m_inv)
		memcpy(cdf_m_inv, a->cdf_marginal_inverse, hh * sizeof(float));
	if (cdf_c_inv)
		memcpy(cdf_c_inv, a->cdf_conditional_inverse, w * hh * sizeof(float));
	if (column_average)
		*column_average = a->column_average;
	return (1);
}

/* Calls calc_inverse_transform_sampling_uv/dir (get_dir.c:15,29) n times. */
int	refh_env_sample(void *hv, int64_t n, double *uv, double *dir)
{
	t_refh	*h;
	t_vec2	s;
	t_vec3	d;

	h = hv;
	for (int64_t i = 0; i < n; i++)
	{
		s = calc_inverse_transform_sampling_uv(&h->m->scene);
		d = calc_inverse_transform_sampling_dir(&s);
		uv[2 * i] = s.x;
		uv[2 * i + 1] = s.y;
		dir[3 * i] = d.x;
		dir[3 * i + 1] = d.y;
		dir[3 * i + 2] = d.z;
	}
	return (0);
}

/* Sky radiance for directions (get_background_color[_clamp], background.c:62,72). */
int	refh_background(void *hv, const double *dirs, int64_t n, int clamp,
	double *rgb)
{
	t_refh		*h;
	t_ray		r;
	t_fcolor	c;

	h = hv;
	for (int64_t i = 0; i < n; i++)
	{
		r.orig = (t_vec3){0, 0, 0};
		r.dir = v3(dirs + 3 * i);
		c = clamp ? get_background_color_clamp(h->m, r)
			: get_background_color(h->m, r);
		rgb[3 * i] = c.r;
		rgb[3 * i + 1] = c.g;
		rgb[3 * i + 2] = c.b;
	}
	return (0);
}

/* Photon map: photons stored in the kd-tree array (kd_tree_build.c:85-94). */
int64_t	refh_photon_count(void *hv)
{
	return ((int64_t)((t_refh *)hv)->m->scene.photon_map.photon_count);
}

int	refh_photons(void *hv, double *pos3, double *pow3, int32_t *in_leaf)
{
	t_kd_tree	*k;

	k = &((t_refh *)hv)->m->scene.photon_map;
	for (size_t i = 0; i < k->photon_count; i++)
	{
		pos3[3 * i] = k->photons[i].position.x;
		pos3[3 * i + 1] = k->photons[i].position.y;
		pos3[3 * i + 2] = k->photons[i].position.z;
		pow3[3 * i] = k->photons[i].power.r;
		pow3[3 * i + 1] = k->photons[i].power.g;
		pow3[3 * i + 2] = k->photons[i].power.b;
	}
	if (in_leaf)
	{
		memset(in_leaf, 0, sizeof(int32_t) * k->photon_count);
		for (size_t n = 0; n < k->node_count; n++)
		{
			if (k->nodes[n].axis != -1)
				continue ;
			for (int j = 0; j < k->nodes[n].u_data.t_leaf.photon_count; j++)
				in_leaf[k->nodes[n].u_data.t_leaf.photon_start_idx + j] = 1;
		}
	}
	return (0);
}

/* estimate_caustics_physically_based (get_caustic.c:67) at query points. */
int	refh_caustic_query(void *hv, const double *pts, int64_t n, int k,
	double *rgb)
{
	t_refh		*h;
	t_fcolor	c;

	h = hv;
	for (int64_t i = 0; i < n; i++)
	{
		c = estimate_caustics_physically_based(&h->m->scene.photon_map,
				v3(pts + 3 * i), k, h->m);
		rgb[3 * i] = c.r;
		rgb[3 * i + 1] = c.g;
		rgb[3 * i + 2] = c.b;
	}
	return (0);
}

/* Accessors for driving the miniRT drop-in adapter on the harness's own
 * t_minirt (tests call the adapter's entry points with these pointers). */
void	*refh_minirt(void *hv)
{
	return (((t_refh *)hv)->m);
}

void	*refh_scene_ptr(void *hv)
{
	return (&((t_refh *)hv)->m->scene);
}

void	*refh_viewport_ptr(void *hv)
{
	return (&((t_refh *)hv)->m->viewport);
}

void	*refh_shader_data(void *hv)
{
	return (&((t_refh *)hv)->m->shaders_data);
}

void	*refh_gpu_structs(void *hv)
{
	return (&((t_refh *)hv)->m->shaders_data.scene);
}

int	refh_sample_counters(void *hv, int *out3)
{
	t_minirt	*m;

	m = ((t_refh *)hv)->m;
	out3[0] = m->screen.sample;
	out3[1] = m->screen.sample_total_anim;
	out3[2] = m->screen.last_sample_am;
	return (0);
}

int	refh_gpu_counts(void *hv, int *out6)
{
	t_gpu_structs	*g;

	g = &((t_refh *)hv)->m->shaders_data.scene;
	out6[0] = g->valid;
	out6[1] = g->spheres_am;
	out6[2] = g->planes_am;
	out6[3] = g->triangles_am;
	out6[4] = g->lights_am;
	out6[5] = g->mat_am;
	return (0);
}

/* The reference's own calc_one_sample with an explicit offset. */
void	refh_calc_one_sample(void *hv, double ox, double oy, int max_bounces)
{
	calc_one_sample(((t_refh *)hv)->m, (t_vec3){ox, oy, 0}, max_bounces);
}
