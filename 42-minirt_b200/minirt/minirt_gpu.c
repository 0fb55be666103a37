/*
 * minirt_gpu.c — miniRT's GPU render entry points over the CUDA library.
 *
 * Drop-in replacement for the OpenGL implementations in miniRT's src/gpu
 * (init_shader.c, gpu_scene.c, use_shader.c, clean_shaders.c,
 * send_uniforms.c, importance_sampling.c) and for the CPU sample loop
 * calc_one_sample (src/ray_tracing/calc_sample.c:73). Compiled against
 * miniRT's own headers, with include/minirt_compat/gpu*.h in place of its GL
 * bridge headers; linked against libmrt.so instead of -lGL -lGLEW -lglfw.
 * Same names, arguments, return values and side effects as the reference:
 *   - int functions return 0 / -1 and print an "[Error]" line on failure;
 *   - compute_frame_gpu adds one sample per pixel into
 *     minirt->screen.float_render (or the BVH heat map into
 *     viewport.depth_buffer in render_mode 1) and on success bumps
 *     screen.sample, sample_total_anim and last_sample_am (use_shader.c:96-98);
 *   - calc_one_sample adds one sample with the caller's shared offset and
 *     leaves the counters to the caller (render.c:33-37).
 * The scene is read from t_scene after init_viewport, i.e. with the BVH
 * list built and custom-object vertices already re-transformed
 * (bvh_make_lst.c:34), and copied: no pointer into t_scene is kept.
 */
#include "minirt.h"
#include "gpu.h"
#include "mrt.h"
#include <stdio.h>
#include <string.h>

/* gpu_bvh_sah(1): build this library's SAH tree instead of the
 * reference's (faster on large meshes; exact-t ties may then resolve to
 * another of the tied primitives). render_mode 1 always uses the
 * reference's tree. */
static int	g_sah_bvh = 0;

void	gpu_bvh_sah(int on)
{
	g_sah_bvh = on != 0;
}

static void	err_line(const char *what)
{
	fprintf(stderr, "\033[0;31m[Error]\033[0m %s: %s\n", what, mrt_last_error());
}

/* init_shader (init_shader.c:133): device context + W*H accumulator. */
int	init_shader(t_shader_data *sd, size_t w, size_t h, t_scene *scene)
{
	(void)scene;
	memset(sd, 0, sizeof(*sd));
	sd->ctx = mrt_create(0, (int)w, (int)h);
	if (!sd->ctx)
	{
		err_line("init_shader");
		return (-1);
	}
	sd->render_width = w;
	sd->render_height = h;
	return (0);
}

typedef struct s_flat
{
	mrt_scene_desc	d;
	mrt_material	*mats;
	mrt_sphere		*sph;
	mrt_plane		*pl;
	mrt_light		*li;
	mrt_mesh		*me;
	mrt_cylinder	*cy;
	mrt_cone		*co;
	mrt_hyperboloid	*hy;
	mrt_texture		*tx;
	double			**buf;
	int				nbuf;
}	t_flat;

static int	mat_index(t_scene *s, t_mat *m)
{
	if (!m || m < s->materials || m >= s->materials + s->mat_amount)
		return (-1);
	return ((int)(m - s->materials));
}

/* 1 + the index of t in the scene's t_tex array, 0 for none */
static int	tex_index(t_scene *s, t_tex *t)
{
	if (!t || t < s->textures || t >= s->textures + s->tex_amount)
		return (0);
	return ((int)(t - s->textures) + 1);
}

static void	c3(uint8_t *o, t_color c)
{
	o[0] = c.r;
	o[1] = c.g;
	o[2] = c.b;
}

static void	v3(double *o, t_vec3 v)
{
	o[0] = v.x;
	o[1] = v.y;
	o[2] = v.z;
}

static void	free_flat(t_flat *f)
{
	for (int i = 0; i < f->nbuf; i++)
		free(f->buf[i]);
	free(f->buf);
	free(f->mats);
	free(f->sph);
	free(f->pl);
	free(f->li);
	free(f->me);
	free(f->cy);
	free(f->co);
	free(f->hy);
	free(f->tx);
}

/* t_custom_object triangles (after ft_update_obj_position) -> a
 * non-indexed mesh; bvh_make_lst gives every triangle its object's material
 * (bvh_make_lst.c:16-27). */
static int	add_custom(t_flat *f, t_scene *s, t_custom_object *o, mrt_mesh *m)
{
	size_t	n = o->triangle_count;
	double	*pos = malloc(sizeof(double) * 9 * (n ? n : 1));
	double	*nrm = malloc(sizeof(double) * 9 * (n ? n : 1));
	double	*uv = malloc(sizeof(double) * 6 * (n ? n : 1));

	if (!pos || !nrm || !uv)
		return (free(pos), free(nrm), free(uv), -1);
	f->buf[f->nbuf++] = pos;
	f->buf[f->nbuf++] = nrm;
	f->buf[f->nbuf++] = uv;
	for (size_t t = 0; t < n; t++)
	{
		t_vertex	*vs[3] = {&o->triangles[t].v0, &o->triangles[t].v1,
			&o->triangles[t].v2};

		for (int c = 0; c < 3; c++)
		{
			v3(pos + 9 * t + 3 * c, vs[c]->pos);
			v3(nrm + 9 * t + 3 * c, vs[c]->normal);
			uv[6 * t + 2 * c] = vs[c]->u;
			uv[6 * t + 2 * c + 1] = vs[c]->v;
		}
	}
	memset(m, 0, sizeof(*m));
	m->n_vertices = (uint32_t)(3 * n);
	m->n_triangles = (uint32_t)n;
	m->positions = pos;
	m->normals = nrm;
	m->uvs = uv;
	m->material = mat_index(s, o->material);
	c3(m->color, o->color);
	return (0);
}

static int	flatten(t_minirt *mrt, t_scene *s, t_flat *f)
{
	int	ns = 0, np = 0, nl = 0, nm = 0, nc = 0, nk = 0, nh = 0;

	memset(f, 0, sizeof(*f));
	for (int i = 0; i < s->el_amount; i++)
	{
		t_objects	ty = s->elements[i].type;

		ns += ty == SPHERE;
		np += ty == PLANE;
		nl += ty == LIGHT || ty == DIRECTIONAL_LIGHT;
		nm += ty == CUSTOM;
		nc += ty == CYLINDER;
		nk += ty == CONE;
		nh += ty == HYPERBOLOID;
	}
	f->mats = calloc(s->mat_amount + 1, sizeof(mrt_material));
	f->sph = calloc(ns + 1, sizeof(mrt_sphere));
	f->pl = calloc(np + 1, sizeof(mrt_plane));
	f->li = calloc(nl + 1, sizeof(mrt_light));
	f->me = calloc(nm + 1, sizeof(mrt_mesh));
	f->tx = calloc(s->tex_amount + 1, sizeof(mrt_texture));
	f->cy = calloc(nc + 1, sizeof(mrt_cylinder));
	f->co = calloc(nk + 1, sizeof(mrt_cone));
	f->hy = calloc(nh + 1, sizeof(mrt_hyperboloid));
	f->buf = calloc(3 * nm + 1, sizeof(double *));
	if (!f->mats || !f->sph || !f->pl || !f->li || !f->me || !f->buf
		|| !f->cy || !f->co || !f->hy || !f->tx)
		return (-1);
	for (int i = 0; i < s->tex_amount; i++)
	{
		t_tex		*t = &s->textures[i];
		mrt_texture	*o = &f->tx[i];

		o->type = (int32_t)t->type;
		if (t->img.rgba && t->img.width && t->img.height)
		{
			o->rgba = (const uint8_t *)t->img.rgba;
			o->width = t->img.width;
			o->height = t->img.height;
		}
		o->checker_scale = t->checker.scale;
		c3(o->c1, t->checker.c1);
		c3(o->c2, t->checker.c2);
	}
	for (int i = 0; i < s->mat_amount; i++)
	{
		t_mat			*m = &s->materials[i];
		mrt_material	*o = &f->mats[i];

		c3(o->color, m->color_value);
		c3(o->emission_color, m->emission_color_tmp);
		o->metallic = m->metallic_value;
		o->roughness = m->roughness_value;
		o->ior = m->ior;
		o->transmission = m->transmission_value;
		o->ao = m->ao_value;
		o->emission_strength = m->emission_strength;
		o->scale = m->scale;
		o->color_tex = tex_index(s, m->color_tex);
		o->metallic_tex = tex_index(s, m->metallic_tex);
		o->roughness_tex = tex_index(s, m->roughness_tex);
		o->transmission_tex = tex_index(s, m->transmission_tex);
		o->ao_tex = tex_index(s, m->ao_tex);
		o->emission_strength_tex = tex_index(s, m->emission_strength_tex);
		o->emission_color_tex = tex_index(s, m->emission_color_tex);
		o->normal_tex = tex_index(s, m->normal);
		o->normal_intensity = m->normal_intensity;
	}
	ns = np = nl = nm = nc = nk = nh = 0;
	for (int i = 0; i < s->el_amount; i++)
	{
		void	*ob = s->elements[i].object;

		if (s->elements[i].type == SPHERE)
		{
			t_sphere	*sp = ob;

			v3(f->sph[ns].center, sp->position);
			f->sph[ns].radius = sp->radius;
			f->sph[ns].material = mat_index(s, sp->material);
			c3(f->sph[ns++].color, sp->color);
		}
		else if (s->elements[i].type == PLANE)
		{
			t_plane	*p = ob;

			v3(f->pl[np].point, p->position);
			v3(f->pl[np].normal, p->normal);
			f->pl[np].material = mat_index(s, p->material);
			c3(f->pl[np++].color, p->color);
		}
		else if (s->elements[i].type == LIGHT)
		{
			t_light	*l = ob;

			f->li[nl].type = MRT_LIGHT_POINT;
			v3(f->li[nl].position, l->position);
			f->li[nl].brightness = l->brightness;
			f->li[nl].radius = l->radius;
			f->li[nl].shadow_sample = l->shadow_sample;
			c3(f->li[nl++].color, l->color);
		}
		else if (s->elements[i].type == DIRECTIONAL_LIGHT)
		{
			t_dlight	*l = ob;

			f->li[nl].type = MRT_LIGHT_DIRECTIONAL;
			v3(f->li[nl].position, l->orientation);
			f->li[nl].brightness = l->brightness;
			c3(f->li[nl++].color, l->color);
		}
		else if (s->elements[i].type == CYLINDER)
		{
			t_cylinder	*c = ob;

			v3(f->cy[nc].position, c->position);
			v3(f->cy[nc].orientation, c->orientation);
			f->cy[nc].diameter = c->diameter;
			f->cy[nc].height = c->height;
			f->cy[nc].material = mat_index(s, c->material);
			f->cy[nc].material_top = mat_index(s, c->material_top);
			f->cy[nc].material_bot = mat_index(s, c->material_bot);
			c3(f->cy[nc++].color, c->color);
		}
		else if (s->elements[i].type == CONE)
		{
			t_cone	*c = ob;

			v3(f->co[nk].position, c->position);
			v3(f->co[nk].orientation, c->orientation);
			f->co[nk].diameter = c->diameter;
			f->co[nk].height = c->height;
			f->co[nk].material = mat_index(s, c->material);
			f->co[nk].material_top = mat_index(s, c->material_top);
			c3(f->co[nk++].color, c->color);
		}
		else if (s->elements[i].type == HYPERBOLOID)
		{
			t_hyperboloid	*c = ob;

			v3(f->hy[nh].position, c->position);
			v3(f->hy[nh].orientation, c->orientation);
			f->hy[nh].a = c->a;
			f->hy[nh].b = c->b;
			f->hy[nh].c = c->c;
			f->hy[nh].shape = c->shape;
			f->hy[nh].height = c->height;
			f->hy[nh].material = mat_index(s, c->material);
			c3(f->hy[nh++].color, c->color);
		}
		else if (s->elements[i].type == CUSTOM)
		{
			if (add_custom(f, s, ob, &f->me[nm++]))
				return (-1);
		}
	}
	f->d.abi_version = MRT_ABI_VERSION;
	f->d.render_width = s->render_width;
	f->d.render_height = s->render_height;
	f->d.max_bounces = (int)mrt->controls.max_bounces;
	f->d.triangle_one_sided = mrt->options.triangle_one_sided;
	f->d.ior_all = s->ior_all;
	v3(f->d.camera.position, s->camera.position);
	v3(f->d.camera.orientation, s->camera.orientation);
	f->d.camera.fov = s->camera.fov;
	f->d.camera.focus_dist = s->camera.focus_dist;
	f->d.camera.defocus_angle = s->camera.defocus_angle;
	f->d.ambient.ratio = s->amb_light.ratio;
	c3(f->d.ambient.color, s->amb_light.skybox_c);
	if (s->amb_light.skybox_t && s->amb_light.skybox_t->type == HDR
		&& s->amb_light.skybox_t->hdr.pixels)
	{
		t_hdr	*h = &s->amb_light.skybox_t->hdr;

		f->d.ambient.hdr_rgbe = (const uint8_t *)h->pixels;
		f->d.ambient.hdr_width = h->width;
		f->d.ambient.hdr_height = h->height;
		f->d.ambient.hdr_exposure = h->exposure;
		f->d.ambient.hdr_gamma = h->gamma;
	}
	if (mrt->options.caustic.caustic_enable)
	{
		f->d.caustic.enable = 1;
		f->d.caustic.passes = 1;
		f->d.caustic.photons_per_light = mrt->options.caustic.nb_photon;
		f->d.caustic.radius = mrt->options.caustic.caustic_radius;
		f->d.caustic.norm_factor = mrt->options.caustic.norm_factor;
		f->d.caustic.knn = 15;
	}
	f->d.materials = f->mats;
	f->d.n_materials = s->mat_amount;
	f->d.spheres = f->sph;
	f->d.n_spheres = ns;
	f->d.planes = f->pl;
	f->d.n_planes = np;
	f->d.lights = f->li;
	f->d.n_lights = nl;
	f->d.meshes = f->me;
	f->d.n_meshes = nm;
	f->d.cylinders = f->cy;
	f->d.n_cylinders = nc;
	f->d.cones = f->co;
	f->d.n_cones = nk;
	f->d.hyperboloids = f->hy;
	f->d.n_hyperboloids = nh;
	f->d.textures = f->tx;
	f->d.n_textures = s->tex_amount;
	return (0);
}

/* The reference's BVH object list (bvh_make_lst.c:52-69) as flat
 * primitive ids (spheres, cylinders, cones, hyperboloids, then the meshes'
 * triangles, as flatten lays them out), with the position its median split
 * sorts by (get_obj_position, bvh_utils.c:88: the object's position, or a
 * triangle's centre as its loader stored it). Selects the reference's own
 * tree for the next build, traversed left child first: the first hit
 * among primitives at exactly the same t is then the one hit_bvh keeps
 * (bvh_hit.c:31-36, the left subtree wins a tie), e.g. the coincident
 * wall faces of scenes/obj/cube.rt, and render_mode 1 reports hit_bvh's
 * visit counts (bvh_hit.c:16). */
static int	set_reference_bvh(t_minirt *mrt, t_scene *s, const t_flat *f)
{
	const int64_t	tb = f->d.n_spheres + f->d.n_cylinders + f->d.n_cones
		+ f->d.n_hyperboloids;
	int64_t			n = tb, i = 0, it = 0;
	int64_t			k4[4] = {0, f->d.n_spheres, f->d.n_spheres + f->d.n_cylinders,
		f->d.n_spheres + f->d.n_cylinders + f->d.n_cones};
	int32_t			*order;
	double			*pos;
	mrt_bvh_options	o;
	int				rc;

	for (int m = 0; m < f->d.n_meshes; m++)
		n += f->me[m].n_triangles;
	order = malloc(sizeof(int32_t) * (n ? n : 1));
	pos = malloc(sizeof(double) * 3 * (n ? n : 1));
	if (!order || !pos)
		return (free(order), free(pos), -1);
	for (int e = 0; e < s->el_amount; e++)
	{
		t_objects	ty = s->elements[e].type;
		void		*ob = s->elements[e].object;
		int64_t		id;

		if (ty == SPHERE || ty == CYLINDER || ty == CONE || ty == HYPERBOLOID)
		{
			int	kind = ty == SPHERE ? 0 : ty == CYLINDER ? 1 : ty == CONE ? 2 : 3;

			id = k4[kind]++;
			order[i++] = (int32_t)id;
			if (ty == SPHERE)
				v3(pos + 3 * id, ((t_sphere *)ob)->position);
			else if (ty == CYLINDER)
				v3(pos + 3 * id, ((t_cylinder *)ob)->position);
			else if (ty == CONE)
				v3(pos + 3 * id, ((t_cone *)ob)->position);
			else
				v3(pos + 3 * id, ((t_hyperboloid *)ob)->position);
		}
		else if (ty == CUSTOM)
		{
			t_custom_object	*c = ob;

			for (size_t k = 0; k < c->triangle_count; k++)
			{
				t_triangle	*t = c->obj_list[k].object;

				id = tb + it + (t - c->triangles);
				order[i++] = (int32_t)id;
				v3(pos + 3 * id, t->center);
			}
			it += c->triangle_count;
		}
	}
	o = (mrt_bvh_options){MRT_BVH_REFERENCE, 0, n, order, pos};
	(void)mrt;
	rc = mrt_set_bvh_options(mrt->shaders_data.ctx, &o);
	free(order);
	free(pos);
	return (rc == MRT_OK ? 0 : -1);
}

/* convert_scene_build (gpu_scene.c:104): full repack and upload. */
int	convert_scene_build(t_minirt *minirt, t_scene *scene, t_viewport *vp,
	t_gpu_structs *gpu)
{
	t_flat	f;
	int		rc;

	(void)vp;
	if (!minirt->shaders_data.ctx)
	{
		fprintf(stderr, "\033[0;31m[Error]\033[0m convert_scene_build: "
			"init_shader was not called\n");
		return (-1);
	}
	if (flatten(minirt, scene, &f))
	{
		free_flat(&f);
		return (-1);
	}
	if (!g_sah_bvh || minirt->render_mode == 1)
	{
		if (set_reference_bvh(minirt, scene, &f))
		{
			free_flat(&f);
			err_line("convert_scene_build");
			return (-1);
		}
	}
	else
	{
		mrt_bvh_options	o = {MRT_BVH_SAH, 0, 0, NULL, NULL};

		mrt_set_bvh_options(minirt->shaders_data.ctx, &o);
	}
	rc = mrt_scene_build(minirt->shaders_data.ctx, &f.d);
	if (rc == MRT_OK)
	{
		memset(gpu, 0, sizeof(*gpu));
		gpu->valid = 1;
		gpu->mat_am = f.d.n_materials;
		gpu->spheres_am = f.d.n_spheres;
		gpu->planes_am = f.d.n_planes;
		gpu->lights_am = f.d.n_lights;
		for (int i = 0; i < f.d.n_meshes; i++)
			gpu->triangles_am += (int)f.me[i].n_triangles;
		gpu->photon_am = (uint32_t)mrt_photon_count(minirt->shaders_data.ctx);
	}
	else
		err_line("convert_scene_build");
	free_flat(&f);
	return (rc == MRT_OK ? 0 : -1);
}

/* convert_scene (gpu_scene.c:62): camera / ior / ambient only. */
void	convert_scene(t_minirt *minirt, t_scene *scene, t_viewport *vp,
	t_gpu_structs *gpu)
{
	mrt_camera	cam;

	(void)vp;
	(void)gpu;
	memset(&cam, 0, sizeof(cam));
	v3(cam.position, scene->camera.position);
	v3(cam.orientation, scene->camera.orientation);
	cam.fov = scene->camera.fov;
	cam.focus_dist = scene->camera.focus_dist;
	cam.defocus_angle = scene->camera.defocus_angle;
	if (mrt_set_camera(minirt->shaders_data.ctx, &cam, scene->ior_all,
			scene->amb_light.ratio) != MRT_OK)
		err_line("convert_scene");
}

static int	one_sample(t_minirt *m, const double *offset, int max_bounces)
{
	mrt_render_params	p;
	mrt_ctx				*c = m->shaders_data.ctx;

	memset(&p, 0, sizeof(p));
	p.spp = 1;
	p.sample_base = m->screen.sample_total_anim;
	p.seed = 0x6d696e6952545f31ull;
	p.max_bounces = max_bounces;
	p.render_mode = m->render_mode;
	p.form = MRT_FORM_AUTO;
	p.offset = offset;
	if (mrt_render(c, &p, NULL) != MRT_OK)
		return (-1);
	if (m->render_mode == 1)
	{
		if (!m->viewport.depth_buffer)
			return (0);
		return (mrt_read_depth(c, m->viewport.depth_buffer) == MRT_OK ? 0 : -1);
	}
	return (mrt_accumulate_double(c, (double *)m->screen.float_render)
		== MRT_OK ? 0 : -1);
}

/* compute_frame_gpu (use_shader.c:81-100). */
void	compute_frame_gpu(t_minirt *m)
{
	if (!m->shaders_data.ctx || one_sample(m, NULL,
			(int)m->controls.max_bounces) != 0)
	{
		err_line("compute_frame_gpu");
		return ;
	}
	m->screen.sample++;
	m->screen.sample_total_anim++;
	m->screen.last_sample_am = m->screen.sample;
}

/* calc_one_sample (calc_sample.c:73): the CPU loop's contract, on the GPU.
 * The first call (and every call at sample 0, after init_viewport rebuilt
 * the scene) uploads the scene. The counters stay with the caller. */
void	calc_one_sample(t_minirt *m, t_vec3 offset, int max_bounces)
{
	double	off[2] = {offset.x, offset.y};

	if (!m->shaders_data.ctx && init_shader(&m->shaders_data,
			m->scene.render_width, m->scene.render_height, &m->scene))
		return ;
	if (m->screen.sample == 0 || !m->shaders_data.scene.valid)
	{
		if (convert_scene_build(m, &m->scene, &m->viewport,
				&m->shaders_data.scene))
			return ;
	}
	if (one_sample(m, off, max_bounces) != 0)
		err_line("calc_one_sample");
	if (m->render_mode == 1)
		set_heat_map_color(m);
}

/* set_heat_map_color (calc_sample.c:16-42): the adapter replaces
 * calc_sample.c, so it also provides its other export (render_gpu.c:27 calls
 * it after compute_frame_gpu in render_mode 1). */
void	set_heat_map_color(t_minirt *minirt)
{
	const size_t	tpi = (size_t)minirt->viewport.render_w
		* minirt->viewport.render_h;
	int				mx;

	if (!minirt->viewport.depth_buffer)
		return ;
	mx = 0;
	for (size_t i = 0; i < tpi; i++)
		if (mx < minirt->viewport.depth_buffer[i])
			mx = minirt->viewport.depth_buffer[i];
	for (size_t i = 0; i < tpi; i++)
		if (minirt->viewport.depth_buffer[i] >= 0)
			minirt->screen.float_render[i] = add_fcolor(
					minirt->screen.float_render[i],
					get_heatmap_fcolor(minirt->viewport.depth_buffer[i], mx));
}

/* clean_shaders / clean_scene (clean_shaders.c:69,32). */
void	clean_shaders(t_shader_data *sd)
{
	mrt_destroy(sd->ctx);
	sd->ctx = NULL;
}

void	clean_scene(t_gpu_structs *gpu)
{
	memset(gpu, 0, sizeof(*gpu));
}

/* send_uniforms (send_uniforms.c:63), send_importance_sampling
 * (importance_sampling.c:69): the parameters travel with convert_scene /
 * convert_scene_build, so there is nothing left to send. */
void	send_uniforms(t_minirt *minirt)
{
	(void)minirt;
}

void	send_importance_sampling(t_minirt *minirt, t_scene *scene)
{
	(void)minirt;
	(void)scene;
}
