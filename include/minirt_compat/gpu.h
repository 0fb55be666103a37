/*
 * Drop-in replacement for miniRT's includes/gpu.h: the GPU render entry
 * points with the reference's names and signatures (includes/gpu.h:25-93),
 * implemented over the CUDA library (libmrt) instead of OpenGL compute.
 */
#ifndef GPU_H
# define GPU_H

# include <stdlib.h>
# include "gpu_struct.h"
# include "structs.h"

/* init_shader.c:133 — create the device context and the W*H frame buffer. */
int		init_shader(t_shader_data *shader_data, size_t render_width,
			size_t render_height, t_scene *scene);
/* gpu_scene.c:104 — repack and upload the whole scene (BVH, materials,
 * lights, planes, photon map, HDRI tables). 0 on success, -1 on error. */
int		convert_scene_build(t_minirt *minirt, t_scene *scene,
			t_viewport *viewport, t_gpu_structs *gpu_structs);
/* gpu_scene.c:62 — camera / viewport / ambient only. */
void	convert_scene(t_minirt *minirt, t_scene *scene,
			t_viewport *viewport, t_gpu_structs *gpu);
/* use_shader.c:81 — one sample per pixel, added into
 * minirt->screen.float_render; bumps the sample counters on success. */
void	compute_frame_gpu(t_minirt *minirt);
/* clean_shaders.c:69 / :32 */
void	clean_shaders(t_shader_data *shader_data);
void	clean_scene(t_gpu_structs *gpu_structs);
/* Not in the reference: the BVH that convert_scene_build builds. By
 * default the reference's own median-split tree (bvh_build.c:104), so that
 * exact-t ties resolve as on the CPU; gpu_bvh_sah(1) selects this
 * library's SAH tree (faster on large meshes). */
void	gpu_bvh_sah(int on);
/* send_uniforms.c:63, importance_sampling.c:69 — parameters now travel with
 * convert_scene / convert_scene_build, so these are kept as no-ops. */
void	send_uniforms(t_minirt *minirt);
void	send_importance_sampling(t_minirt *minirt, t_scene *scene);

#endif
