/*
 * Drop-in replacement for miniRT's includes/gpu_struct.h.
 *
 * The reference's version (includes/gpu_struct.h:16-27) holds a GLFW window,
 * a GL program id and the frame SSBO id. With the CUDA library those become
 * one opaque render context; the rest of the reference's host code only
 * passes &minirt->shaders_data and &minirt->shaders_data.scene around
 * (main_shader.c:62, render_gpu.c:54-59), so recompiling it against this
 * header is all it takes. No GL, GLEW or GLFW header is needed any more.
 */
#ifndef GPU_STRUCT_H
# define GPU_STRUCT_H

# include "gpu_scene.h"

struct mrt_ctx;

typedef struct s_shader_data
{
	struct mrt_ctx	*ctx;		/* replaces window + program + ssbo */
	size_t			render_width;
	size_t			render_height;
	t_gpu_structs	scene;
	t_gpu_textures	tex;
}	t_shader_data;

#endif
