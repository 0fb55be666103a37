/*
 * Drop-in replacement for miniRT's includes/gpu_scene.h.
 *
 * The reference's t_gpu_structs (includes/gpu_scene.h:209-253) is a host-side
 * staging area of std430 arrays plus GL buffer ids. The CUDA library keeps its
 * device arrays inside its own context, so here t_gpu_structs only records
 * what was uploaded (counts and bytes) for callers that print or inspect it.
 * Field names follow the reference where the meaning is the same.
 */
#ifndef GPU_SCENE_H
# define GPU_SCENE_H

# include <stddef.h>
# include <stdint.h>
# include "scene_structs.h"

typedef struct s_gpu_structs
{
	int			valid;			/* 1 after a successful convert_scene_build */
	int			mat_am;
	int			spheres_am;
	int			planes_am;
	int			triangles_am;
	int			lights_am;
	int			bvh_node_am;
	uint32_t	photon_am;
	size_t		device_bytes;	/* scene bytes resident in device memory */
}	t_gpu_structs;

typedef struct s_gpu_textures
{
	int		hdr_width;
	int		hdr_height;
}	t_gpu_textures;

#endif
