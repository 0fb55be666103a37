/* Empty stand-in for minilibx's mlx.h for headless builds: miniRT's headers
 * include it, the path-tracing code and the adapter call nothing from it. */
#ifndef MLX_H
# define MLX_H
#endif
