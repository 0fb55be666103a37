/* Empty stand-in for minilibx's mlx.h: the oracle build is headless and the
 * path-tracing sources only need the header to exist. Test infrastructure. */
#ifndef MLX_H
# define MLX_H
#endif
