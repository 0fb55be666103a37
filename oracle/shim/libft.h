/*
 * Minimal stand-in for the miniRT project's libft interface (the libft git
 * submodule of the reference is not vendored). Test infrastructure only: it
 * lets the reference's own CPU path (src/ray_tracing, src/material,
 * src/caustic, src/math) compile into the oracle library. Only the types and
 * functions that path uses are declared; the implementations are in
 * libft_shim.c and follow the libft contracts the reference relies on
 * (ft_calloc zeroes, vector_add grows and returns -1 on failure, ...).
 */
#ifndef LIBFT_H
# define LIBFT_H

# include <stddef.h>
# include <stdint.h>
# include <stdlib.h>
# include <unistd.h>
# include <sys/types.h>

/* terminal colour codes used by print_error / print_warn */
# define RED "\033[0;31m"
# define GREEN "\033[0;32m"
# define YELLOW "\033[0;33m"
# define BLUE "\033[0;34m"
# define NC "\033[0m"

typedef unsigned int	t_uint;
typedef unsigned char	t_uchar;
typedef char			t_bool;

typedef struct s_bin
{
	unsigned char	*data;
	size_t			size;
}	t_bin;

/* growable array: vector_init / vector_add / at_vector (bvh_build.c:76-86,
 * caustic_manager.c:57-58, kd_tree_build.c) */
typedef struct s_vector
{
	void	*data;
	size_t	element_size;
	size_t	num_elements;
	size_t	capacity;
}	t_vector;

int		vector_init(t_vector *v, size_t element_size, size_t capacity);
int		vector_add(t_vector *v, void *element);
void	*at_vector(t_vector *v, size_t index);

void	*ft_calloc(size_t nmemb, size_t size);
void	ft_bzero(void *s, size_t n);
void	*ft_memcpy(void *dst, const void *src, size_t n);
size_t	ft_strlcpy(char *dst, const char *src, size_t size);
int		ft_printf(const char *fmt, ...);
int		ft_dprintf(int fd, const char *fmt, ...);
char	*ft_sprintf(const char *fmt, ...);
ssize_t	get_cpu_time(void);

#endif
