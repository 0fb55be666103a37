/*
 * Minimal stand-in for miniRT's libft.h (the libft git submodule of miniRT is
 * not vendored here). It declares the types and functions miniRT's headers
 * and its path-tracing sources need, so that the drop-in adapter
 * (minirt_gpu.c) and the test oracle can be compiled headless. A project that
 * has the real libft compiles against that instead; the adapter itself calls
 * no libft function. Implementations for the oracle build live in
 * oracle/shim/libft_shim.c.
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

/* string / number / file helpers of the scene parser (src/parsing, src/utils
 * loaders); restated in oracle/shim/libft_parse_shim.c */
int		ft_strcmp(const char *a, const char *b);
int		ft_strncmp(const char *a, const char *b, size_t n);
size_t	ft_strlen(const char *s);
ssize_t	ft_sstrlen(const char *s);
char	*ft_strchr(const char *s, int c);
char	*ft_strrchr(const char *s, int c);
char	*ft_strnstr(const char *h, const char *n, size_t len);
char	*ft_strdup(const char *s);
int		ft_isdigit(int c);
int		ft_isalpha(int c);
int		ft_isalnum(int c);
int		ft_atoi(const char *s);
int		ft_abs(int x);
double	ft_atod(const char *s);
float	ft_atof(const char *s);
int		is_valid_float(const char *s);
char	**ft_split_in_line(char *s, const char *set);
void	ft_free_tab_null_term(char **tab);
char	*get_next_line(int fd);
int		read_bin_file(t_bin *bin, const char *path);
int		read_uint8_move(t_bin *bin, size_t *i, uint8_t *out);
int		read_uint16_move(t_bin *bin, size_t *i, uint16_t *out);
int		read_uint16_move_little(t_bin *bin, size_t *i, uint16_t *out);
int		read_uint32_move(t_bin *bin, size_t *i, uint32_t *out);
int		read_uint32_move_little(t_bin *bin, size_t *i, uint32_t *out);
int		read_uint64_move_little(t_bin *bin, size_t *i, uint64_t *out);

#endif
