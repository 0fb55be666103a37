/*
 * Implementations of the libft subset declared in shim/libft.h, plus no-op
 * stand-ins for the UI hooks (link_float_input) that init_viewport calls
 * (viewport.c:26-35). Test infrastructure for the oracle build only.
 */
#include "libft.h"
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <time.h>

int	oracle_quiet = 1;

int	vector_init(t_vector *v, size_t element_size, size_t capacity)
{
	if (capacity == 0)
		capacity = 1;
	v->data = malloc(element_size * capacity);
	v->element_size = element_size;
	v->num_elements = 0;
	v->capacity = capacity;
	return (v->data ? 0 : -1);
}

int	vector_add(t_vector *v, void *element)
{
	void	*grown;

	if (v->num_elements == v->capacity)
	{
		grown = realloc(v->data, v->element_size * v->capacity * 2);
		if (!grown)
			return (-1);
		v->data = grown;
		v->capacity *= 2;
	}
	memcpy((char *)v->data + v->num_elements * v->element_size, element,
		v->element_size);
	v->num_elements++;
	return (0);
}

/* No check against num_elements: the BVH builder pops with
 * at_vector(v, --v->num_elements) (bvh_build.c:80-81). */
void	*at_vector(t_vector *v, size_t index)
{
	if (index >= v->capacity)
		return (NULL);
	return ((char *)v->data + index * v->element_size);
}

void	*ft_calloc(size_t nmemb, size_t size)
{
	if (nmemb == 0 || size == 0)
		return (malloc(1));
	return (calloc(nmemb, size));
}

void	ft_bzero(void *s, size_t n)
{
	memset(s, 0, n);
}

void	*ft_memcpy(void *dst, const void *src, size_t n)
{
	return (memcpy(dst, src, n));
}

size_t	ft_strlcpy(char *dst, const char *src, size_t size)
{
	size_t	len = strlen(src);

	if (size)
	{
		size_t	n = len < size - 1 ? len : size - 1;
		memcpy(dst, src, n);
		dst[n] = 0;
	}
	return (len);
}

int	ft_printf(const char *fmt, ...)
{
	va_list	ap;
	int		r;

	if (oracle_quiet)
		return (0);
	va_start(ap, fmt);
	r = vprintf(fmt, ap);
	va_end(ap);
	return (r);
}

int	ft_dprintf(int fd, const char *fmt, ...)
{
	va_list	ap;
	int		r;

	va_start(ap, fmt);
	r = vdprintf(fd, fmt, ap);
	va_end(ap);
	return (r);
}

char	*ft_sprintf(const char *fmt, ...)
{
	va_list	ap;
	char	*out;

	va_start(ap, fmt);
	if (vasprintf(&out, fmt, ap) < 0)
		out = NULL;
	va_end(ap);
	return (out);
}

ssize_t	get_cpu_time(void)
{
	struct timespec	ts;

	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ((ssize_t)ts.tv_sec * 1000 + ts.tv_nsec / 1000000);
}

/* UI float-input binding: the headless oracle has no UI, so this is a no-op. */
struct s_float_input;
void	link_float_input(struct s_float_input *in, double *number)
{
	(void)in;
	(void)number;
}
