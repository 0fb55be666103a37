/*
 * TEST INFRASTRUCTURE — stand-ins for the libft functions that miniRT's
 * scene parser and file loaders call (src/parsing, src/utils/{hdr,obj,png,
 * bmp}). libft is an un-vendored git submodule of the reference; these are
 * restated from the contracts their call sites rely on:
 *   - ft_split_in_line(s, set) splits s IN PLACE at any character of set
 *     (separators become '\0', empty fields are skipped) and returns a
 *     malloc'd NULL-terminated array of pointers into s: callers free only
 *     the array (parse_elements_utils2.c:27-31);
 *   - ft_atod / ft_atof read [+-]digits[.digits] (the syntax is_valid_float
 *     admits first, parse_elements_utils2.c:17);
 *   - get_next_line returns each line of fd with its '\n', NULL at the end;
 *   - read_bin_file loads a whole file into a t_bin; read_uintN_move reads
 *     at *i (big-endian, or little-endian for the _little forms), advances
 *     *i and returns -1 past the end.
 * Used only to build oracle/_ref (the reference compiled from its sources)
 * for the .rt end-to-end tests; nothing of the library calls them.
 */
#include "libft.h"
#include <fcntl.h>
#include <string.h>

int	ft_strcmp(const char *a, const char *b)
{
	return (strcmp(a, b));
}

int	ft_strncmp(const char *a, const char *b, size_t n)
{
	return (strncmp(a, b, n));
}

size_t	ft_strlen(const char *s)
{
	return (strlen(s));
}

ssize_t	ft_sstrlen(const char *s)
{
	return ((ssize_t)strlen(s));
}

char	*ft_strchr(const char *s, int c)
{
	return (strchr(s, c));
}

char	*ft_strrchr(const char *s, int c)
{
	return (strrchr(s, c));
}

char	*ft_strnstr(const char *h, const char *n, size_t len)
{
	size_t	ln = strlen(n);

	if (!ln)
		return ((char *)h);
	for (size_t i = 0; h[i] && i + ln <= len; i++)
		if (strncmp(h + i, n, ln) == 0)
			return ((char *)h + i);
	return (NULL);
}

char	*ft_strdup(const char *s)
{
	return (strdup(s));
}

int	ft_isdigit(int c)
{
	return (c >= '0' && c <= '9');
}

int	ft_isalpha(int c)
{
	return ((c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z'));
}

int	ft_isalnum(int c)
{
	return (ft_isdigit(c) || ft_isalpha(c));
}

int	ft_atoi(const char *s)
{
	return (atoi(s));
}

int	ft_abs(int x)
{
	return (x < 0 ? -x : x);
}

/* [+-]digits[.digits]: integer part and fraction accumulated in double */
double	ft_atod(const char *s)
{
	double	sign = 1.0, v = 0.0, scale = 0.1;

	while (*s == ' ' || *s == '\t')
		s++;
	if (*s == '+' || *s == '-')
		sign = (*s++ == '-') ? -1.0 : 1.0;
	while (ft_isdigit(*s))
		v = v * 10.0 + (*s++ - '0');
	if (*s == '.')
	{
		s++;
		while (ft_isdigit(*s))
		{
			v += (*s++ - '0') * scale;
			scale *= 0.1;
		}
	}
	return (sign * v);
}

float	ft_atof(const char *s)
{
	return ((float)ft_atod(s));
}

int	is_valid_float(const char *s)
{
	int	digits = 0;

	if (*s == '+' || *s == '-')
		s++;
	while (ft_isdigit(*s) && ++digits)
		s++;
	if (*s == '.')
	{
		s++;
		while (ft_isdigit(*s) && ++digits)
			s++;
	}
	return (digits > 0 && *s == '\0');
}

char	**ft_split_in_line(char *s, const char *set)
{
	size_t	n = 0, cap = 8;
	char	**out = malloc(sizeof(char *) * cap);
	size_t	i = 0;

	if (!out)
		return (NULL);
	while (s[i])
	{
		while (s[i] && strchr(set, s[i]))
			s[i++] = '\0';
		if (!s[i])
			break ;
		if (n + 2 > cap)
		{
			char	**t = realloc(out, sizeof(char *) * (cap *= 2));

			if (!t)
				return (free(out), NULL);
			out = t;
		}
		out[n++] = s + i;
		while (s[i] && !strchr(set, s[i]))
			i++;
	}
	out[n] = NULL;
	return (out);
}

void	ft_free_tab_null_term(char **tab)
{
	if (!tab)
		return ;
	for (size_t i = 0; tab[i]; i++)
		free(tab[i]);
	free(tab);
}

/* one line per call, '\n' kept; a small per-fd buffer (one fd at a time) */
char	*get_next_line(int fd)
{
	static char		buf[4096];
	static ssize_t	len = 0, pos = 0;
	static int		last_fd = -1;
	char			*line = NULL;
	size_t			n = 0;

	if (fd != last_fd)
	{
		len = pos = 0;
		last_fd = fd;
	}
	while (1)
	{
		if (pos >= len)
		{
			len = read(fd, buf, sizeof(buf));
			pos = 0;
			if (len <= 0)
			{
				len = 0;
				return (line);
			}
		}
		{
			char	c = buf[pos++];
			char	*t = realloc(line, n + 2);

			if (!t)
				return (free(line), NULL);
			line = t;
			line[n++] = c;
			line[n] = '\0';
			if (c == '\n')
				return (line);
		}
	}
}

int	read_bin_file(t_bin *bin, const char *path)
{
	int				fd = open(path, O_RDONLY);
	unsigned char	chunk[65536];
	ssize_t			r;

	bin->data = NULL;
	bin->size = 0;
	if (fd < 0)
		return (0);
	while ((r = read(fd, chunk, sizeof(chunk))) > 0)
	{
		unsigned char	*t = realloc(bin->data, bin->size + r);

		if (!t)
			return (close(fd), 0);
		bin->data = t;
		memcpy(bin->data + bin->size, chunk, r);
		bin->size += r;
	}
	close(fd);
	return (r == 0);
}

static int	take(t_bin *bin, size_t *i, size_t n, int little, uint64_t *v)
{
	if (*i + n > bin->size)
		return (-1);
	*v = 0;
	for (size_t k = 0; k < n; k++)
	{
		uint64_t	b = bin->data[*i + k];

		*v |= little ? b << (8 * k) : b << (8 * (n - 1 - k));
	}
	*i += n;
	return (0);
}

int	read_uint8_move(t_bin *bin, size_t *i, uint8_t *out)
{
	uint64_t	v;

	if (take(bin, i, 1, 0, &v) < 0)
		return (-1);
	*out = (uint8_t)v;
	return (0);
}

int	read_uint16_move(t_bin *bin, size_t *i, uint16_t *out)
{
	uint64_t	v;

	if (take(bin, i, 2, 0, &v) < 0)
		return (-1);
	*out = (uint16_t)v;
	return (0);
}

int	read_uint16_move_little(t_bin *bin, size_t *i, uint16_t *out)
{
	uint64_t	v;

	if (take(bin, i, 2, 1, &v) < 0)
		return (-1);
	*out = (uint16_t)v;
	return (0);
}

int	read_uint32_move(t_bin *bin, size_t *i, uint32_t *out)
{
	uint64_t	v;

	if (take(bin, i, 4, 0, &v) < 0)
		return (-1);
	*out = (uint32_t)v;
	return (0);
}

int	read_uint32_move_little(t_bin *bin, size_t *i, uint32_t *out)
{
	uint64_t	v;

	if (take(bin, i, 4, 1, &v) < 0)
		return (-1);
	*out = (uint32_t)v;
	return (0);
}

int	read_uint64_move_little(t_bin *bin, size_t *i, uint64_t *out)
{
	return (take(bin, i, 8, 1, out));
}
