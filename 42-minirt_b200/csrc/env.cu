// env.cu — HDRI importance-sampling tables built on the device in FP64.
//
// Reproduces make_importance_sampling_map (importance_sampling_manager.c:41)
// bit for bit: grey values (calc_pdf.c:16-38), row averages (:53-71), the
// column average, pdf_joint / pdf_marginal / pdf_conditional (:73-115), the
// normalised marginal and per-row conditional CDFs and their inverse tables
// (calc_cdf.c:16-129). Sums keep the reference's sequential order (one
// thread per row), products and sums use explicitly rounded intrinsics so
// the compiler cannot fuse them, and the reference's O(n) inverse search
// becomes a binary search for the same "first index with cdf >= u".
//
// It then derives the exact outcome distribution of the two-step lookup of
// get_dir.c:15-27 (row = floor(r1 (H-1)), column index = floor(A + r2 (W-1)),
// A = v (H-1) W). The host turns those probabilities into an alias table
// (Vose 1991) and records, per outcome, the direction, pdf and sky radiance
// the reference computes for it.
#include "kernels.h"

namespace mrt {

namespace {

__global__ void grey_kernel(EnvBuild E) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t n = (size_t)E.W * E.H;
  if (i >= n) return;
  if (E.rgb) {
    const double r = __dmul_rn((double)E.rgb[3 * i], 255.0), g = __dmul_rn((double)E.rgb[3 * i + 1], 255.0),
                 b = __dmul_rn((double)E.rgb[3 * i + 2], 255.0);
    E.gray[i] = __dadd_rn(__dadd_rn(__dmul_rn(0.2126, r), __dmul_rn(0.7152, g)), __dmul_rn(0.0722, b));
    return;
  }
  uint32_t px = E.rgbe[i];
  int e = (int)(px >> 24);
  double scale = ldexp(1.0, e - 128);
  if (!E.exposure_zero) scale = __dmul_rn(scale, E.exposure_scale);
  double r = (double)(px & 255u), g = (double)((px >> 8) & 255u), b = (double)((px >> 16) & 255u);
  double t = __dadd_rn(__dadd_rn(__dmul_rn(0.2126, __dmul_rn(r, scale)),
                                 __dmul_rn(0.7152, __dmul_rn(g, scale))),
                       __dmul_rn(0.0722, __dmul_rn(b, scale)));
  E.gray[i] = t;
}

// Row averages, one thread per row (sequential order of calc_raw_average).
__global__ void row_average_kernel(EnvBuild E) {
  int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= E.H) return;
  const double* row = E.gray + (size_t)y * E.W;
  double sum = 0.0;
  for (int x = 0; x < E.W; ++x) sum = __dadd_rn(sum, row[x]);
  E.raw[y] = __ddiv_rn(sum, (double)E.W);
}

// Column average, marginal pdf/cdf and its inverse: small, one thread.
__global__ void marginal_kernel(EnvBuild E) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const int H = E.H;
  double sum = 0.0;
  for (int i = 0; i < H; ++i) sum = __dadd_rn(sum, E.raw[i]);
  const double col = __ddiv_rn(sum, (double)H);
  E.scal[0] = col;
  const double denom = __ddiv_rn(col, 255.0);
  sum = 0.0;
  for (int i = 0; i < H; ++i) {
    sum = __dadd_rn(sum, __ddiv_rn(E.raw[i], denom));
    E.cdf_h[i] = sum;
  }
  if (sum > 0.0)
    for (int i = 0; i < H; ++i) E.cdf_h[i] = __ddiv_rn(E.cdf_h[i], sum);
  int valid = H;                       // NaN tail: no index there satisfies ">= u"
  for (int i = 0; i < H; ++i)
    if (E.cdf_h[i] != E.cdf_h[i]) { valid = i; break; }
  for (int i = 0; i < H; ++i) {
    double u = __ddiv_rn((double)i, (double)(H - 1));
    int lo = 0, hi = valid;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      if (E.cdf_h[mid] >= u) hi = mid; else lo = mid + 1;
    }
    E.cdf_m_inv[i] = lo < valid ? __double2float_rn(__ddiv_rn((double)lo, (double)(H - 1))) : 0.0f;
  }
}

__global__ void pdf_joint_kernel(EnvBuild E) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)E.W * E.H) return;
  E.pdf_joint[i] = __double2float_rn(__ddiv_rn(E.gray[i], E.scal[0]));
}

// Conditional CDF per row (sequential prefix, one thread per row).
__global__ void conditional_cdf_kernel(EnvBuild E) {
  int y = blockIdx.x * blockDim.x + threadIdx.x;
  if (y >= E.H) return;
  const int W = E.W;
  const double* g = E.gray + (size_t)y * W;
  double* c = E.row_cdf + (size_t)y * W;
  const double denom = __ddiv_rn(E.raw[y], 255.0);
  double sum = 0.0;
  for (int x = 0; x < W; ++x) {
    sum = __dadd_rn(sum, __ddiv_rn(g[x], denom));
    c[x] = sum;
  }
  if (sum > 0.0)
    for (int x = 0; x < W; ++x) c[x] = __ddiv_rn(c[x], sum);
}

// Inverse conditional tables: one thread per (row, i).
__global__ void conditional_inv_kernel(EnvBuild E) {
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int W = E.W;
  if (k >= (size_t)W * E.H) return;
  const int y = (int)(k / W), i = (int)(k % W);
  const double* c = E.row_cdf + (size_t)y * W;
  // prefix sums are non-decreasing until a NaN appears; NaN never satisfies ">= u"
  int valid = W;
  if (c[W - 1] != c[W - 1]) {
    int lo = 0, hi = W;
    while (lo < hi) {          // first NaN (NaNs form a suffix of the prefix sums)
      int mid = (lo + hi) >> 1;
      if (c[mid] != c[mid]) hi = mid; else lo = mid + 1;
    }
    valid = lo;
  }
  const double u = __ddiv_rn((double)i, (double)(W - 1));
  int lo = 0, hi = valid;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (c[mid] >= u) hi = mid; else lo = mid + 1;
  }
  E.cdf_c_inv[k] = lo < valid ? __double2float_rn(__ddiv_rn((double)lo, (double)(W - 1))) : 0.0f;
}

// Outcome (iy, d): probability of the two-step lookup landing there.
__global__ void outcome_kernel(EnvBuild E) {
  size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int W = E.W, H = E.H;
  if (k >= (size_t)(H - 1) * W) return;
  const int iy = (int)(k / W), d = (int)(k % W);
  const double v = (double)E.cdf_m_inv[iy];
  const double A = __dmul_rn(__dmul_rn(v, (double)(H - 1)), (double)W);
  const double j0 = floor(A);
  double lo = (j0 + d - A) / (double)(W - 1);
  double hi = (j0 + d + 1 - A) / (double)(W - 1);
  lo = lo < 0.0 ? 0.0 : lo;
  hi = hi > 1.0 ? 1.0 : hi;
  double p = hi > lo ? (hi - lo) / (double)(H - 1) : 0.0;
  const long long j = (long long)j0 + d;
  if (j < 0 || j >= (long long)W * H) p = 0.0;
  E.out_prob[k] = p;
}

}  // namespace

cudaError_t launch_env_tables(const EnvBuild& E, cudaStream_t st) {
  const size_t n = (size_t)E.W * E.H;
  const unsigned b = 256;
  grey_kernel<<<(unsigned)((n + b - 1) / b), b, 0, st>>>(E);
  row_average_kernel<<<(E.H + 63) / 64, 64, 0, st>>>(E);
  marginal_kernel<<<1, 1, 0, st>>>(E);
  pdf_joint_kernel<<<(unsigned)((n + b - 1) / b), b, 0, st>>>(E);
  conditional_cdf_kernel<<<(E.H + 63) / 64, 64, 0, st>>>(E);
  conditional_inv_kernel<<<(unsigned)((n + b - 1) / b), b, 0, st>>>(E);
  const size_t no = (size_t)(E.H - 1) * E.W;
  if (!E.out_prob) return cudaGetLastError();
  outcome_kernel<<<(unsigned)((no + b - 1) / b), b, 0, st>>>(E);
  return cudaGetLastError();
}

}  // namespace mrt
