// env_noalloc.cu — the HDRI importance-sampling table build for callers that
// cannot allocate GPU memory.
//
// Some hosts may not call cudaMalloc (or anything that allocates) at the
// point where they need the tables: a host that owns all device memory in
// its own pre-sized arena or pool, a real-time loop that must not hit the
// allocator, or code that runs where allocation is forbidden. They hand in
// device buffers for the RGBE sky and the three tables; the build's scratch
// (grey values, row CDFs, row averages, the marginal CDF) lives in the
// fixed array below instead of in per-call allocations.
//
// The array is a file-scope __device__ variable: every GPU that loads this
// module holds it (about 4 MiB) until the process exits. With lazy module
// loading the module loads on the first call on a device, so that first call
// takes the array's memory through the driver; later calls allocate nothing.
// Its host-side name is only a stand-in for the symbol, not a device
// address, so the device address is looked up once per device with
// cudaGetSymbolAddress and cached; the cache is not refreshed after
// cudaDeviceReset, which this entry point does not support.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/mrt.h"
#include "kernels.h"

namespace mrt {

int set_error_message(int code, const char* msg);

namespace {

// Scratch layout, in doubles: grey (W*H) | row CDFs (W*H) | row averages (H)
// | marginal CDF (H) | 8 scalars.
constexpr size_t kScratchDoubles =
    2 * (size_t)MRT_ENV_NOALLOC_MAX_TEXELS + 2 * (size_t)MRT_ENV_NOALLOC_MAX_ROWS + 8;

static __device__ __align__(256) double g_env_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// mrt_last_error's message (api.cu).
int fail(int code, const char* msg, cudaError_t e = cudaSuccess) {
  std::string m = msg;
  if (e != cudaSuccess) {
    m += ": ";
    m += cudaGetErrorString(e);
  }
  return set_error_message(code, m.c_str());
}

// Device address of the scratch array on the current device (set-up on the
// first call per device).
cudaError_t scratch_on(int device, double** out) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_env_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_ptr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[device];
  return cudaSuccess;
}

}  // namespace

}  // namespace mrt

using namespace mrt;

extern "C" int mrt_env_tables_noalloc(int device, const uint8_t* rgbe, int32_t width, int32_t height,
                                      float hdr_exposure, float* pdf_joint, float* cdf_marginal_inverse,
                                      float* cdf_conditional_inverse, void* stream) {
  if (!rgbe || !pdf_joint || !cdf_marginal_inverse || !cdf_conditional_inverse)
    return fail(MRT_ERR_INVALID, "mrt_env_tables_noalloc: null buffer");
  if (reinterpret_cast<uintptr_t>(rgbe) % 4 != 0)
    return fail(MRT_ERR_INVALID, "mrt_env_tables_noalloc: rgbe must be 4-byte aligned");
  if (width < 2 || height < 2)
    return fail(MRT_ERR_INVALID, "mrt_env_tables_noalloc: the sky must be at least 2x2 texels");
  if ((int64_t)width * height > MRT_ENV_NOALLOC_MAX_TEXELS || height > MRT_ENV_NOALLOC_MAX_ROWS) {
    char buf[200];
    snprintf(buf, sizeof(buf),
             "mrt_env_tables_noalloc: %dx%d sky exceeds the fixed scratch (at most %d texels and %d rows)",
             width, height, MRT_ENV_NOALLOC_MAX_TEXELS, MRT_ENV_NOALLOC_MAX_ROWS);
    return fail(MRT_ERR_INVALID, buf);
  }
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(MRT_ERR_NO_DEVICE, "mrt_env_tables_noalloc: no CUDA device", e);
  if (device < 0 || device >= n || device >= kMaxDevices)
    return fail(MRT_ERR_INVALID, "mrt_env_tables_noalloc: device out of range");
  int prev = 0;
  cudaGetDevice(&prev);
  if ((e = cudaSetDevice(device)) != cudaSuccess)
    return fail(MRT_ERR_CUDA, "mrt_env_tables_noalloc: cudaSetDevice", e);
  double* s = nullptr;
  if ((e = scratch_on(device, &s)) != cudaSuccess) {
    cudaSetDevice(prev);
    return fail(MRT_ERR_CUDA, "mrt_env_tables_noalloc: cudaGetSymbolAddress", e);
  }
  // Every scratch element the build reads it has written first in the same
  // call (grey values, row sums and CDFs are fully rewritten), so nothing
  // left by an earlier call needs clearing.
  const size_t t = (size_t)width * height;
  EnvBuild E{};
  E.rgbe = reinterpret_cast<const uint32_t*>(rgbe);
  E.rgb = nullptr;
  E.W = width;
  E.H = height;
  E.exposure_zero = hdr_exposure == 0.0f;
  E.exposure_scale = (double)powf(2.0f, hdr_exposure);
  E.gray = s;
  E.row_cdf = s + t;
  E.raw = s + 2 * t;
  E.cdf_h = s + 2 * t + height;
  E.scal = s + 2 * t + 2 * (size_t)height;
  E.pdf_joint = pdf_joint;
  E.cdf_m_inv = cdf_marginal_inverse;
  E.cdf_c_inv = cdf_conditional_inverse;
  E.out_prob = nullptr;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e = launch_env_tables(E, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaSetDevice(prev);
  if (e != cudaSuccess) return fail(MRT_ERR_CUDA, "mrt_env_tables_noalloc: table build", e);
  return MRT_OK;
}
