// readback.cu — frame read-back kernels, in a translation unit of their own:
// with lazy module loading (the CUDA 12 default) the first launch of a
// kernel loads its module, and render.cu's module (every megakernel
// instantiation) took 150 ms to load when a process had only run the
// wavefront so far. This module is a few kilobytes.
#include "kernels.h"

namespace mrt {

__global__ void accumulate_double_kernel(float4* accum, double* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 a = accum[i];
  out[3 * i] += a.x;
  out[3 * i + 1] += a.y;
  out[3 * i + 2] += a.z;
  accum[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void accum_to_rgb_kernel(const float4* accum, float* rgb, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 a = accum[i];
  rgb[3 * i] = a.x;
  rgb[3 * i + 1] = a.y;
  rgb[3 * i + 2] = a.z;
}

cudaError_t launch_accumulate_double(float4* accum, double* out, int n, cudaStream_t st) {
  accumulate_double_kernel<<<(n + 255) / 256, 256, 0, st>>>(accum, out, n);
  return cudaGetLastError();
}

cudaError_t launch_accum_to_rgb(const float4* accum, float* rgb, int n, cudaStream_t st) {
  accum_to_rgb_kernel<<<(n + 255) / 256, 256, 0, st>>>(accum, rgb, n);
  return cudaGetLastError();
}

}  // namespace mrt
