// render.cu — host launchers of the megakernel forms and the probes: each
// dispatches on the scene's view type (SceneView, or SceneViewQ / SceneViewT
// when the scene has quadrics / textures) to the per-view launcher
// instantiated by render_inst.cu.
#include <type_traits>

#include "kernels.h"
#include "path.cuh"
#include "render_views.h"

namespace mrt {

static int sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

cudaError_t launch_megakernel(const SceneView& S, const LaunchParams& L, float4* accum, int* depth,
                              int* status, unsigned long long* counters, int block,
                              cudaStream_t st) {
  if (L.n_paths == 0) return cudaSuccess;
  block = block > 0 ? block : 128;
  return with_view(S, [&](const auto& v) -> cudaError_t {
    using VT = std::decay_t<decltype(v)>;
    return counters ? launch_megakernel_v<true, VT>(v, L, accum, depth, status, counters, block, st)
                    : launch_megakernel_v<false, VT>(v, L, accum, depth, status, counters, block, st);
  });
}

cudaError_t launch_megakernel_regen(const SceneView& S, const LaunchParams& L, float4* accum,
                                    int* status, unsigned long long* work, int block, int blocks_per_sm,
                                    cudaStream_t st) {
  if (L.n_paths == 0) return cudaSuccess;
  block = block > 0 ? block : 128;
  cudaError_t e = cudaMemsetAsync(work, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const int sms = sm_count();
  return with_view(S, [&](const auto& v) -> cudaError_t {
    return launch_regen_v(v, L, accum, status, work, block, blocks_per_sm, sms, st);
  });
}

cudaError_t launch_megakernel_batch(const SceneView* views, const BatchItem* items, int n_items,
                                    uint64_t total, int* status, unsigned long long* work, int block,
                                    int kind, cudaStream_t st) {
  if (total == 0 || n_items == 0) return cudaSuccess;
  block = block > 0 ? block : 128;
  cudaError_t e = cudaMemsetAsync(work, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  const int sms = sm_count();
  if (kind == 2) return launch_batch_v<SceneViewT>(views, items, n_items, total, status, work, block, sms, st);
  if (kind == 1) return launch_batch_v<SceneViewQ>(views, items, n_items, total, status, work, block, sms, st);
  return launch_batch_v<SceneView>(views, items, n_items, total, status, work, block, sms, st);
}

cudaError_t launch_path_events(const SceneView& S, const LaunchParams& L, const int* pix, const int* smp,
                               int n, float* ev, float* rgb, int* status, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  return with_view(S, [&](const auto& v) -> cudaError_t {
    return launch_path_events_v(v, L, pix, smp, n, ev, rgb, status, st);
  });
}

cudaError_t launch_first_hit(const SceneView& S, const double* rays, int64_t n, HitOut* out,
                             int* status, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  return with_view(S, [&](const auto& v) -> cudaError_t {
    return launch_first_hit_v(v, rays, n, out, status, st);
  });
}

__global__ void env_sample_kernel(SceneView S, int64_t n, uint64_t seed, int* k_out, float4* out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Rng rng{path_seed(seed, (uint32_t)i, (uint32_t)(i >> 32))};
  const int k = env_sample(S, rng);
  k_out[i] = k;
  out[i] = __ldg(S.env_rec0 + k);
}

cudaError_t launch_env_sample(const SceneView& S, int64_t n, uint64_t seed, int* k_out, float4* out,
                              cudaStream_t st) {
  env_sample_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(S, n, seed, k_out, out);
  return cudaGetLastError();
}

}  // namespace mrt
