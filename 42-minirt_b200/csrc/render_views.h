// render_views.h — per-view-type launchers of the megakernel forms and
// probes (render_kernels.cuh), declared here and instantiated by
// render_inst.cu, which is compiled once per (view type, kernel group).
#pragma once
#include "kernels.h"

namespace mrt {

template <bool kCount, class V>
cudaError_t launch_megakernel_v(const V& v, const LaunchParams& L, float4* accum, int* depth,
                                int* status, unsigned long long* counters, int block, cudaStream_t st);
template <class V>
cudaError_t launch_regen_v(const V& v, const LaunchParams& L, float4* accum, int* status,
                           unsigned long long* work, int block, int blocks_per_sm, int sms, cudaStream_t st);
template <class V>
cudaError_t launch_batch_v(const SceneView* views, const BatchItem* items, int n_items, uint64_t total,
                           int* status, unsigned long long* work, int block, int sms, cudaStream_t st);
template <class V>
cudaError_t launch_path_events_v(const V& v, const LaunchParams& L, const int* pix, const int* smp, int n,
                                 float* ev, float* rgb, int* status, cudaStream_t st);
template <class V>
cudaError_t launch_first_hit_v(const V& v, const double* rays, int64_t n, HitOut* out, int* status,
                               cudaStream_t st);

}  // namespace mrt
