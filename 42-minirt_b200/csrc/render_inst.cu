// render_inst.cu — explicit instantiations of the megakernel launchers for
// one scene view type and one kernel group, chosen at compile time:
//   -DMRT_VIEW=SceneView | SceneViewQ | SceneViewT
//   -DMRT_GROUP=0  plain megakernel          1  plain megakernel with counters
//               2  regenerating megakernel and the probes
//               3  multi-scene batch megakernel
// The build compiles this file once per combination (twelve objects), so the
// instantiations build in parallel.
#include "render_kernels.cuh"

#if !defined(MRT_VIEW) || !defined(MRT_GROUP)
#error "render_inst.cu needs -DMRT_VIEW=<view type> -DMRT_GROUP=<0..3>"
#endif

namespace mrt {

#if MRT_GROUP == 0 || MRT_GROUP == 1
template cudaError_t launch_megakernel_v<MRT_GROUP == 1, MRT_VIEW>(const MRT_VIEW&, const LaunchParams&, float4*,
                                                                   int*, int*, unsigned long long*, int,
                                                                   cudaStream_t);
#elif MRT_GROUP == 2
template cudaError_t launch_regen_v<MRT_VIEW>(const MRT_VIEW&, const LaunchParams&, float4*, int*,
                                              unsigned long long*, int, int, int, cudaStream_t);
template cudaError_t launch_path_events_v<MRT_VIEW>(const MRT_VIEW&, const LaunchParams&, const int*, const int*,
                                                    int, float*, float*, int*, cudaStream_t);
template cudaError_t launch_first_hit_v<MRT_VIEW>(const MRT_VIEW&, const double*, int64_t, HitOut*, int*,
                                                  cudaStream_t);
#elif MRT_GROUP == 3
template cudaError_t launch_batch_v<MRT_VIEW>(const SceneView*, const BatchItem*, int, uint64_t, int*,
                                              unsigned long long*, int, int, cudaStream_t);
#else
#error "MRT_GROUP must be 0..3"
#endif

}  // namespace mrt
