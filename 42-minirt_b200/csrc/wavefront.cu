// wavefront.cu — placeholder until the wavefront form lands.
#include "../../include/mrt.h"
#include "kernels.h"

int mrt_render_wavefront(mrt_ctx*, const mrt::SceneView&, const mrt::LaunchParams&, int,
                         const mrt_render_params*, mrt_render_stats*) {
  return MRT_ERR_INVALID;
}
