// kernels.h — host-side declarations of the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "mrt_internal.h"

namespace mrt {

struct LaunchParams {
  uint64_t n_paths;      // paths in this launch (npix * spp)
  uint64_t seed;
  uint32_t sample_base;
  int max_bounces;
  int jitter;            // 0 shared per sample, 1 per pixel
  int render_mode;
  int has_offset;        // explicit shared offset (compute_frame / calc_one_sample)
  float ox, oy;
};

// One scene of a multi-scene batch launch.
struct BatchItem {
  uint64_t start;          // first global path index of this scene
  uint64_t paths;
  uint64_t seed;
  uint32_t sample_base;
  int view;                // index into the device SceneView array
  int max_bounces;
  int jitter;
  float4* accum;           // the scene's accumulator
};

// Matches mrt_hit (include/mrt.h) field for field.
struct HitOut {
  int prim;
  int front_face;
  float t, u, v;
  float n[3];
  float p[3];
  int visits;
};

cudaError_t launch_megakernel(const SceneView& S, const LaunchParams& L, float4* accum, int* depth,
                              int* status, unsigned long long* counters, int block,
                              cudaStream_t st);
cudaError_t launch_megakernel_regen(const SceneView& S, const LaunchParams& L, float4* accum,
                                    int* status, unsigned long long* work, int block, int blocks_per_sm,
                                    cudaStream_t st);
cudaError_t launch_megakernel_batch(const SceneView* views, const BatchItem* items, int n_items,
                                    uint64_t total, int* status, unsigned long long* work, int block,
                                    cudaStream_t st);
cudaError_t launch_path_events(const SceneView& S, const LaunchParams& L, const int* pix, const int* smp,
                               int n, float* ev, float* rgb, int* status, cudaStream_t st);
cudaError_t launch_first_hit(const SceneView& S, const double* rays, int64_t n, HitOut* out,
                             int* status, cudaStream_t st);
cudaError_t launch_accumulate_double(float4* accum, double* out, int n, cudaStream_t st);
cudaError_t launch_env_sample(const SceneView& S, int64_t n, uint64_t seed, int* k_out, float4* out,
                              cudaStream_t st);
cudaError_t launch_accum_to_rgb(const float4* accum, float* rgb, int n, cudaStream_t st);

// HDRI tables (env.cu). Inputs: RGBE texels on the device. Outputs on the
// device: pdf_joint (W*H f32), cdf_m_inv (H f32), cdf_c_inv (W*H f32) and the
// outcome probabilities / records of the two-step sampler ((H-1)*W entries).
struct EnvBuild {
  const uint32_t* rgbe;
  int W, H;
  double exposure_scale;   // powf(2, exposure) widened, used when exposure != 0
  int exposure_zero;
  // scratch + outputs (device)
  double* gray;            // W*H
  double* raw;             // H
  double* row_cdf;         // W*H
  double* scal;            // [0] column_average, [1] marginal sum ... (8 doubles)
  double* cdf_h;           // H
  float* pdf_joint;
  float* cdf_m_inv;
  float* cdf_c_inv;
  double* out_prob;        // (H-1)*W
};
cudaError_t launch_env_tables(const EnvBuild& E, cudaStream_t st);

// Photons (photon.cu)
struct PhotonEmit {
  uint64_t seed;
  uint32_t pass;
  uint64_t per_light;
  int n_point_lights;
  const int* light_index;    // point lights, index into S.lights
  float4* pos;               // capacity entries
  float4* pow;
  unsigned int* count;       // device counter
  uint64_t capacity;
};
cudaError_t launch_photon_emit(const SceneView& S, const PhotonEmit& P, int* status, cudaStream_t st);

struct GridBuild {
  const float4* pos_in;
  const float4* pow_in;
  uint32_t n;
  float4* pos_out;
  float4* pow_out;
  uint32_t* cell_of;         // n
  uint32_t* cell_start;      // n_cells + 1
  uint32_t* cursor;          // n_cells
  uint32_t n_cells;
  float grid_min[3];
  float inv_cell;
  int dim[3];
};
cudaError_t launch_grid_build(const GridBuild& G, cudaStream_t st);

struct CausticQuery {
  const double* pts;
  int64_t n;
  double* out;
};
cudaError_t launch_caustic_query(const SceneView& S, const CausticQuery& Q, cudaStream_t st);

}  // namespace mrt
