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
  // when set (the differentiable forward), path radiance is added here as
  // 64-bit fixed point (kFrameFxScale), 3 per pixel, instead of into the
  // float4 accumulator: integer sums do not depend on the order in which
  // paths finish, so the image is the same on every run
  unsigned long long* accum_fx;
};

// Fixed-point scale of accum_fx: 2^32 per unit radiance (resolution
// 2.3e-10; a pixel sum stays below 2^63 up to 2^31 units).
constexpr double kFrameFxScale = 4294967296.0;

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
// kind: 2 when some scene of the batch has textures, 1 when some has
// cylinders, cones or hyperboloids, else 0 (the view type instantiated)
cudaError_t launch_megakernel_batch(const SceneView* views, const BatchItem* items, int n_items,
                                    uint64_t total, int* status, unsigned long long* work, int block,
                                    int kind, cudaStream_t st);
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
  const float* rgb;        // when set: linear float RGB per texel instead of rgbe
                           // (grey = 0.2126*255r + 0.7152*255g + 0.0722*255b)
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
  double* out_prob;        // (H-1)*W, or null to skip the outcome probabilities
};
cudaError_t launch_env_tables(const EnvBuild& E, cudaStream_t st);

// Differentiable rendering (adjoint.cu).
constexpr int kMaxTape = 16;       // bounces a differentiable path may take
constexpr int kDiffMaxMats = 1024; // materials (shared-memory gradient accumulators)

struct DiffEnvRecords {
  const float* cdf_m_inv;  // H
  const float* cdf_c_inv;  // W*H
  const float* pdf_joint;  // W*H
  const float4* grid;      // W*H: direction .xyz and texel (int bits) per (row, column) index
  const float* sky;        // W*H*3 linear radiance
  int W, H;
  float4* rec0;            // (H-1)*W outputs
  float4* rec1;
  int2* aux;               // (radiance texel, pdf_joint index)
};

struct AdjointArgs {
  uint64_t n_paths;
  uint64_t seed;
  uint32_t sample_base;
  int max_bounces;         // <= kMaxTape
  int jitter;
  int n_mats;
  int n_texels;
  float inv_spp;
  float pdf_dgray;         // d grey / d (lum-weighted channel): 255
  const double* col;       // column average of the grey values (device)
  const float* dimg;       // d loss / d image, W*H*3
  const int2* env_aux;
  // gradient sums as 64-bit fixed point (value * q_scale): integer
  // additions are associative, so the sums do not depend on the order in
  // which threads add, and one seed gives one gradient
  long long* q_mats;       // [albedo M*3 | roughness M | emission M]
  long long* q_sky;        // W*H*3
  long long* q_col;        // one value
  double q_scale;          // 2^S with S chosen from max |d loss / d image|
};

// Tape of the backward: one entry per bounce, tape[k * n_paths + path].
struct __align__(16) TapeEntry {   // 80 B
  float4 o_t;          // ray origin, hit distance (root choice for spheres)
  float4 d_ra;         // ray direction as traced (not normalised), sampler random 1
  float4 P_rb;         // path power before shading, sampler random 2
  float4 T;            // direct-light + caustic term of default_mat (detached)
  int4 meta;           // primitive, material, flags, HDRI NEE outcome
};

cudaError_t launch_diff_mats(const MaterialD* base, const float* theta, int M, MaterialD* out,
                             cudaStream_t st);
cudaError_t launch_diff_env_records(const DiffEnvRecords& E, cudaStream_t st);
cudaError_t launch_diff_image(const unsigned long long* accum_fx, float* img, int npix, int spp,
                              cudaStream_t st);
// max |x| over n floats into *out (device), which must start at 0
cudaError_t launch_abs_max(const float* x, size_t n, float* out, cudaStream_t st);
// out[i] = q[i] / scale for i < n; then the dense pdf term of the sky
cudaError_t launch_diff_grad_out(const AdjointArgs& A, float* out_mats, float* out_sky, int64_t n_mats5,
                                 cudaStream_t st);
cudaError_t launch_diff_sky_init(const SceneView& S, float* out, cudaStream_t st);
// Backward of the paths [sample_base, sample_base + n_paths / W*H) of one
// chunk: replay writing the tape (n_paths * max_bounces entries) and the
// per-path state (4 float4 per path), then one reverse launch per bounce
// level. Gradients accumulate into A.g_*.
cudaError_t launch_adjoint_chunk(const SceneView& S, const AdjointArgs& A, TapeEntry* tape, float4* state,
                                 unsigned long long* work, int* status, cudaStream_t st);
// The dense term of the pdf gradient (after all chunks).

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

// Photon map (photon.cu): sorts the photons by the 63-bit Morton code of
// their position (CUB radix sort of (code, index), deterministic) and builds
// the linear BVH of SceneView.photon_nodes over them.
struct PhotonTree {
  const float4* pos_in;
  const float4* pow_in;
  uint32_t n;
  float4* pos_out;           // n
  float4* pow_out;           // n
  float4* nodes;             // 4 * max(n - 1, 1)
};
cudaError_t launch_photon_tree(const PhotonTree& T, cudaStream_t st);

struct CausticQuery {
  const double* pts;
  int64_t n;
  double* out;
};
cudaError_t launch_caustic_query(const SceneView& S, const CausticQuery& Q, cudaStream_t st);

}  // namespace mrt
