// path.cuh — one camera path through the reference's estimator
// (calc_one_sample_task -> path_trace -> material_manager_v3), in float.
#pragma once
#include "caustic.cuh"
#include "shade.cuh"

namespace mrt {

struct PathCounters {
  uint32_t segments;
  uint32_t shadow;
  uint32_t visits;
};

// importance_sampling (material_default.c:41-69): HDRI next-event estimate.
template <class V>
__device__ __forceinline__ void env_nee(const V& S, PathState& P, const Surf& s,
                                        int* status, PathCounters& C) {
  const int k = env_sample(S, P.rng);
  const float4 e = __ldg(S.env_rec0 + k);
  const float3 dir = f3(e.x, e.y, e.z);
  P.d = dir;
  C.shadow++;
  if (any_hit(S, s.p, dir, INFINITY, status, P.rng.s)) return;
  float ct = dot(s.n, dir);
  float pdf = e.w;
  if (pdf <= 0.0f) return;
  const float4 r = __ldg(S.env_rec1 + k);
  float3 rad = f3(r.x, r.y, r.z);
  if (s.mat >= 0) rad = rad * surf_mat(S, s).ao;
  rad = rad * P.power;
  rad = rad * (ct / pdf);
  P.acc = P.acc + rad;
  P.power = P.power * (1.0f - ct);
}

// default_mat (material_default.c:71-92).
template <class V>
__device__ __forceinline__ void default_mat(const V& S, PathState& P, const Surf& s,
                                            int* status, PathCounters& C) {
  float3 direct = compute_light(S, P.rng, s, status, C.shadow);
  float3 caus = caustic_estimate(S, s.p);
  float3 total = direct + caus;
  P.acc = P.acc + (s.color * P.power) * total;
  P.power = P.power * s.color;
  if (S.env_nee) env_nee(S, P, s, status, C);
  P.d = cos_hemisphere(P.rng, s.n);
}

// dielectric_mat (dielectric.c:37-64) with reflected_dielectric_color (:15-33).
template <class V>
__device__ __forceinline__ void dielectric_mat(const V& S, const MaterialD& M, PathState& P,
                                               const Surf& s, int* status, PathCounters& C) {
  if (M.ior > 0.0f) {
    float ct = -dot(unit(P.d), s.n);
    float refl = M.f0 + (1.0f - M.f0) * pow5(1.0f - ct);
    if (refl >= P.rng.next() && M.ior != 1.0f) {
      float3 m = M.roughness > 0.0f ? ggx_sample(P.rng, s.n, M.alpha4) : s.n;
      P.d = unit(P.d - m * (2.0f * dot(P.d, m)));
    } else if (M.transmission == 1.0f) {
      refract(S, M, P, s);
    } else if (M.transmission == 0.0f) {
      default_mat(S, P, s, status, C);
    } else if (M.transmission < P.rng.next()) {
      default_mat(S, P, s, status, C);
    } else {
      refract(S, M, P, s);
    }
  } else {
    default_mat(S, P, s, status, C);
  }
}

// material_manager_v3 (path_trace.c:15-35).
template <class V>
__device__ __forceinline__ void material_manager(const V& S, PathState& P, const Surf& s,
                                                 int* status, PathCounters& C) {
  if (s.mat < 0) {
    default_mat(S, P, s, status, C);
    return;
  }
  const MaterialD& M = surf_mat(S, s);
  if (M.emission_strength > 0.0f)
    P.acc = P.acc + (ld3(M.emission) * M.emission_strength) * P.power;
  if (M.metallic == 1.0f) metallic(M, P, s);
  else if (M.metallic == 0.0f) dielectric_mat(S, M, P, s, status, C);
  else if (M.metallic > P.rng.next()) metallic(M, P, s);
  else dielectric_mat(S, M, P, s, status, C);
}

// Camera ray of calc_one_sample_task (calc_sample.c:44-59) plus the shared
// (render.c:33) or per-pixel sub-pixel offset, and focus.c:31 defocus.
__device__ __forceinline__ void camera_ray(const SceneView& S, PathState& P, uint32_t pixel,
                                           float ox, float oy) {
  float3 orig = ld3(S.cam);
  if (S.defocus_angle > 0.0f) {
    float px, py;
    for (int it = 0; it < 64; ++it) {       // rejection in the unit disk, bounded
      px = -1.0f + P.rng.next() * 2.0f;
      py = -1.0f + P.rng.next() * 2.0f;
      if (px * px + py * py < 1.0f) break;
      px = py = 0.0f;
    }
    orig = orig + ld3(S.defocus_u) * px + ld3(S.defocus_v) * py;
  }
  float fx = (float)(pixel % (uint32_t)S.width) + ox;
  float fy = (float)(pixel / (uint32_t)S.width) + oy;
  P.o = orig;
  P.d = ld3(S.pixel00) + ld3(S.pdu) * fx + ld3(S.pdv) * fy - orig;
}

// path_trace + add_skybox (path_trace.c:37-76). render_mode 2 returns the
// normal colour of the first hit (path_trace_normal, :78-89); render_mode 1
// returns the node-visit count in .x (path_trace_bvh, :91-102).
// Event record of one bounce (debug probe): flat prim id, t, hit point,
// shading normal, then direction, power and radiance after shading.
constexpr int kEventFloats = 20;
constexpr int kMaxEvents = 16;

__device__ __forceinline__ void write_event(float* ev, int k, const SceneView& S, const HitInfo& h,
                                            const Surf& s, const PathState& P) {
  float* e = ev + k * kEventFloats;
  int flat = h.prim >= 0 ? __ldg(S.meta + h.prim).x : (h.prim == kMiss ? -1 : S.planes[-1 - h.prim].meta.x);
  e[0] = (float)flat; e[1] = h.t;
  e[2] = s.p.x; e[3] = s.p.y; e[4] = s.p.z;
  e[5] = s.n.x; e[6] = s.n.y; e[7] = s.n.z;
  e[8] = P.d.x; e[9] = P.d.y; e[10] = P.d.z;
  e[11] = P.power.x; e[12] = P.power.y; e[13] = P.power.z;
  e[14] = P.acc.x; e[15] = P.acc.y; e[16] = P.acc.z;
  e[17] = (float)s.mat;
}

template <class V>
__device__ __forceinline__ float3 trace_path(const V& S, PathState& P, int max_depth,
                                             int render_mode, int* status, PathCounters& C,
                                             float* ev = nullptr) {
  P.power = f3(1.f, 1.f, 1.f);
  P.acc = f3(0.f, 0.f, 0.f);
  P.last_mat = -1;
  if (render_mode != 0) {
    HitInfo h;
    int visits = 0;
    bool hit = closest_hit<true>(S, P.o, P.d, h, visits, status, P.rng.s);
    C.segments++;
    C.visits += visits;
    if (render_mode == 1) {
      if (S.ref_boxes) {          // the reference's count on its own tree
        bool any_leaf;
        const int cnt = ref_visit_count(S, P.o, P.d, any_leaf, status);
        return f3(hit ? (any_leaf ? (float)cnt : 0.0f) : -1.0f, 0.f, 0.f);
      }
      return f3(hit ? (float)visits : -1.0f, 0.f, 0.f);
    }
    if (!hit) return f3(0.f, 0.f, 0.f);
    return make_surf(S, h, P.o, P.d, 2).color;
  }
  int ev_k = 0;
  while (--max_depth >= 0) {
    HitInfo h;
    int visits = 0;
    C.segments++;
    bool hit = closest_hit<true>(S, P.o, P.d, h, visits, status, P.rng.s);
    C.visits += visits;
    if (!hit) {
      float3 bg = background(S, P.d, true);
      if (P.last_mat >= 0) bg = bg * last_hit_ao(S, P);
      P.acc = P.acc + bg * P.power;
      if (ev && ev_k < kMaxEvents) {
        Surf z{};
        z.mat = -1;
        h.prim = kMiss;
        write_event(ev, ev_k, S, h, z, P);
      }
      break;
    }
    Surf s = make_surf(S, h, P.o, P.d, 0);
    P.o = s.p;
    set_last_hit(S, P, s);
    material_manager(S, P, s, status, C);
    if (ev && ev_k < kMaxEvents) write_event(ev, ev_k++, S, h, s, P);
    // Every later term is multiplied by the path power: a path whose power
    // reached exactly zero contributes nothing more.
    if (P.power.x == 0.0f && P.power.y == 0.0f && P.power.z == 0.0f) break;
  }
  return P.acc;
}

// One bounce of path_trace (path_trace.c:58-72) for a path whose state lives
// in P. Returns false when the path ended (miss, depth exhausted, or zero
// power); P.acc then holds its radiance.
template <class V>
__device__ __forceinline__ bool bounce(const V& S, PathState& P, int& depth_left,
                                       int* status, PathCounters& C) {
  HitInfo h;
  int visits = 0;
  C.segments++;
  const bool hit = closest_hit<false>(S, P.o, P.d, h, visits, status, P.rng.s);
  if (!hit) {
    float3 bg = background(S, P.d, true);
    if (P.last_mat >= 0) bg = bg * last_hit_ao(S, P);
    P.acc = P.acc + bg * P.power;
    return false;
  }
  Surf s = make_surf(S, h, P.o, P.d, 0);
  P.o = s.p;
  set_last_hit(S, P, s);
  material_manager(S, P, s, status, C);
  --depth_left;
  if (P.power.x == 0.0f && P.power.y == 0.0f && P.power.z == 0.0f) return false;
  return depth_left > 0;
}

// Pixel of the lin-th path of a sample: 8x4 tiles so that a warp traces
// neighbouring primary rays.
__device__ __forceinline__ uint32_t tile_pixel(uint32_t lin, int W, int H) {
  // 8x4 tiles in row-major tile order; ragged edge tiles fall back to row-major
  const uint32_t tw = 8, th = 4;
  const uint32_t tiles_x = (W + tw - 1) / tw;
  const uint32_t full_h = (H / th) * th;
  const uint32_t full_rows_pixels = full_h * W;
  if (lin < full_rows_pixels && (W % tw) == 0) {
    uint32_t tile = lin / (tw * th), in = lin % (tw * th);
    uint32_t tx = tile % tiles_x, ty = tile / tiles_x;
    return (ty * th + in / tw) * W + tx * tw + in % tw;
  }
  return lin;
}

// Sub-pixel offset of a sample: shared by every pixel of the sample
// (draw_pixels, render.c:33) or per pixel, from the path's own stream.
__device__ __forceinline__ void sample_offset(uint64_t seed, uint32_t sample, int jitter, Rng& rng,
                                              float& ox, float& oy) {
  if (jitter == 0) {
    Rng j{path_seed(seed, 0xFFFFFFFFu, sample)};
    ox = j.next();
    oy = j.next();
  } else {
    ox = rng.next();
    oy = rng.next();
  }
}

}  // namespace mrt
