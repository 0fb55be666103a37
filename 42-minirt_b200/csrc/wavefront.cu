// wavefront.cu — the wavefront form of the path tracer.
//
// Same estimator as the megakernel (path.cuh), split into stages so that the
// traversal kernels run lean (few registers, high occupancy) and the shading
// kernels see material-coherent warps:
//
//   generate : camera paths of one wave into the path-state arrays (SoA)
//   per bounce:
//     extend   : persistent closest-hit for every live path
//     classify : misses add the sky and retire; hits are bucketed by material
//                kind (warp-aggregated appends into per-kind queues) when the
//                queue is longer than the sort threshold
//     sample   : material_manager_v3 up to the point where light visibility
//                matters: emission, metal / dielectric bounces, and for the
//                diffuse branch every shadow ray it needs (point lights,
//                soft-shadow targets, the HDRI importance sample) plus the
//                next cosine-weighted direction, drawing random numbers in
//                the reference's order
//     connect  : persistent any-hit for the shadow-ray queue
//     finish   : the visibility-dependent part of default_mat: Phong point /
//                directional terms with the reference's truncating sums,
//                caustic gather, env NEE weight and power update
//   retire   : accumulates finished paths into the frame
// A whole wave (generate + depth x stages) is captured once in a CUDA graph
// and replayed; kernels read their queue lengths from device counters.
#include <type_traits>
#include <algorithm>
#include <atomic>
#include <vector>

#include "../../include/mrt.h"
#include "kernels.h"
#include "path.cuh"

namespace mrt {

constexpr int kKinds = 4;   // 0 diffuse/default, 1 metal, 2 dielectric, 3 mixed metallic
constexpr int kWfBlock = 128;

// Traversal kernels are capped at 40 registers (12 blocks of 128 per SM):
// measured 1.2 % faster on c1 than the 54-register build, despite a few
// bytes of spills.
// (The quadric and textured instantiations keep the compiler's choice: at
// 40 registers they spill.)
#ifndef MRT_TRAV_MIN_BLOCKS
#define MRT_TRAV_MIN_BLOCKS 12
#endif
constexpr int kTravMinBlocks = MRT_TRAV_MIN_BLOCKS;
// The 8-wide tree's traversal (MRT_BVH_WIDE) measured faster at 64
// registers (8 blocks per SM) than at 40.
template <class V, int kTree>
constexpr int trav_min_blocks() { return V::kQuadrics ? 1 : (kTree == kTreeWide ? 8 : kTravMinBlocks); }

struct WfState {
  // path state, indexed by path slot
  float4* o;          // origin.xyz, pixel (int bits)
  float4* d;          // dir.xyz, remaining bounces (int bits)
  float4* pw;         // power.xyz, last material (int bits)
  float4* acc;        // radiance.xyz, ao of the last hit (the sky on a miss is scaled by it)
  uint64_t* rng;
  float4* hit;        // t, u, v, prim (int bits)
  float4* sp;         // surface point .xyz, material
  float4* sn;         // surface normal .xyz, -
  float4* sc;         // surface colour .xyz, env pdf
  float4* env;        // env radiance * ao .xyz, env cos
  unsigned* vis;      // visible-sample counts, 8 bits per light: word w of path i at
                      // vis[w * capacity + i] holds lights 4w..4w+3
  unsigned* vis_env;  // per path: env visibility (0/1)
  // queues (path slot indices) and counters
  int* q_live[2];     // ping-pong extend queues
  int* q_kind;        // kKinds regions of capacity
  int* q_def;         // default-pending paths for finish
  float4* sh_o;       // shadow ray origin.xyz, tmax
  float4* sh_d;       // shadow ray dir.xyz, tag (see slot_bits)
  uint64_t* sh_key;   // textured scenes: the path's random state at each shadow ray (alpha test)
  int* counters;      // see Cnt
  float4* frame;      // accumulator (W*H)
  int capacity;
  int sh_capacity;
  int rays_per_path;  // shadow rays a diffuse event may emit
  int vis_words;      // ceil(n_lights / 4)
  int slot_bits;      // light-index bits of a shadow ray's tag
};

// A shadow ray's tag (the int bits of sh_d.w): the path slot above
// WfState::slot_bits bits of light index, the all-ones slot being the HDRI
// sample. slot_bits is the fewest bits that hold the scene's light indices
// and that slot (1 with no lights, 10 for the maximum of 1023 lights), so
// path slots stay below 2^(31 - slot_bits): 2^30 for a scene lit by its sky
// alone, 2^21 at the light maximum.
constexpr int kMaxSlotBits = 10;
constexpr int kMaxWfLights = (1 << kMaxSlotBits) - 1;

__host__ __device__ inline int slot_bits_for(int n_lights) {
  int b = 1;
  while ((1 << b) < n_lights + 1) ++b;
  return b;
}

enum Cnt : int {
  C_LIVE0 = 0, C_LIVE1 = 1, C_KIND = 2,          // C_KIND..C_KIND+3
  C_DEF = 6, C_SH = 7, C_WORK = 8, C_WAVE = 9, C_GEN = 10, C_SEG = 11, C_SHADOW = 12,
  C_WORK_SH = 13,      // work counter of connect (runs beside the next extend)
  C_WORK_FIN = 14,     // work counter of finish (after connect, on the same stream)
  C_COUNT = 16
};

struct WfParams {
  uint64_t seed;
  uint32_t sample_base;
  uint64_t total_paths;   // npix * spp of this call
  int jitter;
  int max_bounces;
  int sort_threshold;
};

__device__ __forceinline__ int warp_append(int* counter, bool pred) {
  const unsigned mask = __ballot_sync(__activemask(), pred);
  if (!pred) return -1;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane) - 1u));
}

// ------------------------------------------------------------ generate
__global__ void __launch_bounds__(kWfBlock) wf_generate(SceneView S, WfState W, const WfParams* __restrict__ Pp) {
  const WfParams P = *Pp;
  const uint64_t wave = (uint64_t)W.counters[C_WAVE];
  const uint64_t npix = (uint64_t)S.width * S.height;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < W.capacity; i += gridDim.x * blockDim.x) {
    const uint64_t g = wave * (uint64_t)W.capacity + i;
    const bool live = g < P.total_paths;
    if (live) {
      const uint32_t lin = (uint32_t)(g % npix);
      const uint32_t sample = P.sample_base + (uint32_t)(g / npix);
      uint32_t pixel = lin;
      {
        const uint32_t tw = 8, th = 4;
        const uint32_t tiles_x = (S.width + tw - 1) / tw;
        const uint32_t full = (uint32_t)(S.height / th) * th * S.width;
        if (lin < full && (S.width % tw) == 0) {
          uint32_t tile = lin / (tw * th), in = lin % (tw * th);
          pixel = ((tile / tiles_x) * th + in / tw) * S.width + (tile % tiles_x) * tw + in % tw;
        }
      }
      PathState ps;
      ps.rng.s = path_seed(P.seed, pixel, sample);
      float ox, oy;
      sample_offset(P.seed, sample, P.jitter, ps.rng, ox, oy);
      camera_ray(S, ps, pixel, ox, oy);
      W.o[i] = make_float4(ps.o.x, ps.o.y, ps.o.z, __int_as_float((int)pixel));
      W.d[i] = make_float4(ps.d.x, ps.d.y, ps.d.z, __int_as_float(P.max_bounces));
      W.pw[i] = make_float4(1.f, 1.f, 1.f, __int_as_float(-1));
      W.acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      W.rng[i] = ps.rng.s;
    }
    int slot = warp_append(&W.counters[C_LIVE0], live);
    if (live) W.q_live[0][slot] = i;
  }
}

// --------------------------------------------------------------- extend
template <int kBounceParity, class V, int kTree>
__global__ void __launch_bounds__(kWfBlock, trav_min_blocks<V, kTree>()) wf_extend(V S, WfState W, int* status) {
  const int n = W.counters[kBounceParity ? C_LIVE1 : C_LIVE0];
  const int* q = W.q_live[kBounceParity];
  const int lane = threadIdx.x & 31;
  LocalStack stack;
  while (true) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&W.counters[C_WORK], 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const int k = base + lane;
    if (k < n) {
      const int i = q[k];
      const float4 o = W.o[i], d = W.d[i];
      HitInfo h;
      int visits = 0;
      // textured scenes: the alpha test draws from the path's random state
      const uint64_t akey = V::kTextures ? W.rng[i] : 0;
      bool hit = closest_hit_compact<false, kTree>(S, f3(o.x, o.y, o.z), f3(d.x, d.y, d.z), h, visits, status,
                                                   stack, akey);
      W.hit[i] = make_float4(h.t, h.u, h.v, __int_as_float(hit ? h.prim : kMiss));
    }
  }
}

// retire: add the path radiance into the frame
__device__ __forceinline__ void retire(const WfState& W, int i) {
  const float4 a = W.acc[i];
  const int pixel = __float_as_int(W.o[i].w);
  atomicAdd(W.frame + pixel, make_float4(a.x, a.y, a.z, 1.0f));
}

__device__ __forceinline__ int material_kind(const SceneView& S, int mat) {
  if (mat < 0) return 0;
  const float m = S.mats[mat].metallic;
  if (m == 1.0f) return 1;
  if (m == 0.0f) return S.mats[mat].ior > 0.0f ? 2 : 0;
  return 3;
}

// ------------------------------------------------------------- classify
template <int kBounceParity>
__global__ void __launch_bounds__(kWfBlock) wf_classify(SceneView S, WfState W, const WfParams* __restrict__ Pp) {
  const WfParams P = *Pp;
  const int n = W.counters[kBounceParity ? C_LIVE1 : C_LIVE0];
  const int* q = W.q_live[kBounceParity];
  const bool sort = n >= P.sort_threshold;
  for (int k0 = blockIdx.x * blockDim.x; k0 < n; k0 += gridDim.x * blockDim.x) {
    const int k = k0 + threadIdx.x;
    int i = -1, kind = -1;
    if (k < n) {
      i = q[k];
      const float4 h = W.hit[i];
      const int prim = __float_as_int(h.w);
      if (prim == kMiss) {
        // add_skybox (path_trace.c:37-48): clamped sky, scaled by the last ao
        const float4 d = W.d[i], p = W.pw[i];
        float3 bg = background(S, f3(d.x, d.y, d.z), true);
        const int last = __float_as_int(p.w);
        if (last >= 0) bg = bg * W.acc[i].w;
        float4 a = W.acc[i];
        a.x += bg.x * p.x; a.y += bg.y * p.y; a.z += bg.z * p.z;
        W.acc[i] = a;
        retire(W, i);
      } else {
        int mat;
        if (prim >= 0) mat = __ldg(S.meta + prim).y;
        else mat = S.planes[-1 - prim].meta.y;
        kind = sort ? material_kind(S, mat) : 0;
      }
    }
    for (int c = 0; c < kKinds; ++c) {
      const int slot = warp_append(&W.counters[C_KIND + c], kind == c);
      if (kind == c) W.q_kind[(size_t)c * W.capacity + slot] = i;
    }
  }
}

// --------------------------------------------------------------- sample
// Emits the shadow rays of a diffuse event and records what finish needs.
__device__ __forceinline__ void emit_shadow(const WfState& W, int path, int slot, float3 o, float3 d,
                                            float tmax, int* status, uint64_t key) {
  const int s = atomicAdd(&W.counters[C_SH], 1);
  if (s >= W.sh_capacity) {
    atomicOr(status, ST_QUEUE);
    return;
  }
  W.sh_o[s] = make_float4(o.x, o.y, o.z, tmax);
  W.sh_d[s] = make_float4(d.x, d.y, d.z, __int_as_float((path << W.slot_bits) | slot));
  if (W.sh_key) W.sh_key[s] = key;
}

template <int kBounceParity, class V>
__global__ void __launch_bounds__(kWfBlock) wf_sample(V S, WfState W, const WfParams* __restrict__ Pp, int* status) {
  int cum[kKinds + 1];
  cum[0] = 0;
  for (int c = 0; c < kKinds; ++c) cum[c + 1] = cum[c] + W.counters[C_KIND + c];
  const int n = cum[kKinds];
  int* q_next = W.q_live[kBounceParity ^ 1];
  int* c_next = &W.counters[kBounceParity ? C_LIVE0 : C_LIVE1];
  for (int k0 = blockIdx.x * blockDim.x; k0 < n; k0 += gridDim.x * blockDim.x) {
    const int k = k0 + threadIdx.x;
    bool cont = false, pend = false;
    int i = -1;
    if (k < n) {
      int c = 0;
      while (k >= cum[c + 1]) ++c;
      i = W.q_kind[(size_t)c * W.capacity + (k - cum[c])];
      const float4 o = W.o[i], d = W.d[i], h4 = W.hit[i];
      float4 p4 = W.pw[i];
      PathState ps;
      ps.o = f3(o.x, o.y, o.z);
      ps.d = f3(d.x, d.y, d.z);
      ps.power = f3(p4.x, p4.y, p4.z);
      const float4 a4 = W.acc[i];
      ps.acc = f3(a4.x, a4.y, a4.z);
      ps.rng.s = W.rng[i];
      HitInfo h;
      h.t = h4.x; h.u = h4.y; h.v = h4.z; h.prim = __float_as_int(h4.w);
      const Surf s = make_surf(S, h, ps.o, ps.d, 0);
      ps.o = s.p;
      int depth_left = __float_as_int(d.w) - 1;
      bool diffuse = false;
      // material_manager_v3 (path_trace.c:15-35) with the diffuse branch deferred
      if (s.mat < 0) {
        diffuse = true;
      } else {
        const MaterialD& M = surf_mat(S, s);
        if (M.emission_strength > 0.0f) ps.acc = ps.acc + (ld3(M.emission) * M.emission_strength) * ps.power;
        bool metal;
        if (M.metallic == 1.0f) metal = true;
        else if (M.metallic == 0.0f) metal = false;
        else metal = M.metallic > ps.rng.next();
        if (metal) {
          metallic(M, ps, s);
        } else if (M.ior > 0.0f) {
          const float ct = -dot(unit(ps.d), s.n);
          const float refl = M.f0 + (1.0f - M.f0) * pow5(1.0f - ct);
          if (refl >= ps.rng.next() && M.ior != 1.0f) {
            const float3 m = M.roughness > 0.0f ? ggx_sample(ps.rng, s.n, M.alpha4) : s.n;
            ps.d = unit(ps.d - m * (2.0f * dot(ps.d, m)));
          } else if (M.transmission == 1.0f) {
            refract(S, M, ps, s);
          } else if (M.transmission == 0.0f) {
            diffuse = true;
          } else if (M.transmission < ps.rng.next()) {
            diffuse = true;
          } else {
            refract(S, M, ps, s);
          }
        } else {
          diffuse = true;
        }
      }
      if (diffuse) {
        // default_mat (material_default.c:71-92): shadow rays of compute_light
        // (light order, soft-shadow targets drawn now), the HDRI sample, the
        // next direction; visibility-dependent terms are applied in finish.
        for (int l = 0; l < S.n_lights; ++l) {
          const LightD L = S.lights[l];
          const float3 lp = ld3(L.pos);
          if (L.type == 0) {
            if (L.radius == 0.0f || L.shadow_sample <= 1) {
              const float3 to = lp - s.p;
              emit_shadow(W, i, l, s.p, unit(to), sqrtf(len2(to)), status, ps.rng.s);
            } else {
              for (int t = 0; t < L.shadow_sample; ++t) {
                const float3 tgt = lp + rnd_in_unit_sphere(ps.rng) * L.radius;
                const float3 to = tgt - s.p;
                emit_shadow(W, i, l, s.p, unit(to), sqrtf(len2(to)), status, ps.rng.s);
              }
            }
          } else {
            emit_shadow(W, i, l, s.p, unit(-lp), INFINITY, status, ps.rng.s);
          }
        }
        for (int w = 0; w < W.vis_words; ++w) W.vis[(size_t)w * W.capacity + i] = 0u;
        W.vis_env[i] = 0u;
        float env_pdf = 0.f, env_ct = 0.f;
        float3 env_rad = f3(0.f, 0.f, 0.f);
        if (S.env_nee) {
          const int kk = env_sample(S, ps.rng);
          const float4 e = __ldg(S.env_rec0 + kk);
          const float3 dir = f3(e.x, e.y, e.z);
          env_ct = dot(s.n, dir);
          env_pdf = e.w;
          const float4 r = __ldg(S.env_rec1 + kk);
          env_rad = f3(r.x, r.y, r.z);
          if (s.mat >= 0) env_rad = env_rad * surf_mat(S, s).ao;
          emit_shadow(W, i, (1 << W.slot_bits) - 1, s.p, dir, INFINITY, status, ps.rng.s);
        }
        ps.d = cos_hemisphere(ps.rng, s.n);
        W.sp[i] = make_float4(s.p.x, s.p.y, s.p.z, __int_as_float(s.mat));
        W.sn[i] = make_float4(s.n.x, s.n.y, s.n.z, 0.f);
        W.sc[i] = make_float4(s.color.x, s.color.y, s.color.z, env_pdf);
        W.env[i] = make_float4(env_rad.x, env_rad.y, env_rad.z, env_ct);
        pend = true;
      }
      p4 = make_float4(ps.power.x, ps.power.y, ps.power.z, __int_as_float(s.mat));
      W.pw[i] = p4;
      // the ao of this hit scales the sky if the next segment misses
      W.acc[i] = make_float4(ps.acc.x, ps.acc.y, ps.acc.z, s.mat >= 0 ? surf_mat(S, s).ao : 1.0f);
      W.d[i] = make_float4(ps.d.x, ps.d.y, ps.d.z, __int_as_float(depth_left));
      W.o[i] = make_float4(ps.o.x, ps.o.y, ps.o.z, o.w);
      W.rng[i] = ps.rng.s;
      if (!pend) {
        const bool dead = ps.power.x == 0.0f && ps.power.y == 0.0f && ps.power.z == 0.0f;
        cont = depth_left > 0 && !dead;
        if (!cont) retire(W, i);
      } else {
        // a diffuse path continues whatever its shadow rays find: its next
        // segment is traced while connect and finish complete this bounce
        cont = depth_left > 0;
      }
    }
    const int slot = warp_append(c_next, cont);
    if (cont) q_next[slot] = i;
    const int ds = warp_append(&W.counters[C_DEF], pend);
    if (pend) W.q_def[ds] = i;
  }
}

// -------------------------------------------------------------- connect
template <class V, int kTree>
__global__ void __launch_bounds__(kWfBlock, trav_min_blocks<V, kTree>()) wf_connect(V S, WfState W, int* status) {
  const int n = min(W.counters[C_SH], W.sh_capacity);
  const int lane = threadIdx.x & 31;
  LocalStack stack;
  while (true) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&W.counters[C_WORK_SH], 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const int k = base + lane;
    if (k < n) {
      const float4 o = W.sh_o[k], d = W.sh_d[k];
      const uint64_t akey = V::kTextures ? W.sh_key[k] : 0;
      const bool blocked = any_hit_compact<kTree>(S, f3(o.x, o.y, o.z), f3(d.x, d.y, d.z), o.w, status, stack, akey);
      if (!blocked) {
        const int tag = __float_as_int(d.w);
        const int env_slot = (1 << W.slot_bits) - 1;
        const int path = tag >> W.slot_bits, slot = tag & env_slot;
        if (slot == env_slot) W.vis_env[path] = 1u;
        else atomicAdd(&W.vis[(size_t)(slot >> 2) * W.capacity + path], 1u << (8 * (slot & 3)));
      }
    }
  }
}

// --------------------------------------------------------------- finish
// finish: persistent, 7 blocks per SM (72 registers), warps taking 32
// diffuse events at a time from a work counter. The caustic gather makes
// event costs uneven (dense caustic regions walk far more of the photon
// tree); against a grid-stride loop at the compiler's 113 registers this
// measured c2 282 -> 339 Mpaths/s and c2p 173 -> 236 on B200 (6 blocks:
// 339 / 228, 5: 326 / 195, 8: 334 with 324 B of spills).
constexpr int kFinishMinBlocks = 7;
__device__ __forceinline__ void finish_one(const SceneView& S, const WfState& W, int i);

__global__ void __launch_bounds__(kWfBlock, kFinishMinBlocks) wf_finish(SceneView S, WfState W) {
  const int n = W.counters[C_DEF];
  const int lane = threadIdx.x & 31;
  while (true) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&W.counters[C_WORK_FIN], 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const int k = base + lane;
    if (k < n) finish_one(S, W, W.q_def[k]);
  }
}

// Direct light (with connect's visibility), the caustic gather and the
// sky NEE term of one diffuse event, then retirement of a finished path.
__device__ __forceinline__ void finish_one(const SceneView& S, const WfState& W, int i) {
  {
    {
      const float4 sp = W.sp[i], sn = W.sn[i], sc = W.sc[i], ev = W.env[i];
      const float3 p = f3(sp.x, sp.y, sp.z), nrm = f3(sn.x, sn.y, sn.z), col = f3(sc.x, sc.y, sc.z);
      float4 pw4 = W.pw[i];
      float3 power = f3(pw4.x, pw4.y, pw4.z);
      float4 a4 = W.acc[i];
      float3 acc = f3(a4.x, a4.y, a4.z);
      // compute_light_v2 with the visibility found by connect
      float lc0 = 0.f, lc1 = 0.f, lc2 = 0.f;
      if (S.n_lights) {
        const float3 view = unit(ld3(S.cam) - p);
        unsigned vis = 0u;
        for (int l = 0; l < S.n_lights; ++l) {
          const LightD L = S.lights[l];
          const float3 lp = ld3(L.pos);
          if ((l & 3) == 0) vis = W.vis[(size_t)(l >> 2) * W.capacity + i];
          const int seen = (int)((vis >> (8 * (l & 3))) & 255u);
          if (L.type == 0) {
            float sf;
            bool ok;
            if (L.radius == 0.0f || L.shadow_sample <= 1) { sf = 1.0f; ok = seen > 0; }
            else { sf = (float)seen / (float)L.shadow_sample; ok = sf > 0.0f; }
            if (!ok) continue;
            const float3 ld = unit(lp - p);
            const float ndl = dot(nrm, ld);
            if (ndl > 0.0f) {
              const float di = L.brightness * ndl * sf;
              lc0 = floorf(lc0 + L.color[0] * di);
              lc1 = floorf(lc1 + L.color[1] * di);
              lc2 = floorf(lc2 + L.color[2] * di);
              const float rdv = fmaxf(dot(reflect_v(-ld, nrm), view), 0.0f);
              const float spec = powf(rdv, 64.0f) * sf;
              lc0 = floorf(lc0 + L.color[0] * L.brightness * spec);
              lc1 = floorf(lc1 + L.color[1] * L.brightness * spec);
              lc2 = floorf(lc2 + L.color[2] * L.brightness * spec);
            }
          } else {
            if (seen == 0) continue;
            const float3 ld = -lp;
            const float ndl = dot(nrm, ld);
            if (ndl > 0.0f) {
              lc0 = floorf(lc0 + L.color[0] * L.brightness * ndl);
              lc1 = floorf(lc1 + L.color[1] * L.brightness * ndl);
              lc2 = floorf(lc2 + L.color[2] * L.brightness * ndl);
              const float rdv = fmaxf(dot(reflect_v(-ld, nrm), view), 0.0f);
              const float spec = powf(rdv, 64.0f);
              lc0 = floorf(lc0 + L.color[0] * L.brightness * spec);
              lc1 = floorf(lc1 + L.color[1] * L.brightness * spec);
              lc2 = floorf(lc2 + L.color[2] * L.brightness * spec);
            }
          }
        }
      }
      const float3 direct = f3(lc0 / 255.0f, lc1 / 255.0f, lc2 / 255.0f);
      const float3 caus = caustic_estimate(S, p);
      acc = acc + (col * power) * (direct + caus);
      power = power * col;
      if (S.env_nee && W.vis_env[i] && sc.w > 0.0f) {
        const float3 rad = f3(ev.x, ev.y, ev.z) * power * (ev.w / sc.w);
        acc = acc + rad;
        power = power * (1.0f - ev.w);
      }
      W.acc[i] = make_float4(acc.x, acc.y, acc.z, a4.w);
      W.pw[i] = make_float4(power.x, power.y, power.z, pw4.w);
      // the path continues (sample queued it) unless this was its last bounce
      if (__float_as_int(W.d[i].w) <= 0) retire(W, i);
    }
  }
}

// Resets the counters of bounce parity kBounceParity once its connect and
// finish are done: its consumed live queue, the kind queues, the diffuse and
// shadow-ray queues.
template <int kBounceParity>
__global__ void wf_reset(WfState W) {
  if (threadIdx.x == 0) {
    W.counters[kBounceParity ? C_LIVE1 : C_LIVE0] = 0;   // the queue extend consumed
    for (int c = 0; c < kKinds; ++c) W.counters[C_KIND + c] = 0;
    W.counters[C_DEF] = 0;
    W.counters[C_SH] = 0;
  }
}

__global__ void wf_work_reset(WfState W) {
  if (threadIdx.x == 0) W.counters[C_WORK] = 0;
}

__global__ void wf_sh_work_reset(WfState W) {
  if (threadIdx.x == 0) {
    W.counters[C_WORK_SH] = 0;
    W.counters[C_WORK_FIN] = 0;
  }
}

__global__ void wf_wave_begin(WfState W) {
  if (threadIdx.x == 0) {
    W.counters[C_LIVE0] = 0;
    W.counters[C_LIVE1] = 0;
    for (int c = 0; c < kKinds; ++c) W.counters[C_KIND + c] = 0;
    W.counters[C_DEF] = 0;
    W.counters[C_SH] = 0;
    W.counters[C_WORK] = 0;
    W.counters[C_WORK_SH] = 0;
    W.counters[C_WORK_FIN] = 0;
  }
}

__global__ void wf_wave_end(WfState W) {
  if (threadIdx.x == 0) W.counters[C_WAVE] += 1;
}

}  // namespace mrt

// ----------------------------------------------------------------- host

using namespace mrt;

struct WfHost {
  int capacity = 0, sh_capacity = 0;
  int vis_words = 0;
  int sms = 0;
  WfState st{};
  WfParams* dparams = nullptr;
  std::vector<void*> allocs;
  cudaGraphExec_t graph = nullptr;
  // the side stream of each bounce's connect and finish, which run beside
  // the next bounce's extend; fork / join events
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  int graph_bounces = -1;
  unsigned graph_launches = 0;   // kernels per replay of the graph
  uint64_t graph_key = 0;
};

static cudaError_t wf_alloc(WfHost* H, int capacity, int n_lights, bool env) {
  for (void* p : H->allocs) cudaFree(p);
  H->allocs.clear();
  if (H->graph) { cudaGraphExecDestroy(H->graph); H->graph = nullptr; }
  H->graph_bounces = -1;
  H->sh_capacity = 0;          // the shadow queue went with the other buffers
  const int rays = n_lights * 1 + (env ? 1 : 0);
  const int vis_words = std::max(1, (n_lights + 3) / 4);
  H->capacity = capacity;
  H->vis_words = vis_words;
  WfState& s = H->st;
  s = WfState{};
  s.capacity = capacity;
  s.rays_per_path = rays;
  s.vis_words = vis_words;
  auto A = [&](void** p, size_t bytes) -> cudaError_t {
    cudaError_t e = cudaMalloc(p, bytes > 0 ? bytes : 16);
    if (e == cudaSuccess) H->allocs.push_back(*p);
    return e;
  };
  const size_t n = (size_t)capacity;
  cudaError_t e;
#define AL(field, bytes) if ((e = A((void**)&s.field, (bytes))) != cudaSuccess) return e
  AL(o, n * 16); AL(d, n * 16); AL(pw, n * 16); AL(acc, n * 16); AL(rng, n * 8); AL(hit, n * 16);
  AL(sp, n * 16); AL(sn, n * 16); AL(sc, n * 16); AL(env, n * 16);
  AL(vis, n * 4 * vis_words); AL(vis_env, n * 4);
  AL(q_live[0], n * 4); AL(q_live[1], n * 4); AL(q_kind, n * 4 * kKinds); AL(q_def, n * 4);
  AL(counters, sizeof(int) * C_COUNT);
  if ((e = A((void**)&H->dparams, sizeof(WfParams))) != cudaSuccess) return e;
#undef AL
  return cudaMemset(s.counters, 0, sizeof(int) * C_COUNT);
}

// Shadow-ray queue of sh_cap rays; keys: the per-ray random state the alpha
// test of textured scenes needs.
static cudaError_t wf_shadow_alloc(WfHost* H, size_t sh_cap, bool keys) {
  if ((size_t)H->sh_capacity >= sh_cap && (!keys || H->st.sh_key)) return cudaSuccess;
  sh_cap = std::max(sh_cap, (size_t)H->sh_capacity);
  cudaError_t e;
  float4 *o = nullptr, *d = nullptr;
  uint64_t* key = nullptr;
  if ((e = cudaMalloc(&o, sh_cap * 16)) != cudaSuccess) return e;
  H->allocs.push_back(o);
  if ((e = cudaMalloc(&d, sh_cap * 16)) != cudaSuccess) return e;
  H->allocs.push_back(d);
  if (keys || H->st.sh_key) {
    if ((e = cudaMalloc(&key, sh_cap * 8)) != cudaSuccess) return e;
    H->allocs.push_back(key);
  }
  H->st.sh_o = o;
  H->st.sh_d = d;
  H->st.sh_key = key;
  H->st.sh_capacity = (int)sh_cap;
  H->sh_capacity = (int)sh_cap;
  if (H->graph) { cudaGraphExecDestroy(H->graph); H->graph = nullptr; }
  return cudaSuccess;
}

// One wave: generate, then per bounce classify and sample on the main
// stream, connect and finish (the shadow rays of the bounce and the terms
// they decide) on the side stream while the main stream traces the next
// bounce's extension rays (extend), joined before the next classify, which
// reads the power and radiance finish updates. The two branches touch
// disjoint path state: extend writes the hit records, finish the power and
// radiance, connect the visibility words.
template <class VT>
static void wf_enqueue_wave_t(WfHost* H, const VT& v, const WfParams& P, int* status,
                              cudaStream_t st, unsigned* launches) {
  const WfParams* dP = H->dparams;
  const int gen_blocks = std::max(1, std::min((H->capacity + kWfBlock - 1) / kWfBlock, H->sms * 16));
  const int pers = H->sms * kTravMinBlocks, pers_wide = H->sms * 8;
  const WfState s = H->st;
  cudaStream_t sd = H->side;
  unsigned n = 0;
  // the tree's own traversal kernels (the wide tree: SceneView only)
  bool wide = false;
  if constexpr (!VT::kQuadrics) wide = v.wnodes != nullptr;
  auto extend = [&](int par) {
    wf_work_reset<<<1, 32, 0, st>>>(s);
    if constexpr (!VT::kQuadrics) {
      if (wide) {
        if (par) wf_extend<1, VT, kTreeWide><<<pers_wide, kWfBlock, 0, st>>>(v, s, status);
        else wf_extend<0, VT, kTreeWide><<<pers_wide, kWfBlock, 0, st>>>(v, s, status);
        n += 2;
        return;
      }
    }
    if (par) wf_extend<1, VT, kTreeBinary><<<pers, kWfBlock, 0, st>>>(v, s, status);
    else wf_extend<0, VT, kTreeBinary><<<pers, kWfBlock, 0, st>>>(v, s, status);
    n += 2;
  };
  auto connect = [&]() {
    if constexpr (!VT::kQuadrics) {
      if (wide) {
        wf_connect<VT, kTreeWide><<<pers_wide, kWfBlock, 0, sd>>>(v, s, status);
        return;
      }
    }
    wf_connect<VT, kTreeBinary><<<pers, kWfBlock, 0, sd>>>(v, s, status);
  };
  wf_wave_begin<<<1, 32, 0, st>>>(s);
  wf_generate<<<gen_blocks, kWfBlock, 0, st>>>(v, s, dP);
  n += 2;
  extend(0);
  for (int b = 0; b < P.max_bounces; ++b) {
    const int par = b & 1;
    if (par) {
      wf_classify<1><<<gen_blocks, kWfBlock, 0, st>>>(v, s, dP);
      wf_sample<1, VT><<<gen_blocks, kWfBlock, 0, st>>>(v, s, dP, status);
    } else {
      wf_classify<0><<<gen_blocks, kWfBlock, 0, st>>>(v, s, dP);
      wf_sample<0, VT><<<gen_blocks, kWfBlock, 0, st>>>(v, s, dP, status);
    }
    cudaEventRecord(H->ev_fork, st);
    cudaStreamWaitEvent(sd, H->ev_fork, 0);
    wf_sh_work_reset<<<1, 32, 0, sd>>>(s);
    connect();
    wf_finish<<<H->sms * kFinishMinBlocks, kWfBlock, 0, sd>>>(v, s);
    cudaEventRecord(H->ev_join, sd);
    n += 5;
    if (b + 1 < P.max_bounces) extend(par ^ 1);
    cudaStreamWaitEvent(st, H->ev_join, 0);
    if (par) wf_reset<1><<<1, 32, 0, st>>>(s);
    else wf_reset<0><<<1, 32, 0, st>>>(s);
    n += 1;
  }
  // paths still live after the last bounce retire with what they gathered
  wf_wave_end<<<1, 32, 0, st>>>(s);
  n += 1;
  if (launches) *launches += n;
}

static void wf_enqueue_wave(WfHost* H, const SceneView& v, const WfParams& P, int* status,
                            cudaStream_t st, unsigned* launches) {
  with_view(v, [&](const auto& vt) {
    wf_enqueue_wave_t(H, vt, P, status, st, launches);
    return 0;
  });
}

__global__ void wf_retire_remaining(WfState W, int parity_count_index, int parity) {
  const int n = W.counters[parity_count_index];
  const int* q = W.q_live[parity];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) retire(W, q[k]);
}

size_t wf_device_bytes(const WfHost* H);

// Device bytes of all wavefront states of the process (many contexts, as in a
// batch of scenes, each keep theirs): their default capacities together stay
// within kWfTotalBudget.
static std::atomic<size_t> g_wf_bytes{0};
constexpr size_t kWfTotalBudget = 48ull << 30;

int wf_render(WfHost* H, const SceneView& v, const LaunchParams& L, int spp, int capacity,
              int sort_threshold, int use_graph, float4* frame, int* status, cudaStream_t st,
              unsigned* launches, const char** err) {
  if (!H->sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&H->sms, cudaDevAttrMultiProcessorCount, dev);
  }
  if (!H->side) {
    cudaError_t e0 = cudaStreamCreateWithFlags(&H->side, cudaStreamNonBlocking);
    if (e0 == cudaSuccess) e0 = cudaEventCreateWithFlags(&H->ev_fork, cudaEventDisableTiming);
    if (e0 == cudaSuccess) e0 = cudaEventCreateWithFlags(&H->ev_join, cudaEventDisableTiming);
    if (e0 != cudaSuccess) { *err = cudaGetErrorString(e0); return MRT_ERR_CUDA; }
  }
  const uint64_t npix = (uint64_t)v.width * v.height;
  const uint64_t total = npix * (uint64_t)spp;
  if (total == 0) return MRT_OK;
  if (v.n_lights > kMaxWfLights) {
    *err = "wavefront form supports up to 1023 lights (use the megakernel)";
    return MRT_ERR_INVALID;
  }
  // shadow rays per diffuse event: hard lights 1, soft lights shadow_sample, env 1
  size_t per_path = v.env_nee ? 1 : 0;
  {
    std::vector<LightD> ls(v.n_lights);
    if (v.n_lights) cudaMemcpy(ls.data(), v.lights, sizeof(LightD) * v.n_lights, cudaMemcpyDeviceToHost);
    for (auto& Lh : ls) {
      int k = (Lh.type == 0 && Lh.radius != 0.0f && Lh.shadow_sample > 1) ? Lh.shadow_sample : 1;
      if (k > 255) { *err = "wavefront form supports up to 255 soft-shadow samples"; return MRT_ERR_INVALID; }
      per_path += k;
    }
  }
  // Path slots: by default every path of the call at once, up to 2^25 and
  // within min(16 GiB, a quarter of free memory) of path state and shadow
  // queue. Fewer, larger waves mean fewer queue drains (the last bounces of
  // a wave run with few live paths): on c1 (33 M paths per 16-spp step) one
  // wave of 2^25 slots traced 511 Mpaths/s against 381 with 2^22.
  const int slot_bits = slot_bits_for(v.n_lights);
  if (capacity <= 0) {
    const size_t per_slot = 16 * 10 + 8 + 4 * (4 + std::max(1, (v.n_lights + 3) / 4)) + 4 * kKinds +
                            per_path * (32 + (v.has_textures ? 8 : 0));
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t have = wf_device_bytes(H);
    const size_t others = g_wf_bytes.load() - std::min(g_wf_bytes.load(), have);
    const size_t budget = std::min<size_t>({16ull << 30, (free_b + have) / 4,
                                            kWfTotalBudget - std::min(kWfTotalBudget, others)});
    capacity = (int)std::max<size_t>(1 << 20, std::min<size_t>(1 << 25, budget / per_slot));
  }
  capacity = std::min(capacity, 1 << (31 - slot_bits));
  capacity = (int)std::min<uint64_t>((uint64_t)capacity, std::max<uint64_t>(total, 1024));
  cudaError_t e = cudaSuccess;
  const size_t before = wf_device_bytes(H);
  if (H->capacity != capacity || H->vis_words != std::max(1, (v.n_lights + 3) / 4))
    e = wf_alloc(H, capacity, v.n_lights, v.env_nee);
  if (e == cudaSuccess) e = wf_shadow_alloc(H, std::max<size_t>(per_path * capacity, 1024), v.has_textures != 0);
  g_wf_bytes += wf_device_bytes(H);
  g_wf_bytes -= before;
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return MRT_ERR_OOM;
  }
  H->st.frame = frame;
  H->st.slot_bits = slot_bits;
  WfParams P{};
  P.seed = L.seed;
  P.sample_base = L.sample_base;
  P.total_paths = total;
  P.jitter = L.jitter;
  P.max_bounces = L.max_bounces;
  P.sort_threshold = sort_threshold > 0 ? sort_threshold : 1 << 16;
  const uint64_t waves = (total + capacity - 1) / capacity;
  // this call's parameters and a zero wave counter, ahead of the (re)played graph
  static thread_local WfParams host_params;
  host_params = P;
  if ((e = cudaMemcpyAsync(H->dparams, &host_params, sizeof(WfParams), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
      (e = cudaMemsetAsync(H->st.counters + C_WAVE, 0, sizeof(int), st)) != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return MRT_ERR_CUDA;
  }
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { *err = cudaGetErrorString(e); return MRT_ERR_CUDA; }
  // the graph bakes in the scene view, buffers and bounce count
  uint64_t key = 1469598103934665603ull;
  {
    const unsigned char* b = reinterpret_cast<const unsigned char*>(&v);
    for (size_t k = 0; k < sizeof(SceneView); ++k) key = (key ^ b[k]) * 1099511628211ull;
    key ^= ((uint64_t)P.max_bounces << 48) ^ (uint64_t)(uintptr_t)status ^ (uint64_t)(uintptr_t)frame;
  }
  if (use_graph) {
    if (!H->graph || H->graph_key != key) {
      if (H->graph) { cudaGraphExecDestroy(H->graph); H->graph = nullptr; }
      cudaGraph_t g;
      if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) { *err = cudaGetErrorString(e); return MRT_ERR_CUDA; }
      unsigned count = 1;   // wf_retire_remaining below
      wf_enqueue_wave(H, v, P, status, st, &count);
      // the paths alive after max_bounces retire (parity of the last bounce)
      const int par = P.max_bounces & 1;
      wf_retire_remaining<<<H->sms * 4, kWfBlock, 0, st>>>(H->st, par ? C_LIVE1 : C_LIVE0, par);
      if ((e = cudaStreamEndCapture(st, &g)) != cudaSuccess) { *err = cudaGetErrorString(e); return MRT_ERR_CUDA; }
      e = cudaGraphInstantiate(&H->graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) { *err = cudaGetErrorString(e); return MRT_ERR_CUDA; }
      H->graph_key = key;
      H->graph_bounces = P.max_bounces;
      H->graph_launches = count;
    }
    for (uint64_t w = 0; w < waves; ++w) {
      if ((e = cudaGraphLaunch(H->graph, st)) != cudaSuccess) { *err = cudaGetErrorString(e); return MRT_ERR_CUDA; }
      if (launches) *launches += H->graph_launches;
    }
  } else {
    for (uint64_t w = 0; w < waves; ++w) {
      wf_enqueue_wave(H, v, P, status, st, launches);
      const int par = P.max_bounces & 1;
      wf_retire_remaining<<<H->sms * 4, kWfBlock, 0, st>>>(H->st, par ? C_LIVE1 : C_LIVE0, par);
      if (launches) *launches += 1;
    }
    if ((e = cudaGetLastError()) != cudaSuccess) { *err = cudaGetErrorString(e); return MRT_ERR_CUDA; }
  }
  return MRT_OK;
}

WfHost* wf_create() { return new WfHost(); }

size_t wf_device_bytes(const WfHost* H) {
  if (!H) return 0;
  const size_t cap = (size_t)H->capacity, sh = (size_t)H->sh_capacity;
  return cap * (16 * 10 + 8 + 4 * (4 + H->vis_words) + 4 * kKinds) + sh * (H->st.sh_key ? 40 : 32);
}

void wf_destroy(WfHost* H) {
  if (!H) return;
  g_wf_bytes -= wf_device_bytes(H);
  for (void* p : H->allocs) cudaFree(p);
  if (H->graph) cudaGraphExecDestroy(H->graph);
  if (H->side) cudaStreamDestroy(H->side);
  if (H->ev_fork) cudaEventDestroy(H->ev_fork);
  if (H->ev_join) cudaEventDestroy(H->ev_join);
  delete H;
}
