// render_kernels.cuh — the megakernel forms and the single-path probes as
// templates on the scene view type, with one launcher template per kernel.
//
// Megakernel: one thread = one camera path (pixel, sample), all bounces in
// registers, one vector atomic into the float4 accumulator at the end.
// Threads are laid out so that a warp covers an 8x4 pixel tile of one
// sample (coherent primary rays), and samples vary slowest.
//
// Each launcher template is instantiated for one view type and one kernel
// group per object file (render_inst.cu, compiled once per combination), so
// the heavy instantiations compile in parallel; render.cu dispatches on the
// scene's view type at run time.
#pragma once
#include <algorithm>

#include "kernels.h"
#include "path.cuh"
#include "render_views.h"

namespace mrt {

template <bool kCount, int kBlock, class V>
__global__ void __launch_bounds__(kBlock) megakernel(V S, LaunchParams L, float4* accum,
                                                   int* depth, int* status,
                                                   unsigned long long* counters) {
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  PathCounters C{0, 0, 0};
  if (idx < L.n_paths) {
    const uint32_t npix = (uint32_t)S.width * (uint32_t)S.height;
    const uint32_t lin = (uint32_t)(idx % npix);
    const uint32_t sample = L.sample_base + (uint32_t)(idx / npix);
    const uint32_t pixel = tile_pixel(lin, S.width, S.height);
    PathState P;
    P.rng.s = path_seed(L.seed, pixel, sample);
    float ox, oy;
    if (L.has_offset) { ox = L.ox; oy = L.oy; }
    else sample_offset(L.seed, sample, L.jitter, P.rng, ox, oy);
    camera_ray(S, P, pixel, ox, oy);
    float3 c = trace_path(S, P, L.max_bounces, L.render_mode, status, C);
    if (L.render_mode == 1) {
      depth[pixel] = (int)c.x;
    } else {
      atomicAdd(accum + pixel, make_float4(c.x, c.y, c.z, 1.0f));
    }
  }
  if (kCount) {
    // warp-aggregated counters
    unsigned long long seg = C.segments, sh = C.shadow, vi = C.visits;
    for (int off = 16; off > 0; off >>= 1) {
      seg += __shfl_down_sync(0xffffffffu, seg, off);
      sh += __shfl_down_sync(0xffffffffu, sh, off);
      vi += __shfl_down_sync(0xffffffffu, vi, off);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(counters + 0, seg);
      atomicAdd(counters + 1, sh);
      atomicAdd(counters + 2, vi);
    }
  }
}

// A finished path's radiance into the frame: the float4 accumulator, or the
// fixed-point one of the differentiable forward (LaunchParams::accum_fx).
__device__ __forceinline__ void add_path(const LaunchParams& L, float4* accum, uint32_t pixel, float3 c) {
  if (L.accum_fx) {
    unsigned long long* q = L.accum_fx + 3 * (size_t)pixel;
    const float v[3] = {c.x, c.y, c.z};
    for (int k = 0; k < 3; ++k) {
      double x = (double)v[k] * kFrameFxScale;
      if (!(x == x)) x = 0.0;
      x = fmin(fmax(x, -4.0e18), 4.0e18);
      const long long iq = __double2ll_rn(x);
      if (iq) atomicAdd(q + k, (unsigned long long)iq);
    }
  } else {
    atomicAdd(accum + pixel, make_float4(c.x, c.y, c.z, 1.0f));
  }
}

// Persistent megakernel with path regeneration: every lane advances its path
// by one bounce per loop iteration; lanes whose path ended take the next path
// index (one atomic per warp for all idle lanes), so warps stay full until
// the launch runs out of paths.
// The regenerating and batch megakernels run at 44 registers per thread:
// the whole path loop spills to local memory, which stays in L1, and the SM
// keeps up to 46 warps of latency-bound traversal in flight instead of 16 at
// the compiler's 128. Measured on B200 (regenerating megakernel, Mpaths/s,
// 128 / 96 / 64 / 44 / 40 / 32 registers): c1 235 / 278 / 369 / 401 / 410 /
// 384, c4 480 / 558 / 682 / 740 / 734 / 700, c0 4,288 / 4,608 / 5,742 /
// 6,050 / 5,607 / 5,532, c2 81 / 90 / 97 / 98 / 103 / 65; the batch
// megakernel on c3's 64 scenes 500 -> 703 (64 registers: 712). The plain
// megakernel keeps the compiler's choice: it is the untuned baseline form.
constexpr int kMegaRegs = 44;

template <int kBlock, class V>
__global__ void __maxnreg__(kMegaRegs) megakernel_regen(V S, LaunchParams L, float4* accum,
                                                        int* status, unsigned long long* work) {
  const uint32_t npix = (uint32_t)S.width * (uint32_t)S.height;
  const int lane = threadIdx.x & 31;
  PathCounters C{0, 0, 0};
  PathState P;
  int depth_left = 0;
  uint32_t pixel = 0;
  bool active = false, done = false;
  while (true) {
    const bool need = !active && !done;
    const unsigned need_mask = __ballot_sync(0xffffffffu, need);
    if (need_mask) {
      unsigned long long base = 0;
      const int leader = __ffs(need_mask) - 1;
      if (lane == leader) base = atomicAdd(work, (unsigned long long)__popc(need_mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const uint64_t idx = base + __popc(need_mask & ((1u << lane) - 1u));
        if (idx >= L.n_paths) {
          done = true;
        } else {
          const uint32_t lin = (uint32_t)(idx % npix);
          const uint32_t sample = L.sample_base + (uint32_t)(idx / npix);
          pixel = tile_pixel(lin, S.width, S.height);
          P.rng.s = path_seed(L.seed, pixel, sample);
          float ox, oy;
          sample_offset(L.seed, sample, L.jitter, P.rng, ox, oy);
          camera_ray(S, P, pixel, ox, oy);
          P.power = f3(1.f, 1.f, 1.f);
          P.acc = f3(0.f, 0.f, 0.f);
          P.last_mat = -1;
          depth_left = L.max_bounces;
          active = depth_left > 0;
          if (!active) add_path(L, accum, pixel, f3(0.f, 0.f, 0.f));
        }
      }
    }
    if (__all_sync(0xffffffffu, done)) break;
    if (active) {
      if (!bounce(S, P, depth_left, status, C)) {
        active = false;
        add_path(L, accum, pixel, P.acc);
      }
    }
  }
}

// Multi-scene batch: one persistent launch over the paths of many scenes.
// Scenes are ordered longest-first by the host (LPT); path index g maps to
// the scene whose [start, start + paths) range holds it (binary search over
// <= a few hundred prefix sums). Otherwise the regenerating loop above.
template <int kBlock, class V>
__global__ void __maxnreg__(kMegaRegs) megakernel_batch(const SceneView* __restrict__ views,
                                                           const BatchItem* __restrict__ items,
                                                           int n_items, uint64_t total,
                                                           int* status, unsigned long long* work) {
  const int lane = threadIdx.x & 31;
  PathCounters C{0, 0, 0};
  PathState P;
  int depth_left = 0, item = 0;
  uint32_t pixel = 0;
  bool active = false, done = false;
  while (true) {
    const bool need = !active && !done;
    const unsigned need_mask = __ballot_sync(0xffffffffu, need);
    if (need_mask) {
      unsigned long long base = 0;
      const int leader = __ffs(need_mask) - 1;
      if (lane == leader) base = atomicAdd(work, (unsigned long long)__popc(need_mask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const uint64_t g = base + __popc(need_mask & ((1u << lane) - 1u));
        if (g >= total) {
          done = true;
        } else {
          int lo = 0, hi = n_items - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (items[mid].start <= g) lo = mid; else hi = mid - 1;
          }
          item = lo;
          const BatchItem it = items[item];
          const V& S = static_cast<const V&>(views[it.view]);
          const uint64_t idx = g - it.start;
          const uint32_t npix = (uint32_t)S.width * (uint32_t)S.height;
          const uint32_t lin = (uint32_t)(idx % npix);
          const uint32_t sample = it.sample_base + (uint32_t)(idx / npix);
          pixel = tile_pixel(lin, S.width, S.height);
          P.rng.s = path_seed(it.seed, pixel, sample);
          float ox, oy;
          sample_offset(it.seed, sample, it.jitter, P.rng, ox, oy);
          camera_ray(S, P, pixel, ox, oy);
          P.power = f3(1.f, 1.f, 1.f);
          P.acc = f3(0.f, 0.f, 0.f);
          P.last_mat = -1;
          depth_left = it.max_bounces;
          active = depth_left > 0;
          if (!active) atomicAdd(it.accum + pixel, make_float4(0.f, 0.f, 0.f, 1.0f));
        }
      }
    }
    if (__all_sync(0xffffffffu, done)) break;
    if (active) {
      const BatchItem& it = items[item];
      if (!bounce(static_cast<const V&>(views[it.view]), P, depth_left, status, C)) {
        active = false;
        atomicAdd(it.accum + pixel, make_float4(P.acc.x, P.acc.y, P.acc.z, 1.0f));
      }
    }
  }
}

// Debug probe: full event record of single paths (pixel, sample).
template <class V>
__global__ void path_events_kernel(V S, LaunchParams L, const int* pix, const int* smp, int n,
                                   float* ev, float* rgb, int* status) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  PathCounters C{0, 0, 0};
  PathState P;
  const uint32_t pixel = (uint32_t)pix[i], sample = (uint32_t)smp[i];
  P.rng.s = path_seed(L.seed, pixel, sample);
  float ox, oy;
  sample_offset(L.seed, sample, L.jitter, P.rng, ox, oy);
  camera_ray(S, P, pixel, ox, oy);
  float* e = ev + (size_t)i * kMaxEvents * kEventFloats;
  for (int k = 0; k < kMaxEvents * kEventFloats; ++k) e[k] = 0.0f;
  for (int k = 0; k < kMaxEvents; ++k) e[k * kEventFloats] = -2.0f;
  float3 c = trace_path(S, P, L.max_bounces, 0, status, C, e);
  rgb[3 * i] = c.x;
  rgb[3 * i + 1] = c.y;
  rgb[3 * i + 2] = c.z;
}

template <class V>
__global__ void first_hit_kernel(V S, const double* rays, int64_t n, HitOut* out,
                                 int* status) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* r = rays + 6 * i;
  float3 o = f3((float)r[0], (float)r[1], (float)r[2]);
  float3 d = f3((float)r[3], (float)r[4], (float)r[5]);
  HitInfo h;
  int visits = 0;
  HitOut res;
  bool hit = closest_hit<true>(S, o, d, h, visits, status);
  res.visits = visits;
  if (!hit) {
    res.prim = -1;
    res.front_face = 0;
    res.t = res.u = res.v = 0.f;
    res.n[0] = res.n[1] = res.n[2] = 0.f;
    res.p[0] = res.p[1] = res.p[2] = 0.f;
  } else {
    Surf s = make_surf(S, h, o, d, 0);
    res.prim = h.prim >= 0 ? __ldg(S.meta + h.prim).x : S.planes[-1 - h.prim].meta.x;
    res.front_face = s.front;
    res.t = h.t;
    res.u = h.u;
    res.v = h.v;
    res.n[0] = s.n.x; res.n[1] = s.n.y; res.n[2] = s.n.z;
    res.p[0] = s.p.x; res.p[1] = s.p.y; res.p[2] = s.p.z;
  }
  out[i] = res;
}

template <bool kCount, class V>
cudaError_t launch_megakernel_v(const V& v, const LaunchParams& L, float4* accum, int* depth,
                                int* status, unsigned long long* counters, int block, cudaStream_t st) {
  const unsigned grid = (unsigned)((L.n_paths + block - 1) / block);
#define MRT_MK(B)                                                                                 \
  if (block <= B) {                                                                               \
    megakernel<kCount, B, V><<<grid, block, 0, st>>>(v, L, accum, depth, status, counters);       \
    return cudaGetLastError();                                                                    \
  }
  MRT_MK(64)
  MRT_MK(128)
  MRT_MK(256)
#undef MRT_MK
  return cudaErrorInvalidValue;
}

template <class V>
cudaError_t launch_regen_v(const V& v, const LaunchParams& L, float4* accum, int* status,
                           unsigned long long* work, int block, int blocks_per_sm, int sms, cudaStream_t st) {
#define MRT_RG(B)                                                                                 \
  if (block <= B) {                                                                               \
    int occ = 0;                                                                                  \
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, megakernel_regen<B, V>, B, 0);            \
    int per = blocks_per_sm > 0 ? std::min(blocks_per_sm, std::max(occ, 1)) : std::max(occ, 1);   \
    unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)sms * per, (L.n_paths + B - 1) / B);   \
    megakernel_regen<B, V><<<grid, B, 0, st>>>(v, L, accum, status, work);                        \
    return cudaGetLastError();                                                                    \
  }
  MRT_RG(64)
  MRT_RG(128)
  MRT_RG(256)
#undef MRT_RG
  return cudaErrorInvalidValue;
}

template <class V>
cudaError_t launch_batch_v(const SceneView* views, const BatchItem* items, int n_items, uint64_t total,
                           int* status, unsigned long long* work, int block, int sms, cudaStream_t st) {
#define MRT_BT(B)                                                                                 \
  if (block <= B) {                                                                               \
    int occ = 0;                                                                                  \
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, megakernel_batch<B, V>, B, 0);            \
    unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)sms * std::max(occ, 1), (total + B - 1) / B); \
    megakernel_batch<B, V><<<grid, B, 0, st>>>(views, items, n_items, total, status, work);       \
    return cudaGetLastError();                                                                    \
  }
  MRT_BT(64)
  MRT_BT(128)
  MRT_BT(256)
#undef MRT_BT
  return cudaErrorInvalidValue;
}

template <class V>
cudaError_t launch_path_events_v(const V& v, const LaunchParams& L, const int* pix, const int* smp, int n,
                                 float* ev, float* rgb, int* status, cudaStream_t st) {
  path_events_kernel<<<(n + 63) / 64, 64, 0, st>>>(v, L, pix, smp, n, ev, rgb, status);
  return cudaGetLastError();
}

template <class V>
cudaError_t launch_first_hit_v(const V& v, const double* rays, int64_t n, HitOut* out, int* status,
                               cudaStream_t st) {
  first_hit_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(v, rays, n, out, status);
  return cudaGetLastError();
}

}  // namespace mrt
