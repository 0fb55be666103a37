// photon.cu — photon emission and the uniform-grid photon map.
//
// Emission follows caustic_manager / emit_photon_from_one_light /
// trace_single_photon_path / material_manager_v3_phothon
// (caustic_manager.c:30-105, trace_photon_path.c:18-72,
// dielectric.c:66-91, material_default.c:94-98): per point light N photons
// of power colour * brightness / N (0..255 scale), uniform directions, at
// most 10 bounces, stored at the first diffuse event if at least one
// specular bounce preceded it (`return depth != 0`). One thread per photon,
// warp-aggregated append into the photon buffer.
//
// The grid sorts photons by cell (CUB radix sort of (cell, index), so the
// order is deterministic) and records each cell's start.
#include <cub/device/device_radix_sort.cuh>

#include "kernels.h"
#include "path.cuh"

namespace mrt {

namespace {

constexpr uint32_t kPhotonSalt = 0x9E3779B9u;

// vec3_random_unit (vec3_random.c:33-44), bounded rejection loop.
__device__ __forceinline__ float3 rnd_unit(Rng& rng) {
  for (int it = 0; it < 64; ++it) {
    float3 p = f3(-1.0f + rng.next() * 2.0f, -1.0f + rng.next() * 2.0f, -1.0f + rng.next() * 2.0f);
    float l2 = len2(p);
    if (l2 > 1e-30f && l2 <= 1.0f) return p * rsqrtf(l2);
  }
  return f3(0.f, 1.f, 0.f);
}

__global__ void photon_emit_kernel(SceneView S, PhotonEmit E, int* status) {
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t total = E.per_light * (uint64_t)E.n_point_lights;
  bool store = false;
  float3 pos = f3(0.f, 0.f, 0.f), pw = f3(0.f, 0.f, 0.f);
  if (g < total) {
    const int l = (int)(g / E.per_light);
    const LightD L = S.lights[E.light_index[l]];
    Rng rng{path_seed(E.seed ^ ((uint64_t)kPhotonSalt << 32), (uint32_t)g, E.pass ^ (uint32_t)(g >> 32))};
    const float inv_n = 1.0f / (float)E.per_light;
    PathState P;
    P.power = f3(L.color[0] * L.brightness * inv_n, L.color[1] * L.brightness * inv_n,
                 L.color[2] * L.brightness * inv_n);
    P.d = rnd_unit(rng);
    P.o = ld3(L.pos);
    P.rng = rng;
    for (int depth = 0; depth < 10; ++depth) {
      HitInfo h;
      int visits = 0;
      if (!closest_hit<false>(S, P.o, P.d, h, visits, status)) break;
      Surf s = make_surf(S, h, P.o, P.d, 0);
      P.o = s.p;
      bool diffuse = false;
      if (s.mat < 0) {
        diffuse = true;
      } else {
        const MaterialD& M = S.mats[s.mat];
        bool as_metal;
        if (M.metallic == 1.0f) as_metal = true;
        else if (M.metallic == 0.0f) as_metal = false;
        else as_metal = M.metallic > P.rng.next();
        if (as_metal) {
          metallic(M, P, s);
        } else if (M.ior > 0.0f) {
          float ct = -dot(unit(P.d), s.n);
          float refl = M.f0 + (1.0f - M.f0) * pow5(1.0f - ct);
          if (refl >= P.rng.next() && M.ior != 1.0f) {
            float3 m = M.roughness > 0.0f ? ggx_sample(P.rng, s.n, M.alpha4) : s.n;
            P.d = unit(P.d - m * (2.0f * dot(P.d, m)));
          } else if (M.transmission == 1.0f) {
            refract(S, M, P, s);
          } else if (M.transmission == 0.0f) {
            diffuse = true;
          } else if (M.transmission < P.rng.next()) {
            diffuse = true;
          } else {
            refract(S, M, P, s);
          }
        } else {
          diffuse = true;
        }
      }
      if (diffuse) {
        P.power = P.power * s.color;
        if (depth != 0) { store = true; pos = s.p; pw = P.power; }
        break;
      }
    }
  }
  // warp-aggregated append
  const unsigned mask = __ballot_sync(0xffffffffu, store);
  if (mask == 0) return;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(E.count, (unsigned)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (store) {
    const unsigned slot = base + __popc(mask & ((1u << lane) - 1u));
    if (slot < E.capacity) {
      E.pos[slot] = make_float4(pos.x, pos.y, pos.z, 0.f);
      E.pow[slot] = make_float4(pw.x, pw.y, pw.z, 0.f);
    } else {
      atomicOr(status, ST_QUEUE);
    }
  }
}

__global__ void cell_of_kernel(GridBuild G, uint32_t* idx) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G.n) return;
  float4 p = G.pos_in[i];
  int x = min(max((int)floorf((p.x - G.grid_min[0]) * G.inv_cell), 0), G.dim[0] - 1);
  int y = min(max((int)floorf((p.y - G.grid_min[1]) * G.inv_cell), 0), G.dim[1] - 1);
  int z = min(max((int)floorf((p.z - G.grid_min[2]) * G.inv_cell), 0), G.dim[2] - 1);
  G.cell_of[i] = (uint32_t)((z * G.dim[1] + y) * G.dim[0] + x);
  idx[i] = i;
}

__global__ void gather_kernel(GridBuild G, const uint32_t* sorted_cell, const uint32_t* sorted_idx) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= G.n) return;
  uint32_t s = sorted_idx[i];
  G.pos_out[i] = G.pos_in[s];
  G.pow_out[i] = G.pow_in[s];
  uint32_t c = sorted_cell[i];
  if (i == 0 || sorted_cell[i - 1] != c) {
    uint32_t prev = i == 0 ? 0 : sorted_cell[i - 1] + 1;
    for (uint32_t k = prev; k <= c; ++k) G.cell_start[k] = i;
  }
  if (i == G.n - 1)
    for (uint32_t k = c + 1; k <= G.n_cells; ++k) G.cell_start[k] = G.n;
}

__global__ void empty_grid_kernel(GridBuild G) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k <= G.n_cells) G.cell_start[k] = 0;
}

__global__ void caustic_query_kernel(SceneView S, CausticQuery Q) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Q.n) return;
  float3 p = f3((float)Q.pts[3 * i], (float)Q.pts[3 * i + 1], (float)Q.pts[3 * i + 2]);
  float3 c = caustic_estimate(S, p);
  Q.out[3 * i] = c.x;
  Q.out[3 * i + 1] = c.y;
  Q.out[3 * i + 2] = c.z;
}

}  // namespace

cudaError_t launch_photon_emit(const SceneView& S, const PhotonEmit& P, int* status, cudaStream_t st) {
  const uint64_t total = P.per_light * (uint64_t)P.n_point_lights;
  if (total == 0) return cudaSuccess;
  const unsigned b = 128;
  photon_emit_kernel<<<(unsigned)((total + b - 1) / b), b, 0, st>>>(S, P, status);
  return cudaGetLastError();
}

// Scratch: cell_of (n), idx (n), sorted cell (n), sorted idx (n), CUB temp.
cudaError_t launch_grid_build(const GridBuild& G, cudaStream_t st) {
  if (G.n == 0) {
    empty_grid_kernel<<<(G.n_cells + 256) / 256, 256, 0, st>>>(G);
    return cudaGetLastError();
  }
  uint32_t *idx = nullptr, *scell = nullptr, *sidx = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  cudaError_t e;
  if ((e = cudaMallocAsync(&idx, sizeof(uint32_t) * G.n, st)) != cudaSuccess) return e;
  if ((e = cudaMallocAsync(&scell, sizeof(uint32_t) * G.n, st)) != cudaSuccess) return e;
  if ((e = cudaMallocAsync(&sidx, sizeof(uint32_t) * G.n, st)) != cudaSuccess) return e;
  const unsigned b = 256;
  cell_of_kernel<<<(G.n + b - 1) / b, b, 0, st>>>(G, idx);
  int bits = 1;
  while (bits < 32 && (1ull << bits) <= G.n_cells) ++bits;
  cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, G.cell_of, scell, idx, sidx, (int)G.n, 0, bits, st);
  if ((e = cudaMallocAsync(&tmp, tmp_bytes, st)) != cudaSuccess) return e;
  cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, G.cell_of, scell, idx, sidx, (int)G.n, 0, bits, st);
  gather_kernel<<<(G.n + b - 1) / b, b, 0, st>>>(G, scell, sidx);
  cudaFreeAsync(tmp, st);
  cudaFreeAsync(idx, st);
  cudaFreeAsync(scell, st);
  cudaFreeAsync(sidx, st);
  return cudaGetLastError();
}

cudaError_t launch_caustic_query(const SceneView& S, const CausticQuery& Q, cudaStream_t st) {
  if (Q.n == 0) return cudaSuccess;
  caustic_query_kernel<<<(unsigned)((Q.n + 127) / 128), 128, 0, st>>>(S, Q);
  return cudaGetLastError();
}

}  // namespace mrt
