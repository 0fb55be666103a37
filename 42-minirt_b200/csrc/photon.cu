// photon.cu — photon emission and the photon map.
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
// The map sorts the photons by the 63-bit Morton code of their position in
// the photons' bounding box (21 bits per axis: a few stray photons land
// hundreds of metres from the caustics, and a coarser code would leave the
// caustics in a handful of cells; CUB radix sort of (code, index), so the
// order is deterministic) and builds a linear BVH over them (Karras,
// "Maximizing parallelism in the construction of BVHs, octrees, and k-d
// trees", HPG 2012): internal node i covers a Morton range and splits it at
// its highest differing bit, so every node is a spatial cell of the code's
// implicit octree; boxes and power sums are filled bottom-up, the second
// child to finish completing its parent. A uniform grid was the first form:
// the caustics of configuration 2 are clustered (the densest 10 cm of floor
// holds ~180x the median) and the stray photons stretched its cells, so
// every gather scanned thousands of photons. The hierarchy adapts: a kNN
// gather prunes by its k-th distance, a fixed-radius gather adds whole nodes
// that lie inside the sphere.

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

template <class V>
__global__ void photon_emit_kernel(V S, PhotonEmit E, int* status) {
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
      if (!closest_hit<false>(S, P.o, P.d, h, visits, status, P.rng.s)) break;
      // photon paths trace with is_light set (trace_photon_path.c:42)
      Surf s = make_surf(S, h, P.o, P.d, 0, true);
      P.o = s.p;
      bool diffuse = false;
      if (s.mat < 0) {
        diffuse = true;
      } else {
        const MaterialD& M = surf_mat(S, s);
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

// Float min / max through int atomics: the order-preserving map of a float
// to an int (negative values have their magnitude bits flipped).
__device__ __forceinline__ int ordered(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float unordered(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// bounds[0..2] min, [3..5] max as ordered ints (initialised by the host).
__global__ void photon_bounds_kernel(PhotonTree T, int* bounds) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (i < T.n) {
    const float4 p = T.pos_in[i];
    mn[0] = mx[0] = p.x;
    mn[1] = mx[1] = p.y;
    mn[2] = mx[2] = p.z;
  }
  for (int k = 0; k < 3; ++k)
    for (int off = 16; off > 0; off >>= 1) {
      mn[k] = fminf(mn[k], __shfl_down_sync(0xffffffffu, mn[k], off));
      mx[k] = fmaxf(mx[k], __shfl_down_sync(0xffffffffu, mx[k], off));
    }
  if ((threadIdx.x & 31) == 0 && mn[0] <= mx[0])
    for (int k = 0; k < 3; ++k) {
      atomicMin(bounds + k, ordered(mn[k]));
      atomicMax(bounds + 3 + k, ordered(mx[k]));
    }
}

// Spreads the low 21 bits of v to every third bit.
__device__ __forceinline__ uint64_t spread3(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__global__ void morton_kernel(PhotonTree T, const int* bounds, uint64_t* code, uint32_t* idx) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T.n) return;
  const float4 p = T.pos_in[i];
  const float q[3] = {p.x, p.y, p.z};
  // one scale for the three axes (cubic cells): photons on a plane have a
  // near-zero extent across it, and scaling that axis by its own extent
  // would give float noise the top bits of the code
  double ext = 0.0;
  for (int k = 0; k < 3; ++k) ext = fmax(ext, (double)unordered(bounds[3 + k]) - (double)unordered(bounds[k]));
  uint64_t c[3];
  for (int k = 0; k < 3; ++k) {
    const double u = ext > 0.0 ? ((double)q[k] - (double)unordered(bounds[k])) / ext : 0.0;
    c[k] = (uint64_t)min(max((long long)(u * 2097151.0), 0ll), 2097151ll);
  }
  code[i] = (spread3(c[0]) << 2) | (spread3(c[1]) << 1) | spread3(c[2]);
  idx[i] = i;
}

__global__ void photon_gather_kernel(PhotonTree T, const uint32_t* sorted_idx) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T.n) return;
  const uint32_t s = sorted_idx[i];
  T.pos_out[i] = T.pos_in[s];
  T.pow_out[i] = T.pow_in[s];
}

// Length of the common prefix of the keys of photons i and j (index as a
// tie-break for equal codes); -1 outside [0, n).
__device__ __forceinline__ int common_prefix(const uint64_t* code, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  const uint64_t a = code[i], b = code[j];
  if (a != b) return __clzll((long long)(a ^ b));
  return 64 + __clz((int)((uint32_t)i ^ (uint32_t)j));
}

// Internal node i of the radix tree: its range, split and children.
__global__ void lbvh_internal_kernel(PhotonTree T, const uint64_t* code, int* parent_node, int* parent_leaf) {
  const int n = (int)T.n;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = common_prefix(code, n, i, i + 1) - common_prefix(code, n, i, i - 1) >= 0 ? 1 : -1;
  const int dmin = common_prefix(code, n, i, i - d);
  int lmax = 2;
  while (common_prefix(code, n, i, i + lmax * d) > dmin) lmax *= 2;   // bounded by the range end
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (common_prefix(code, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = common_prefix(code, n, i, j);
  int s = 0;
  for (int div = 2;; div *= 2) {
    const int t = (l + div - 1) / div;
    if (common_prefix(code, n, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
  }
  const int g = i + s * d + min(d, 0);
  const int lo = min(i, j), hi = max(i, j);
  const int left = lo == g ? ~g : g;
  const int right = hi == g + 1 ? ~(g + 1) : g + 1;
  T.nodes[4 * (size_t)i + 3] = make_float4(__int_as_float(left), __int_as_float(right), 0.f, 0.f);
  if (left >= 0) parent_node[left] = i; else parent_leaf[~left] = i;
  if (right >= 0) parent_node[right] = i; else parent_leaf[~right] = i;
  if (i == 0) parent_node[0] = -1;
}

__device__ __forceinline__ void child_box(const PhotonTree& T, int c, float3& lo, float3& hi, float3& pw) {
  if (c < 0) {
    const float4 p = __ldcg(T.pos_out + ~c), w = __ldcg(T.pow_out + ~c);
    lo = hi = f3(p.x, p.y, p.z);
    pw = f3(w.x, w.y, w.z);
  } else {
    const float4 a = __ldcg(T.nodes + 4 * (size_t)c), b = __ldcg(T.nodes + 4 * (size_t)c + 1),
                 w = __ldcg(T.nodes + 4 * (size_t)c + 2);
    lo = f3(a.x, a.y, a.z);
    hi = f3(b.x, b.y, b.z);
    pw = f3(w.x, w.y, w.z);
  }
}

// Bottom-up boxes: one thread per photon walks to the root; at each node the
// first child to arrive stops, the second fills the node.
__global__ void lbvh_bounds_kernel(PhotonTree T, const int* parent_node, const int* parent_leaf,
                                   unsigned* arrived) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (int)T.n) return;
  int node = parent_leaf[j];
  for (int guard = 0; node >= 0 && guard < 64 + (int)T.n; ++guard) {
    __threadfence();
    if (atomicAdd(arrived + node, 1u) == 0u) return;
    const float4 ch = __ldcg(T.nodes + 4 * (size_t)node + 3);
    float3 la, ha, pa, lb, hb, pb;
    child_box(T, __float_as_int(ch.x), la, ha, pa);
    child_box(T, __float_as_int(ch.y), lb, hb, pb);
    T.nodes[4 * (size_t)node] = make_float4(fminf(la.x, lb.x), fminf(la.y, lb.y), fminf(la.z, lb.z), 0.f);
    T.nodes[4 * (size_t)node + 1] = make_float4(fmaxf(ha.x, hb.x), fmaxf(ha.y, hb.y), fmaxf(ha.z, hb.z), 0.f);
    T.nodes[4 * (size_t)node + 2] = make_float4(pa.x + pb.x, pa.y + pb.y, pa.z + pb.z, 0.f);
    node = parent_node[node];
  }
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
  with_view(S, [&](const auto& v) {
    photon_emit_kernel<<<(unsigned)((total + b - 1) / b), b, 0, st>>>(v, P, status);
    return 0;
  });
  return cudaGetLastError();
}


// ------------------------------------------------------------ radix sort
// Stable LSD radix sort of the photons' 64-bit Morton codes with their
// indices, 8 bits per pass: per tile of kSortTile elements a 256-bin
// histogram (stored bin-major, so one exclusive scan over all of them gives
// every (bin, tile) its first output slot in stable order), the scan, then a
// scatter that ranks equal digits within each 256-element chunk of a tile
// with warp matching and running per-digit counters.
constexpr int kSortThreads = 256;
constexpr int kSortTile = 4096;

__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const uint64_t* key, int n, int shift,
                                                                  unsigned* hist, int tiles) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int t0 = blockIdx.x * kSortTile;
  for (int i = t0 + threadIdx.x; i < min(n, t0 + kSortTile); i += kSortThreads)
    atomicAdd(&h[(key[i] >> shift) & 255u], 1u);
  __syncthreads();
  hist[(size_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of m counters in place, one block.
__global__ void __launch_bounds__(1024) radix_scan_kernel(unsigned* c, int m) {
  __shared__ unsigned part[1024];
  const int per = (m + 1023) / 1024;
  const int a = threadIdx.x * per, b = min(m, a + per);
  unsigned sum = 0;
  for (int i = a; i < b; ++i) sum += c[i];
  part[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    const unsigned v = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  unsigned run = part[threadIdx.x] - sum;
  for (int i = a; i < b; ++i) {
    const unsigned x = c[i];
    c[i] = run;
    run += x;
  }
}

__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const uint64_t* key, const uint32_t* val,
                                                                     uint64_t* okey, uint32_t* oval, int n,
                                                                     int shift, const unsigned* hist, int tiles) {
  constexpr int kWarps = kSortThreads / 32;
  __shared__ unsigned base[256];            // next output slot of each digit in this tile
  __shared__ unsigned wcount[kWarps][256];  // digit counts per warp in the current chunk
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  base[threadIdx.x] = hist[(size_t)threadIdx.x * tiles + blockIdx.x];
  const int t0 = blockIdx.x * kSortTile;
  for (int c0 = t0; c0 < min(n, t0 + kSortTile); c0 += kSortThreads) {
    for (int w = 0; w < kWarps; ++w) wcount[w][threadIdx.x] = 0;
    __syncthreads();
    const int i = c0 + threadIdx.x;
    const bool ok = i < n && i < t0 + kSortTile;
    uint64_t k = 0;
    uint32_t v = 0;
    unsigned d = 256;                        // no digit: beyond the tile
    if (ok) {
      k = key[i];
      v = val[i];
      d = (unsigned)((k >> shift) & 255u);
    }
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned rank = __popc(peers & ((1u << lane) - 1u));
    if (ok && lane == __ffs(peers) - 1) wcount[warp][d] = __popc(peers);
    __syncthreads();
    unsigned before = 0;                     // this digit in earlier warps of the chunk
    if (ok)
      for (int w = 0; w < warp; ++w) before += wcount[w][d];
    if (ok) {
      const unsigned dst = base[d] + before + rank;
      okey[dst] = k;
      oval[dst] = v;
    }
    __syncthreads();
    unsigned tot = 0;
    for (int w = 0; w < kWarps; ++w) tot += wcount[w][threadIdx.x];
    base[threadIdx.x] += tot;
    __syncthreads();
  }
}

// Scratch: bounds (6 ints), code (n, 64-bit), idx (n), sorted code, sorted idx
// (n), radix-sort histograms; stream-ordered allocations released at the end.
cudaError_t launch_photon_tree(const PhotonTree& T, cudaStream_t st) {
  if (T.n == 0) return cudaSuccess;
  int* bounds = nullptr;
  uint64_t *code = nullptr, *scode = nullptr;
  uint32_t *idx = nullptr, *sidx = nullptr;
  void* tmp = nullptr;
  size_t tmp_bytes = 0;
  cudaError_t e;
  if ((e = cudaMallocAsync(&bounds, sizeof(int) * 6, st)) != cudaSuccess) return e;
  if ((e = cudaMallocAsync(&code, sizeof(uint64_t) * T.n, st)) != cudaSuccess) return e;
  if ((e = cudaMallocAsync(&idx, sizeof(uint32_t) * T.n, st)) != cudaSuccess) return e;
  if ((e = cudaMallocAsync(&scode, sizeof(uint64_t) * T.n, st)) != cudaSuccess) return e;
  if ((e = cudaMallocAsync(&sidx, sizeof(uint32_t) * T.n, st)) != cudaSuccess) return e;
  // ordered(+inf) for the minima, ordered(-inf) for the maxima
  const int init[6] = {0x7f800000, 0x7f800000, 0x7f800000, (int)(0xff800000u ^ 0x7fffffffu),
                       (int)(0xff800000u ^ 0x7fffffffu), (int)(0xff800000u ^ 0x7fffffffu)};
  if ((e = cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  const unsigned b = 256;
  const unsigned g = (T.n + b - 1) / b;
  photon_bounds_kernel<<<g, b, 0, st>>>(T, bounds);
  morton_kernel<<<g, b, 0, st>>>(T, bounds, code, idx);
  {
    // eight 8-bit passes over the 63-bit codes, ping-pong: the result lands
    // back in (code, idx)
    const int n = (int)T.n;
    const int tiles = (n + kSortTile - 1) / kSortTile;
    tmp_bytes = sizeof(unsigned) * 256 * (size_t)tiles;
    if ((e = cudaMallocAsync(&tmp, tmp_bytes, st)) != cudaSuccess) return e;
    unsigned* hist = static_cast<unsigned*>(tmp);
    uint64_t* kin = code;
    uint64_t* kout = scode;
    uint32_t* vin = idx;
    uint32_t* vout = sidx;
    for (int pass = 0; pass < 8; ++pass) {
      radix_hist_kernel<<<tiles, kSortThreads, 0, st>>>(kin, n, 8 * pass, hist, tiles);
      radix_scan_kernel<<<1, 1024, 0, st>>>(hist, 256 * tiles);
      radix_scatter_kernel<<<tiles, kSortThreads, 0, st>>>(kin, vin, kout, vout, n, 8 * pass, hist, tiles);
      std::swap(kin, kout);
      std::swap(vin, vout);
    }
    scode = kin;   // sorted codes and indices
    sidx = vin;
    code = kout;   // the other buffers, freed below like these
    idx = vout;
  }
  photon_gather_kernel<<<g, b, 0, st>>>(T, sidx);
  if (T.n > 1) {
    int *parent_node = nullptr, *parent_leaf = nullptr;
    unsigned* arrived = nullptr;
    if ((e = cudaMallocAsync(&parent_node, sizeof(int) * (T.n - 1), st)) != cudaSuccess) return e;
    if ((e = cudaMallocAsync(&parent_leaf, sizeof(int) * T.n, st)) != cudaSuccess) return e;
    if ((e = cudaMallocAsync(&arrived, sizeof(unsigned) * (T.n - 1), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(arrived, 0, sizeof(unsigned) * (T.n - 1), st)) != cudaSuccess) return e;
    lbvh_internal_kernel<<<(T.n - 1 + b - 1) / b, b, 0, st>>>(T, scode, parent_node, parent_leaf);
    lbvh_bounds_kernel<<<g, b, 0, st>>>(T, parent_node, parent_leaf, arrived);
    cudaFreeAsync(parent_node, st);
    cudaFreeAsync(parent_leaf, st);
    cudaFreeAsync(arrived, st);
  }
  cudaFreeAsync(tmp, st);
  cudaFreeAsync(bounds, st);
  cudaFreeAsync(code, st);
  cudaFreeAsync(idx, st);
  cudaFreeAsync(scode, st);
  cudaFreeAsync(sidx, st);
  return cudaGetLastError();
}

cudaError_t launch_caustic_query(const SceneView& S, const CausticQuery& Q, cudaStream_t st) {
  if (Q.n == 0) return cudaSuccess;
  caustic_query_kernel<<<(unsigned)((Q.n + 127) / 128), 128, 0, st>>>(S, Q);
  return cudaGetLastError();
}

}  // namespace mrt
