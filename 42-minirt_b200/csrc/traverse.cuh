// traverse.cuh — closest-hit and any-hit queries over the BVH (the binary
// tree, or the 8-wide tree in the SceneView instantiation) + planes.
//
// Semantics follow hit_register_all (hit_register.c:79-120): BVH primitives
// (spheres, triangles, and in the SceneViewQ instantiation cylinders, cones
// and hyperboloids) count when t in [0.001, 1000) (valid_t.c:16 and the
// closest_t = 1000 start, hit_register.c:21), then every infinite plane is
// tested and replaces the BVH hit only with a strictly smaller t
// (hit_plane.c:43-71, t in [0.001, 1000]). The tree is walked near child
// first with boxes culled beyond the best t; the stack (64 entries; the
// builder keeps the depth below that) is a per-thread array (LocalStack).
#pragma once
#include "device_common.cuh"
#include "quadric.cuh"
#include "texture.cuh"

namespace mrt {

struct HitInfo {
  float t;
  float u, v;        // barycentrics (triangles)
  int prim;          // leaf-order primitive index, -1 - plane index, or INT_MIN for a miss
};

constexpr int kMiss = -2147483647 - 1;

__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ int4 ldg4(const int4* p) { return __ldg(p); }

// Slab test against one child box; returns entry distance or +inf.
__device__ __forceinline__ float box_hit(float x0, float x1, float y0, float y1, float z0, float z1,
                                         float3 oi, float3 inv, float tmax) {
  // t = b * inv - o * inv, NaN-tolerant through fminf/fmaxf
  float tx0 = fmaf(x0, inv.x, -oi.x), tx1 = fmaf(x1, inv.x, -oi.x);
  float ty0 = fmaf(y0, inv.y, -oi.y), ty1 = fmaf(y1, inv.y, -oi.y);
  float tz0 = fmaf(z0, inv.z, -oi.z), tz1 = fmaf(z1, inv.z, -oi.z);
  float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), 0.0f));
  float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
  return tn <= tf ? tn : INFINITY;
}

// Moller-Trumbore with the reference's epsilon and windows (hit_triangle.c:38-93).
__device__ __forceinline__ bool tri_hit(const float4& a, const float4& b, const float4& c, float3 o,
                                        float3 d, int one_sided, float tbest, float& t, float& u,
                                        float& v) {
  float3 v0 = f3(a.x, a.y, a.z), e1 = f3(b.x, b.y, b.z), e2 = f3(c.x, c.y, c.z);
  float3 h = cross(d, e2);
  float det = dot(e1, h);
  if (one_sided ? (det < 1e-6f) : (fabsf(det) < 1e-6f)) return false;
  float f = 1.0f / det;
  float3 s = o - v0;
  u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return false;
  float3 q = cross(s, e1);
  v = f * dot(d, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  t = f * dot(e2, q);
  return t >= kTMin && t < tbest;
}

// Sphere: quadratic of init_sphere_quadratic (quadratique.c:32) in a
// cancellation-free form, nearer root first then the farther one (valid_t.c:16).
__device__ __forceinline__ bool sphere_hit(const float4& a, const float4& b, float3 o, float3 d,
                                           float tbest, float& t) {
  float3 oc = o - f3(a.x, a.y, a.z);
  float A = dot(d, d);
  float bh = dot(d, oc);
  float3 l = oc - d * (bh / A);
  float disc = A * (b.y - dot(l, l));
  if (disc < 0.0f) return false;
  float sq = sqrtf(disc);
  float qv = -(bh + copysignf(sq, bh));
  float c = dot(oc, oc) - b.y;
  float r0 = qv / A, r1 = (qv != 0.0f) ? c / qv : r0;
  float t0 = fminf(r0, r1), t1 = fmaxf(r0, r1);
  if (t0 >= kTMin && t0 <= kTMax) t = t0;
  else if (t1 >= kTMin && t1 <= kTMax) t = t1;
  else return false;
  return t < tbest;
}

__device__ __forceinline__ bool plane_hit(const PlaneD& p, float3 o, float3 d, float& t) {
  float3 n = f3(p.nn.x, p.nn.y, p.nn.z);
  float denom = dot(n, d);
  if (fabsf(denom) < 1e-8f) return false;
  t = dot(f3(p.pn.x, p.pn.y, p.pn.z) - o, n) / denom;
  return t >= kTMin && t <= kTMax;
}

// One primitive of a leaf: triangle, sphere or (SceneViewQ) quadric. u, v
// receive a triangle's barycentrics, or u the part of a quadric that was hit.
// akey: the path stream's state, for the alpha test of textured scenes.
template <class V>
__device__ __forceinline__ bool prim_hit_geom(const V& S, int i, int type, const float4& a, const float4& b,
                                              const float4* g, float3 o, float3 d, float tbest, float& t,
                                              float& u, float& v) {
  if (type == PRIM_TRI) {
    const float4 c = ldg4(g + 2);
    return tri_hit(a, b, c, o, d, S.one_sided, tbest, t, u, v);
  }
  if constexpr (V::kQuadrics) {
    if (type != PRIM_SPHERE) {
      const QuadricHit q = quadric_hit(type, a, b, ldg4(g + 2), o, d, tbest);
      if (q.t < 0.0f) return false;
      t = q.t;
      u = (float)q.part;
      v = 0.f;
      return true;
    }
  }
  return sphere_hit(a, b, o, d, tbest, t);
}

template <class V>
__device__ __forceinline__ bool prim_hit(const V& S, int i, float3 o, float3 d, float tbest, float& t,
                                         float& u, float& v, uint64_t akey = 0) {
  const float4* g = S.geom + 3 * (size_t)i;
  const float4 a = ldg4(g), b = ldg4(g + 1);
  const int type = __float_as_int(a.w);
  if (!prim_hit_geom(S, i, type, a, b, g, o, d, tbest, t, u, v)) return false;
  if constexpr (V::kTextures) {
    if (alpha_drops(S, i, type, o, d, t, u, v, akey)) return false;
  }
  return true;
}

// The traversal stack: a per-thread array (registers / local memory, which
// L1 caches). A shared-memory short stack (24 entries per thread, spilling
// to local memory) measured 2.7 % slower in the wavefront on c1, so the
// traversal loops take the stack as a parameter and every caller passes this
// one.
struct LocalStack {
  int s[kStackSize];
  __device__ __forceinline__ void put(int i, int v) { s[i] = v; }
  __device__ __forceinline__ int get(int i) const { return s[i]; }
};

// 8-wide tree (WNode). One node per iteration: its up-to-8 quantised child
// boxes are tested against the ray clipped to [0, tbest]; hit leaves are
// intersected at once, near to far; the nearest hit internal child is
// visited next and the node's other hit internal children are pushed as
// one group entry (child_base, remaining hit bits << 8 | imask), two ints
// of the stack. Visit order is the ray's octant applied to the slots (key
// = slot ^ sign bits, lowest key first). Slab test per child and axis:
// t = q * (2^e / d) + (p - o) / d, one fma.
struct WideHits {
  uint32_t inner;    // hit internal children, bit = key
  uint32_t leaf;     // hit leaves, bit = key
};

// Byte j of w as a float, exactly: the byte under the exponent of 2^23
// (one byte permute) minus 2^23 (one add), instead of an integer-to-float
// conversion, which issues at a fraction of the FP32 rate.
__device__ __forceinline__ float qbyte(uint32_t w, int j) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u + (uint32_t)j)) - 8388608.0f;
}

__device__ __forceinline__ WideHits wide_children(const WNode* nd, float3 o, float3 inv, uint32_t oct,
                                                  float tmax, int4& b, uint32_t& imask) {
  const float4 a = ldg4(&nd->a);
  b = ldg4(&nd->b);
  const int4 c = ldg4(&nd->c), d = ldg4(&nd->d), e = ldg4(&nd->e);
  const uint32_t w = __float_as_uint(a.w);
  imask = w >> 24;
  const float ax = __uint_as_float((w & 0xffu) << 23) * inv.x;
  const float ay = __uint_as_float(((w >> 8) & 0xffu) << 23) * inv.y;
  const float az = __uint_as_float(((w >> 16) & 0xffu) << 23) * inv.z;
  const float bx = (a.x - o.x) * inv.x, by = (a.y - o.y) * inv.y, bz = (a.z - o.z) * inv.z;
  WideHits h{0u, 0u};
  // near and far planes per axis: the low bytes for a non-negative direction
  // component, the high bytes for a negative one (NaNs of zero components
  // drop out of fminf / fmaxf, leaving the box conservative)
  const bool fx = oct & 1u, fy = oct & 2u, fz = oct & 4u;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const uint32_t meta = (uint32_t)(half ? b.w : b.z);
    const uint32_t lx = (uint32_t)(half ? c.y : c.x), ly = (uint32_t)(half ? c.w : c.z);
    const uint32_t lz = (uint32_t)(half ? d.y : d.x), hx = (uint32_t)(half ? d.w : d.z);
    const uint32_t hy = (uint32_t)(half ? e.y : e.x), hz = (uint32_t)(half ? e.w : e.z);
    const uint32_t nx = fx ? hx : lx, ny = fy ? hy : ly, nz = fz ? hz : lz;
    const uint32_t gx = fx ? lx : hx, gy = fy ? ly : hy, gz = fz ? lz : hz;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int sh = 8 * j;
      const float tnx = fmaf(qbyte(nx, j), ax, bx), tfx = fmaf(qbyte(gx, j), ax, bx);
      const float tny = fmaf(qbyte(ny, j), ay, by), tfy = fmaf(qbyte(gy, j), ay, by);
      const float tnz = fmaf(qbyte(nz, j), az, bz), tfz = fmaf(qbyte(gz, j), az, bz);
      const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, 0.0f));
      const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tmax));
      const int slot = 4 * half + j;
      if (((meta >> sh) & 0x80u) && tn <= tf) {
        const uint32_t bit = 1u << ((uint32_t)slot ^ oct);
        if ((imask >> slot) & 1u) h.inner |= bit;
        else h.leaf |= bit;
      }
    }
  }
  return h;
}

__device__ __forceinline__ int wide_child(int base, uint32_t imask, uint32_t key, uint32_t oct) {
  const uint32_t slot = key ^ oct;
  return base + __popc(imask & ((1u << slot) - 1u));
}

// Leaf slot `key` of a node: its primitive range.
__device__ __forceinline__ void wide_leaf(const int4& b, uint32_t key, uint32_t oct, int& first, int& count) {
  const uint32_t slot = key ^ oct;
  const uint32_t m = ((uint32_t)(slot < 4 ? b.z : b.w) >> (8 * (slot & 3))) & 0xffu;
  first = b.y + (int)(m & 31u);
  count = (int)((m >> 5) & 3u) + 1;
}

template <bool kCount, class V, class Stack>
__device__ __forceinline__ void wide_closest(const V& S, float3 o, float3 d, float& tbest, int& best, float& bu,
                                             float& bv, int& visits, int* status, Stack& stack, uint64_t akey) {
  const float3 inv = f3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  int sp = 0;
  int cur = 0;
  int budget = 2 * S.n_wnodes + S.n_prims + 64;
  while (true) {
    if (--budget < 0) {
      if (status) atomicOr(status, ST_BUDGET);
      return;
    }
    int4 b;
    uint32_t imask;
    if (kCount) visits++;
    WideHits h = wide_children(S.wnodes + cur, o, inv, oct, tbest, b, imask);
    while (h.leaf) {
      const uint32_t key = (uint32_t)(__ffs(h.leaf) - 1);
      h.leaf &= h.leaf - 1u;
      int first, count;
      wide_leaf(b, key, oct, first, count);
      for (int i = first; i < first + count; ++i) {
        float t, u = 0.f, v = 0.f;
        if (prim_hit(S, i, o, d, tbest, t, u, v, akey)) { tbest = t; best = i; bu = u; bv = v; }
      }
    }
    if (h.inner) {
      const uint32_t key = (uint32_t)(__ffs(h.inner) - 1);
      h.inner &= h.inner - 1u;
      if (h.inner) {
        if (sp < kWideStack) {
          stack.put(2 * sp, b.x);
          stack.put(2 * sp + 1, (int)((h.inner << 8) | imask));
          ++sp;
        } else if (status) {
          atomicOr(status, ST_STACK);
        }
      }
      cur = wide_child(b.x, imask, key, oct);
      continue;
    }
    if (sp == 0) return;
    const int base = stack.get(2 * sp - 2);
    const uint32_t g = (uint32_t)stack.get(2 * sp - 1);
    uint32_t rest = g >> 8;
    const uint32_t im = g & 0xffu;
    const uint32_t key = (uint32_t)(__ffs(rest) - 1);
    rest &= rest - 1u;
    if (rest) stack.put(2 * sp - 1, (int)((rest << 8) | im));
    else --sp;
    cur = wide_child(base, im, key, oct);
  }
}

template <class V, class Stack>
__device__ __forceinline__ bool wide_any(const V& S, float3 o, float3 d, float tlim, int* status, Stack& stack,
                                         uint64_t akey) {
  const float3 inv = f3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  const uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  int sp = 0;
  int cur = 0;
  int budget = 2 * S.n_wnodes + S.n_prims + 64;
  while (true) {
    if (--budget < 0) {
      if (status) atomicOr(status, ST_BUDGET);
      return false;
    }
    int4 b;
    uint32_t imask;
    WideHits h = wide_children(S.wnodes + cur, o, inv, oct, tlim, b, imask);
    while (h.leaf) {
      const uint32_t key = (uint32_t)(__ffs(h.leaf) - 1);
      h.leaf &= h.leaf - 1u;
      int first, count;
      wide_leaf(b, key, oct, first, count);
      for (int i = first; i < first + count; ++i) {
        float t, u, v;
        if (prim_hit(S, i, o, d, tlim, t, u, v, akey)) return true;
      }
    }
    if (h.inner) {
      const uint32_t key = (uint32_t)(__ffs(h.inner) - 1);
      h.inner &= h.inner - 1u;
      if (h.inner) {
        if (sp < kWideStack) {
          stack.put(2 * sp, b.x);
          stack.put(2 * sp + 1, (int)((h.inner << 8) | imask));
          ++sp;
        } else if (status) {
          atomicOr(status, ST_STACK);
        }
      }
      cur = wide_child(b.x, imask, key, oct);
      continue;
    }
    if (sp == 0) return false;
    const int base = stack.get(2 * sp - 2);
    const uint32_t g = (uint32_t)stack.get(2 * sp - 1);
    uint32_t rest = g >> 8;
    const uint32_t im = g & 0xffu;
    const uint32_t key = (uint32_t)(__ffs(rest) - 1);
    rest &= rest - 1u;
    if (rest) stack.put(2 * sp - 1, (int)((rest << 8) | im));
    else --sp;
    cur = wide_child(base, im, key, oct);
  }
}

// Closest hit. `visits` counts node fetches (heat-map / roofline counter).
// Returns false on a miss. `status` receives ST_BUDGET if the bounded loop
// ran out (a corrupted tree), never hangs.
//
// One node or one leaf per iteration, near child first, boxes culled beyond
// the best t. The wavefront's extend and connect kernels and the
// megakernels all use this loop: on B200 it measured 5 % faster in the
// wavefront (c1) than the while-while loop with speculative leaf
// postponement (Aila & Laine, HPG 2009) that the wavefront used first.
// kTree: kTreeAny picks the tree at run time (S.wnodes); kTreeBinary and
// kTreeWide compile one traversal only (the wavefront's extend and connect
// kernels, launched per tree, so that neither carries the other's registers).
enum TreeSel : int { kTreeAny = 0, kTreeBinary = 1, kTreeWide = 2 };

template <bool kCount, int kTree = kTreeAny, class V, class Stack>
__device__ __forceinline__ bool closest_hit_compact(const V& S, float3 o, float3 d, HitInfo& hit,
                                                    int& visits, int* status, Stack& stack,
                                                    uint64_t akey = 0) {
  float tbest = kTMax;
  int best = kMiss;
  float bu = 0.f, bv = 0.f;
  bool wide = false;
  if constexpr (!V::kQuadrics && kTree != kTreeBinary) {
    if (S.has_bvh && (kTree == kTreeWide || S.wnodes)) {
      wide_closest<kCount>(S, o, d, tbest, best, bu, bv, visits, status, stack, akey);
      wide = true;
    }
  }
  if (kTree != kTreeWide && S.has_bvh && !wide) {
    float3 inv = f3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float3 oi = o * inv;
    int sp = 0;
    int cur = 0;
    int budget = 4 * S.n_nodes + 4 * S.n_prims + 64;
    while (true) {
      if (--budget < 0) {
        if (status) atomicOr(status, ST_BUDGET);
        break;
      }
      if (cur >= 0) {
        const Node* nd = S.nodes + cur;
        float4 lxy = ldg4(&nd->lxy), rxy = ldg4(&nd->rxy), z = ldg4(&nd->z);
        int4 ln = ldg4(&nd->link);
        if (kCount) visits++;
        float tl = box_hit(lxy.x, lxy.y, lxy.z, lxy.w, z.x, z.y, oi, inv, tbest);
        float tr = box_hit(rxy.x, rxy.y, rxy.z, rxy.w, z.z, z.w, oi, inv, tbest);
        bool hl = tl < INFINITY, hr = tr < INFINITY;
        if (hl && hr) {
          // nearer child first; the reference-topology tree keeps the
          // reference's left-first order, so exact-t ties resolve as there
          const bool left_near = S.left_first || tl <= tr;
          int nearc = left_near ? ln.x : ln.y;
          int farc = left_near ? ln.y : ln.x;
          if (sp < kStackSize) stack.put(sp++, farc);
          else if (status) atomicOr(status, ST_STACK);
          cur = nearc;
          continue;
        }
        if (hl) { cur = ln.x; continue; }
        if (hr) { cur = ln.y; continue; }
      } else {
        int code = ~cur;
        int first = code >> 3, count = (code & 7) + 1;
        for (int i = first; i < first + count; ++i) {
          float t, u = 0.f, v = 0.f;
          if (prim_hit(S, i, o, d, tbest, t, u, v, akey)) { tbest = t; best = i; bu = u; bv = v; }
        }
      }
      if (sp == 0) break;
      cur = stack.get(--sp);
    }
  }
  for (int i = 0; i < S.n_planes; ++i) {
    float t;
    if (plane_hit(S.planes[i], o, d, t) && (best == kMiss || t < tbest)) {
      tbest = t;
      best = -1 - i;
    }
  }
  hit.t = tbest;
  hit.u = bu;
  hit.v = bv;
  hit.prim = best;
  return best != kMiss;
}

// Any hit, compact loop.
template <int kTree = kTreeAny, class V, class Stack>
__device__ __forceinline__ bool any_hit_compact(const V& S, float3 o, float3 d, float tmax,
                                                int* status, Stack& stack, uint64_t akey = 0) {
  for (int i = 0; i < S.n_planes; ++i) {
    float t;
    if (plane_hit(S.planes[i], o, d, t) && t < tmax) return true;
  }
  if (!S.has_bvh) return false;
  const float tlim = fminf(tmax, kTMax);
  if constexpr (!V::kQuadrics && kTree != kTreeBinary) {
    if (kTree == kTreeWide || S.wnodes) return wide_any(S, o, d, tlim, status, stack, akey);
  }
  float3 inv = f3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  float3 oi = o * inv;
  int sp = 0;
  int cur = 0;
  int budget = 4 * S.n_nodes + 4 * S.n_prims + 64;
  while (true) {
    if (--budget < 0) {
      if (status) atomicOr(status, ST_BUDGET);
      return false;
    }
    if (cur >= 0) {
      const Node* nd = S.nodes + cur;
      float4 lxy = ldg4(&nd->lxy), rxy = ldg4(&nd->rxy), z = ldg4(&nd->z);
      int4 ln = ldg4(&nd->link);
      float tl = box_hit(lxy.x, lxy.y, lxy.z, lxy.w, z.x, z.y, oi, inv, tlim);
      float tr = box_hit(rxy.x, rxy.y, rxy.z, rxy.w, z.z, z.w, oi, inv, tlim);
      bool hl = tl < INFINITY, hr = tr < INFINITY;
      if (hl && hr) {
        if (sp < kStackSize) stack.put(sp++, ln.y);
        else if (status) atomicOr(status, ST_STACK);
        cur = ln.x;
        continue;
      }
      if (hl) { cur = ln.x; continue; }
      if (hr) { cur = ln.y; continue; }
    } else {
      int code = ~cur;
      int first = code >> 3, count = (code & 7) + 1;
      for (int i = first; i < first + count; ++i) {
        float t, u, v;
        if (prim_hit(S, i, o, d, tlim, t, u, v, akey)) return true;
      }
    }
    if (sp == 0) return false;
    cur = stack.get(--sp);
  }
}

// The reference's node-visit count for render_mode 1 on the reference-topology
// tree (S.ref_boxes): hit_bvh (bvh_hit.c:16-43) visits the root and both
// children of every internal node whose box the ray hits, without culling,
// and counts every visit; boxes are tested in double with intersect_aabb's
// formula (bvh_utils.c:38-59). any_leaf receives whether a leaf primitive was
// hit, on which hit_register_all keeps the count (hit_register.c:113-121).
__device__ __forceinline__ bool ref_box_hit(const double* b, double3 o, double3 d) {
  double t1 = fmin((b[0] - o.x) / d.x, (b[3] - o.x) / d.x);
  double tmin = fmax(t1, fmin((b[1] - o.y) / d.y, (b[4] - o.y) / d.y));
  t1 = fmin((b[2] - o.z) / d.z, (b[5] - o.z) / d.z);
  tmin = fmax(tmin, t1);
  t1 = fmax((b[0] - o.x) / d.x, (b[3] - o.x) / d.x);
  double tmax = fmin(t1, fmax((b[1] - o.y) / d.y, (b[4] - o.y) / d.y));
  t1 = fmax((b[2] - o.z) / d.z, (b[5] - o.z) / d.z);
  tmax = fmin(tmax, t1);
  return tmax >= fmax(tmin, 0.0) && tmin < 1000.0;
}

template <class V>
__device__ int ref_visit_count(const V& S, float3 of, float3 df, bool& any_leaf, int* status) {
  const double3 o = make_double3(of.x, of.y, of.z), d = make_double3(df.x, df.y, df.z);
  any_leaf = false;
  int count = 1;
  if (!S.has_bvh || !ref_box_hit(S.ref_boxes, o, d)) return count;
  auto leaf = [&](int link) {
    const int first = (~link) >> 3;
    float t, u, v;
    if (prim_hit(S, first, of, df, kTMax, t, u, v)) any_leaf = true;
  };
  if (S.root_leaf) {
    leaf(S.root_leaf);
    return count;
  }
  int stack[kStackSize];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const int k = stack[--sp];
    count += 2;
    const int4 ln = __ldg(&S.nodes[k].link);
    const double* b = S.ref_boxes + 6 + 12 * (size_t)k;
    const int child[2] = {ln.x, ln.y};
    for (int c = 1; c >= 0; --c) {          // right pushed first: left popped first
      if (!ref_box_hit(b + 6 * c, o, d)) continue;
      if (child[c] < 0) leaf(child[c]);
      else if (sp < kStackSize) stack[sp++] = child[c];
      else if (status) atomicOr(status, ST_STACK);
    }
  }
  return count;
}

// Entry points of the shading code (megakernels, probes, photon emission);
// the wavefront's extend and connect kernels call the compact loops directly.
template <bool kCount, class V>
__device__ __forceinline__ bool closest_hit(const V& S, float3 o, float3 d, HitInfo& hit,
                                            int& visits, int* status, uint64_t akey = 0) {
  LocalStack stack;
  return closest_hit_compact<kCount>(S, o, d, hit, visits, status, stack, akey);
}

template <class V>
__device__ __forceinline__ bool any_hit(const V& S, float3 o, float3 d, float tmax, int* status,
                                        uint64_t akey = 0) {
  LocalStack stack;
  return any_hit_compact(S, o, d, tmax, status, stack, akey);
}

}  // namespace mrt
