// texture.cuh — textures and maps of the SceneViewT instantiation.
//
//   get_tex_color (get_tex_color.c:27-48): IMAGE nearest texel
//     rgba[w * (int)(v (h-1)) + (int)(u (w-1))] / 255, a missing image reads
//     the fallback checker (get_solid_texture_default, scale 2, black /
//     magenta); CHECKER_LOCAL by floor(u s) + floor(v s); CHECKER_GLOBAL by
//     floor(p s) with y + 0.5 (get_solid_texture.c:31); HDR and COLOR black.
//     Texel indices are clamped to the image (the reference reads outside it
//     for mesh uvs outside [0, 1]).
//   texture coordinates per object: get_sphere_uv (hit_sphere.c:15),
//     get_uv_plane (hit_plane.c:18), the triangle's interpolated vertex uvs
//     (hit_triangle.c:93), cylinder_uv.c, hit_cone.c:14-52,
//     hit_hyperboloid.c:14-34; tiled by the material's scale.
//   apply_normal_map (apply_map.c:38-58) and the alpha test of
//     hit_register_bvh (hit_register.c:62-72): a texel of alpha a drops the
//     candidate with probability 1 - a/255. The draw is a hash of the path
//     stream's state at the traversal and the object's flat id
//     (alpha_uniform, also in the oracle), not the reference's global
//     random_double, whose order follows its exhaustive leaf recursion.
#pragma once
#include "device_common.cuh"
#include "quadric.cuh"

namespace mrt {

constexpr float kPiF = 3.14159265358979f;

__device__ __forceinline__ float clamp01f(float x) { return x < 0.f ? 0.f : (x > 1.f ? 1.f : x); }

// solid checker of the hit point (get_solid_texture.c:15-43)
__device__ __forceinline__ float3 solid_checker(float3 p, float scale, float3 c1, float3 c2) {
  p = p * scale;
  const int a = (int)floorf(p.x), b = (int)floorf(p.y + 0.5f), c = (int)floorf(p.z);
  return ((a + b + c) % 2 == 0) ? c1 : c2;
}

// Texture k (1-based): rgb and alpha / 255.
// The texel the reference reads for (u, v): one linear index,
// width * (int)(v * (h - 1)) + (int)(u * (w - 1)) (get_tex_color.c:37,
// apply_map.c:45-47), so a u beyond [0, 1] runs on into the neighbouring
// row rather than clamping to the edge. Where that index leaves the image
// (the reference then reads outside its buffer) it is clamped to it.
__device__ __forceinline__ uchar4 texel_at(const SceneView& S, const TexD& t, float u, float v) {
  long long i = (long long)t.w * (int)(v * (float)(t.h - 1)) + (int)(u * (float)(t.w - 1));
  const long long n = (long long)t.w * t.h;
  i = i < 0 ? 0 : (i >= n ? n - 1 : i);
  return __ldg(S.texels + t.offset + (size_t)i);
}

__device__ __forceinline__ float4 tex_lookup(const SceneView& S, int k, float u, float v, float3 p) {
  const TexD& t = S.texs[k - 1];
  if (t.type == 0) {   // IMAGE
    if (t.w <= 0) {
      const float3 c = solid_checker(p, 2.0f, f3(0.f, 0.f, 0.f), f3(243.f / 255.f, 0.f, 243.f / 255.f));
      return make_float4(c.x, c.y, c.z, 1.f);
    }
    const uchar4 q = texel_at(S, t, u, v);
    const float s = 1.0f / 255.0f;
    return make_float4(q.x * s, q.y * s, q.z * s, q.w * s);
  }
  if (t.type == 3) {   // CHECKER_LOCAL
    const int a = (int)floorf(u * t.scale), b = (int)floorf(v * t.scale);
    return ((a + b) % 2 == 0) ? make_float4(t.c1[0], t.c1[1], t.c1[2], 1.f)
                              : make_float4(t.c2[0], t.c2[1], t.c2[2], 1.f);
  }
  if (t.type == 4) {   // CHECKER_GLOBAL
    const float3 c = solid_checker(p, t.scale, f3(t.c1[0], t.c1[1], t.c1[2]), f3(t.c2[0], t.c2[1], t.c2[2]));
    return make_float4(c.x, c.y, c.z, 1.f);
  }
  return make_float4(0.f, 0.f, 0.f, 1.f);
}

__device__ __forceinline__ void uv_tile(float scale, float& u, float& v) {
  if (scale != 1.0f) {
    u *= scale;
    v *= scale;
    u -= truncf(u);
    v -= truncf(v);
  }
}

__device__ __forceinline__ float3 uv_right(float3 ori) {
  return fabsf(ori.y) < 0.99f ? unit(cross(f3(0.f, 1.f, 0.f), ori)) : unit(cross(f3(1.f, 0.f, 0.f), ori));
}

__device__ __forceinline__ float uv_angle(float3 rel, float3 ori) {
  const float3 r = uv_right(ori);
  return clamp01f((atan2f(dot(rel, cross(ori, r)), dot(rel, r)) + kPiF) / (2.0f * kPiF));
}

__device__ __forceinline__ void uv_cap(float3 p, float3 centre, float3 ori, float diam, float& u, float& v) {
  const float3 r = uv_right(ori);
  const float3 rel = p - centre;
  u = clamp01f(dot(rel, r) / diam + 0.5f);
  v = clamp01f(dot(rel, cross(ori, r)) / diam + 0.5f);
}

// Texture coordinates of BVH primitive i hit at p; bu, bv are the hit's
// barycentrics (triangles) or part (quadrics, in bu); scale = the hit
// material's uv scale.
__device__ __forceinline__ void prim_uv(const SceneView& S, int i, float3 p, float bu, float bv, float scale,
                                        float& u, float& v) {
  const float4* g = S.geom + 3 * (size_t)i;
  const float4 a = __ldg(g), b = __ldg(g + 1);
  const int type = __float_as_int(a.w);
  if (type == PRIM_TRI) {
    const float4* sh = S.shade + 4 * (size_t)i;
    const float4 s0 = __ldg(sh), s1 = __ldg(sh + 1), s2 = __ldg(sh + 2), vv = __ldg(sh + 3);
    const float w = 1.0f - bu - bv;
    u = w * s0.w + bu * s1.w + bv * s2.w;
    v = w * vv.x + bu * vv.y + bv * vv.z;
    return;
  }
  const float3 c = f3(a.x, a.y, a.z);
  if (type == PRIM_SPHERE) {
    const float r = b.x;
    u = clamp01f((atan2f((-p.z + c.z) / r, (p.x - c.x) / r) + kPiF) / (2.0f * kPiF));
    v = clamp01f(acosf(fminf(fmaxf((-p.y + c.y) / r, -1.f), 1.f)) / kPiF);
    uv_tile(scale, u, v);
    return;
  }
  const float4 cc = __ldg(g + 2);
  const float3 ori = f3(b.x, b.y, b.z);
  const int part = (int)bu;
  if (type == PRIM_CYL) {
    if (part == PART_SIDE) {
      u = uv_angle(p - c, ori);
      v = clamp01f(dot(p - c, ori) / cc.x + 0.5f);
    } else {
      uv_cap(p, c + ori * (cc.x * 0.5f * (part == PART_TOP ? 1.f : -1.f)), ori, 2.0f * b.w, u, v);
    }
  } else if (type == PRIM_CONE) {
    if (part == PART_SIDE) {
      u = uv_angle(p - c, ori);
      v = clamp01f(dot(p - c, ori) / cc.x);
    } else {
      uv_cap(p, c + ori * (cc.x * 0.5f), ori, 2.0f * b.w, u, v);
    }
  } else {
    u = uv_angle(p - c, ori);
    v = clamp01f((dot(p - c, ori) / (cc.w * 0.5f)) * 0.5f + 0.5f);
  }
  uv_tile(scale, u, v);
}

// get_uv_plane (hit_plane.c:18-41).
__device__ __forceinline__ void plane_uv(const PlaneD& pl, float3 p, float scale, bool has_mat, float& u, float& v) {
  const float3 n = f3(pl.nn.x, pl.nn.y, pl.nn.z);
  const float3 up = fabsf(n.y) < 0.99f ? f3(0.f, 1.f, 0.f) : f3(1.f, 0.f, 0.f);
  const float3 tg = unit(cross(up, n));
  const float3 local = p - f3(pl.pn.x, pl.pn.y, pl.pn.z);
  u = dot(local, tg);
  v = dot(local, cross(n, tg));
  if (has_mat) {
    u *= scale * 0.1f;
    v *= scale * 0.1f;
  }
  u -= floorf(u);
  v -= floorf(v);
}

// Material of BVH primitive i at the part hit (cylinder / cone caps).
__device__ __forceinline__ int prim_material(const SceneView& S, int i, int type, float part) {
  int mat = __ldg(S.meta + i).y;
  if (type == PRIM_CYL || type == PRIM_CONE) {
    const float4 c = __ldg(S.geom + 3 * (size_t)i + 2);
    const int p = (int)part;
    const int top = __float_as_int(c.y), bot = __float_as_int(c.z);
    if (p == PART_TOP && top >= 0) mat = top;
    else if (type == PRIM_CYL && p == PART_BOTTOM && bot >= 0) mat = bot;
  }
  return mat;
}

// Uniform in [0, 1) of the partial-transparency test: splitmix64's
// finalizer of key ^ (flat + 1) * golden ratio, 24 bits.
__device__ __forceinline__ float alpha_uniform(uint64_t key, uint32_t flat) {
  uint64_t z = key ^ ((uint64_t)(flat + 1) * 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (float)(z >> 40) * (1.0f / 16777216.0f);
}

// The alpha test of a candidate hit of primitive i at t: true when dropped.
__device__ __forceinline__ bool alpha_drops(const SceneView& S, int i, int type, float3 o, float3 d, float t,
                                            float bu, float bv, uint64_t key) {
  const int mat = prim_material(S, i, type, bu);
  if (mat < 0) return false;
  const MatTexD& mt = S.mat_tex[mat];
  if (!mt.alpha) return false;
  const float3 p = o + d * t;
  float u, v;
  prim_uv(S, i, p, bu, bv, mt.uv_scale, u, v);
  const float tr = 1.0f - tex_lookup(S, mt.tex[TS_COLOR], u, v, p).w;
  if (tr == 1.0f) return true;
  if (tr == 0.0f) return false;
  return alpha_uniform(key, (uint32_t)__ldg(S.meta + i).x) < tr;
}

// apply_normal_map (apply_map.c:38-58) on the faced normal n.
__device__ __forceinline__ float3 normal_map(const SceneView& S, const MatTexD& mt, float u, float v, float3 n) {
  const TexD& t = S.texs[mt.tex[TS_NORMAL] - 1];
  if (t.w <= 0) return n;           // any type, as long as it has an image
  const uchar4 q = texel_at(S, t, u, v);
  const float3 mp = f3(q.x / 127.5f - 1.0f, q.y / 127.5f - 1.0f, q.z / 127.5f - 1.0f);
  float3 tg = cross(n, f3(0.f, -1.f, 0.f));
  if (len2(tg) == 0.0f) tg = cross(n, f3(0.f, 0.f, 1.f));
  tg = unit(tg);
  const float3 bt = unit(cross(n, tg));
  const float3 res = tg * mp.x + bt * mp.y + n * mp.z;
  if (mt.normal_intensity == 1.0f) return unit(res);
  const float w = mt.normal_intensity;
  return unit(n * (1.0f - w) + unit(res) * w);
}

}  // namespace mrt
