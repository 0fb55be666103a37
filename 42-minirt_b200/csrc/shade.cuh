// shade.cuh — surface reconstruction, BSDF sampling, lights, sky and HDRI
// next-event estimation, in float, with the reference's estimator.
//
// Each function names the reference function it implements. Random numbers
// are drawn in the same order as the reference so that a path here and the
// same path in the FP64 oracle (counter-RNG mode) consume identical numbers.
#pragma once
#include "traverse.cuh"

namespace mrt {

struct Surf {
  float3 p, n;
  float3 color;
  int mat;
  int front;
  // SceneViewT only: this hit's material values with its texels applied
  // (apply_all_map writes them into the shared t_mat, apply_map.c:60-85)
  int has_hm;
  MaterialD hm;
};

struct PathState {
  float3 o, d;
  float3 power, acc;
  Rng rng;
  int last_mat;     // material of the last hit (sky * ao on a miss, path_trace.c:37-48)
  float last_ao;    // SceneViewT: that hit's ao value
};

// The material values of a hit: its own copy in a textured scene, else the
// material table's entry.
template <class V>
__device__ __forceinline__ const MaterialD& surf_mat(const V& S, const Surf& s) {
  if constexpr (V::kTextures) {
    if (s.has_hm) return s.hm;
  }
  return S.mats[s.mat];
}

// ao of the last hit for the sky term of a miss (path_trace.c:37-48).
template <class V>
__device__ __forceinline__ float last_hit_ao(const V& S, const PathState& P) {
  if constexpr (V::kTextures) return P.last_ao;
  return S.mats[P.last_mat].ao;
}

template <class V>
__device__ __forceinline__ void set_last_hit(const V& S, PathState& P, const Surf& s) {
  P.last_mat = s.mat;
  if constexpr (V::kTextures) P.last_ao = s.mat >= 0 ? surf_mat(S, s).ao : 1.0f;
}

// ----------------------------------------------------------------- sky

// get_hdr_pixel_skybox (get_hdr_value.c:43-68), texel (x, y).
__device__ __forceinline__ float3 sky_texel(const SceneView& S, int x, int y) {
  uint32_t px = __ldg(S.rgbe + (size_t)y * S.env_w + x);
  int e = (int)(px >> 24);
  float scale = ldexpf(1.0f, e - 128);
  if (!S.env_exposure_zero) scale *= S.env_scale_exp;
  float3 c = f3((float)(px & 255u) * scale / 255.0f, (float)((px >> 8) & 255u) * scale / 255.0f,
                (float)((px >> 16) & 255u) * scale / 255.0f);
  if (S.env_inv_gamma != 1.0f)
    c = f3(powf(c.x, S.env_inv_gamma), powf(c.y, S.env_inv_gamma), powf(c.z, S.env_inv_gamma));
  return c;
}

// Texel (x, y) of direction d: the spherical mapping of get_background_color
// (background.c:15-70).
__device__ __forceinline__ void sky_xy(const SceneView& S, float3 d, int& x, int& y) {
  d = unit(d);
  float v = 0.5f + asinf(fminf(fmaxf(d.y, -1.f), 1.f)) / (float)MRT_PI_D;
  float u = 0.5f - atan2f(d.z, d.x) / (float)(2.0 * MRT_PI_D);
  x = (int)(u * (S.env_w - 1));
  y = (int)(v * (S.env_h - 1));
  x = min(max(x, 0), S.env_w - 1);
  y = min(max(y, 0), S.env_h - 1);
}

// get_background_color[_clamp] (background.c:15-84).
__device__ __forceinline__ float3 background(const SceneView& S, float3 d, bool clamp) {
  if (!S.has_env) return f3(S.amb_const[0], S.amb_const[1], S.amb_const[2]);
  int x, y;
  sky_xy(S, d, x, y);
  float3 c;
  if (S.sky_rgb) {
    const float* t = S.sky_rgb + 3 * ((size_t)y * S.env_w + x);
    c = f3(t[0], t[1], t[2]);
  } else {
    c = sky_texel(S, x, y);
  }
  if (clamp) c = f3(fminf(fmaxf(c.x, 0.f), 16.f), fminf(fmaxf(c.y, 0.f), 16.f), fminf(fmaxf(c.z, 0.f), 16.f));
  return c;
}

// ------------------------------------------------------------- surface

// Normal, facing and material of a cylinder, cone or hyperboloid hit
// (hit_cylinder.c, hit_cone.c, hit_hyperboloid.c, hit_obj.c:16-49): the
// hit point is already in s.p, the part hit in h.u.
__device__ __forceinline__ void quadric_surf(const SceneView& S, const HitInfo& h, int type, float3 d, Surf& s) {
  const float4* g = S.geom + 3 * (size_t)h.prim;
  const float4 a = __ldg(g), b = __ldg(g + 1), c = __ldg(g + 2);
  const float3 pos = f3(a.x, a.y, a.z), ori = f3(b.x, b.y, b.z);
  const float3 axis = unit(ori);
  const int part = (int)h.u;
  float3 n;
  if (type == PRIM_CYL) {
    if (part == PART_SIDE) {
      // the lateral normal is faced twice (set_normal_face, then once more
      // at the end of hit_cylinder): it always ends facing the ray, front 1
      const float3 base = pos - axis * (c.x * 0.5f);
      const float3 out = unit((s.p - base) - axis * dot(s.p - base, axis));
      s.n = dot(d, out) < 0.0f ? out : -out;
      s.front = 1;
    } else {
      n = part == PART_TOP ? ori : -ori;
      s.front = dot(d, n) < 0.0f;
      s.n = s.front ? n : -n;
    }
    const int top = __float_as_int(c.y), bot = __float_as_int(c.z);
    if (part == PART_TOP && top >= 0) s.mat = top;
    else if (part == PART_BOTTOM && bot >= 0) s.mat = bot;
    return;
  }
  if (type == PRIM_CONE) {
    if (part == PART_SIDE) {
      const float rr = b.w / c.x;
      n = unit((s.p - pos) - axis * ((1.0f + rr * rr) * dot(s.p - pos, axis)));
    } else {
      n = axis;
    }
    s.front = dot(d, n) < 0.0f;
    s.n = s.front ? n : -n;
    const int top = __float_as_int(c.y);
    if (part == PART_TOP && top >= 0) s.mat = top;
    return;
  }
  // hyperboloid: gradient of the quadric in the frame of compute_normal
  // (hit_hyperboloid.c:36-52)
  const float3 to_p = s.p - pos;
  const float3 tmp = fabsf(axis.y) < 0.99f ? f3(0.f, 1.f, 0.f) : f3(1.f, 0.f, 0.f);
  const float3 u = unit(cross(tmp, axis));
  const float3 v = cross(axis, u);
  n = unit(u * (2.0f * dot(to_p, u) / (b.w * b.w)) + v * (2.0f * dot(to_p, v) / (c.x * c.x)) -
           axis * (2.0f * dot(to_p, axis) / (c.y * c.y)));
  s.front = dot(d, n) < 0.0f;
  s.n = s.front ? n : -n;
}

// Hit record of handle_hit / hit_all_planes + get_hit_register_color
// (hit_obj.c:68, hit_register.c:79-107, get_hit_color.c:17-36), untextured.
template <class V>
__device__ __forceinline__ Surf make_surf(const V& S, const HitInfo& h, float3 o, float3 d,
                                          int render_mode, bool is_light = false) {
  Surf s;
  s.p = o + d * h.t;
  s.has_hm = 0;
  uint32_t col;
  if (h.prim >= 0) {
    int4 m = __ldg(S.meta + h.prim);
    s.mat = m.y;
    col = (uint32_t)m.w;
    if (m.z == PRIM_TRI) {
      const float4* sh = S.shade + 4 * (size_t)h.prim;
      float4 n0 = __ldg(sh), n1 = __ldg(sh + 1), n2 = __ldg(sh + 2);
      float w = 1.0f - h.u - h.v;
      float3 n = unit(f3(w * n0.x + h.u * n1.x + h.v * n2.x, w * n0.y + h.u * n1.y + h.v * n2.y,
                         w * n0.z + h.u * n1.z + h.v * n2.z));
      if (!S.one_sided && dot(d, n) > 0.0f) { s.front = 0; s.n = -n; }
      else { s.front = 1; s.n = n; }
    } else if (!V::kQuadrics || m.z == PRIM_SPHERE) {
      float4 a = __ldg(S.geom + 3 * (size_t)h.prim), b = __ldg(S.geom + 3 * (size_t)h.prim + 1);
      float3 out = (s.p - f3(a.x, a.y, a.z)) * (1.0f / b.x);
      s.front = dot(d, out) < 0.0f;
      s.n = s.front ? out : -out;
    } else if constexpr (V::kQuadrics) {
      quadric_surf(S, h, m.z, d, s);
    }
  } else {
    const PlaneD& pl = S.planes[-1 - h.prim];
    float3 n = f3(pl.nn.x, pl.nn.y, pl.nn.z);
    s.front = dot(d, n) < 0.0f;
    s.n = s.front ? n : -n;
    s.mat = pl.meta.y;
    col = (uint32_t)pl.meta.w;
  }
  if constexpr (V::kTextures) {
    if (s.mat >= 0 && S.mat_tex[s.mat].any) {
      // apply_all_map (apply_map.c:60-85) into this hit's copy
      const MatTexD& mt = S.mat_tex[s.mat];
      float u, v;
      if (h.prim >= 0) prim_uv(S, h.prim, s.p, h.u, h.v, mt.uv_scale, u, v);
      else plane_uv(S.planes[-1 - h.prim], s.p, mt.uv_scale, true, u, v);
      s.hm = S.mats[s.mat];
      s.has_hm = 1;
      if (mt.tex[TS_NORMAL]) s.n = normal_map(S, mt, u, v, s.n);
      if (mt.tex[TS_TRANSMISSION]) s.hm.transmission = tex_lookup(S, mt.tex[TS_TRANSMISSION], u, v, s.p).x;
      if (!is_light) {
        if (mt.tex[TS_ROUGHNESS]) {
          const float r = tex_lookup(S, mt.tex[TS_ROUGHNESS], u, v, s.p).x;
          s.hm.roughness = r;
          s.hm.alpha4 = (r * r) * (r * r);
        }
        if (mt.tex[TS_METALLIC]) s.hm.metallic = tex_lookup(S, mt.tex[TS_METALLIC], u, v, s.p).x;
        if (mt.tex[TS_AO]) s.hm.ao = tex_lookup(S, mt.tex[TS_AO], u, v, s.p).x;
        if (mt.tex[TS_EMIS_STRENGTH])
          s.hm.emission_strength = tex_lookup(S, mt.tex[TS_EMIS_STRENGTH], u, v, s.p).x;
        if (mt.tex[TS_EMIS_COLOR]) {
          const float4 e = tex_lookup(S, mt.tex[TS_EMIS_COLOR], u, v, s.p);
          s.hm.emission[0] = e.x;
          s.hm.emission[1] = e.y;
          s.hm.emission[2] = e.z;
        }
      }
      if (render_mode != 2 && mt.tex[TS_COLOR]) {
        const float4 c = tex_lookup(S, mt.tex[TS_COLOR], u, v, s.p);
        s.color = f3(c.x, c.y, c.z);
        return s;
      }
    }
  }
  if (render_mode == 2)
    s.color = f3((s.n.x + 1) * 0.5f, (s.n.z + 1) * 0.5f, (s.n.y + 1) * 0.5f);
  else if (s.mat >= 0)
    s.color = ld3(S.mats[s.mat].color);
  else
    s.color = unpack_rgb8(col);
  return s;
}

// ------------------------------------------------------------- BSDFs

// ggx_sample_hemisphere (material/utils.c:39-62).
__device__ __forceinline__ float3 ggx_sample(Rng& rng, float3 n, float alpha4) {
  float u2 = rng.next();
  float r = rng.next();
  float ct = sqrtf((1.0f - u2) / (1.0f + (alpha4 - 1.0f) * u2));
  float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  float sp, cp;
  sincospif(2.0f * r, &sp, &cp);
  float3 tg = unit(cross(n, f3(1.f, 0.f, 0.f)));
  if (len2(tg) < 0.0001f) tg = unit(cross(n, f3(0.f, 1.f, 0.f)));
  return n * ct + (tg * (cp * st) + unit(cross(n, tg)) * (sp * st));
}

__device__ __forceinline__ float pow5(float x) { float x2 = x * x; return x2 * x2 * x; }

// metallic_color (metallic.c:25-46) with fresnel_schlick_color (fresnel_schlick.c:19).
__device__ __forceinline__ void metallic(const MaterialD& M, PathState& P, const Surf& s) {
  float ct = -dot(unit(P.d), s.n);
  float3 m = M.roughness > 0.0f ? ggx_sample(P.rng, s.n, M.alpha4) : s.n;
  P.d = unit(P.d - m * (2.0f * dot(P.d, m)));
  float k = pow5(1.0f - ct);
  P.power = P.power * (s.color + (f3(1.f, 1.f, 1.f) - s.color) * k);
}

// refracted_ray / refracted_value / refracted_v (refraction.c:15-78).
__device__ __forceinline__ void refract(const SceneView& S, const MaterialD& M, PathState& P,
                                        const Surf& s) {
  float eta = s.front ? S.ior_all / M.ior : M.ior / S.ior_all;
  P.d = unit(P.d);
  float ct = fminf(-dot(P.d, s.n), 1.0f);
  float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  if (eta * st > 1.0f) {
    metallic(M, P, s);
    return;
  }
  float3 perp = (P.d + s.n * fminf(dot(-P.d, s.n), 1.0f)) * eta;
  float3 dir = unit(s.n * (-sqrtf(fabsf(1.0f - len2(perp)))) + perp);
  if (M.roughness > 0.0f) dir = ggx_sample(P.rng, dir, M.alpha4);
  P.d = dir;
  P.power = P.power * s.color;
}

// cos_weighted_sample_hemishphere (material_default.c:20-38).
__device__ __forceinline__ float3 cos_hemisphere(Rng& rng, float3 n) {
  float r1 = rng.next();
  float r2 = rng.next();
  float sp, cp;
  sincospif(2.0f * r1, &sp, &cp);
  float sr = sqrtf(r2);
  float3 l = f3(cp * sr, sqrtf(1.0f - r2), sp * sr);
  n = unit(n);
  float3 u = fabsf(n.y) < 0.999f ? unit(cross(f3(0.f, 1.f, 0.f), n)) : unit(cross(f3(1.f, 0.f, 0.f), n));
  return unit((u * l.x + n * l.y) + cross(n, u) * l.z);
}

// ------------------------------------------------------------- lights

// random_in_unit_sphere (random.c:42-50).
__device__ __forceinline__ float3 rnd_in_unit_sphere(Rng& rng) {
  float3 p;
  p.x = rng.next() * 2 - 1.0f;
  p.y = rng.next() * 2 - 1.0f;
  p.z = rng.next() * 2 - 1.0f;
  if (len2(p) >= 1.0f) p = unit(p) * cbrtf(rng.next());
  return p;
}

// reflection_vec (material/utils.c:21).
__device__ __forceinline__ float3 reflect_v(float3 v, float3 n) { return v - n * (2.0f * dot(v, n)); }

// compute_light_v2 (light_manager.c:59-71) and its point / directional
// terms (p_light.c:19-89, d_light.c:19-55). The reference sums into uint64
// channels (t_lcolor), truncating every addition; floorf reproduces that.
template <class V>
__device__ __forceinline__ float3 compute_light(const V& S, Rng& rng, const Surf& s,
                                                int* status, uint32_t& shadow_rays) {
  float lc0 = 0.f, lc1 = 0.f, lc2 = 0.f;
  if (S.n_lights == 0) return f3(0.f, 0.f, 0.f);
  float3 view = unit(ld3(S.cam) - s.p);
  for (int i = 0; i < S.n_lights; ++i) {
    const LightD L = S.lights[i];
    float3 lp = ld3(L.pos);
    if (L.type == 0) {
      float sf;
      bool vis;
      if (L.radius == 0.0f || L.shadow_sample <= 1) {
        sf = 1.0f;
        float3 to = lp - s.p;
        float dist = sqrtf(len2(to));
        shadow_rays++;
        vis = !any_hit(S, s.p, unit(to), dist, status, rng.s);
      } else {
        int hits = 0;
        for (int k = 0; k < L.shadow_sample; ++k) {
          float3 tgt = lp + rnd_in_unit_sphere(rng) * L.radius;
          float3 to = tgt - s.p;
          shadow_rays++;
          if (!any_hit(S, s.p, unit(to), sqrtf(len2(to)), status, rng.s)) hits++;
        }
        sf = (float)hits / (float)L.shadow_sample;
        vis = sf > 0.0f;
      }
      if (vis) {
        float3 ld = unit(lp - s.p);
        float ndl = dot(s.n, ld);
        if (ndl > 0.0f) {
          float di = L.brightness * ndl * sf;
          lc0 = floorf(lc0 + L.color[0] * di);
          lc1 = floorf(lc1 + L.color[1] * di);
          lc2 = floorf(lc2 + L.color[2] * di);
          float rdv = fmaxf(dot(reflect_v(-ld, s.n), view), 0.0f);
          float spec = powf(rdv, 64.0f) * sf;
          lc0 = floorf(lc0 + L.color[0] * L.brightness * spec);
          lc1 = floorf(lc1 + L.color[1] * L.brightness * spec);
          lc2 = floorf(lc2 + L.color[2] * L.brightness * spec);
        }
      }
    } else {
      shadow_rays++;
      if (!any_hit(S, s.p, unit(-lp), INFINITY, status, rng.s)) {
        float3 ld = -lp;
        float ndl = dot(s.n, ld);
        if (ndl > 0.0f) {
          lc0 = floorf(lc0 + L.color[0] * L.brightness * ndl);
          lc1 = floorf(lc1 + L.color[1] * L.brightness * ndl);
          lc2 = floorf(lc2 + L.color[2] * L.brightness * ndl);
          float rdv = fmaxf(dot(reflect_v(-ld, s.n), view), 0.0f);
          float spec = powf(rdv, 64.0f);
          lc0 = floorf(lc0 + L.color[0] * L.brightness * spec);
          lc1 = floorf(lc1 + L.color[1] * L.brightness * spec);
          lc2 = floorf(lc2 + L.color[2] * L.brightness * spec);
        }
      }
    }
  }
  return f3(lc0 / 255.0f, lc1 / 255.0f, lc2 / 255.0f);
}

// ------------------------------------------------------------ env NEE

// Outcome index of one importance sample. Alias mode: one bucket of the
// alias table built from the exact outcome distribution of the reference's
// two-step inverse-CDF lookup (get_dir.c:15-27). Lookup mode: that two-step
// lookup itself, with the reference's double arithmetic, on the same tables.
// Outcome k = row * W + (column index - floor(v (H-1) W)).
__device__ __forceinline__ int env_sample(const SceneView& S, Rng& rng) {
  float r1 = rng.next();
  float r2 = rng.next();
  if (!S.env_lookup) {
    int n = S.n_env_outcomes;
    int i = min((int)(r1 * (float)n), n - 1);
    float2 e = __ldg(S.alias + i);
    return r2 < e.x ? i : __float_as_int(e.y);
  }
  const int H = S.env_h, W = S.env_w;
  const int iy = min((int)((double)r1 * (double)(H - 1)), H - 2);
  const double vy = (double)__ldg(S.cdf_m_inv + iy);
  // (int)(n.y * (H-1) * W + r.y * (W-1)) in double, without fused multiply-adds
  const double A = __dmul_rn(__dmul_rn(vy, (double)(H - 1)), (double)W);
  const double j = floor(__dadd_rn(A, __dmul_rn((double)r2, (double)(W - 1))));
  const int d = min(max((int)(j - floor(A)), 0), W - 1);
  return iy * W + d;
}

}  // namespace mrt
