// adjoint.cu — differentiable rendering: parameter views and the
// path-replay adjoint.
//
// Parameters theta are float shadows of reference fields that are 8-bit
// colours or RGBE texels there. Layout (M materials, sky W x H):
//   [albedo M*3 | roughness M | emission strength M | sky radiance H*W*3]
// albedo is t_mat.color_value / 255, roughness roughness_value,
// emission emission_strength, and sky the linear radiance that
// get_hdr_pixel_skybox returns per texel (get_hdr_value.c:43).
//
// Forward: the production renderer over a SceneView whose materials, sky and
// HDRI sampling tables are rebuilt from theta (diff_mats_kernel, the FP64
// table build of env.cu fed with the float sky, diff_env_records_kernel),
// so a forward at the scene's own values is the ordinary render.
//
// Backward, in wavefront form: a replay kernel traces every path again
// with the production shading functions (persistent, lanes regenerate
// paths) and writes one 80-byte tape entry per bounce to HBM (ray, power,
// hit, branch, random numbers, NEE outcome); then one reverse kernel per
// bounce level, deepest first, turns the adjoint state of each path
// (d loss / d power, origin, direction after the bounce) into the state
// before it. The reverse step needs the vector-Jacobian product of the
// bounce's outputs (hit point, next direction, the geometry-dependent
// cosines) with their adjoints, with respect to its inputs (incoming origin
// and direction) and the material roughness. It is computed in forward
// mode: the bounce's geometry is re-evaluated once in Dual<7> arithmetic
// (slots: origin xyz, direction xyz, roughness) on the scalar
// phi = sum(adjoint * output), whose seven derivative slots are exactly
// that product.
//
// What carries gradient (all for fixed random numbers, i.e. the derivative
// that central differences with common random numbers converge to as the
// step shrinks):
//   * albedo: the power multipliers (diffuse, Schlick-tinted metal,
//     refraction) and the radiance terms of default_mat;
//   * emission strength: the emitted term of material_manager_v3;
//   * sky texels: the NEE radiance, the miss radiance (inside the [0, 16]
//     clamp), and pdf_joint = luminance / mean luminance (calc_pdf.c:93),
//     through the sampled texel's luminance and through the mean, which
//     every texel shares (a dense term added at the end);
//   * roughness: through the GGX-sampled directions (material/utils.c:39)
//     and everything they move downstream: hit points, interpolated
//     normals, later sampled directions, NEE cosines, Fresnel factors.
// Detached, because their derivative is zero almost everywhere: the
// discrete choices (which primitive is hit, which branch, the inverse-CDF
// table lookups, visibility, the nearest-texel sky lookup of a direction),
// the point/directional-light term (its channels are truncated to
// integers, light_manager.c:103) and the photon estimate (treated as a
// constant field).
#include <algorithm>
#include <type_traits>

#include "dual.cuh"
#include "kernels.h"
#include "path.cuh"

namespace mrt {

namespace {

constexpr int kSlots = 7;          // origin xyz, direction xyz, roughness
using D7 = Dual<kSlots>;

enum TapeFlags : int {
  TF_BRANCH = 3,       // 0 diffuse, 1 metal, 2 dielectric reflection, 3 refraction
  TF_FRONT = 4,
  TF_EMIT = 8,
  TF_NEE = 16,         // HDRI NEE contributed (visible, pdf > 0)
  TF_GGX = 32,         // a GGX sample was drawn (roughness > 0)
  TF_PART_SHIFT = 6,   // bits 6-7: part of a quadric hit (QuadricPart)
};
enum Branch : int { BR_DIFFUSE = 0, BR_METAL = 1, BR_REFLECT = 2, BR_REFRACT = 3 };

// ------------------------------------------------------------ dual helpers

__device__ __forceinline__ V3T<D7> dv3(float x, float y, float z) { return V3T<D7>{D7(x), D7(y), D7(z)}; }
__device__ __forceinline__ V3T<D7> dv3(float3 a) { return dv3(a.x, a.y, a.z); }
__device__ __forceinline__ V3T<D7> dunit(const V3T<D7>& a) {
  const D7 l2 = vdot(a, a);
  if (l2.v > 0.f) return a * (D7(1.0f) / dsqrt(l2));
  return dv3(0.f, 0.f, 0.f);
}
__device__ __forceinline__ D7 dot_c(const V3T<D7>& a, float3 w) { return a.x * w.x + a.y * w.y + a.z * w.z; }

// Outward normal of a quadric part at p (quadric_surf's formulas, before
// facing): the lateral normals depend on p, the caps' do not.
__device__ __forceinline__ V3T<D7> quadric_normal_dual(int type, int part, const float4& a, const float4& b,
                                                       const float4& c, const V3T<D7>& p) {
  const float3 pos = f3(a.x, a.y, a.z), ori = f3(b.x, b.y, b.z), axis = unit(ori);
  if (type == PRIM_CYL) {
    if (part == PART_TOP) return dv3(ori);
    if (part == PART_BOTTOM) return dv3(-ori);
    const V3T<D7> q = p - dv3(pos - axis * (c.x * 0.5f));
    return dunit(q - dv3(axis) * dot_c(q, axis));
  }
  if (type == PRIM_CONE) {
    if (part != PART_SIDE) return dv3(axis);
    const float rr = b.w / c.x;
    const V3T<D7> q = p - dv3(pos);
    return dunit(q - dv3(axis) * (dot_c(q, axis) * (1.0f + rr * rr)));
  }
  const float3 tmp = fabsf(axis.y) < 0.99f ? f3(0.f, 1.f, 0.f) : f3(1.f, 0.f, 0.f);
  const float3 u = unit(cross(tmp, axis));
  const float3 v = cross(axis, u);
  const V3T<D7> q = p - dv3(pos);
  return dunit(dv3(u) * (dot_c(q, u) * (2.0f / (b.w * b.w))) + dv3(v) * (dot_c(q, v) * (2.0f / (c.x * c.x))) -
               dv3(axis) * (dot_c(q, axis) * (2.0f / (c.y * c.y))));
}

// Hit point and shading normal of a known primitive for the ray (o, d):
// make_surf's formulas with t (and u, v) recomputed from the ray. For a
// quadric, t follows the implicit surface F(o + t d) = 0 to first order:
// dt = -N . (do + t dd) / (N . d) with N the normal at the recorded hit,
// which is the derivative of t through the tangent plane there; the value
// of t stays the recorded one.
template <class V>
__device__ __forceinline__ void surf_dual(const V& S, int prim, float t_rec, int flags,
                                          const V3T<D7>& o, const V3T<D7>& d, V3T<D7>& p, V3T<D7>& n) {
  const int front = (flags & TF_FRONT) != 0;
  if (prim >= 0) {
    const float4* g = S.geom + 3 * (size_t)prim;
    const float4 a = __ldg(g), b = __ldg(g + 1);
    const int type = __float_as_int(a.w);
    if constexpr (V::kQuadrics) {
      if (type >= PRIM_CYL) {
        const float4 c = __ldg(g + 2);
        const int part = (flags >> TF_PART_SHIFT) & 3;
        const float3 o0 = f3(o.x.v, o.y.v, o.z.v), d0 = f3(d.x.v, d.y.v, d.z.v);
        const float3 p0 = o0 + d0 * t_rec;
        const V3T<D7> n0 = quadric_normal_dual(type, part, a, b, c, dv3(p0));
        const float3 N = f3(n0.x.v, n0.y.v, n0.z.v);
        D7 t = dot_c(dv3(p0) - o, N) / dot_c(d, N);
        t.v = t_rec;
        p = o + d * t;
        const V3T<D7> out = quadric_normal_dual(type, part, a, b, c, p);
        // the cylinder's lateral normal faces the ray with front_face 1
        const bool keep = (type == PRIM_CYL && part == PART_SIDE)
                              ? (d.x.v * out.x.v + d.y.v * out.y.v + d.z.v * out.z.v) < 0.0f
                              : front != 0;
        n = keep ? out : -out;
        return;
      }
    }
    if (type == PRIM_TRI) {
      const float4 c = __ldg(g + 2);
      const V3T<D7> v0 = dv3(a.x, a.y, a.z), e1 = dv3(b.x, b.y, b.z), e2 = dv3(c.x, c.y, c.z);
      const V3T<D7> h = vcross(d, e2);
      const D7 f = D7(1.0f) / vdot(e1, h);
      const V3T<D7> s = o - v0;
      const D7 u = f * vdot(s, h);
      const V3T<D7> q = vcross(s, e1);
      const D7 v = f * vdot(d, q);
      const D7 t = f * vdot(e2, q);
      p = o + d * t;
      const float4* sh = S.shade + 4 * (size_t)prim;
      const float4 n0 = __ldg(sh), n1 = __ldg(sh + 1), n2 = __ldg(sh + 2);
      const D7 w = D7(1.0f) - u - v;
      V3T<D7> nn = dv3(n0.x, n0.y, n0.z) * w + dv3(n1.x, n1.y, n1.z) * u + dv3(n2.x, n2.y, n2.z) * v;
      nn = dunit(nn);
      n = front ? nn : -nn;
    } else {
      const V3T<D7> cc = dv3(a.x, a.y, a.z);
      const V3T<D7> oc = o - cc;
      const D7 A = vdot(d, d), bh = vdot(d, oc);
      const V3T<D7> l = oc - d * (bh / A);
      const D7 disc = A * (D7(b.y) - vdot(l, l));
      const D7 sq = dsqrt(disc);
      const D7 qv = bh.v >= 0.f ? -(bh + sq) : sq - bh;
      const D7 cq = vdot(oc, oc) - D7(b.y);
      const D7 r0 = qv / A;
      const D7 r1 = qv.v != 0.f ? cq / qv : r0;
      const D7 t = fabsf(r0.v - t_rec) <= fabsf(r1.v - t_rec) ? r0 : r1;
      p = o + d * t;
      const V3T<D7> out = (p - cc) * (1.0f / b.x);
      n = front ? out : -out;
    }
  } else {
    const PlaneD& pl = S.planes[-1 - prim];
    const float3 pn = f3(pl.nn.x, pl.nn.y, pl.nn.z);
    const D7 t = dot_c(dv3(pl.pn.x, pl.pn.y, pl.pn.z) - o, pn) / dot_c(d, pn);
    p = o + d * t;
    n = front ? dv3(pn) : dv3(-pn);
  }
}

// ggx_sample_hemisphere (material/utils.c:39-62) with its random numbers given.
// sin(theta) comes from 1 - ct^2 = alpha4 u / (1 + (alpha4 - 1) u), the same
// value without the cancellation of 1 - ct^2 at small roughness (alpha4 of
// 6e-6 at roughness 0.05), which would cost its derivative two digits.
__device__ __forceinline__ V3T<D7> ggx_dual(const V3T<D7>& n, const D7& alpha4, float u2, float r) {
  const D7 den = D7(1.0f) + (alpha4 - D7(1.0f)) * u2;
  const D7 ct = dsqrt(D7(1.0f - u2) / den);
  const D7 st = dsqrt(alpha4 * u2 / den);
  float sp, cp;
  sincospif(2.0f * r, &sp, &cp);
  V3T<D7> tg = dunit(vcross(n, dv3(1.f, 0.f, 0.f)));
  if (vdot(tg, tg).v < 0.0001f) tg = dunit(vcross(n, dv3(0.f, 1.f, 0.f)));
  return n * ct + (tg * (st * cp) + dunit(vcross(n, tg)) * (st * sp));
}

// cos_weighted_sample_hemishphere (material_default.c:20-38), random numbers given.
__device__ __forceinline__ V3T<D7> coshemi_dual(V3T<D7> n, float r1, float r2) {
  float sp, cp;
  sincospif(2.0f * r1, &sp, &cp);
  const float sr = sqrtf(r2);
  const float lx = cp * sr, ly = sqrtf(1.0f - r2), lz = sp * sr;
  n = dunit(n);
  const V3T<D7> u = fabsf(n.y.v) < 0.999f ? dunit(vcross(dv3(0.f, 1.f, 0.f), n))
                                          : dunit(vcross(dv3(1.f, 0.f, 0.f), n));
  return dunit((u * lx + n * ly) + vcross(n, u) * lz);
}

// Reflection about the microfacet normal: metallic_color (metallic.c:25-46)
// and reflected_dielectric_color (dielectric.c:15-33).
__device__ __forceinline__ V3T<D7> reflect_dual(const V3T<D7>& d, const V3T<D7>& m) {
  return dunit(d - m * (D7(2.0f) * vdot(d, m)));
}

// ----------------------------------------------------------- replay (float)

// What the replay records of one bounce besides the ray and power.
struct Rec {
  int flags;
  float ra, rb;        // the sampler's two random numbers
  int nee;             // HDRI outcome of the NEE sample, -1 none
  float3 T;            // direct-light + caustic term of default_mat (detached)
};

__device__ __forceinline__ void record_pair(const Rng& r, Rec& rec) {
  Rng c = r;
  rec.ra = c.next();
  rec.rb = c.next();
}

// default_mat (material_default.c:71-92), recording.
template <class V>
__device__ __forceinline__ void default_rec(const V& S, PathState& P, const Surf& s, int* status,
                                            PathCounters& C, Rec& rec) {
  const float3 direct = compute_light(S, P.rng, s, status, C.shadow);
  const float3 total = direct + caustic_estimate(S, s.p);
  rec.T = total;
  P.acc = P.acc + (s.color * P.power) * total;
  P.power = P.power * s.color;
  if (S.env_nee) {   // env_nee (path.cuh), recording the outcome
    const int k = env_sample(S, P.rng);
    rec.nee = k;
    const float4 e = __ldg(S.env_rec0 + k);
    const float3 dir = f3(e.x, e.y, e.z);
    P.d = dir;
    if (!any_hit(S, s.p, dir, INFINITY, status)) {
      const float ct = dot(s.n, dir);
      const float pdf = e.w;
      if (pdf > 0.0f) {
        const float4 r = __ldg(S.env_rec1 + k);
        float3 rad = f3(r.x, r.y, r.z);
        if (s.mat >= 0) rad = rad * S.mats[s.mat].ao;
        rad = rad * P.power;
        rad = rad * (ct / pdf);
        P.acc = P.acc + rad;
        P.power = P.power * (1.0f - ct);
        rec.flags |= TF_NEE;
      }
    }
  }
  record_pair(P.rng, rec);
  P.d = cos_hemisphere(P.rng, s.n);
  rec.flags = (rec.flags & ~TF_BRANCH) | BR_DIFFUSE;
}

__device__ __forceinline__ void metal_rec(const MaterialD& M, PathState& P, const Surf& s, Rec& rec) {
  if (M.roughness > 0.0f) { record_pair(P.rng, rec); rec.flags |= TF_GGX; }
  rec.flags = (rec.flags & ~TF_BRANCH) | BR_METAL;
  metallic(M, P, s);
}

__device__ __forceinline__ void refract_rec(const SceneView& S, const MaterialD& M, PathState& P,
                                            const Surf& s, Rec& rec) {
  // refracted_ray's total-internal-reflection test (refraction.c:15-40)
  const float eta = s.front ? S.ior_all / M.ior : M.ior / S.ior_all;
  const float3 dn = unit(P.d);
  const float ct = fminf(-dot(dn, s.n), 1.0f);
  const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  if (M.roughness > 0.0f) { record_pair(P.rng, rec); rec.flags |= TF_GGX; }
  rec.flags = (rec.flags & ~TF_BRANCH) | (eta * st > 1.0f ? BR_METAL : BR_REFRACT);
  refract(S, M, P, s);
}

// material_manager_v3 (path_trace.c:15-35) + dielectric_mat (dielectric.c:37-64).
template <class V>
__device__ __forceinline__ void material_rec(const V& S, PathState& P, const Surf& s, int* status,
                                             PathCounters& C, Rec& rec) {
  if (s.mat < 0) { default_rec(S, P, s, status, C, rec); return; }
  const MaterialD& M = S.mats[s.mat];
  if (M.emission_strength > 0.0f) {
    P.acc = P.acc + (ld3(M.emission) * M.emission_strength) * P.power;
    rec.flags |= TF_EMIT;
  }
  bool metal;
  if (M.metallic == 1.0f) metal = true;
  else if (M.metallic == 0.0f) metal = false;
  else metal = M.metallic > P.rng.next();
  if (metal) { metal_rec(M, P, s, rec); return; }
  if (M.ior > 0.0f) {
    const float ct = -dot(unit(P.d), s.n);
    const float refl = M.f0 + (1.0f - M.f0) * pow5(1.0f - ct);
    if (refl >= P.rng.next() && M.ior != 1.0f) {
      if (M.roughness > 0.0f) { record_pair(P.rng, rec); rec.flags |= TF_GGX; }
      rec.flags = (rec.flags & ~TF_BRANCH) | BR_REFLECT;
      const float3 m = M.roughness > 0.0f ? ggx_sample(P.rng, s.n, M.alpha4) : s.n;
      P.d = unit(P.d - m * (2.0f * dot(P.d, m)));
    } else if (M.transmission == 1.0f) {
      refract_rec(S, M, P, s, rec);
    } else if (M.transmission == 0.0f) {
      default_rec(S, P, s, status, C, rec);
    } else if (M.transmission < P.rng.next()) {
      default_rec(S, P, s, status, C, rec);
    } else {
      refract_rec(S, M, P, s, rec);
    }
  } else {
    default_rec(S, P, s, status, C, rec);
  }
}

// Gradient sums are 64-bit fixed point (AdjointArgs::q_scale): each value is
// rounded to an integer once, and integer additions give the same total in
// any order, so the result does not depend on thread scheduling.
__device__ __forceinline__ long long fx_q(float v, double scale) {
  double x = (double)v * scale;
  if (!(x == x)) x = 0.0;                      // NaN contributes nothing
  x = fmin(fmax(x, -4.0e18), 4.0e18);
  return __double2ll_rn(x);
}

// atomicAdd with the lanes of a warp that target the same address summed
// first (one atomic per distinct address): HDRI NEE concentrates on the few
// texels of a sun, and a warp's paths often share a material.
__device__ __forceinline__ void agg_add_q(long long* addr, long long q) {
  const unsigned active = __activemask();
  const unsigned peers = __match_any_sync(active, (unsigned long long)addr);
  const int leader = __ffs(peers) - 1;
  long long sum = 0;
  for (unsigned m = peers; m; m &= m - 1) sum += __shfl_sync(peers, q, __ffs(m) - 1);
  if ((int)(threadIdx.x & 31) == leader && sum != 0)
    atomicAdd(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)sum);
}

__device__ __forceinline__ void add_sky_grad(const AdjointArgs& A, int texel, int c, float v) {
  agg_add_q(A.q_sky + 3 * (size_t)texel + c, fx_q(v, A.q_scale));
}

// Shared-memory accumulators of the per-material gradients of one block.
struct MatGrad {
  long long* s;   // [albedo M*3 | roughness M | emission M], fixed point
  int M;
  double scale;
  __device__ __forceinline__ void albedo(int m, int c, float v) { agg_add_q(s + 3 * m + c, fx_q(v, scale)); }
  __device__ __forceinline__ void rough(int m, float v) { agg_add_q(s + 3 * M + m, fx_q(v, scale)); }
  __device__ __forceinline__ void emis(int m, float v) { agg_add_q(s + 4 * M + m, fx_q(v, scale)); }
};

// One reverse step: the adjoint state (Pb, ob, db) after bounce k becomes
// the state before it; gradients of the bounce's parameters are added.
template <class V>
__device__ __forceinline__ void reverse_step(const V& S, const AdjointArgs& A, MatGrad& G,
                                             const TapeEntry& te, float3 g, float inv_col, float3& Pb,
                                             float3& ob, float3& db, float& gcol) {
  const float lw[3] = {0.2126f, 0.7152f, 0.0722f};
  const int prim = te.meta.x, mat = te.meta.y, flags = te.meta.z, nee_k = te.meta.w;
  const int br = flags & TF_BRANCH;
  const bool ggx = (flags & TF_GGX) != 0;
  const MaterialD* M = mat >= 0 ? S.mats + mat : nullptr;
  float3 col;
  if (mat >= 0) col = ld3(M->color);
  else col = unpack_rgb8((uint32_t)(prim >= 0 ? __ldg(S.meta + prim).w : S.planes[-1 - prim].meta.w));
  const float3 Pk = f3(te.P_rb.x, te.P_rb.y, te.P_rb.z);
  const float ra = te.d_ra.w, rb = te.P_rb.w;
  // dual inputs
  const V3T<D7> o{D7::seed(te.o_t.x, 0), D7::seed(te.o_t.y, 1), D7::seed(te.o_t.z, 2)};
  const V3T<D7> d{D7::seed(te.d_ra.x, 3), D7::seed(te.d_ra.y, 4), D7::seed(te.d_ra.z, 5)};
  V3T<D7> p, n;
  surf_dual(S, prim, te.o_t.w, flags, o, d, p, n);
  // phi = ob . p + db . next_direction + (scalar weights) . (cosines)
  D7 phi = dot_c(p, ob);
  float3 a = f3(0.f, 0.f, 0.f);   // radiance added per unit power: c_k = P_k * a
  float3 Mv = f3(1.f, 1.f, 1.f);  // power multiplier values
  float3 dMdC = f3(0.f, 0.f, 0.f);
  float3 dadC = f3(0.f, 0.f, 0.f);
  if (mat >= 0 && M->emission_strength >= 0.0f) {
    // the emitted term e * E * P is added for e > 0 and is 0 at e = 0:
    // its (right) derivative E * P holds for every e >= 0
    const float3 E = ld3(M->emission);
    if (flags & TF_EMIT) a = a + E * M->emission_strength;
    G.emis(mat, g.x * Pk.x * E.x + g.y * Pk.y * E.y + g.z * Pk.z * E.z);
  }
  if (br == BR_DIFFUSE) {
    const float3 T = f3(te.T.x, te.T.y, te.T.z);
    a = a + col * T;
    dadC = T;
    Mv = col;
    dMdC = f3(1.f, 1.f, 1.f);
    if (flags & TF_NEE) {
      const float4 e = __ldg(S.env_rec0 + nee_k);
      const float4 r = __ldg(S.env_rec1 + nee_k);
      const int2 ax = __ldg(A.env_aux + nee_k);
      const float ao = mat >= 0 ? M->ao : 1.0f;
      const float pdf = e.w;
      const D7 ct = dot_c(n, f3(e.x, e.y, e.z));
      const float3 R = f3(r.x, r.y, r.z) * ao;
      const float w = ct.v / pdf;
      a = a + col * R * w;
      dadC = dadC + R * w;
      Mv = col * (1.0f - ct.v);
      dMdC = f3(1.0f - ct.v, 1.0f - ct.v, 1.0f - ct.v);
      // d/d ct of  g.(P*C*R*ct/pdf)  and of  Pb.(P*C*(1 - ct))
      const float3 PC = Pk * col;
      const float gR = g.x * PC.x * R.x + g.y * PC.y * R.y + g.z * PC.z * R.z;
      phi = phi + ct * (gR / pdf - (Pb.x * PC.x + Pb.y * PC.y + Pb.z * PC.z));
      // sky: radiance texel, and pdf_joint = gray[pi] / column average
      const float3 gr = g * PC * (ao * w);
      add_sky_grad(A, ax.x, 0, gr.x);
      add_sky_grad(A, ax.x, 1, gr.y);
      add_sky_grad(A, ax.x, 2, gr.z);
      const float gpdf = -gR * w / pdf;              // d loss / d pdf
      for (int c = 0; c < 3; ++c) add_sky_grad(A, ax.y, c, gpdf * A.pdf_dgray * lw[c] * inv_col);
      gcol += gpdf * (-pdf * inv_col);
    }
    phi = phi + vdot(coshemi_dual(n, ra, rb), dv3(db));
  } else {
    const D7 al = D7::seed(M->roughness, 6);
    const D7 a4 = (al * al) * (al * al);
    if (br == BR_REFRACT) {
      const float eta = (flags & TF_FRONT) ? S.ior_all / M->ior : M->ior / S.ior_all;
      const V3T<D7> du = dunit(d);
      const D7 c0 = -vdot(du, n);
      const D7 ctp = c0.v <= 1.0f ? c0 : D7(1.0f);
      const V3T<D7> perp = (du + n * ctp) * eta;
      const D7 k2 = D7(1.0f) - vdot(perp, perp);
      V3T<D7> dir = dunit(n * (-dsqrt(dabs(k2))) + perp);
      if (ggx) dir = ggx_dual(dir, a4, ra, rb);
      phi = phi + vdot(dir, dv3(db));
      Mv = col;
      dMdC = f3(1.f, 1.f, 1.f);
    } else {
      const V3T<D7> m = ggx ? ggx_dual(n, a4, ra, rb) : n;
      phi = phi + vdot(reflect_dual(d, m), dv3(db));
      if (br == BR_METAL) {
        // fresnel_schlick_color (fresnel_schlick.c:19): M = C + (1 - C) (1 - ct)^5
        const D7 ctm = -vdot(dunit(d), n);
        const D7 q = dpow5(D7(1.0f) - ctm);
        const float3 omc = f3(1.f, 1.f, 1.f) - col;
        Mv = col + omc * q.v;
        dMdC = f3(1.0f - q.v, 1.0f - q.v, 1.0f - q.v);
        phi = phi + q * (Pb.x * Pk.x * omc.x + Pb.y * Pk.y * omc.y + Pb.z * Pk.z * omc.z);
      }
    }
  }
  if (mat >= 0) {
    G.albedo(mat, 0, g.x * Pk.x * dadC.x + Pb.x * Pk.x * dMdC.x);
    G.albedo(mat, 1, g.y * Pk.y * dadC.y + Pb.y * Pk.y * dMdC.y);
    G.albedo(mat, 2, g.z * Pk.z * dadC.z + Pb.z * Pk.z * dMdC.z);
    if (ggx) G.rough(mat, phi.g[6]);
  }
  Pb = g * a + Pb * Mv;
  ob = f3(phi.g[0], phi.g[1], phi.g[2]);
  db = f3(phi.g[3], phi.g[4], phi.g[5]);
}

// Path state of the backward between kernels (4 float4 per path):
// (g.xyz, bounces K as int bits), Pb, ob, db.
__device__ __forceinline__ void finish_path(const SceneView& S, const AdjointArgs& A, float4* state,
                                            uint64_t idx, float3 g, int K, const PathState& P, bool miss) {
  float3 Pb = f3(0.f, 0.f, 0.f);
  if (miss) {
    const float ao = P.last_mat >= 0 ? S.mats[P.last_mat].ao : 1.0f;
    Pb = g * background(S, P.d, true) * ao;
    if (S.has_env && S.sky_rgb) {
      int x, y;
      sky_xy(S, P.d, x, y);
      const int tx = y * S.env_w + x;
      const float* sk = S.sky_rgb + 3 * (size_t)tx;
      const float3 gp = g * P.power * ao;
      add_sky_grad(A, tx, 0, sk[0] > 0.f && sk[0] < 16.f ? gp.x : 0.f);
      add_sky_grad(A, tx, 1, sk[1] > 0.f && sk[1] < 16.f ? gp.y : 0.f);
      add_sky_grad(A, tx, 2, sk[2] > 0.f && sk[2] < 16.f ? gp.z : 0.f);
    }
  }
  state[4 * idx] = make_float4(g.x, g.y, g.z, __int_as_float(K));
  state[4 * idx + 1] = make_float4(Pb.x, Pb.y, Pb.z, 0.f);
  state[4 * idx + 2] = make_float4(0.f, 0.f, 0.f, 0.f);
  state[4 * idx + 3] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Replay: the paths of the forward again (persistent, lanes regenerate
// paths as in the regenerating megakernel), writing one tape entry per
// bounce to tape[k * n_paths + path].
// The replay kernel traces like the regenerating megakernel and, like it,
// runs faster at 44 registers than at the compiler's 128 (c4 512x512x64 spp
// backward: 57.9 -> 46.8 ms; 64 registers: 49.7 ms). The per-level kernel
// keeps its registers (its Dual<7> arithmetic needs them; 128: no change).
constexpr int kReplayRegs = 44;
template <int kBlock, class V>
__global__ void __maxnreg__(kReplayRegs) adj_replay_kernel(V S, AdjointArgs A, TapeEntry* tape,
                                                            float4* state, int* status,
                                                            unsigned long long* work) {
  const uint32_t npix = (uint32_t)S.width * (uint32_t)S.height;
  const int lane = threadIdx.x & 31;
  PathCounters C{0, 0, 0};
  PathState P;
  uint64_t idx = 0;
  float3 g = f3(0.f, 0.f, 0.f);
  int K = 0;
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
        idx = base + __popc(need_mask & ((1u << lane) - 1u));
        if (idx >= A.n_paths) {
          done = true;
        } else {
          const uint32_t lin = (uint32_t)(idx % npix);
          const uint32_t sample = A.sample_base + (uint32_t)(idx / npix);
          const uint32_t pixel = tile_pixel(lin, S.width, S.height);
          g = f3(A.dimg[3 * (size_t)pixel] * A.inv_spp, A.dimg[3 * (size_t)pixel + 1] * A.inv_spp,
                 A.dimg[3 * (size_t)pixel + 2] * A.inv_spp);
          K = 0;
          if (g.x == 0.f && g.y == 0.f && g.z == 0.f) {
            finish_path(S, A, state, idx, g, 0, P, false);
          } else {
            P.rng.s = path_seed(A.seed, pixel, sample);
            float ox, oy;
            sample_offset(A.seed, sample, A.jitter, P.rng, ox, oy);
            camera_ray(S, P, pixel, ox, oy);
            P.power = f3(1.f, 1.f, 1.f);
            P.acc = f3(0.f, 0.f, 0.f);
            P.last_mat = -1;
            active = true;
          }
        }
      }
    }
    if (__all_sync(0xffffffffu, done)) break;
    if (active) {
      HitInfo h;
      int visits = 0;
      if (!closest_hit<false>(S, P.o, P.d, h, visits, status)) {
        finish_path(S, A, state, idx, g, K, P, true);
        active = false;
      } else {
        const Surf s = make_surf(S, h, P.o, P.d, 0);
        TapeEntry te;
        te.o_t = make_float4(P.o.x, P.o.y, P.o.z, h.t);
        int fl = s.front ? (int)TF_FRONT : 0;
        if (V::kQuadrics && h.prim >= 0 && __ldg(S.meta + h.prim).z >= PRIM_CYL)
          fl |= ((int)h.u) << TF_PART_SHIFT;
        Rec rec{fl, 0.f, 0.f, -1, f3(0.f, 0.f, 0.f)};
        const float3 d0 = P.d, p0 = P.power;
        P.o = s.p;
        P.last_mat = s.mat;
        material_rec(S, P, s, status, C, rec);
        te.d_ra = make_float4(d0.x, d0.y, d0.z, rec.ra);
        te.P_rb = make_float4(p0.x, p0.y, p0.z, rec.rb);
        te.T = make_float4(rec.T.x, rec.T.y, rec.T.z, 0.f);
        te.meta = make_int4(h.prim, s.mat, rec.flags, rec.nee);
        tape[(size_t)K * A.n_paths + idx] = te;
        ++K;
        const bool dead = P.power.x == 0.0f && P.power.y == 0.0f && P.power.z == 0.0f;
        if (dead || K >= A.max_bounces) {
          finish_path(S, A, state, idx, g, K, P, false);
          active = false;
        }
      }
    }
  }
}

// Reverse sweep of bounce level k for every path that reached it.
template <int kBlock, class V>
__global__ void __launch_bounds__(kBlock) adj_level_kernel(V S, AdjointArgs A, const TapeEntry* tape,
                                                           float4* state, int k) {
  extern __shared__ long long smem_q[];
  MatGrad G{smem_q, A.n_mats, A.q_scale};
  for (int i = threadIdx.x; i < 5 * A.n_mats; i += kBlock) smem_q[i] = 0;
  __syncthreads();
  const float inv_col = A.col ? (float)(1.0 / *A.col) : 0.f;
  float gcol = 0.f;
  for (uint64_t idx = (uint64_t)blockIdx.x * kBlock + threadIdx.x; idx < A.n_paths;
       idx += (uint64_t)gridDim.x * kBlock) {
    const float4 s0 = state[4 * idx];
    if (__float_as_int(s0.w) <= k) continue;
    const float4 s1 = state[4 * idx + 1], s2 = state[4 * idx + 2], s3 = state[4 * idx + 3];
    float3 Pb = f3(s1.x, s1.y, s1.z), ob = f3(s2.x, s2.y, s2.z), db = f3(s3.x, s3.y, s3.z);
    const TapeEntry te = tape[(size_t)k * A.n_paths + idx];
    reverse_step(S, A, G, te, f3(s0.x, s0.y, s0.z), inv_col, Pb, ob, db, gcol);
    if (k > 0) {
      state[4 * idx + 1] = make_float4(Pb.x, Pb.y, Pb.z, 0.f);
      state[4 * idx + 2] = make_float4(ob.x, ob.y, ob.z, 0.f);
      state[4 * idx + 3] = make_float4(db.x, db.y, db.z, 0.f);
    }
  }
  long long qcol = fx_q(gcol, A.q_scale);
  for (int off = 16; off > 0; off >>= 1) qcol += __shfl_down_sync(0xffffffffu, qcol, off);
  if ((threadIdx.x & 31) == 0 && qcol != 0)
    atomicAdd(reinterpret_cast<unsigned long long*>(A.q_col), (unsigned long long)qcol);
  __syncthreads();
  for (int i = threadIdx.x; i < 5 * A.n_mats; i += kBlock)
    if (smem_q[i] != 0) atomicAdd(reinterpret_cast<unsigned long long*>(A.q_mats + i), (unsigned long long)smem_q[i]);
}

// theta -> MaterialD array (colour, roughness, alpha4, emission strength
// replaced; metallic, ior, f0, transmission, ao, emission colour kept).
__global__ void diff_mats_kernel(const MaterialD* base, const float* theta, int M, MaterialD* out) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  MaterialD o = base[m];
  o.color[0] = theta[3 * m];
  o.color[1] = theta[3 * m + 1];
  o.color[2] = theta[3 * m + 2];
  const float r = theta[3 * M + m];
  o.roughness = r;
  const double rd = (double)r;
  o.alpha4 = (float)((rd * rd) * (rd * rd));
  o.emission_strength = theta[4 * M + m];
  out[m] = o;
}

// Per-outcome records of the two-step sampler for the current tables:
// direction and texel from the (row index, column index) grid that the
// host computed once with the reference's double-precision libm calls,
// pdf_joint at the reference's index (material_default.c:57-59).
__global__ void diff_env_records_kernel(DiffEnvRecords E) {
  const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int W = E.W, H = E.H;
  if (k >= (size_t)(H - 1) * W) return;
  const int iy = (int)(k / W), dcol = (int)(k % W);
  const double v = (double)E.cdf_m_inv[iy];
  const double A = __dmul_rn(__dmul_rn(v, (double)(H - 1)), (double)W);
  const long long j = (long long)floor(A) + dcol;
  float4 r0 = make_float4(0.f, 1.f, 0.f, 0.f), r1 = make_float4(0.f, 0.f, 0.f, 0.f);
  int2 ax = make_int2(0, 0);
  if (j >= 0 && j < (long long)W * H) {
    const double u = (double)E.cdf_c_inv[j];
    const int iv = min(max(__double2int_rn(v * (double)(H - 1)), 0), H - 1);
    const int iu = min(max(__double2int_rn(u * (double)(W - 1)), 0), W - 1);
    const float4 gr = E.grid[(size_t)iv * W + iu];
    const int tx = __float_as_int(gr.w);
    const long long pi = (long long)__dadd_rn(A, __dmul_rn(u, (double)(W - 1)));
    const bool ok = pi >= 0 && pi < (long long)W * H;
    r0 = make_float4(gr.x, gr.y, gr.z, ok ? E.pdf_joint[pi] : 0.0f);
    const float* sk = E.sky + 3 * (size_t)tx;
    r1 = make_float4(sk[0], sk[1], sk[2], 0.f);
    ax = make_int2(tx, ok ? (int)pi : 0);
  }
  E.rec0[k] = r0;
  E.rec1[k] = r1;
  E.aux[k] = ax;
}

__global__ void diff_image_kernel(const unsigned long long* q, float* img, int npix, double inv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npix) return;
  for (int c = 0; c < 3; ++c) img[3 * i + c] = (float)((double)(long long)q[3 * i + c] * inv);
}

__global__ void abs_max_kernel(const float* x, size_t n, float* out) {
  float m = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float a = fabsf(x[i]);
    if (a > m && a < INFINITY) m = a;
  }
  for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, off));
  // non-negative floats order like their bit patterns
  if ((threadIdx.x & 31) == 0 && m > 0.f) atomicMax(reinterpret_cast<int*>(out), __float_as_int(m));
}

// Fixed-point sums to the float gradient, with the dense part of the
// pdf_joint gradient: every texel's luminance enters the column average that
// divides every pdf (d column_average / d texel channel c = 255 * lum[c] /
// (W * H)).
__global__ void diff_grad_out_kernel(AdjointArgs A, float* out_mats, float* out_sky, int64_t n_mats5,
                                     float dense) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const double inv = 1.0 / A.q_scale;
  if (i < n_mats5) out_mats[i] = (float)((double)A.q_mats[i] * inv);
  if (i < A.n_texels) {
    const float s = (float)((double)*A.q_col * inv) * dense;
    const float lw[3] = {0.2126f, 0.7152f, 0.0722f};
    for (int c = 0; c < 3; ++c) out_sky[3 * i + c] = (float)((double)A.q_sky[3 * i + c] * inv) + s * lw[c];
  }
}

// Linear sky radiance of every texel as the renderer decodes it (RGBE,
// exposure, gamma: get_hdr_pixel_skybox, get_hdr_value.c:43-68).
__global__ void diff_sky_init_kernel(SceneView S, float* out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)S.env_w * S.env_h) return;
  const float3 c = sky_texel(S, (int)(i % S.env_w), (int)(i / S.env_w));
  out[3 * i] = c.x;
  out[3 * i + 1] = c.y;
  out[3 * i + 2] = c.z;
}

}  // namespace

cudaError_t launch_diff_sky_init(const SceneView& S, float* out, cudaStream_t st) {
  const size_t n = (size_t)S.env_w * S.env_h;
  if (n == 0) return cudaSuccess;
  diff_sky_init_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(S, out);
  return cudaGetLastError();
}

cudaError_t launch_diff_mats(const MaterialD* base, const float* theta, int M, MaterialD* out,
                             cudaStream_t st) {
  if (M == 0) return cudaSuccess;
  diff_mats_kernel<<<(M + 127) / 128, 128, 0, st>>>(base, theta, M, out);
  return cudaGetLastError();
}

cudaError_t launch_diff_env_records(const DiffEnvRecords& E, cudaStream_t st) {
  const size_t no = (size_t)(E.H - 1) * E.W;
  if (no == 0) return cudaSuccess;
  diff_env_records_kernel<<<(unsigned)((no + 255) / 256), 256, 0, st>>>(E);
  return cudaGetLastError();
}

cudaError_t launch_diff_image(const unsigned long long* accum_fx, float* img, int npix, int spp,
                              cudaStream_t st) {
  diff_image_kernel<<<(npix + 255) / 256, 256, 0, st>>>(accum_fx, img, npix,
                                                       1.0 / (kFrameFxScale * (double)std::max(spp, 1)));
  return cudaGetLastError();
}

cudaError_t launch_abs_max(const float* x, size_t n, float* out, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 1184);
  abs_max_kernel<<<blocks, 256, 0, st>>>(x, n, out);
  return cudaGetLastError();
}

cudaError_t launch_diff_grad_out(const AdjointArgs& A, float* out_mats, float* out_sky, int64_t n_mats5,
                                 cudaStream_t st) {
  const int64_t n = std::max<int64_t>(n_mats5, A.n_texels);
  if (n == 0) return cudaSuccess;
  const float dense = A.n_texels ? A.pdf_dgray / (float)A.n_texels : 0.f;
  diff_grad_out_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A, out_mats, out_sky, n_mats5, dense);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_chunk(const SceneView& S, const AdjointArgs& A, TapeEntry* tape, float4* state,
                                 unsigned long long* work, int* status, cudaStream_t st) {
  if (A.n_paths == 0) return cudaSuccess;
  constexpr int kBlock = 128;
  int dev = 0, sms = 0, occ = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaMemsetAsync(work, 0, sizeof(unsigned long long), st);
  if (e != cudaSuccess) return e;
  return with_view(S, [&](const auto& v) -> cudaError_t {
    using VT = std::decay_t<decltype(v)>;
    if constexpr (VT::kTextures) {
      return cudaErrorNotSupported;   // mrt_forward / mrt_backward refuse textured scenes
    } else {
    cudaError_t e2 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, adj_replay_kernel<kBlock, VT>, kBlock, 0);
    if (e2 != cudaSuccess) return e2;
    const uint64_t want = (A.n_paths + kBlock - 1) / kBlock;
    unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)sms * std::max(occ, 1), want);
    adj_replay_kernel<kBlock, VT><<<grid, kBlock, 0, st>>>(v, A, tape, state, status, work);
    if ((e2 = cudaGetLastError()) != cudaSuccess) return e2;
    const size_t smem = (size_t)5 * A.n_mats * sizeof(long long);
    e2 = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, adj_level_kernel<kBlock, VT>, kBlock, smem);
    if (e2 != cudaSuccess) return e2;
    grid = (unsigned)std::min<uint64_t>((uint64_t)sms * std::max(occ, 1), want);
    for (int k = A.max_bounces - 1; k >= 0; --k) {
      adj_level_kernel<kBlock, VT><<<grid, kBlock, smem, st>>>(v, A, tape, state, k);
      if ((e2 = cudaGetLastError()) != cudaSuccess) return e2;
    }
    return cudaSuccess;
    }
  });
}

}  // namespace mrt
