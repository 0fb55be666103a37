// quadric.cuh — cylinder, cone and hyperboloid intersection, with the
// reference's arithmetic in double and its choice of root and part:
//   hit_cylinder (hit_cylinder.c:110-134): the lateral root valid_t picks
//     (t0 if in [IT_MIN, IT_MAX], else t1; valid_t.c:16) kept only if its
//     projection on the axis lies within the height, then the bottom and the
//     top cap (discs, |d . axis| >= 1e-6) replace it only when strictly
//     nearer;
//   hit_cone (hit_cone.c:108-129): no hit at all without a real root; the
//     lateral root of valid_t if within the height, else the cap disc;
//   hit_hyperboloid (hit_hyperboloid.c:80-104): both roots in the open
//     interval (IT_MIN, IT_MAX), the nearer one that lies within |z| <= h/2.
// Geometry records (48 B, geom):
//   cylinder   (centre, type) (orientation, radius) (height, top material,
//              bottom material, -)   materials as int bits, < 0 none
//   cone       (apex, type) (orientation, radius) (height, top material, -, -)
//   hyperboloid (centre, type) (orientation, a) (b, c, shape, height)
// The part hit (0 lateral, 1 top cap, 2 bottom cap) is returned for the
// shading normal and the per-part material.
//
// Only the SceneViewQ instantiation of the kernels includes these tests:
// their double arithmetic needs about twice the registers of the triangle
// test, which scenes without quadrics should not pay for.
#pragma once
#include "device_common.cuh"

namespace mrt {

enum QuadricPart : int { PART_SIDE = 0, PART_TOP = 1, PART_BOTTOM = 2 };

struct Dv3 {
  double x, y, z;
};
__device__ __forceinline__ Dv3 dv(float3 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ Dv3 dv(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ Dv3 operator+(Dv3 a, Dv3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ Dv3 operator-(Dv3 a, Dv3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ Dv3 operator*(Dv3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double ddot(Dv3 a, Dv3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ Dv3 dcross(Dv3 a, Dv3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ Dv3 dunitv(Dv3 a) {   // vec3_unit: zero stays zero
  const double l = sqrt(ddot(a, a));
  return l > 0.0 ? a * (1.0 / l) : Dv3{0.0, 0.0, 0.0};
}

constexpr double kItMinD = 0.001, kItMaxD = 1000.0;

// solve_quadratic (quadratique.c:17) + valid_t (valid_t.c:16).
__device__ __forceinline__ bool quad_roots(double A, double B, double C, double& t0, double& t1) {
  const double disc = B * B - 4.0 * A * C;
  if (disc < 0.0) return false;
  const double den = 2.0 * A, sq = sqrt(disc);
  t0 = (-B - sq) / den;
  t1 = (-B + sq) / den;
  return true;
}
__device__ __forceinline__ bool valid_root(double t0, double t1, double& th) {
  th = t0;
  if (th < kItMinD || th > kItMaxD) {
    th = t1;
    if (th < kItMinD || th > kItMaxD) return false;
  }
  return true;
}

// Disc of radius r centred at c with normal n (not necessarily unit, as the
// reference passes the orientation): t of the hit or -1.
__device__ __forceinline__ double disc_hit(Dv3 o, Dv3 d, Dv3 c, Dv3 n, double r, bool plus_form) {
  const double den = ddot(d, n);
  if (fabs(den) < 1e-6) return -1.0;
  // cylinder caps: t = -((o - c) . n) / den ; cone cap: t = ((c - o) . n) / den
  const double t = plus_form ? ddot(c - o, n) / den : -ddot(o - c, n) / den;
  if (t < kItMinD || t > kItMaxD) return -1.0;
  const Dv3 hp = o + d * t;
  const Dv3 e = hp - c;
  if (sqrt(ddot(e, e)) > r) return -1.0;
  return t;
}

__device__ __forceinline__ bool cylinder_hit(const float4& a, const float4& b, const float4& c, float3 of,
                                             float3 df, float tbest, float& t_out, int& part) {
  const Dv3 o = dv(of), d = dv(df), pos = dv(a.x, a.y, a.z), ori = dv(b.x, b.y, b.z);
  const double r = b.w, h = c.x;
  const Dv3 axis = dunitv(ori);
  bool hit = false;
  double tb = 0.0;
  int pb = PART_SIDE;
  {
    const Dv3 oc = o - pos;
    const double dd = ddot(d, ori), oo = ddot(oc, ori);
    double t0, t1, th;
    if (quad_roots(ddot(d, d) - dd * dd, 2.0 * (ddot(d, oc) - dd * oo), ddot(oc, oc) - oo * oo - r * r, t0, t1) &&
        valid_root(t0, t1, th)) {
      const Dv3 p = o + d * th;
      const Dv3 base = pos - axis * (h * 0.5);
      const double proj = ddot(p - base, axis);
      if (!(proj < 0.0 || proj > h)) {
        hit = true;
        tb = th;
      }
    }
  }
  const double tbot = disc_hit(o, d, pos - axis * (h * 0.5), ori, r, false);
  if (tbot >= 0.0 && (!hit || tbot < tb)) { hit = true; tb = tbot; pb = PART_BOTTOM; }
  const double ttop = disc_hit(o, d, pos + axis * (h * 0.5), ori, r, false);
  if (ttop >= 0.0 && (!hit || ttop < tb)) { hit = true; tb = ttop; pb = PART_TOP; }
  if (!hit) return false;
  const float t = (float)tb;
  if (!(t < tbest)) return false;
  t_out = t;
  part = pb;
  return true;
}

__device__ __forceinline__ bool cone_hit(const float4& a, const float4& b, const float4& c, float3 of, float3 df,
                                         float tbest, float& t_out, int& part) {
  const Dv3 o = dv(of), d = dv(df), apex = dv(a.x, a.y, a.z), ori = dv(b.x, b.y, b.z);
  const double r = b.w, h = c.x;
  const double q = r / h;
  const double k = q * q;             // pow((diameter / 2) / height, 2)
  const Dv3 oc = o - apex;
  const double dd = ddot(d, ori), oo = ddot(oc, ori);
  double t0, t1, th;
  if (!quad_roots(ddot(d, d) - (1.0 + k) * dd * dd, 2.0 * (ddot(d, oc) - (1.0 + k) * dd * oo),
                  ddot(oc, oc) - (1.0 + k) * oo * oo, t0, t1) ||
      !valid_root(t0, t1, th))
    return false;
  const Dv3 axis = dunitv(ori);
  const Dv3 p = o + d * th;
  const double proj = ddot(p - apex, axis);
  double tb;
  int pb;
  if (!(proj < 0.0 || proj > h)) {
    tb = th;
    pb = PART_SIDE;
  } else {
    tb = disc_hit(o, d, apex + axis * h, axis, r, true);
    if (tb < 0.0) return false;
    pb = PART_TOP;
  }
  const float t = (float)tb;
  if (!(t < tbest)) return false;
  t_out = t;
  part = pb;
  return true;
}

// Orthonormal frame of the hyperboloid's quadratic (quadratique_hyperboloid.c:15-26).
__device__ __forceinline__ void hyp_basis(Dv3 ori, Dv3& x, Dv3& y, Dv3& z) {
  z = dunitv(ori);
  const Dv3 tmp = fabs(z.x) > 0.9 ? Dv3{0.0, 1.0, 0.0} : Dv3{1.0, 0.0, 0.0};
  x = dunitv(dcross(tmp, z));
  y = dcross(z, x);
}

__device__ __forceinline__ bool hyperboloid_hit(const float4& a, const float4& b, const float4& c, float3 of,
                                                float3 df, float tbest, float& t_out, int& part) {
  const Dv3 o = dv(of), d = dv(df), pos = dv(a.x, a.y, a.z), ori = dv(b.x, b.y, b.z);
  const double ha = b.w, hb = c.x, hc = c.y, shape = c.z, h = c.w;
  Dv3 x, y, z;
  hyp_basis(ori, x, y, z);
  const Dv3 rel = o - pos;
  const Dv3 ld = {ddot(d, x), ddot(d, y), ddot(d, z)}, lo = {ddot(rel, x), ddot(rel, y), ddot(rel, z)};
  const double aa = ha * ha, bb = hb * hb, cc = hc * hc;
  double t0, t1;
  if (!quad_roots(ld.x * ld.x / aa + ld.y * ld.y / bb - ld.z * ld.z / cc,
                  2.0 * (ld.x * lo.x / aa + ld.y * lo.y / bb - ld.z * lo.z / cc),
                  lo.x * lo.x / aa + lo.y * lo.y / bb - lo.z * lo.z / cc - shape, t0, t1))
    return false;
  const Dv3 axis = dunitv(ori);
  double imax = kItMaxD, tb = 0.0;
  bool hit = false;
  if (t0 > kItMinD && t0 < imax && fabs(ddot(o + d * t0 - pos, axis)) <= h * 0.5) {
    hit = true;
    tb = t0;
    imax = t0;
  }
  if (t1 > kItMinD && t1 < imax && fabs(ddot(o + d * t1 - pos, axis)) <= h * 0.5) {
    hit = true;
    tb = t1;
  }
  if (!hit) return false;
  const float t = (float)tb;
  if (!(t < tbest)) return false;
  t_out = t;
  part = PART_SIDE;
  return true;
}

// One quadric of type PRIM_CYL, PRIM_CONE or PRIM_HYP: t < 0 for no hit
// nearer than tbest, else t and the part hit.
struct QuadricHit {
  float t;
  int part;
};
__device__ __forceinline__ QuadricHit quadric_hit(int type, const float4& a, const float4& b, const float4& c,
                                                  float3 o, float3 d, float tbest) {
  QuadricHit q{-1.0f, PART_SIDE};
  float t;
  int part = PART_SIDE;
  bool ok;
  if (type == PRIM_CYL) ok = cylinder_hit(a, b, c, o, d, tbest, t, part);
  else if (type == PRIM_CONE) ok = cone_hit(a, b, c, o, d, tbest, t, part);
  else ok = hyperboloid_hit(a, b, c, o, d, tbest, t, part);
  if (ok) {
    q.t = t;
    q.part = part;
  }
  return q;
}

}  // namespace mrt
