// caustic.cuh — photon-map radiance estimate over the photon hierarchy.
//
// Reference: estimate_caustics_physically_based + calculate_caustic_radiance
// (get_caustic.c:37-88) over a median kd-tree (kd_tree_find_near.c:93). The
// estimate is non-zero only when the k-th nearest photon lies within
// r_max^2 = caustic_radius (the option value is compared against squared
// distances, get_caustic.c:45), so only photons inside r_max matter.
//
// The photons are in Morton order with a linear BVH over them
// (SceneView.photon_nodes). The kNN walk visits the nearer child first and
// skips every node farther than the current k-th distance (or r_max until k
// are found), keeping the k nearest in a register-resident sorted list. The
// fixed-radius walk (the progressive mode) adds the summed power of a node
// whose box lies entirely inside the sphere without visiting its photons.
#pragma once
#include "device_common.cuh"

namespace mrt {

constexpr int kKnnMax = 32;
// A depth-first walk keeps at most one pending node per level; the radix
// tree is at most 63 code bits + 32 index bits deep.
constexpr int kPhotonStack = 100;

__device__ __forceinline__ float node_dist2(const float4& lo, const float4& hi, float3 p) {
  const float dx = fmaxf(fmaxf(lo.x - p.x, p.x - hi.x), 0.f);
  const float dy = fmaxf(fmaxf(lo.y - p.y, p.y - hi.y), 0.f);
  const float dz = fmaxf(fmaxf(lo.z - p.z, p.z - hi.z), 0.f);
  return dx * dx + dy * dy + dz * dz;
}
__device__ __forceinline__ float node_far2(const float4& lo, const float4& hi, float3 p) {
  const float dx = fmaxf(fabsf(p.x - lo.x), fabsf(p.x - hi.x));
  const float dy = fmaxf(fabsf(p.y - lo.y), fabsf(p.y - hi.y));
  const float dz = fmaxf(fabsf(p.z - lo.z), fabsf(p.z - hi.z));
  return dx * dx + dy * dy + dz * dz;
}

// The k nearest photons with k <= kKnnReg: the sorted list lives in
// registers (every index compile-time: a new distance bubbles in through one
// compare-and-swap per slot, equal distances keeping their visit order), so
// none of it goes to local memory. Same photons, same order and the same
// estimate as the general walk below.
constexpr int kKnnReg = 16;

__device__ __forceinline__ float3 knn_estimate_reg(const SceneView& S, float3 p, float r2max) {
  const int n = S.n_photons, k = S.knn;
  int stack[kPhotonStack];
  int sp = 0;
  int kids[2] = {n == 1 ? ~0 : 0, n == 1 ? ~0 : 0};
  int n_kids = n == 1 ? 1 : 0;
  if (n > 1) stack[sp++] = 0;
  int guard = 2 * n + 8;
  float bd[kKnnReg];
  int bi[kKnnReg];
#pragma unroll
  for (int t = 0; t < kKnnReg; ++t) { bd[t] = INFINITY; bi[t] = 0; }
  int cnt = 0;
  float kth = INFINITY;                  // bd[k - 1]
  while ((sp > 0 || n_kids > 0) && --guard > 0) {
    const float bound = cnt == k ? fminf(r2max, kth) : r2max;
    if (n_kids == 0) {
      const int nd = stack[--sp];
      const float4 lo = __ldg(S.photon_nodes + 4 * nd), hi = __ldg(S.photon_nodes + 4 * nd + 1);
      if (node_dist2(lo, hi, p) > bound) continue;
      const float4 ch = __ldg(S.photon_nodes + 4 * nd + 3);
      const int c0 = __float_as_int(ch.x), c1 = __float_as_int(ch.y);
      // internal children pushed farther first; photon children next
      float d0 = INFINITY, d1 = INFINITY;
      if (c0 >= 0) d0 = node_dist2(__ldg(S.photon_nodes + 4 * c0), __ldg(S.photon_nodes + 4 * c0 + 1), p);
      if (c1 >= 0) d1 = node_dist2(__ldg(S.photon_nodes + 4 * c1), __ldg(S.photon_nodes + 4 * c1 + 1), p);
      if (c0 >= 0 && c1 >= 0) {
        const bool swap = d0 < d1;
        const int fa = swap ? c1 : c0, ne = swap ? c0 : c1;
        const float dfa = swap ? d1 : d0, dne = swap ? d0 : d1;
        if (dfa <= bound && sp < kPhotonStack) stack[sp++] = fa;
        if (dne <= bound && sp < kPhotonStack) stack[sp++] = ne;
      } else if (c0 >= 0) {
        if (d0 <= bound && sp < kPhotonStack) stack[sp++] = c0;
      } else if (c1 >= 0) {
        if (d1 <= bound && sp < kPhotonStack) stack[sp++] = c1;
      }
      n_kids = 0;
      if (c0 < 0) kids[n_kids++] = c0;
      if (c1 < 0) kids[n_kids++] = c1;
      continue;
    }
    const int i = ~kids[--n_kids];
    const float4 q = __ldg(S.photon_pos + i);
    const float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
    float d2 = dx * dx + dy * dy + dz * dz;
    if (d2 > r2max) continue;
    if (cnt == k && d2 >= kth) continue;
    if (cnt < k) ++cnt;
    int id = i;
#pragma unroll
    for (int t = 0; t < kKnnReg; ++t) {
      if (d2 < bd[t]) {
        const float td = bd[t]; bd[t] = d2; d2 = td;
        const int ti = bi[t]; bi[t] = id; id = ti;
      }
    }
#pragma unroll
    for (int t = 0; t < kKnnReg; ++t)
      if (t == k - 1) kth = bd[t];
  }
  if (cnt < k) return f3(0.f, 0.f, 0.f);
  const float area = 3.14159265358979f * kth;
  if (area < 1e-9f) return f3(0.f, 0.f, 0.f);
  float3 sum = f3(0.f, 0.f, 0.f);
#pragma unroll
  for (int t = 0; t < kKnnReg; ++t) {
    if (t < k) {
      const float4 w = __ldg(S.photon_pow + bi[t]);
      sum = sum + f3(w.x, w.y, w.z);
    }
  }
  return sum * (S.inv_norm / area);
}

// kNN mode: sum of the k nearest photon powers / (pi r_k^2) / norm when the
// k-th distance^2 <= caustic_radius; fixed-radius mode: sum within the
// pass radius / (pi r^2) / norm.
__device__ __forceinline__ float3 caustic_estimate(const SceneView& S, float3 p) {
  if (!S.caustic || S.n_photons == 0) return f3(0.f, 0.f, 0.f);
  const float r2max = S.caustic_mode ? S.fixed_radius2 : S.caustic_radius2;
  const int n = S.n_photons;
  int stack[kPhotonStack];
  int sp = 0;
  // children of the node being expanded (a single photon is its own root)
  int kids[2] = {n == 1 ? ~0 : 0, n == 1 ? ~0 : 0};
  int n_kids = n == 1 ? 1 : 0;
  if (n > 1) stack[sp++] = 0;
  int guard = 2 * n + 8;                  // every node is visited at most once
  if (S.caustic_mode) {
    float3 sum = f3(0.f, 0.f, 0.f);
    while ((sp > 0 || n_kids > 0) && --guard > 0) {
      if (n_kids == 0) {
        const int nd = stack[--sp];
        const float4 lo = __ldg(S.photon_nodes + 4 * nd), hi = __ldg(S.photon_nodes + 4 * nd + 1);
        if (node_dist2(lo, hi, p) > r2max) continue;
        if (node_far2(lo, hi, p) <= r2max) {
          const float4 w = __ldg(S.photon_nodes + 4 * nd + 2);
          sum = sum + f3(w.x, w.y, w.z);
          continue;
        }
        const float4 ch = __ldg(S.photon_nodes + 4 * nd + 3);
        kids[0] = __float_as_int(ch.x);
        kids[1] = __float_as_int(ch.y);
        n_kids = 2;
      }
      const int c = kids[--n_kids];
      if (c < 0) {
        const float4 q = __ldg(S.photon_pos + ~c);
        const float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        if (dx * dx + dy * dy + dz * dz <= r2max) {
          const float4 w = __ldg(S.photon_pow + ~c);
          sum = sum + f3(w.x, w.y, w.z);
        }
      } else if (sp < kPhotonStack) {
        stack[sp++] = c;
      }
    }
    const float area = 3.14159265358979f * r2max;
    return sum * (S.inv_norm / area);
  }
  if (S.knn <= kKnnReg) return knn_estimate_reg(S, p, r2max);
  const int k = S.knn;
  float bd[kKnnMax];
  int bi[kKnnMax];
  int cnt = 0;
  while ((sp > 0 || n_kids > 0) && --guard > 0) {
    float bound = cnt == k ? fminf(r2max, bd[k - 1]) : r2max;
    if (n_kids == 0) {
      const int nd = stack[--sp];
      const float4 lo = __ldg(S.photon_nodes + 4 * nd), hi = __ldg(S.photon_nodes + 4 * nd + 1);
      if (node_dist2(lo, hi, p) > bound) continue;
      const float4 ch = __ldg(S.photon_nodes + 4 * nd + 3);
      kids[0] = __float_as_int(ch.x);
      kids[1] = __float_as_int(ch.y);
      n_kids = 2;
      // photons first; internal children pushed farther first
      int in[2], m = 0;
      float din[2];
      for (int t = 0; t < 2; ++t) {
        const int c = kids[t];
        if (c >= 0) {
          din[m] = node_dist2(__ldg(S.photon_nodes + 4 * c), __ldg(S.photon_nodes + 4 * c + 1), p);
          in[m++] = c;
        }
      }
      if (m == 2 && din[0] < din[1]) {
        const int ti = in[0]; in[0] = in[1]; in[1] = ti;
        const float td = din[0]; din[0] = din[1]; din[1] = td;
      }
      for (int t = 0; t < m; ++t)
        if (din[t] <= bound && sp < kPhotonStack) stack[sp++] = in[t];
      // keep only the photon children for the loop below
      int np = 0;
      for (int t = 0; t < 2; ++t)
        if (kids[t] < 0) kids[np++] = kids[t];
      n_kids = np;
      continue;
    }
    const int c = kids[--n_kids];
    const int i = ~c;
    const float4 q = __ldg(S.photon_pos + i);
    const float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
    const float d2 = dx * dx + dy * dy + dz * dz;
    if (d2 > r2max) continue;
    if (cnt == k && d2 >= bd[k - 1]) continue;
    int j = cnt < k ? cnt++ : k - 1;
    while (j > 0 && bd[j - 1] > d2) {
      bd[j] = bd[j - 1];
      bi[j] = bi[j - 1];
      --j;
    }
    bd[j] = d2;
    bi[j] = i;
  }
  if (cnt < k) return f3(0.f, 0.f, 0.f);
  float r2 = bd[k - 1];
  float area = 3.14159265358979f * r2;
  if (area < 1e-9f) return f3(0.f, 0.f, 0.f);
  float3 sum = f3(0.f, 0.f, 0.f);
  for (int j = 0; j < k; ++j) {
    float4 w = __ldg(S.photon_pow + bi[j]);
    sum = sum + f3(w.x, w.y, w.z);
  }
  return sum * (S.inv_norm / area);
}

}  // namespace mrt
