// caustic.cuh — photon-map radiance estimate on a uniform hash grid.
//
// Reference: estimate_caustics_physically_based + calculate_caustic_radiance
// (get_caustic.c:37-88) over a median kd-tree (kd_tree_find_near.c:93). The
// estimate is non-zero only when the k-th nearest photon lies within
// r_max^2 = caustic_radius (the option value is compared against squared
// distances, get_caustic.c:45), so only photons inside r_max matter: the grid
// has cells of side >= r_max and the 27 cells around the query hold every
// candidate. The k nearest are kept in a register-resident sorted list.
#pragma once
#include "device_common.cuh"

namespace mrt {

constexpr int kKnnMax = 32;

__device__ __forceinline__ int grid_cell_index(const SceneView& S, int x, int y, int z) {
  return (z * S.grid_dim[1] + y) * S.grid_dim[0] + x;
}

// kNN mode: sum of the k nearest photon powers / (pi r_k^2) / norm when the
// k-th distance^2 <= caustic_radius; fixed-radius mode: sum within the
// pass radius / (pi r^2) / norm.
__device__ __forceinline__ float3 caustic_estimate(const SceneView& S, float3 p) {
  if (!S.caustic || S.n_photons == 0) return f3(0.f, 0.f, 0.f);
  const float r2max = S.caustic_mode ? S.fixed_radius2 : S.caustic_radius2;
  int cx = (int)floorf((p.x - S.grid_min[0]) * S.grid_inv_cell);
  int cy = (int)floorf((p.y - S.grid_min[1]) * S.grid_inv_cell);
  int cz = (int)floorf((p.z - S.grid_min[2]) * S.grid_inv_cell);
  if (cx < -1 || cy < -1 || cz < -1 || cx > S.grid_dim[0] || cy > S.grid_dim[1] || cz > S.grid_dim[2])
    return f3(0.f, 0.f, 0.f);
  if (S.caustic_mode) {
    float3 sum = f3(0.f, 0.f, 0.f);
    for (int z = max(cz - 1, 0); z <= min(cz + 1, S.grid_dim[2] - 1); ++z)
      for (int y = max(cy - 1, 0); y <= min(cy + 1, S.grid_dim[1] - 1); ++y)
        for (int x = max(cx - 1, 0); x <= min(cx + 1, S.grid_dim[0] - 1); ++x) {
          int c = grid_cell_index(S, x, y, z);
          uint32_t b = __ldg(S.cell_start + c), e = __ldg(S.cell_start + c + 1);
          for (uint32_t i = b; i < e; ++i) {
            float4 q = __ldg(S.photon_pos + i);
            float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
            if (dx * dx + dy * dy + dz * dz <= r2max) {
              float4 w = __ldg(S.photon_pow + i);
              sum = sum + f3(w.x, w.y, w.z);
            }
          }
        }
    float area = 3.14159265358979f * r2max;
    return sum * (S.inv_norm / area);
  }
  const int k = S.knn;
  float bd[kKnnMax];
  int bi[kKnnMax];
  int cnt = 0;
  for (int z = max(cz - 1, 0); z <= min(cz + 1, S.grid_dim[2] - 1); ++z)
    for (int y = max(cy - 1, 0); y <= min(cy + 1, S.grid_dim[1] - 1); ++y)
      for (int x = max(cx - 1, 0); x <= min(cx + 1, S.grid_dim[0] - 1); ++x) {
        int c = grid_cell_index(S, x, y, z);
        uint32_t b = __ldg(S.cell_start + c), e = __ldg(S.cell_start + c + 1);
        for (uint32_t i = b; i < e; ++i) {
          float4 q = __ldg(S.photon_pos + i);
          float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
          float d2 = dx * dx + dy * dy + dz * dz;
          if (d2 > r2max) continue;
          if (cnt == k && d2 >= bd[k - 1]) continue;
          int j = cnt < k ? cnt++ : k - 1;
          while (j > 0 && bd[j - 1] > d2) {
            bd[j] = bd[j - 1];
            bi[j] = bi[j - 1];
            --j;
          }
          bd[j] = d2;
          bi[j] = (int)i;
        }
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
