// bvh_build.h — host BVH builder interface (see bvh_build.cpp).
#pragma once
#include <stdint.h>
#include <string>
#include <vector>

#include "mrt_internal.h"

namespace mrt {

struct PrimBox {
  float mn[3], mx[3];   // outward-rounded float bounds
  float c[3];           // centroid used for binning
};

struct BvhResult {
  std::vector<Node> nodes;        // device nodes, root at 0
  std::vector<uint32_t> order;    // leaf order -> input primitive index
  int root_leaf = 0;              // non-zero when the whole scene is one leaf
  int max_depth = 0;
  int leaves = 0;
};

void prim_box_from_double(PrimBox& p, const double* mn, const double* mx);
bool build_bvh(const std::vector<PrimBox>& prims, BvhResult& out, std::string& err);

}  // namespace mrt
