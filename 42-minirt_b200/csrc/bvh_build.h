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
  std::vector<WNode> wnodes;      // 8-wide tree (build_bvh_wide), root at 0
  std::vector<uint32_t> order;    // leaf order -> input primitive index
  int root_leaf = 0;              // non-zero when the whole scene is one leaf
  int max_depth = 0;
  int leaves = 0;
};

void prim_box_from_double(PrimBox& p, const double* mn, const double* mx);
bool build_bvh(const std::vector<PrimBox>& prims, BvhResult& out, std::string& err);
// The 8-wide tree with quantised child boxes (WNode); out.nodes stays empty.
bool build_bvh_wide(const std::vector<PrimBox>& prims, BvhResult& out, std::string& err);
// Structural check of a wide tree against its primitives (host, O(n)).
bool check_bvh_wide(const BvhResult& t, const std::vector<PrimBox>& prims, std::string& err);

// A primitive of the reference-topology build: its bounds as the reference
// computes them (compute_object_bounds, bvh_math.c:17) and the position its
// median split sorts by (get_obj_position, bvh_utils.c:88).
struct RefPrim {
  double mn[3], mx[3];
  double pos[3];
};

// The reference's own tree (bvh_build.c:16-127): list[i] is the input
// primitive at position i of the reference's object list (bvh_make_lst.c).
// dboxes receives the double-precision boxes for the reference's node-visit
// count: 6 for the root, then 12 per device node (left child, right child),
// each as min xyz, max xyz.
bool build_bvh_reference(const std::vector<RefPrim>& prims, const std::vector<uint32_t>& list,
                         BvhResult& out, std::vector<double>& dboxes, std::string& err);

}  // namespace mrt
