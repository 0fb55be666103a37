// bvh_build.cpp — host BVH builder for the device layout in mrt_internal.h.
//
// The reference builds a median-split BVH with one primitive per leaf and
// traverses it exhaustively (bvh_build.c:16-127, bvh_hit.c:16-43). Closest-hit
// results do not depend on the tree, so the library builds its own tree for
// speed: binned SAH (32 bins on each axis, Wald 2007) with up to 8 primitives
// per leaf, object-median splits below depth 40 so the depth stays within the
// traversal stack, and top-level subtrees built on several threads. Boxes are
// rounded outward to float so float traversal never culls a hit that the
// double-precision reference finds inside the box.
#include <algorithm>
#include <array>
#include <functional>
#include <atomic>
#include <cmath>
#include <cstring>
#include <future>
#include <string>
#include <thread>
#include <vector>

#include "bvh_build.h"

namespace mrt {

namespace {

struct Box {
  float mn[3], mx[3];
  void reset() {
    for (int k = 0; k < 3; ++k) { mn[k] = INFINITY; mx[k] = -INFINITY; }
  }
  void grow(const Box& b) {
    for (int k = 0; k < 3; ++k) { mn[k] = std::min(mn[k], b.mn[k]); mx[k] = std::max(mx[k], b.mx[k]); }
  }
  void grow(const float* p) {
    for (int k = 0; k < 3; ++k) { mn[k] = std::min(mn[k], p[k]); mx[k] = std::max(mx[k], p[k]); }
  }
  float area() const {
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = std::max(0.0f, mx[k] - mn[k]);
    return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
  }
};

struct BNode {
  Box box;
  int left = -1, right = -1;
  uint32_t first = 0, count = 0;
  int depth = 0;
};

constexpr int kBins = 32;
constexpr int kMedianDepth = 40;
// Intersection cost 1.5 and leaves of at most 4 primitives were measured
// against these (c1, c4): within 1 % either way.
constexpr float kTraversalCost = 1.0f;
constexpr float kIsectCost = 1.0f;

struct Builder {
  const std::vector<PrimBox>& prims;
  std::vector<uint32_t>& order;
  std::vector<BNode> nodes;
  std::atomic<int> max_depth{0};
  uint32_t leaf_max = kLeafMax;

  Builder(const std::vector<PrimBox>& p, std::vector<uint32_t>& o, uint32_t lm)
      : prims(p), order(o), leaf_max(lm) {}

  Box bounds(uint32_t b, uint32_t e, Box* cbox) const {
    Box bb, cb;
    bb.reset();
    cb.reset();
    for (uint32_t i = b; i < e; ++i) {
      const PrimBox& p = prims[order[i]];
      Box pb;
      std::memcpy(pb.mn, p.mn, sizeof(pb.mn));
      std::memcpy(pb.mx, p.mx, sizeof(pb.mx));
      bb.grow(pb);
      cb.grow(p.c);
    }
    if (cbox) *cbox = cb;
    return bb;
  }

  // Returns split position in [b,e) or 0 for "make a leaf".
  uint32_t split(uint32_t b, uint32_t e, const Box& box, const Box& cb, int depth) {
    const uint32_t n = e - b;
    if (n <= 1) return 0;
    int axis = 0;
    float ext[3];
    for (int k = 0; k < 3; ++k) ext[k] = cb.mx[k] - cb.mn[k];
    if (ext[1] > ext[axis]) axis = 1;
    if (ext[2] > ext[axis]) axis = 2;
    if (depth >= kMedianDepth || ext[axis] <= 0.0f) {
      if (n <= leaf_max && depth < kMedianDepth) return 0;
      uint32_t mid = b + n / 2;
      std::nth_element(order.begin() + b, order.begin() + mid, order.begin() + e,
                       [&](uint32_t x, uint32_t y) { return prims[x].c[axis] < prims[y].c[axis]; });
      return mid;
    }
    float best_cost = INFINITY;
    int best_axis = -1, best_bin = -1;
    for (int a = 0; a < 3; ++a) {
      if (ext[a] <= 0.0f) continue;
      Box bin_box[kBins];
      uint32_t bin_n[kBins] = {};
      for (int i = 0; i < kBins; ++i) bin_box[i].reset();
      const float scale = kBins / ext[a];
      for (uint32_t i = b; i < e; ++i) {
        const PrimBox& p = prims[order[i]];
        int bi = std::min(kBins - 1, (int)((p.c[a] - cb.mn[a]) * scale));
        bi = std::max(0, bi);
        Box pb;
        std::memcpy(pb.mn, p.mn, sizeof(pb.mn));
        std::memcpy(pb.mx, p.mx, sizeof(pb.mx));
        bin_box[bi].grow(pb);
        bin_n[bi]++;
      }
      float right_area[kBins];
      uint32_t right_n[kBins];
      Box acc;
      acc.reset();
      uint32_t cnt = 0;
      for (int i = kBins - 1; i > 0; --i) {
        acc.grow(bin_box[i]);
        cnt += bin_n[i];
        right_area[i] = acc.area();
        right_n[i] = cnt;
      }
      acc.reset();
      cnt = 0;
      for (int i = 0; i < kBins - 1; ++i) {
        acc.grow(bin_box[i]);
        cnt += bin_n[i];
        if (cnt == 0 || right_n[i + 1] == 0) continue;
        float c = acc.area() * cnt + right_area[i + 1] * right_n[i + 1];
        if (c < best_cost) { best_cost = c; best_axis = a; best_bin = i; }
      }
    }
    const float parent_area = std::max(box.area(), 1e-30f);
    const float split_cost = kTraversalCost + kIsectCost * best_cost / parent_area;
    const float leaf_cost = kIsectCost * n;
    if (best_axis < 0 || (n <= leaf_max && leaf_cost <= split_cost)) {
      if (n <= leaf_max) return 0;
      uint32_t mid = b + n / 2;
      std::nth_element(order.begin() + b, order.begin() + mid, order.begin() + e,
                       [&](uint32_t x, uint32_t y) { return prims[x].c[axis] < prims[y].c[axis]; });
      return mid;
    }
    const float scale = kBins / ext[best_axis];
    auto it = std::partition(order.begin() + b, order.begin() + e, [&](uint32_t x) {
      int bi = std::min(kBins - 1, (int)((prims[x].c[best_axis] - cb.mn[best_axis]) * scale));
      return std::max(0, bi) <= best_bin;
    });
    uint32_t mid = (uint32_t)(it - order.begin());
    if (mid == b || mid == e) mid = b + n / 2;
    return mid;
  }

  // Builds the subtree for [b,e) into `out` (its own node vector, root first).
  void build_range(uint32_t b, uint32_t e, int depth0, std::vector<BNode>& out) {
    struct Task { uint32_t b, e; int node; int depth; };
    std::vector<Task> stack;
    out.emplace_back();
    stack.push_back({b, e, 0, depth0});
    while (!stack.empty()) {
      Task t = stack.back();
      stack.pop_back();
      Box cb;
      Box box = bounds(t.b, t.e, &cb);
      out[t.node].box = box;
      out[t.node].depth = t.depth;
      int d = max_depth.load();
      while (t.depth > d && !max_depth.compare_exchange_weak(d, t.depth)) {}
      uint32_t mid = split(t.b, t.e, box, cb, t.depth);
      if (mid == 0) {
        out[t.node].first = t.b;
        out[t.node].count = t.e - t.b;
        continue;
      }
      int l = (int)out.size();
      out.emplace_back();
      int r = (int)out.size();
      out.emplace_back();
      out[t.node].left = l;
      out[t.node].right = r;
      stack.push_back({mid, t.e, r, t.depth + 1});
      stack.push_back({t.b, mid, l, t.depth + 1});
    }
  }
};

inline float round_down(double x) {
  float f = (float)x;
  if ((double)f > x) f = std::nextafter(f, -INFINITY);
  return f;
}
inline float round_up(double x) {
  float f = (float)x;
  if ((double)f < x) f = std::nextafter(f, INFINITY);
  return f;
}

}  // namespace

void prim_box_from_double(PrimBox& p, const double* mn, const double* mx) {
  for (int k = 0; k < 3; ++k) {
    p.mn[k] = round_down(mn[k]);
    p.mx[k] = round_up(mx[k]);
    p.c[k] = (float)(0.5 * (mn[k] + mx[k]));
  }
}

// Flattens a tree of BNodes (root 0) to dual-child device nodes in
// depth-first order; dev_index_out (optional) receives each internal
// node's device index.
static bool flatten(const std::vector<BNode>& nodes, BvhResult& out, std::vector<int>* dev_index_out) {
  if (nodes[0].left < 0) {
    out.root_leaf = leaf_link(nodes[0].first, nodes[0].count);
    Node dn;
    const BNode& r = nodes[0];
    dn.lxy = make_float4(r.box.mn[0], r.box.mx[0], r.box.mn[1], r.box.mx[1]);
    dn.rxy = make_float4(INFINITY, -INFINITY, INFINITY, -INFINITY);
    dn.z = make_float4(r.box.mn[2], r.box.mx[2], INFINITY, -INFINITY);
    dn.link = make_int4(out.root_leaf, out.root_leaf, 0, 0);
    out.nodes.push_back(dn);
    out.leaves = 1;
    return true;
  }
  std::vector<int> local_index;
  std::vector<int>& dev_index = dev_index_out ? *dev_index_out : local_index;
  dev_index.assign(nodes.size(), -1);
  std::vector<int> stack{0};
  std::vector<int> order_nodes;
  while (!stack.empty()) {
    int i = stack.back();
    stack.pop_back();
    dev_index[i] = (int)order_nodes.size();
    order_nodes.push_back(i);
    if (nodes[nodes[i].right].left >= 0) stack.push_back(nodes[i].right);
    if (nodes[nodes[i].left].left >= 0) stack.push_back(nodes[i].left);
  }
  out.nodes.resize(order_nodes.size());
  for (size_t k = 0; k < order_nodes.size(); ++k) {
    const BNode& p = nodes[order_nodes[k]];
    const BNode& L = nodes[p.left];
    const BNode& R = nodes[p.right];
    Node dn;
    dn.lxy = make_float4(L.box.mn[0], L.box.mx[0], L.box.mn[1], L.box.mx[1]);
    dn.rxy = make_float4(R.box.mn[0], R.box.mx[0], R.box.mn[1], R.box.mx[1]);
    dn.z = make_float4(L.box.mn[2], L.box.mx[2], R.box.mn[2], R.box.mx[2]);
    int ll = L.left >= 0 ? dev_index[p.left] : leaf_link(L.first, L.count);
    int rl = R.left >= 0 ? dev_index[p.right] : leaf_link(R.first, R.count);
    if (L.left < 0) out.leaves++;
    if (R.left < 0) out.leaves++;
    dn.link = make_int4(ll, rl, 0, 0);
    out.nodes[k] = dn;
  }
  return true;
}

// The binary SAH tree over prims (root 0, leaves of up to leaf_max
// primitives as ranges of out.order); fills out.order and out.max_depth.
static bool build_tree(const std::vector<PrimBox>& prims, uint32_t leaf_max, BvhResult& out,
                       std::vector<BNode>& tree, std::string& err) {
  const uint32_t n = (uint32_t)prims.size();
  if (n >= (1u << 28)) {
    err = "too many primitives for the leaf encoding (max 2^28)";
    return false;
  }
  out.order.resize(n);
  for (uint32_t i = 0; i < n; ++i) out.order[i] = i;
  Builder B(prims, out.order, leaf_max);

  // Top levels single-threaded down to ~4x hardware threads subtrees, then
  // subtrees in parallel, then stitched into one node vector.
  std::vector<BNode>& nodes = B.nodes;
  struct Pending { uint32_t b, e; int node; int depth; };
  std::vector<Pending> leaves_to_build;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const uint32_t par_threshold = std::max<uint32_t>(4096, n / (4 * hw));
  {
    struct Task { uint32_t b, e; int node; int depth; };
    std::vector<Task> stack;
    nodes.emplace_back();
    stack.push_back({0, n, 0, 0});
    while (!stack.empty()) {
      Task t = stack.back();
      stack.pop_back();
      if (t.e - t.b <= par_threshold && n > par_threshold) {
        leaves_to_build.push_back({t.b, t.e, t.node, t.depth});
        continue;
      }
      Box cb;
      Box box = B.bounds(t.b, t.e, &cb);
      nodes[t.node].box = box;
      nodes[t.node].depth = t.depth;
      uint32_t mid = B.split(t.b, t.e, box, cb, t.depth);
      if (mid == 0) {
        nodes[t.node].first = t.b;
        nodes[t.node].count = t.e - t.b;
        continue;
      }
      int l = (int)nodes.size();
      nodes.emplace_back();
      int r = (int)nodes.size();
      nodes.emplace_back();
      nodes[t.node].left = l;
      nodes[t.node].right = r;
      stack.push_back({mid, t.e, r, t.depth + 1});
      stack.push_back({t.b, mid, l, t.depth + 1});
    }
  }
  if (!leaves_to_build.empty()) {
    std::vector<std::vector<BNode>> parts(leaves_to_build.size());
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (unsigned w = 0; w < hw; ++w)
      pool.emplace_back([&]() {
        for (size_t i; (i = next.fetch_add(1)) < leaves_to_build.size();)
          B.build_range(leaves_to_build[i].b, leaves_to_build[i].e, leaves_to_build[i].depth, parts[i]);
      });
    for (auto& th : pool) th.join();
    for (size_t i = 0; i < parts.size(); ++i) {
      const int base = (int)nodes.size();
      const int dst = leaves_to_build[i].node;
      std::vector<BNode>& p = parts[i];
      nodes[dst] = p[0];
      if (nodes[dst].left >= 0) {
        nodes[dst].left += base - 1;
        nodes[dst].right += base - 1;
      }
      for (size_t k = 1; k < p.size(); ++k) {
        BNode q = p[k];
        if (q.left >= 0) { q.left += base - 1; q.right += base - 1; }
        nodes.push_back(q);
      }
    }
  }
  out.max_depth = B.max_depth.load();
  for (const BNode& b : nodes) out.max_depth = std::max(out.max_depth, b.depth);
  if (out.max_depth >= kMaxTreeDepth) {
    err = "BVH deeper than the traversal stack";
    return false;
  }
  tree = std::move(nodes);
  return true;
}

bool build_bvh(const std::vector<PrimBox>& prims, BvhResult& out, std::string& err) {
  out = BvhResult();
  if (prims.empty()) return true;
  std::vector<BNode> tree;
  if (!build_tree(prims, kLeafMax, out, tree, err)) return false;
  return flatten(tree, out, nullptr);
}


// ---------------------------------------------------------------------------
// The 8-wide tree (WNode, mrt_internal.h): the binary SAH tree built with
// leaves of up to kWideLeafMax primitives, collapsed by the SAH-optimal
// slot distribution below, children placed in slots by octant and their
// boxes quantised to 8 bits on a power-of-two grid (Ylitie, Karras and
// Laine, HPG 2017).
// Wide nodes are numbered breadth first, so the internal children of a node
// are consecutive from its child_base and the primitives of its leaves
// consecutive from its prim_base; out.order is re-laid in that order.
namespace {

// Quantisation grid of one axis of a node box [lo, hi]: a power-of-two step
// s with (hi - lo) / s <= 252 and at least a few ulps of the coordinates,
// and an origin p one step below lo (rounded down to float), so that every
// child keeps a margin of one step on each side within q in 0..255.
struct AxisGrid {
  float p;
  double s;
  uint32_t biased;   // exponent of s + 127
};

inline bool axis_grid(float lo, float hi, AxisGrid& g) {
  const double E = std::max(0.0, (double)hi - (double)lo);
  const double maxabs = std::max(std::fabs((double)lo), std::fabs((double)hi));
  const double want = std::max({E / 252.0, maxabs * std::ldexp(1.0, -21), std::ldexp(1.0, -100)});
  int e = (int)std::ceil(std::log2(want));
  if (std::ldexp(1.0, e) < want) ++e;
  if (e < -126 || e > 127) return false;
  g.s = std::ldexp(1.0, e);
  g.biased = (uint32_t)(e + 127);
  g.p = round_down((double)lo - g.s);
  return std::isfinite(g.p);
}

inline bool quantise(const AxisGrid& g, float lo, float hi, uint32_t& qlo, uint32_t& qhi) {
  double a = std::floor(((double)lo - (double)g.p) / g.s) - 1.0;
  double b = std::ceil(((double)hi - (double)g.p) / g.s) + 1.0;
  a = std::max(0.0, a);
  b = std::min(255.0, b);
  qlo = (uint32_t)a;
  qhi = (uint32_t)b;
  // the decoded box must contain the child's box
  return (double)g.p + qlo * g.s <= (double)lo && (double)g.p + qhi * g.s >= (double)hi && qlo <= qhi;
}

inline void put_byte(int& word, int j, uint32_t v) {
  word = (int)(((uint32_t)word & ~(0xffu << (8 * j))) | ((v & 0xffu) << (8 * j)));
}

}  // namespace

bool build_bvh_wide(const std::vector<PrimBox>& prims, BvhResult& out, std::string& err) {
  out = BvhResult();
  const uint32_t n = (uint32_t)prims.size();
  if (n == 0) return true;
  std::vector<BNode> tree;
  BvhResult bin;
  if (!build_tree(prims, kWideLeafMax, bin, tree, err)) return false;
  // primitive range of every binary subtree (the builder partitions the
  // order array, so a subtree's primitives are contiguous): a subtree of at
  // most kWideLeafMax primitives becomes one leaf slot, so that the bottom
  // wide nodes are full of leaves rather than of 1-primitive binary leaves
  std::vector<uint32_t> sub_first(tree.size()), sub_count(tree.size());
  for (size_t i = tree.size(); i-- > 0;) {   // children after parents in the node vector
    const BNode& b = tree[i];
    if (b.left < 0) {
      sub_first[i] = b.first;
      sub_count[i] = b.count;
    } else {
      sub_first[i] = std::min(sub_first[b.left], sub_first[b.right]);
      sub_count[i] = sub_count[b.left] + sub_count[b.right];
    }
  }
  // SAH-optimal collapse (Ylitie, Karras and Laine 2017, section 3.1): for
  // every binary node n and slot budget i in 1..8, cost[n][i] is the least
  // SAH cost of representing n's subtree with at most i slots of its
  // parent: as one slot (a leaf of at most kWideLeafMax primitives, or a
  // wide node of its own), or by giving j slots to its left subtree and
  // i - j to its right.
  constexpr double kNodeCost = 1.0, kPrimCost = 0.3;
  const size_t nbin = tree.size();
  std::vector<std::array<double, 9>> cost(nbin);
  std::vector<std::array<uint8_t, 9>> give(nbin);   // 0: one slot; j: j slots to the left subtree
  std::vector<uint8_t> as_leaf(nbin), node_left(nbin);
  for (size_t i = nbin; i-- > 0;) {
    const BNode& b = tree[i];
    double d[3];
    for (int a = 0; a < 3; ++a) d[a] = std::max(0.0, (double)b.box.mx[a] - (double)b.box.mn[a]);
    const double area = 2.0 * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    const bool fits = sub_count[i] <= (uint32_t)kWideLeafMax;
    const double leaf = fits ? area * kPrimCost * (double)sub_count[i] : INFINITY;
    double node = INFINITY;
    int nj = 4;
    if (b.left >= 0) {
      for (int j = 1; j < 8; ++j) {
        const double c = cost[b.left][j] + cost[b.right][8 - j];
        if (c < node) { node = c; nj = j; }
      }
      node += area * kNodeCost;
    }
    as_leaf[i] = fits && (leaf <= node || b.left < 0);
    node_left[i] = (uint8_t)nj;
    const double one = std::min(leaf, node);
    for (int k = 1; k <= 8; ++k) {
      double best = one;
      int bj = 0;
      if (b.left >= 0)
        for (int j = 1; j < k; ++j) {
          const double c = cost[b.left][j] + cost[b.right][k - j];
          if (c < best) { best = c; bj = j; }
        }
      cost[i][k] = best;
      give[i][k] = (uint8_t)bj;
    }
  }
  auto is_leaf = [&](int i) { return as_leaf[i] != 0; };
  // the slots that subtree n fills when given k of them
  std::function<void(int, int, std::vector<int>&)> distribute = [&](int n, int k, std::vector<int>& ch) {
    const int j = give[n][k];
    if (j == 0) {
      ch.push_back(n);
      return;
    }
    distribute(tree[n].left, j, ch);
    distribute(tree[n].right, k - j, ch);
  };
  struct Item { int bnode; int depth; };
  std::vector<Item> items{{0, 0}};        // items[i] becomes wide node i
  out.wnodes.reserve(tree.size() / 4 + 1);
  out.order.clear();
  out.order.reserve(n);
  int max_depth = 0;
  for (size_t wi = 0; wi < items.size(); ++wi) {
    const Item it = items[wi];
    max_depth = std::max(max_depth, it.depth);
    if (it.depth >= kWideStack - 2) {
      err = "wide BVH deeper than its traversal stack";
      return false;
    }
    // children: the binary subtrees the collapse gives this node's slots
    std::vector<int> ch;
    const BNode& root = tree[it.bnode];
    if (is_leaf(it.bnode)) {
      ch.push_back(it.bnode);               // the whole scene in one leaf
    } else {
      distribute(root.left, node_left[it.bnode], ch);
      distribute(root.right, 8 - node_left[it.bnode], ch);
    }
    // node box and centre
    Box nb;
    nb.reset();
    for (int c : ch) nb.grow(tree[c].box);
    // octant slots: greedy on cost = -(child centre - node centre) . corner(slot)
    int slot_of[8], child_in[8];
    for (int k = 0; k < 8; ++k) { slot_of[k] = -1; child_in[k] = -1; }
    float cost[8][8];
    for (size_t k = 0; k < ch.size(); ++k) {
      const Box& b = tree[ch[k]].box;
      float dc[3];
      for (int a = 0; a < 3; ++a) dc[a] = 0.5f * (b.mn[a] + b.mx[a]) - 0.5f * (nb.mn[a] + nb.mx[a]);
      for (int sl = 0; sl < 8; ++sl) {
        float c = 0.0f;
        for (int a = 0; a < 3; ++a) c -= dc[a] * (((sl >> a) & 1) ? 1.0f : -1.0f);
        cost[k][sl] = c;
      }
    }
    for (size_t done = 0; done < ch.size(); ++done) {
      int bk = -1, bs = -1;
      float bc = INFINITY;
      for (size_t k = 0; k < ch.size(); ++k) {
        if (slot_of[k] >= 0) continue;
        for (int sl = 0; sl < 8; ++sl)
          if (child_in[sl] < 0 && (bk < 0 || cost[k][sl] < bc)) { bc = cost[k][sl]; bk = (int)k; bs = sl; }
      }
      slot_of[bk] = bs;
      child_in[bs] = bk;
    }
    // quantisation grid
    AxisGrid g[3];
    for (int a = 0; a < 3; ++a)
      if (!axis_grid(nb.mn[a], nb.mx[a], g[a])) {
        err = "wide BVH: node box out of the quantisation range";
        return false;
      }
    WNode w{};
    uint32_t imask = 0;
    const uint32_t child_base = (uint32_t)items.size();
    const uint32_t prim_base = (uint32_t)out.order.size();
    uint32_t prim_off = 0;
    int words[6][2] = {};                   // qlo x y z, qhi x y z; slots 0-3 / 4-7
    int meta[2] = {0, 0};
    for (int sl = 0; sl < 8; ++sl) {
      const int k = child_in[sl];
      if (k < 0) continue;
      const BNode& c = tree[ch[k]];
      uint32_t m = 0x80u;
      if (!is_leaf(ch[k])) {
        imask |= 1u << sl;
        items.push_back({ch[k], it.depth + 1});
      } else {
        const uint32_t cf = sub_first[ch[k]], cn = sub_count[ch[k]];
        if (cn == 0 || cn > (uint32_t)kWideLeafMax || prim_off + cn > 32) {
          err = "wide BVH: leaf does not fit its slot";
          return false;
        }
        m |= prim_off | ((cn - 1) << 5);
        for (uint32_t j = 0; j < cn; ++j) out.order.push_back(bin.order[cf + j]);
        prim_off += cn;
        ++out.leaves;
      }
      put_byte(meta[sl >> 2], sl & 3, m);
      for (int a = 0; a < 3; ++a) {
        uint32_t ql, qh;
        if (!quantise(g[a], c.box.mn[a], c.box.mx[a], ql, qh)) {
          err = "wide BVH: child box quantisation";
          return false;
        }
        put_byte(words[a][sl >> 2], sl & 3, ql);
        put_byte(words[3 + a][sl >> 2], sl & 3, qh);
      }
    }
    uint32_t ebits = g[0].biased | (g[1].biased << 8) | (g[2].biased << 16) | (imask << 24);
    float ew;
    std::memcpy(&ew, &ebits, 4);
    w.a = make_float4(g[0].p, g[1].p, g[2].p, ew);
    w.b = make_int4((int)child_base, (int)prim_base, meta[0], meta[1]);
    w.c = make_int4(words[0][0], words[0][1], words[1][0], words[1][1]);
    w.d = make_int4(words[2][0], words[2][1], words[3][0], words[3][1]);
    w.e = make_int4(words[4][0], words[4][1], words[5][0], words[5][1]);
    out.wnodes.push_back(w);
  }
  if (out.order.size() != n) {
    err = "wide BVH: primitive count mismatch";
    return false;
  }
  out.max_depth = max_depth;
  return true;
}

// Structure of an 8-wide tree: every node reachable exactly once from the
// root through child indices greater than its own, every leaf range inside
// the primitive array, every primitive in exactly one leaf, order a
// permutation, and every slot's decoded box (in double) containing all the
// primitive boxes below it, so that no culling step can drop a hit.
bool check_bvh_wide(const BvhResult& t, const std::vector<PrimBox>& prims, std::string& err) {
  const size_t n = prims.size(), nn = t.wnodes.size();
  if (n == 0) return nn == 0;
  if (nn == 0 || t.order.size() != n) { err = "wide BVH check: empty tree or order size"; return false; }
  std::vector<char> seen_prim(n, 0), seen_node(nn, 0), seen_src(n, 0);
  for (size_t k = 0; k < n; ++k) {
    if (t.order[k] >= n || seen_src[t.order[k]]) { err = "wide BVH check: order is not a permutation"; return false; }
    seen_src[t.order[k]] = 1;
  }
  seen_node[0] = 1;
  std::vector<Box> below(nn);
  for (size_t ii = nn; ii-- > 0;) {
    const WNode& w = t.wnodes[ii];
    uint32_t bits;
    std::memcpy(&bits, &w.a.w, 4);
    const uint32_t imask = bits >> 24;
    const double p[3] = {w.a.x, w.a.y, w.a.z};
    double s[3];
    for (int a = 0; a < 3; ++a) {
      const int e = (int)((bits >> (8 * a)) & 0xffu) - 127;
      if (e < -126 || e > 127) { err = "wide BVH check: exponent"; return false; }
      s[a] = std::ldexp(1.0, e);
    }
    const uint32_t meta[2] = {(uint32_t)w.b.z, (uint32_t)w.b.w};
    const uint32_t lo[3][2] = {{(uint32_t)w.c.x, (uint32_t)w.c.y}, {(uint32_t)w.c.z, (uint32_t)w.c.w},
                               {(uint32_t)w.d.x, (uint32_t)w.d.y}};
    const uint32_t hi[3][2] = {{(uint32_t)w.d.z, (uint32_t)w.d.w}, {(uint32_t)w.e.x, (uint32_t)w.e.y},
                               {(uint32_t)w.e.z, (uint32_t)w.e.w}};
    Box all;
    all.reset();
    int inner = 0;
    for (int sl = 0; sl < 8; ++sl) {
      const int h = sl >> 2, sh = 8 * (sl & 3);
      const uint32_t m = (meta[h] >> sh) & 0xffu;
      const bool is_inner = (imask >> sl) & 1u;
      if (!(m & 0x80u)) {
        if (is_inner) { err = "wide BVH check: empty slot marked internal"; return false; }
        continue;
      }
      Box need;
      need.reset();
      if (is_inner) {
        const size_t c = (size_t)(uint32_t)w.b.x + (size_t)inner++;
        if (c >= nn || c <= ii || seen_node[c]) { err = "wide BVH check: child index"; return false; }
        seen_node[c] = 1;
        need = below[c];
      } else {
        const size_t first = (size_t)(uint32_t)w.b.y + (m & 31u), count = ((m >> 5) & 3u) + 1;
        if (first + count > n) { err = "wide BVH check: leaf range"; return false; }
        for (size_t k = first; k < first + count; ++k) {
          if (seen_prim[k]) { err = "wide BVH check: primitive in two leaves"; return false; }
          seen_prim[k] = 1;
          Box pb;
          std::memcpy(pb.mn, prims[t.order[k]].mn, sizeof(pb.mn));
          std::memcpy(pb.mx, prims[t.order[k]].mx, sizeof(pb.mx));
          need.grow(pb);
        }
      }
      for (int a = 0; a < 3; ++a) {
        const double bl = p[a] + ((lo[a][h] >> sh) & 0xffu) * s[a];
        const double bh = p[a] + ((hi[a][h] >> sh) & 0xffu) * s[a];
        if ((double)need.mn[a] < bl || (double)need.mx[a] > bh) {
          err = "wide BVH check: a slot box does not contain what lies below it";
          return false;
        }
      }
      all.grow(need);
    }
    below[ii] = all;
  }
  for (size_t i = 0; i < nn; ++i)
    if (!seen_node[i]) { err = "wide BVH check: unreachable node"; return false; }
  for (size_t k = 0; k < n; ++k)
    if (!seen_prim[k]) { err = "wide BVH check: primitive in no leaf"; return false; }
  return true;
}

// ---------------------------------------------------------------------------
// The reference's median-split tree, for parity runs (MRT_BVH_REFERENCE).
// Its steps are restated, not redesigned, because the topology must come out
// identical: node bounds are the union of the primitives' double bounds; a
// node of more than one primitive is split on the longest axis of its bounds
// (choose_axis, bvh_build.c:44) at count / 2 after sorting its primitives by
// their position on that axis compared as float (compare_obj_axis_with_bvh,
// bvh_math.c:34); the sort is the reference's (qshort_axis.c: insertion sort
// below 16 elements, else median-of-three quicksort recursing on the smaller
// side), whose handling of equal keys decides the order of ties.
namespace {

struct RefSort {
  const std::vector<RefPrim>& prims;
  const std::vector<uint32_t>& list;
  int axis;
  int cmp(uint32_t a, uint32_t b) const {
    const float va = (float)prims[list[a]].pos[axis], vb = (float)prims[list[b]].pos[axis];
    return va < vb ? -1 : (va > vb ? 1 : 0);
  }
  void insertion(uint32_t* arr, int lo, int hi) const {
    for (int i = lo + 1; i <= hi; ++i) {
      const uint32_t key = arr[i];
      int j = i - 1;
      while (j >= lo && cmp(arr[j], key) > 0) {
        arr[j + 1] = arr[j];
        --j;
      }
      arr[j + 1] = key;
    }
  }
  int partition(uint32_t* arr, int lo, int hi) const {
    const int mid = lo + (hi - lo) / 2;
    if (cmp(arr[lo], arr[mid]) > 0) std::swap(arr[lo], arr[mid]);
    if (cmp(arr[lo], arr[hi]) > 0) std::swap(arr[lo], arr[hi]);
    if (cmp(arr[mid], arr[hi]) > 0) std::swap(arr[mid], arr[hi]);
    std::swap(arr[mid], arr[hi - 1]);
    const uint32_t pivot = arr[hi - 1];
    int i = lo, j = hi - 1;
    while (true) {
      while (cmp(arr[++i], pivot) < 0) {}
      while (cmp(arr[--j], pivot) > 0) {}
      if (i >= j) break;
      std::swap(arr[i], arr[j]);
    }
    std::swap(arr[i], arr[hi - 1]);
    return i;
  }
  void sort(uint32_t* arr, int lo, int hi) const {
    while (lo < hi) {
      if (hi - lo < 16) {
        insertion(arr, lo, hi);
        return;
      }
      const int p = partition(arr, lo, hi);
      if (p - lo < hi - p) {
        sort(arr, lo, p - 1);
        lo = p + 1;
      } else {
        sort(arr, p + 1, hi);
        hi = p - 1;
      }
    }
  }
};

}  // namespace


bool build_bvh_reference(const std::vector<RefPrim>& prims, const std::vector<uint32_t>& list,
                         BvhResult& out, std::vector<double>& dboxes, std::string& err) {
  out = BvhResult();
  dboxes.clear();
  const uint32_t n = (uint32_t)list.size();
  if (n == 0) return true;
  if (n >= (1u << 28) || list.size() != prims.size()) {
    err = n >= (1u << 28) ? "too many primitives for the leaf encoding (max 2^28)"
                          : "reference BVH: object list does not cover the primitives";
    return false;
  }
  std::vector<uint32_t> idx(n);            // prim_indices: positions in the object list
  for (uint32_t i = 0; i < n; ++i) idx[i] = i;
  std::vector<BNode> nodes;
  std::vector<double> dbl;                 // 6 per BNode
  RefSort sorter{prims, list, 0};
  auto make_node = [&](uint32_t start, uint32_t count, int depth) {
    double mn[3], mx[3];
    const RefPrim& f = prims[list[idx[start]]];
    for (int k = 0; k < 3; ++k) { mn[k] = f.mn[k]; mx[k] = f.mx[k]; }
    for (uint32_t i = 0; i < count; ++i) {
      const RefPrim& p = prims[list[idx[start + i]]];
      for (int k = 0; k < 3; ++k) { mn[k] = std::fmin(mn[k], p.mn[k]); mx[k] = std::fmax(mx[k], p.mx[k]); }
    }
    BNode b;
    for (int k = 0; k < 3; ++k) { b.box.mn[k] = round_down(mn[k]); b.box.mx[k] = round_up(mx[k]); }
    b.first = start;
    b.count = count;
    b.depth = depth;
    nodes.push_back(b);
    dbl.insert(dbl.end(), {mn[0], mn[1], mn[2], mx[0], mx[1], mx[2]});
    return (int)nodes.size() - 1;
  };
  struct Task { uint32_t start, count; int node; };
  std::vector<Task> stack;
  stack.push_back({0, n, make_node(0, n, 0)});
  while (!stack.empty()) {
    const Task t = stack.back();
    stack.pop_back();
    if (t.count <= 1) continue;
    const double* b = &dbl[6 * (size_t)t.node];
    const double ex = b[3] - b[0], ey = b[4] - b[1], ez = b[5] - b[2];
    sorter.axis = (ex > ey && ex > ez) ? 0 : (ey > ez ? 1 : 2);
    sorter.sort(idx.data() + t.start, 0, (int)t.count - 1);
    const uint32_t mid = t.start + t.count / 2;
    const int depth = nodes[t.node].depth + 1;
    const int l = make_node(t.start, mid - t.start, depth);
    const int r = make_node(mid, t.start + t.count - mid, depth);
    nodes[t.node].left = l;
    nodes[t.node].right = r;
    stack.push_back({mid, t.start + t.count - mid, r});
    stack.push_back({t.start, mid - t.start, l});
  }
  for (const BNode& q : nodes) out.max_depth = std::max(out.max_depth, q.depth);
  if (out.max_depth >= kMaxTreeDepth) {
    err = "reference BVH deeper than the traversal stack";
    return false;
  }
  // leaves hold one primitive each: leaf order = the sorted object list
  out.order.resize(n);
  for (uint32_t i = 0; i < n; ++i) out.order[i] = list[idx[i]];
  std::vector<int> dev_index;
  if (!flatten(nodes, out, &dev_index)) return false;
  dboxes.assign(6 + 12 * out.nodes.size(), 0.0);
  std::copy(dbl.begin(), dbl.begin() + 6, dboxes.begin());
  if (nodes[0].left < 0) {                 // a single primitive: the root is the leaf
    std::copy(dbl.begin(), dbl.begin() + 6, dboxes.begin() + 6);
    return true;
  }
  for (size_t i = 0; i < nodes.size(); ++i) {
    if (nodes[i].left < 0) continue;
    double* d = &dboxes[6 + 12 * (size_t)dev_index[i]];
    std::copy(dbl.begin() + 6 * nodes[i].left, dbl.begin() + 6 * nodes[i].left + 6, d);
    std::copy(dbl.begin() + 6 * nodes[i].right, dbl.begin() + 6 * nodes[i].right + 6, d + 6);
  }
  return true;
}

}  // namespace mrt
