// mrt_internal.h — device data layout shared by the host repack and the
// kernels. Everything here lives in HBM (or constant memory for the small
// per-scene block) and is read-only while rendering.
//
// Layout (all arrays 16-byte aligned, read with 128-bit loads):
//   nodes   : BVH2 with both child boxes stored in the parent, 64 B per node
//             (float4 x-y of left, float4 x-y of right, float4 z of both,
//             int4 child links). A negative link is a leaf:
//             ~(first_prim << 3 | (count - 1)), up to 8 primitives.
//   wnodes  : the MRT_BVH_WIDE option: 8-wide, 80 B per node (WNode
//             below), leaves of up to 4 primitives, siblings contiguous.
//   geom    : 48 B per primitive in leaf order. Triangle: (v0, type) (e1, -)
//             (e2, -). Sphere: (centre, type) (radius, r^2, -, -) (-).
//   meta    : int4 per primitive in leaf order: (flat id, material, type,
//             packed rgb8 object colour).
//   shade   : 64 B per triangle in leaf order: (n0, u0) (n1, u1) (n2, u2)
//             (v0, v1, v2, -). Read once per closest hit.
//   planes  : 2 float4 + int4 per plane.
//   photons : position / power float4 pairs in Morton order plus a linear
//             BVH over them (4 float4 per internal node).
//   env     : RGBE texels as uint32; for importance sampling an alias table
//             (float prob, int alias) over the outcomes of the reference's
//             two-step lookup and two float4 records per outcome
//             (direction + pdf, sky radiance of that direction).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace mrt {

enum PrimType : int { PRIM_TRI = 0, PRIM_SPHERE = 1, PRIM_CYL = 2, PRIM_CONE = 3, PRIM_HYP = 4 };

constexpr int kLeafMax = 8;          // primitives per leaf (3-bit count)
constexpr int kStackSize = 64;       // traversal stack; the builder bounds depth below it
constexpr int kMaxTreeDepth = 60;
constexpr float kTMin = 0.001f;      // IT_MIN (minirt.h:44)
constexpr float kTMax = 1000.0f;     // IT_MAX and the initial closest_t (hit_register.c:21)

struct __align__(16) Node {
  float4 lxy;   // left  (min.x, max.x, min.y, max.y)
  float4 rxy;   // right (min.x, max.x, min.y, max.y)
  float4 z;     // (left min.z, left max.z, right min.z, right max.z)
  int4 link;    // (left, right, -, -)
};

__host__ __device__ inline int leaf_link(uint32_t first, uint32_t count) {
  return ~(int)((first << 3) | (count - 1));
}

// 8-wide BVH node with 8-bit quantised child boxes (the compressed wide BVH
// of Ylitie, Karras and Laine, HPG 2017, in this library's own packing), 80 B:
//   a: origin p.xyz, w = bits ex | ey << 8 | ez << 16 | imask << 24
//      (child box along x: p.x + q * 2^(ex - 127), q in 0..255)
//   b: (child_base, prim_base, meta of slots 0-3, meta of slots 4-7)
//   c: (qlo.x slots 0-3, qlo.x 4-7, qlo.y 0-3, qlo.y 4-7)
//   d: (qlo.z 0-3, qlo.z 4-7, qhi.x 0-3, qhi.x 4-7)
//   e: (qhi.y 0-3, qhi.y 4-7, qhi.z 0-3, qhi.z 4-7)
// A slot's meta byte is 0 when empty, else has bit 7 set. imask bit s marks
// slot s as an internal child: node child_base + popc(imask below s). A
// leaf slot holds ((meta >> 5) & 3) + 1 primitives from prim_base +
// (meta & 31). Children sit in the slot whose octant they lie towards, so
// visiting slots in the order of slot ^ (the ray's sign bits) is roughly
// near to far.
struct __align__(16) WNode {
  float4 a;
  int4 b;
  int4 c;
  int4 d;
  int4 e;
};
constexpr int kWideLeafMax = 4;      // primitives per leaf slot
constexpr int kWideStack = 32;       // node-group entries (2 ints each) in the 64-int stack

struct MaterialD {
  float color[3];        // color_value / 255
  float metallic;
  float roughness;
  float ior;
  float transmission;
  float ao;
  float emission_strength;
  float emission[3];     // emission_color / 255
  float f0;              // powf(((ior-1)/(ior+1)), 2) (material/utils.c:29-37)
  float alpha4;          // roughness^4 for the GGX-like sampler (utils.c:47-48)
};

// Texture (t_tex): type as mrt_tex_type; an IMAGE's texels are
// texels[offset, offset + w*h) as RGBA8, w = 0 for a missing image.
struct TexD {
  int type;
  int w, h;
  uint32_t offset;
  float c1[3], c2[3];    // checker colours / 255
  float scale;           // checker scale
  int pad;
};

// Texture slots of a material (1 + texture index, 0 none), in the order of
// mrt_material's *_tex fields.
enum TexSlot : int {
  TS_COLOR = 0, TS_METALLIC, TS_ROUGHNESS, TS_TRANSMISSION, TS_AO, TS_EMIS_STRENGTH, TS_EMIS_COLOR,
  TS_NORMAL, TS_COUNT
};
struct MatTexD {
  int tex[TS_COUNT];
  float normal_intensity;
  float uv_scale;        // t_mat.scale (uv tiling)
  int any;               // some slot is set
  int alpha;             // the colour texture is an image with a texel of alpha < 255
};

struct LightD {
  float pos[3];          // point: position; directional: unit orientation
  float brightness;
  float color[3];        // 0..255 scale, as the reference accumulates it
  float radius;
  int type;
  int shadow_sample;
  int pad[2];
};

struct PlaneD {
  float4 pn;             // point.xyz, -
  float4 nn;             // normal.xyz, -
  int4 meta;             // flat id, material, -, packed colour
};

// Everything a kernel needs, passed by value (kernel parameter space).
// Kernels are instantiated for SceneView (spheres, triangles, planes) and for
// SceneViewQ (the same plus cylinders, cones and hyperboloids), chosen per
// scene at launch: the quadric tests compute in double, and their registers
// stay out of the kernels of scenes without quadrics.
struct SceneView {
  static constexpr bool kQuadrics = false;
  static constexpr bool kTextures = false;
  const Node* nodes;
  const float4* geom;
  const int4* meta;
  const float4* shade;
  const PlaneD* planes;
  const MaterialD* mats;
  const LightD* lights;
  int n_nodes;
  int n_prims;
  int n_planes;
  int n_mats;
  int n_lights;
  int one_sided;
  int root_leaf;         // scene with a single leaf: the link of that leaf, else 0
  int has_bvh;
  int has_quadrics;      // launch the SceneViewQ instantiation
  int has_textures;      // launch the SceneViewT instantiation
  int left_first;        // traverse the left child first (reference-topology tree), else the nearer
  const double* ref_boxes;  // reference-topology tree: double child boxes for its node-visit count
  const WNode* wnodes;   // when set: the 8-wide tree, traversed instead of `nodes`
  int n_wnodes;
  const MatTexD* mat_tex;    // per material
  const TexD* texs;
  const uchar4* texels;
  // camera (viewport.c:38-87), float
  float cam[3];
  float pixel00[3];
  float pdu[3];
  float pdv[3];
  float defocus_u[3];
  float defocus_v[3];
  float defocus_angle;
  int width;
  int height;
  int max_bounces;
  float ior_all;
  // ambient / sky
  float amb_const[3];    // colour * ratio / 255 when there is no sky texture
  const uint32_t* rgbe;
  int env_w;
  int env_h;
  float env_scale_exp;   // powf(2, exposure) or 1 (get_hdr_value.c:47-53)
  int env_exposure_zero;
  float env_inv_gamma;   // 1/gamma, 1 = linear
  int has_env;           // sky texture present
  const float* sky_rgb;  // when set: linear sky radiance per texel (W*H*3), used instead of rgbe
  int env_nee;           // importance-sampling tables present
  const float2* alias;   // (prob, alias as int bits), n_env_outcomes entries
  const float4* env_rec0;  // per outcome: direction .xyz, pdf
  const float4* env_rec1;  // per outcome: sky radiance of that direction (unclamped) .rgb
  int n_env_outcomes;
  int env_lookup;        // 1: sample with the two-step inverse-CDF tables instead
  const float* pdf_joint;  // W*H   (calc_pdf.c:93)
  const float* cdf_m_inv;  // H     (calc_cdf.c:39)
  const float* cdf_c_inv;  // W*H   (calc_cdf.c:112)
  // caustics (photon map)
  int caustic;
  int knn;
  float caustic_radius2; // compared against the k-th squared distance (get_caustic.c:45)
  float inv_norm;        // 1 / norm_factor
  const float4* photon_pos;    // in Morton order of their positions
  const float4* photon_pow;
  // Linear BVH over the Morton-ordered photons (Karras 2012): n - 1 internal
  // nodes, node 0 the root, each split at the highest Morton bit that
  // differs within its range; 4 float4 per node: (min.xyz, -), (max.xyz, -),
  // (summed power.rgb, -), (left, right as int bits, -, -) where a child
  // >= 0 is an internal node and ~i is photon i.
  const float4* photon_nodes;
  int caustic_mode;      // 0 kNN, 1 fixed radius
  float fixed_radius2;
  int n_photons;
};

struct SceneViewQ : SceneView {
  static constexpr bool kQuadrics = true;
};
// Scenes with textured materials (and any objects): texture lookups, maps
// and the alpha test, with a per-hit copy of the material values.
struct SceneViewT : SceneView {
  static constexpr bool kQuadrics = true;
  static constexpr bool kTextures = true;
};

// Calls f with the view as the type its kernels are instantiated for.
template <class F>
inline auto with_view(const SceneView& S, F&& f) {
  if (S.has_textures) {
    SceneViewT t;
    static_cast<SceneView&>(t) = S;
    return f(t);
  }
  if (S.has_quadrics) {
    SceneViewQ q;
    static_cast<SceneView&>(q) = S;
    return f(q);
  }
  return f(S);
}

// Device status word bits -> mrt_status on the host.
enum StatusBits : int {
  ST_STACK = 1, ST_BUDGET = 2, ST_QUEUE = 4, ST_ABORT = 8,
};

}  // namespace mrt
