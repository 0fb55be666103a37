// api.cu — the C-ABI of libmrt.so (include/mrt.h).
//
// Host side of the boundary that replaces miniRT's GL bridge (src/gpu):
// mrt_create ~ init_shader (init_shader.c:133), mrt_scene_build ~
// convert_scene_build (gpu_scene.c:104), mrt_set_camera ~ convert_scene
// (gpu_scene.c:62), mrt_render ~ compute_frame_gpu (use_shader.c:81) for many
// samples at once, mrt_destroy ~ clean_shaders / clean_scene
// (clean_shaders.c:32,69). The scene is repacked into the device layout of
// mrt_internal.h; the context owns all device memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mrt.h"
#include "bvh_build.h"
#include "comm.h"
#include "kernels.h"

using namespace mrt;

namespace {

thread_local std::string g_err;

int set_err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return set_err(e_ == cudaErrorMemoryAllocation ? MRT_ERR_OOM : MRT_ERR_CUDA,        \
                     "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaError_t alloc(size_t count) {
    release();
    n = count;
    if (count == 0) return cudaSuccess;
    return cudaMalloc(&p, sizeof(T) * count);
  }
  cudaError_t upload(const T* src, size_t count, cudaStream_t st) {
    cudaError_t e = alloc(count);
    if (e != cudaSuccess || count == 0) return e;
    return cudaMemcpyAsync(p, src, sizeof(T) * count, cudaMemcpyHostToDevice, st);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

struct V3 { double x, y, z; };
inline V3 v3(const double* p) { return {p[0], p[1], p[2]}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 dv(V3 a, double s) { return s != 0.0 ? V3{a.x / s, a.y / s, a.z / s} : V3{0, 0, 0}; }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double len(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline V3 unitv(V3 a) { double l = len(a); return l > 0.0 ? dv(a, l) : V3{0, 0, 0}; }
inline void put3(float* d, V3 a) { d[0] = (float)a.x; d[1] = (float)a.y; d[2] = (float)a.z; }

constexpr double kPiD = 3.1415926535897;

inline float int_bits_as_float(int i) {
  float f;
  std::memcpy(&f, &i, sizeof(f));
  return f;
}

}  // namespace

namespace mrt {
// Sets mrt_last_error's message for entry points defined in other files.
int set_error_message(int code, const char* msg) { return set_err(code, "%s", msg); }
}  // namespace mrt

struct WfHost;
WfHost* wf_create();
void wf_destroy(WfHost* H);
int wf_render(WfHost* H, const SceneView& v, const LaunchParams& L, int spp, int capacity,
              int sort_threshold, int use_graph, float4* frame, int* status, cudaStream_t st,
              unsigned* launches, const char** err);

// Device state of the differentiable forward / backward (mrt_forward,
// mrt_backward), sized for the current scene.
struct DiffState {
  int M = 0, EW = 0, EH = 0;
  bool tables = false;                 // HDRI NEE tables are rebuilt from theta
  DevBuf<float> theta, grad, img, dimg;
  DevBuf<MaterialD> mats;
  DevBuf<float4> grid, rec0, rec1, state;
  DevBuf<TapeEntry> tape;
  DevBuf<int2> aux;
  DevBuf<float> pdf, cm, cc;
  DevBuf<double> gray, raw, rowcdf, scal, cdfh;
  DevBuf<unsigned long long> accum_fx;   // forward image, fixed point (3 per pixel)
  DevBuf<long long> gq;                  // backward sums, fixed point (as grad)
  DevBuf<float> wmax;                    // max |d loss / d image|
  void release() {
    accum_fx.release(); gq.release(); wmax.release();
    theta.release(); grad.release(); img.release(); dimg.release(); mats.release();
    grid.release(); rec0.release(); rec1.release(); aux.release();
    state.release(); tape.release();
    pdf.release(); cm.release(); cc.release();
    gray.release(); raw.release(); rowcdf.release(); scal.release(); cdfh.release();
  }
};

struct mrt_ctx {
  int device = 0;
  DiffState* diff = nullptr;
  WfHost* wf = nullptr;
  int W = 0, H = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevBuf<float4> accum;
  DevBuf<float> rgb_dev;                 // read-back staging: accumulator as rgb floats
  float* rgb_host = nullptr;             // pinned host copy of rgb_dev
  size_t rgb_host_n = 0;
  DevBuf<int> depth;
  DevBuf<int> status;
  DevBuf<unsigned long long> counters;
  int accum_spp = 0;
  bool has_scene = false;
  // scene
  DevBuf<Node> nodes;
  DevBuf<WNode> wnodes;
  DevBuf<float4> geom, shade;
  DevBuf<int4> meta;
  DevBuf<PlaneD> planes;
  DevBuf<MaterialD> mats;
  DevBuf<LightD> lights;
  DevBuf<MatTexD> mat_tex;
  DevBuf<TexD> texs;
  DevBuf<uchar4> texels;
  DevBuf<int> point_lights;
  int n_point_lights = 0;
  DevBuf<uint32_t> rgbe;
  DevBuf<float> pdf_joint, cdf_m, cdf_c;
  DevBuf<float2> alias;
  DevBuf<float4> env_rec0, env_rec1;
  DevBuf<float4> ph_pos, ph_pow, ph_pos_raw, ph_pow_raw;
  DevBuf<float4> ph_nodes;
  DevBuf<unsigned int> ph_count;
  uint64_t photons_per_light = 0;
  int64_t n_photons = 0;
  mrt_caustic caustic{};
  int photon_pass = 0;                   // progressive mode: pass of the current photon map
  SceneView view{};
  size_t scene_bytes = 0;
  int bvh_depth = 0;
  int auto_form = MRT_FORM_MEGAKERNEL;   // choice of the autotuner for this scene
  int auto_block = 0, auto_capacity = 0, auto_sort = 0;
  // multi-GPU sample sharding (mrt_comm_init)
  void* comm = nullptr;
  int comm_rank = 0, comm_world = 1;
  DevBuf<long long> comm_count;          // sample count reduced with the frame
  // BVH build options (mrt_set_bvh_options), applied by mrt_scene_build
  int bvh_mode = MRT_BVH_SAH;
  std::vector<int32_t> bvh_list;         // reference object-list order (flat ids), empty = flat order
  std::vector<double> bvh_pos;           // positions the reference's split sorts by, empty = computed
  DevBuf<double> ref_boxes;
  std::vector<uint32_t> leaf_order;      // flat primitive id of each leaf slot (last build)
  // mrt_render_batch (when this context leads a batch): device arrays of the
  // megakernel groups per view type, and the streams the batch's jobs use
  DevBuf<SceneView> batch_views[3];
  DevBuf<BatchItem> batch_items[3];
  cudaStream_t batch_stream[4] = {};
  cudaEvent_t batch_event[4] = {};
};

constexpr int kBatchStreams = 4;

namespace {

int check_ctx(mrt_ctx* c) {
  if (!c) return set_err(MRT_ERR_INVALID, "null context");
  cudaError_t e = cudaSetDevice(c->device);
  if (e != cudaSuccess) return set_err(MRT_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return MRT_OK;
}

// init_viewport (viewport.c:38-87) in double, stored to float.
void set_viewport(SceneView& v, const mrt_camera& cam, int W, int H) {
  const double focus = cam.focus_dist == 0 ? 1.0 : cam.focus_dist;
  const V3 dir = unitv(v3(cam.orientation));
  const V3 pos = v3(cam.position);
  const float vw = (float)(2.0 * std::tan(cam.fov * (kPiD / 180.0) / 2.0) * focus);
  const float vh = (float)(vw / ((double)W / (double)H));
  V3 up = {0, 1, 0};
  if (std::fabs(dir.y) > 0.999) up = {1, 0, 0};
  const V3 u = unitv(cross(up, mul(dir, -1.0)));
  const V3 vu = mul(u, vw);
  const V3 vv = mul(cross(dir, u), vh);
  const V3 pdu = dv(vu, W), pdv = dv(vv, H);
  const V3 upper = sub(sub(add(pos, mul(dir, focus)), dv(vu, 2)), dv(vv, 2));
  const V3 p00 = add(upper, mul(add(pdu, pdv), 0.5));
  const double rad = focus * std::tan(cam.defocus_angle * kPiD / 360);
  put3(v.cam, pos);
  put3(v.pixel00, p00);
  put3(v.pdu, pdu);
  put3(v.pdv, pdv);
  put3(v.defocus_u, mul(u, rad));
  put3(v.defocus_v, mul(cross(dir, u), rad));
  v.defocus_angle = (float)cam.defocus_angle;
}

void set_ambient(SceneView& v, const mrt_ambient& a, bool has_tex) {
  for (int k = 0; k < 3; ++k) v.amb_const[k] = (float)(a.color[k] / 255.0 * a.ratio);
  const double exposure = (double)a.hdr_exposure + a.ratio - 1;
  v.env_exposure_zero = exposure == 0;
  v.env_scale_exp = powf(2.0f, (float)exposure);
  v.env_inv_gamma = a.hdr_gamma == 1.0f || a.hdr_gamma == 0.0f ? 1.0f : (float)(1.0 / a.hdr_gamma);
  v.has_env = has_tex;
}

uint32_t pack_color(const uint8_t* c) {
  return (uint32_t)c[0] | ((uint32_t)c[1] << 8) | ((uint32_t)c[2] << 16);
}

// Vose's alias method on the outcome probabilities (normalised here).
void build_alias(const std::vector<double>& p, std::vector<float2>& out) {
  const size_t n = p.size();
  out.assign(n, make_float2(1.0f, 0.0f));
  double total = 0;
  for (double x : p) total += x;
  if (total <= 0) return;
  std::vector<double> q(n);
  std::vector<uint32_t> small, large;
  small.reserve(n);
  large.reserve(n);
  for (size_t i = 0; i < n; ++i) {
    q[i] = p[i] / total * (double)n;
    (q[i] < 1.0 ? small : large).push_back((uint32_t)i);
  }
  while (!small.empty() && !large.empty()) {
    uint32_t s = small.back(); small.pop_back();
    uint32_t l = large.back();
    out[s] = make_float2((float)q[s], int_bits_as_float((int)l));
    q[l] = (q[l] + q[s]) - 1.0;
    if (q[l] < 1.0) { large.pop_back(); small.push_back(l); }
  }
  for (uint32_t l : large) out[l] = make_float2(1.0f, int_bits_as_float((int)l));
  for (uint32_t s : small) out[s] = make_float2(1.0f, int_bits_as_float((int)s));
}

// Per-outcome records of the two-step sampler, with the reference's double
// arithmetic: direction of calc_inverse_transform_sampling_dir (get_dir.c:29-41,
// float theta/phi), pdf_joint at the reference's index (material_default.c:57-59)
// and the unclamped sky radiance get_background_color returns for that
// direction (background.c:15-70, get_hdr_value.c:43-68). The sampled
// directions sit exactly on texel boundaries, so the texel choice has to come
// from the same double-precision libm calls as the reference.
void env_records(const mrt_ambient& a, const std::vector<float>& pdf, const std::vector<float>& cm,
                 const std::vector<float>& cc, std::vector<float4>& r0, std::vector<float4>& r1) {
  const int W = a.hdr_width, H = a.hdr_height;
  const size_t no = (size_t)(H - 1) * W;
  r0.assign(no, make_float4(0.f, 1.f, 0.f, 0.f));
  r1.assign(no, make_float4(0.f, 0.f, 0.f, 0.f));
  const double exposure = (double)a.hdr_exposure + a.ratio - 1;
  const double gcorr = 1.0 / a.hdr_gamma;
  auto work = [&](int y0, int y1) {
    for (int iy = y0; iy < y1; ++iy) {
      const double v = (double)cm[iy];
      const double A = v * (H - 1) * W;
      const double j0 = std::floor(A);
      for (int d = 0; d < W; ++d) {
        const long long j = (long long)j0 + d;
        if (j < 0 || j >= (long long)W * H) continue;
        const double u = (double)cc[j];
        const float theta = (float)((v - 0.5) * kPiD);
        const float phi = (float)((0.5 - u) * 2 * kPiD);
        // C's cos/sin on the float values (the double overloads, as the reference calls them)
        const double th = (double)theta, ph = (double)phi;
        V3 dir = {std::cos(th) * std::cos(ph), std::sin(th), std::cos(th) * std::sin(ph)};
        const long long pi = (long long)(v * (H - 1) * W + u * (W - 1));
        const float pd = (pi >= 0 && pi < (long long)W * H) ? pdf[pi] : 0.0f;
        const size_t k = (size_t)iy * W + d;
        r0[k] = make_float4((float)dir.x, (float)dir.y, (float)dir.z, pd);
        const V3 un = unitv(dir);
        const double vv = 0.5 + std::asin(un.y) / kPiD;
        const double uu = 0.5 - std::atan2(un.z, un.x) / (2.0 * kPiD);
        int x = (int)(uu * (W - 1)), yy = (int)(vv * (H - 1));
        x = std::min(std::max(x, 0), W - 1);
        yy = std::min(std::max(yy, 0), H - 1);
        const uint8_t* px = a.hdr_rgbe + 4 * ((size_t)yy * W + x);
        double scale = std::ldexp(1.0, px[3] - 128);
        if (exposure != 0) scale *= powf(2.0f, (float)exposure);
        double c3[3] = {px[0] * scale / 255.0, px[1] * scale / 255.0, px[2] * scale / 255.0};
        if (a.hdr_gamma != 1.0f)
          for (double& q : c3) q = std::pow(q, gcorr);
        r1[k] = make_float4((float)c3[0], (float)c3[1], (float)c3[2], 0.f);
      }
    }
  };
  const int nt = std::max(1, std::min((int)std::thread::hardware_concurrency(), 32));
  std::vector<std::thread> pool;
  const int rows = H - 1;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back(work, rows * t / nt, rows * (t + 1) / nt);
  for (auto& th : pool) th.join();
}

}  // namespace

// ------------------------------------------------------------------ C-ABI

extern "C" {

const char* mrt_last_error(void) { return g_err.c_str(); }
int mrt_version(void) { return MRT_ABI_VERSION; }

int mrt_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

mrt_ctx* mrt_create(int device, int width, int height) {
  if (width <= 0 || height <= 0 || (int64_t)width * height > (1ll << 30)) {
    set_err(MRT_ERR_INVALID, "invalid render size %dx%d", width, height);
    return nullptr;
  }
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    set_err(MRT_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    return nullptr;
  }
  if (device < 0 || device >= n) {
    set_err(MRT_ERR_INVALID, "device %d out of range (%d devices)", device, n);
    return nullptr;
  }
  mrt_ctx* c = new mrt_ctx();
  c->device = device;
  c->W = width;
  c->H = height;
  auto fail = [&](cudaError_t err, const char* what) -> mrt_ctx* {
    set_err(err == cudaErrorMemoryAllocation ? MRT_ERR_OOM : MRT_ERR_CUDA, "%s: %s", what,
            cudaGetErrorString(err));
    mrt_destroy(c);
    return nullptr;
  };
  if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return fail(e, "cudaStreamCreate");
  if ((e = cudaEventCreate(&c->ev0)) != cudaSuccess) return fail(e, "cudaEventCreate");
  if ((e = cudaEventCreate(&c->ev1)) != cudaSuccess) return fail(e, "cudaEventCreate");
  const size_t np = (size_t)width * height;
  if ((e = c->accum.alloc(np)) != cudaSuccess) return fail(e, "accumulator");
  if ((e = c->depth.alloc(np)) != cudaSuccess) return fail(e, "depth buffer");
  if ((e = c->status.alloc(1)) != cudaSuccess) return fail(e, "status word");
  if ((e = c->counters.alloc(8)) != cudaSuccess) return fail(e, "counters");
  // read-back staging, sized with the frame: allocated here, before any
  // scene memory, so that mrt_read_accum / mrt_accumulate_double allocate
  // nothing (a first pinned allocation later, with gigabytes of wavefront
  // state resident, measured 150-180 ms)
  if ((e = c->rgb_dev.alloc(3 * np)) != cudaSuccess) return fail(e, "read-back buffer");
  if ((e = cudaMallocHost(&c->rgb_host, 3 * np * sizeof(float))) != cudaSuccess)
    return fail(e, "pinned read-back buffer");
  c->rgb_host_n = 3 * np;
  cudaMemsetAsync(c->accum.p, 0, c->accum.bytes(), c->stream);
  cudaMemsetAsync(c->depth.p, 0, c->depth.bytes(), c->stream);
  cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream);
  cudaMemsetAsync(c->counters.p, 0, c->counters.bytes(), c->stream);
  if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess) return fail(e, "init");
  c->view.width = width;
  c->view.height = height;
  return c;
}

void mrt_destroy(mrt_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  c->accum.release(); c->depth.release(); c->status.release(); c->counters.release();
  c->nodes.release(); c->wnodes.release(); c->geom.release(); c->shade.release(); c->meta.release();
  c->planes.release(); c->mats.release(); c->lights.release(); c->point_lights.release();
  c->rgbe.release(); c->pdf_joint.release(); c->cdf_m.release(); c->cdf_c.release();
  c->alias.release(); c->env_rec0.release(); c->env_rec1.release();
  c->ph_pos.release(); c->ph_pow.release(); c->ph_pos_raw.release(); c->ph_pow_raw.release();
  c->ph_nodes.release(); c->ph_count.release();
  c->mat_tex.release(); c->texs.release(); c->texels.release(); c->rgb_dev.release();
  if (c->rgb_host) cudaFreeHost(c->rgb_host);
  wf_destroy(c->wf);
  nccl_comm_destroy(c->comm);
  c->comm_count.release();
  if (c->diff) { c->diff->release(); delete c->diff; }
  for (int k = 0; k < 3; ++k) { c->batch_views[k].release(); c->batch_items[k].release(); }
  for (int k = 0; k < kBatchStreams; ++k) {
    if (c->batch_stream[k]) cudaStreamDestroy(c->batch_stream[k]);
    if (c->batch_event[k]) cudaEventDestroy(c->batch_event[k]);
  }
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

}  // extern "C"

// ------------------------------------------------------- photon map build

// Photon map over the emitted photons: Morton order + linear BVH.
static int build_photon_map(mrt_ctx* c) {
  SceneView& v = c->view;
  const uint32_t n = (uint32_t)c->n_photons;
  CK(c->ph_pos.alloc(std::max<size_t>(n, 1)));
  CK(c->ph_pow.alloc(std::max<size_t>(n, 1)));
  CK(c->ph_nodes.alloc(4 * std::max<size_t>(n > 1 ? n - 1 : 1, 1)));
  PhotonTree T{};
  T.pos_in = c->ph_pos_raw.p;
  T.pow_in = c->ph_pow_raw.p;
  T.n = n;
  T.pos_out = c->ph_pos.p;
  T.pow_out = c->ph_pow.p;
  T.nodes = c->ph_nodes.p;
  CK(launch_photon_tree(T, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  v.photon_pos = c->ph_pos.p;
  v.photon_pow = c->ph_pow.p;
  v.photon_nodes = c->ph_nodes.p;
  v.n_photons = (int)n;
  return MRT_OK;
}

// Emits the photons of `pass` and rebuilds the photon map (caustic_manager.c:83).
static int emit_photons(mrt_ctx* c, uint32_t pass) {
  SceneView& v = c->view;
  const uint64_t cap = c->photons_per_light * (uint64_t)c->n_point_lights;
  v.caustic = 0;   // emission traces without gathering
  if (cap == 0) {
    c->n_photons = 0;
    v.n_photons = 0;
    return MRT_OK;
  }
  if (c->ph_pos_raw.n < cap) {
    CK(c->ph_pos_raw.alloc(cap));
    CK(c->ph_pow_raw.alloc(cap));
  }
  if (!c->ph_count.p) CK(c->ph_count.alloc(1));
  CK(cudaMemsetAsync(c->ph_count.p, 0, sizeof(unsigned), c->stream));
  PhotonEmit E{};
  E.seed = 0x5eed5eedULL;
  E.pass = pass;
  E.per_light = c->photons_per_light;
  E.n_point_lights = c->n_point_lights;
  E.light_index = c->point_lights.p;
  E.pos = c->ph_pos_raw.p;
  E.pow = c->ph_pow_raw.p;
  E.count = c->ph_count.p;
  E.capacity = cap;
  CK(launch_photon_emit(v, E, c->status.p, c->stream));
  unsigned cnt = 0;
  CK(cudaMemcpyAsync(&cnt, c->ph_count.p, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->n_photons = std::min<uint64_t>(cnt, cap);
  int rc = build_photon_map(c);
  if (rc != MRT_OK) return rc;
  v.caustic = 1;
  return MRT_OK;
}

// ------------------------------------------------------------ scene build

extern "C" int mrt_scene_build(mrt_ctx* c, const mrt_scene_desc* d) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!d) return set_err(MRT_ERR_INVALID, "null scene");
  if (d->abi_version != MRT_ABI_VERSION)
    return set_err(MRT_ERR_INVALID, "scene abi_version %u != %d", d->abi_version, MRT_ABI_VERSION);
  if (d->render_width != c->W || d->render_height != c->H)
    return set_err(MRT_ERR_INVALID, "scene size %dx%d does not match the context %dx%d",
                   d->render_width, d->render_height, c->W, c->H);
  if (d->n_materials < 0 || d->n_spheres < 0 || d->n_planes < 0 || d->n_meshes < 0 || d->n_lights < 0 ||
      d->n_cylinders < 0 || d->n_cones < 0 || d->n_hyperboloids < 0)
    return set_err(MRT_ERR_INVALID, "negative element count");
  if ((d->n_materials && !d->materials) || (d->n_spheres && !d->spheres) ||
      (d->n_planes && !d->planes) || (d->n_meshes && !d->meshes) || (d->n_lights && !d->lights) ||
      (d->n_cylinders && !d->cylinders) || (d->n_cones && !d->cones) ||
      (d->n_hyperboloids && !d->hyperboloids))
    return set_err(MRT_ERR_INVALID, "null element array with a non-zero count");
  if (d->n_textures < 0 || (d->n_textures && !d->textures))
    return set_err(MRT_ERR_INVALID, "bad texture array");
  for (int i = 0; i < d->n_textures; ++i) {
    const mrt_texture& t = d->textures[i];
    if (t.type < MRT_TEX_IMAGE || t.type > MRT_TEX_CHECKER_GLOBAL)
      return set_err(MRT_ERR_INVALID, "texture %d: unknown type %d", i, t.type);
    if (t.rgba && (uint64_t)t.width * t.height > (1ull << 28))
      return set_err(MRT_ERR_INVALID, "texture %d: %ux%u texels is too large", i, t.width, t.height);
    if (!std::isfinite(t.checker_scale))
      return set_err(MRT_ERR_INVALID, "texture %d: checker scale is not finite", i);
  }
  for (int i = 0; i < d->n_materials; ++i) {
    const int32_t* tx = &d->materials[i].color_tex;   // color_tex .. normal_tex
    for (int k = 0; k < TS_COUNT; ++k)
      if (tx[k] < 0 || tx[k] > d->n_textures)
        return set_err(MRT_ERR_INVALID, "material %d: texture slot %d names texture %d of %d", i, k, tx[k],
                       d->n_textures);
  }
  c->has_scene = false;
  if (c->diff) {
    cudaStreamSynchronize(c->stream);
    c->diff->release();
    delete c->diff;
    c->diff = nullptr;
  }
  SceneView v{};
  v.width = c->W;
  v.height = c->H;
  v.max_bounces = d->max_bounces;
  v.one_sided = d->triangle_one_sided ? 1 : 0;
  v.ior_all = (float)d->ior_all;
  cudaStream_t st = c->stream;

  // materials (t_mat after set_values_mat)
  std::vector<MaterialD> mats(std::max(1, d->n_materials));
  for (int i = 0; i < d->n_materials; ++i) {
    const mrt_material& m = d->materials[i];
    MaterialD& o = mats[i];
    for (int k = 0; k < 3; ++k) {
      o.color[k] = (float)(m.color[k] / 255.0);
      o.emission[k] = (float)(m.emission_color[k] / 255.0);
    }
    auto clamp01 = [](double x) { return x < 0 ? 0.0 : (x > 1 ? 1.0 : x); };
    const double rough = clamp01(m.roughness);
    o.metallic = (float)clamp01(m.metallic);
    o.roughness = (float)rough;
    o.ior = (float)m.ior;
    o.transmission = (float)m.transmission;
    o.ao = (float)m.ao;
    o.emission_strength = (float)m.emission_strength;
    o.f0 = powf((float)((m.ior - 1) / (m.ior + 1)), 2.0f);
    o.alpha4 = (float)((rough * rough) * (rough * rough));
  }

  // primitives in flat-id order: spheres, cylinders, cones, hyperboloids,
  // triangles; double boxes -> float
  size_t n_tris = 0;
  for (int i = 0; i < d->n_meshes; ++i) {
    const mrt_mesh& me = d->meshes[i];
    if (me.n_triangles && (!me.positions || !me.normals))
      return set_err(MRT_ERR_INVALID, "mesh %d has no positions or normals", i);
    if (me.indices)
      for (size_t k = 0; k < 3 * (size_t)me.n_triangles; ++k)
        if (me.indices[k] >= me.n_vertices)
          return set_err(MRT_ERR_INVALID, "mesh %d index %u out of range", i, me.indices[k]);
    if (!me.indices && (uint64_t)me.n_vertices < 3ull * me.n_triangles)
      return set_err(MRT_ERR_INVALID, "mesh %d has too few vertices for implicit indices", i);
    n_tris += me.n_triangles;
  }
  const size_t q_cyl = (size_t)d->n_spheres, q_cone = q_cyl + d->n_cylinders;
  const size_t q_hyp = q_cone + d->n_cones, tri_base = q_hyp + d->n_hyperboloids;
  const size_t n_prims = tri_base + n_tris;
  std::vector<PrimBox> boxes(n_prims);
  // double bounds and split positions for the reference-topology tree
  const bool ref_tree = c->bvh_mode == MRT_BVH_REFERENCE;
  std::vector<RefPrim> refp(ref_tree ? n_prims : 0);
  auto set_box = [&](size_t idx, const double* mn, const double* mx, const double* pos) {
    prim_box_from_double(boxes[idx], mn, mx);
    if (!ref_tree) return;
    for (int k = 0; k < 3; ++k) { refp[idx].mn[k] = mn[k]; refp[idx].mx[k] = mx[k]; refp[idx].pos[k] = pos[k]; }
  };
  struct TriRef { const mrt_mesh* m; uint32_t t; };
  std::vector<TriRef> tris;
  tris.reserve(n_tris);
  for (int i = 0; i < d->n_spheres; ++i) {
    const mrt_sphere& s = d->spheres[i];
    if (!(s.radius >= 0) || !std::isfinite(s.center[0]) || !std::isfinite(s.center[1]) ||
        !std::isfinite(s.center[2]))
      return set_err(MRT_ERR_INVALID, "sphere %d is not finite", i);
    double mn[3], mx[3];
    const double r = (s.radius * 2.0) * 0.5;
    for (int k = 0; k < 3; ++k) { mn[k] = s.center[k] - r; mx[k] = s.center[k] + r; }
    set_box(i, mn, mx, s.center);
  }
  // quadric bounds as bvh_obj_bounds.c computes them (axis-aligned extents of
  // the end discs, :41-96); a zero orientation takes the default the hit
  // functions give it (+y for cylinders and cones, +z for hyperboloids)
  auto finite3 = [](const double* q) { return std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]); };
  auto axis_of = [](const double* o, double dz, V3& axis) {
    V3 a = v3(o);
    if (a.x == 0 && a.y == 0 && a.z == 0) a = dz ? V3{0, 0, 1} : V3{0, 1, 0};
    axis = unitv(a);
  };
  auto disc_box = [&](size_t idx, const V3& p0, const V3& p1, const V3& a, double r, const double* pos) {
    const double e[3] = {r * std::sqrt(std::max(0.0, 1.0 - a.x * a.x)), r * std::sqrt(std::max(0.0, 1.0 - a.y * a.y)),
                         r * std::sqrt(std::max(0.0, 1.0 - a.z * a.z))};
    const double lo[3] = {std::min(p0.x, p1.x), std::min(p0.y, p1.y), std::min(p0.z, p1.z)};
    const double hi[3] = {std::max(p0.x, p1.x), std::max(p0.y, p1.y), std::max(p0.z, p1.z)};
    double mn[3], mx[3];
    for (int k = 0; k < 3; ++k) { mn[k] = lo[k] - e[k]; mx[k] = hi[k] + e[k]; }
    set_box(idx, mn, mx, pos);
  };
  for (int i = 0; i < d->n_cylinders; ++i) {
    const mrt_cylinder& q = d->cylinders[i];
    if (!finite3(q.position) || !finite3(q.orientation) || !(q.diameter >= 0) || !(q.height >= 0) ||
        !std::isfinite(q.diameter) || !std::isfinite(q.height))
      return set_err(MRT_ERR_INVALID, "cylinder %d is not finite or has a negative size", i);
    V3 a;
    axis_of(q.orientation, 0, a);
    const V3 c = v3(q.position), h = mul(a, q.height * 0.5);
    disc_box(q_cyl + i, sub(c, h), add(c, h), a, q.diameter * 0.5, q.position);
  }
  for (int i = 0; i < d->n_cones; ++i) {
    const mrt_cone& q = d->cones[i];
    if (!finite3(q.position) || !finite3(q.orientation) || !(q.diameter >= 0) || !(q.height > 0) ||
        !std::isfinite(q.diameter) || !std::isfinite(q.height))
      return set_err(MRT_ERR_INVALID, "cone %d is not finite or has a non-positive height", i);
    V3 a;
    axis_of(q.orientation, 0, a);
    const V3 c = v3(q.position);
    disc_box(q_cone + i, c, add(c, mul(a, q.height)), a, q.diameter * 0.5, q.position);
  }
  for (int i = 0; i < d->n_hyperboloids; ++i) {
    const mrt_hyperboloid& q = d->hyperboloids[i];
    if (!finite3(q.position) || !finite3(q.orientation) || !std::isfinite(q.a) || !std::isfinite(q.b) ||
        !std::isfinite(q.c) || !std::isfinite(q.shape) || !(q.height >= 0) || !std::isfinite(q.height) ||
        q.a == 0 || q.b == 0 || q.c == 0)
      return set_err(MRT_ERR_INVALID, "hyperboloid %d is not finite or has a zero semi-axis", i);
    V3 a = v3(q.orientation);
    a = (a.x * a.x + a.y * a.y + a.z * a.z) < 1e-6 ? V3{0, 0, 1} : unitv(a);
    const V3 c = v3(q.position), h = mul(a, q.height * 0.5);
    const double hh = q.height * 0.5;
    const double rmax = std::max(std::fabs(q.a), std::fabs(q.b)) *
                        std::sqrt(std::max(0.0, q.shape + (hh * hh) / (q.c * q.c)));
    disc_box(q_hyp + i, sub(c, h), add(c, h), a, rmax, q.position);
  }
  {
    size_t p = tri_base;
    for (int i = 0; i < d->n_meshes; ++i) {
      const mrt_mesh& me = d->meshes[i];
      for (uint32_t t = 0; t < me.n_triangles; ++t, ++p) {
        double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        double sum[3] = {0, 0, 0};      // (v0 + v1) + v2, the centre's order of additions
        for (int cidx = 0; cidx < 3; ++cidx) {
          uint32_t vi = me.indices ? me.indices[3 * (size_t)t + cidx] : 3 * t + cidx;
          const double* q = me.positions + 3 * (size_t)vi;
          for (int k = 0; k < 3; ++k) {
            if (!std::isfinite(q[k]))
              return set_err(MRT_ERR_INVALID, "mesh %d triangle %u has a non-finite vertex", i, t);
            mn[k] = std::min(mn[k], q[k]);
            mx[k] = std::max(mx[k], q[k]);
            sum[k] += q[k];
          }
        }
        // triangle centre as the loaders compute it (obj_finilizer.c:54)
        const double centre[3] = {sum[0] / 3.0, sum[1] / 3.0, sum[2] / 3.0};
        set_box(p, mn, mx, centre);
        tris.push_back({&me, t});
      }
    }
  }
  BvhResult bvh;
  std::string err;
  std::vector<double> dboxes;
  // the wide traversal is compiled into the SceneView kernels only
  bool has_quadrics_or_textures = (d->n_cylinders + d->n_cones + d->n_hyperboloids) > 0;
  for (int i = 0; i < d->n_materials && !has_quadrics_or_textures; ++i) {
    const mrt_material& m = d->materials[i];
    has_quadrics_or_textures = m.color_tex || m.metallic_tex || m.roughness_tex || m.transmission_tex || m.ao_tex ||
                               m.emission_strength_tex || m.emission_color_tex || m.normal_tex;
  }
  if (ref_tree) {
    std::vector<uint32_t> list(n_prims);
    if (!c->bvh_list.empty()) {
      if (c->bvh_list.size() != n_prims)
        return set_err(MRT_ERR_INVALID, "BVH options: object list of %zu entries for %zu primitives",
                       c->bvh_list.size(), n_prims);
      std::vector<char> seen(n_prims, 0);
      for (size_t i = 0; i < n_prims; ++i) {
        const int32_t f = c->bvh_list[i];
        if (f < 0 || (size_t)f >= n_prims || seen[f])
          return set_err(MRT_ERR_INVALID, "BVH options: object list entry %zu (%d) is not a permutation", i, f);
        seen[f] = 1;
        list[i] = (uint32_t)f;
      }
    } else {
      for (size_t i = 0; i < n_prims; ++i) list[i] = (uint32_t)i;
    }
    if (!c->bvh_pos.empty()) {
      if (c->bvh_pos.size() != 3 * n_prims)
        return set_err(MRT_ERR_INVALID, "BVH options: %zu positions for %zu primitives", c->bvh_pos.size() / 3, n_prims);
      for (size_t i = 0; i < n_prims; ++i)
        for (int k = 0; k < 3; ++k) refp[i].pos[k] = c->bvh_pos[3 * i + k];
    }
    if (!build_bvh_reference(refp, list, bvh, dboxes, err))
      return set_err(MRT_ERR_INVALID, "BVH: %s", err.c_str());
  } else if (c->bvh_mode != MRT_BVH_WIDE || has_quadrics_or_textures) {
    if (!build_bvh(boxes, bvh, err)) return set_err(MRT_ERR_INVALID, "BVH: %s", err.c_str());
  } else if (!build_bvh_wide(boxes, bvh, err)) {
    // a tree deeper than the wide stack, or a box beyond the quantisation
    // range: the binary tree instead
    err.clear();
    if (!build_bvh(boxes, bvh, err)) return set_err(MRT_ERR_INVALID, "BVH: %s", err.c_str());
  } else if (!check_bvh_wide(bvh, boxes, err)) {
    return set_err(MRT_ERR_INVALID, "BVH: %s", err.c_str());
  }
  c->bvh_depth = bvh.max_depth;
  c->leaf_order = bvh.order;

  // leaf-order geometry, metadata and shading records
  std::vector<float4> geom(3 * std::max<size_t>(n_prims, 1));
  std::vector<int4> meta(std::max<size_t>(n_prims, 1));
  std::vector<float4> shade(4 * std::max<size_t>(n_prims, 1));
  auto mat_or = [&](int32_t m) { return (m >= 0 && m < d->n_materials) ? m : -1; };
  for (size_t k = 0; k < n_prims; ++k) {
    const uint32_t src = bvh.order[k];
    if (src >= q_cyl && src < tri_base) {
      // quadric records: (position, type) (orientation as given, radius or a) (...)
      const float f0 = 0.f;
      if (src < q_cone) {
        const mrt_cylinder& q = d->cylinders[src - q_cyl];
        V3 o = v3(q.orientation);
        if (o.x == 0 && o.y == 0 && o.z == 0) o = V3{0, 1, 0};
        geom[3 * k] = make_float4((float)q.position[0], (float)q.position[1], (float)q.position[2],
                                  int_bits_as_float(PRIM_CYL));
        geom[3 * k + 1] = make_float4((float)o.x, (float)o.y, (float)o.z, (float)(q.diameter * 0.5));
        geom[3 * k + 2] = make_float4((float)q.height, int_bits_as_float(mat_or(q.material_top)),
                                      int_bits_as_float(mat_or(q.material_bot)), f0);
        meta[k] = make_int4((int)src, q.material < d->n_materials ? q.material : -1, PRIM_CYL,
                            (int)pack_color(q.color));
      } else if (src < q_hyp) {
        const mrt_cone& q = d->cones[src - q_cone];
        V3 o = v3(q.orientation);
        if (o.x == 0 && o.y == 0 && o.z == 0) o = V3{0, 1, 0};
        geom[3 * k] = make_float4((float)q.position[0], (float)q.position[1], (float)q.position[2],
                                  int_bits_as_float(PRIM_CONE));
        geom[3 * k + 1] = make_float4((float)o.x, (float)o.y, (float)o.z, (float)(q.diameter * 0.5));
        geom[3 * k + 2] = make_float4((float)q.height, int_bits_as_float(mat_or(q.material_top)), f0, f0);
        meta[k] = make_int4((int)src, q.material < d->n_materials ? q.material : -1, PRIM_CONE,
                            (int)pack_color(q.color));
      } else {
        const mrt_hyperboloid& q = d->hyperboloids[src - q_hyp];
        V3 o = v3(q.orientation);
        if (o.x * o.x + o.y * o.y + o.z * o.z < 1e-6) o = V3{0, 0, 1};
        geom[3 * k] = make_float4((float)q.position[0], (float)q.position[1], (float)q.position[2],
                                  int_bits_as_float(PRIM_HYP));
        geom[3 * k + 1] = make_float4((float)o.x, (float)o.y, (float)o.z, (float)q.a);
        geom[3 * k + 2] = make_float4((float)q.b, (float)q.c, (float)q.shape, (float)q.height);
        meta[k] = make_int4((int)src, q.material < d->n_materials ? q.material : -1, PRIM_HYP,
                            (int)pack_color(q.color));
      }
    } else if (src < (uint32_t)d->n_spheres) {
      const mrt_sphere& s = d->spheres[src];
      const double r = (s.radius * 2.0) * 0.5;
      geom[3 * k] = make_float4((float)s.center[0], (float)s.center[1], (float)s.center[2],
                                int_bits_as_float(PRIM_SPHERE));
      geom[3 * k + 1] = make_float4((float)r, (float)(r * r), 0.f, 0.f);
      geom[3 * k + 2] = make_float4(0.f, 0.f, 0.f, 0.f);
      const int mat = s.material < d->n_materials ? s.material : -1;
      meta[k] = make_int4((int)src, mat, PRIM_SPHERE, (int)pack_color(s.color));
    } else {
      const TriRef& tr = tris[src - tri_base];
      const mrt_mesh& me = *tr.m;
      uint32_t vi[3];
      for (int cidx = 0; cidx < 3; ++cidx)
        vi[cidx] = me.indices ? me.indices[3 * (size_t)tr.t + cidx] : 3 * tr.t + cidx;
      const double* p0 = me.positions + 3 * (size_t)vi[0];
      const double* p1 = me.positions + 3 * (size_t)vi[1];
      const double* p2 = me.positions + 3 * (size_t)vi[2];
      geom[3 * k] = make_float4((float)p0[0], (float)p0[1], (float)p0[2], int_bits_as_float(PRIM_TRI));
      geom[3 * k + 1] = make_float4((float)(p1[0] - p0[0]), (float)(p1[1] - p0[1]), (float)(p1[2] - p0[2]), 0.f);
      geom[3 * k + 2] = make_float4((float)(p2[0] - p0[0]), (float)(p2[1] - p0[1]), (float)(p2[2] - p0[2]), 0.f);
      float uvv[3][2] = {{0, 0}, {0, 0}, {0, 0}};
      for (int cidx = 0; cidx < 3; ++cidx) {
        const double* nn = me.normals + 3 * (size_t)vi[cidx];
        if (me.uvs) {
          uvv[cidx][0] = (float)me.uvs[2 * (size_t)vi[cidx]];
          uvv[cidx][1] = (float)me.uvs[2 * (size_t)vi[cidx] + 1];
        }
        shade[4 * k + cidx] = make_float4((float)nn[0], (float)nn[1], (float)nn[2], uvv[cidx][0]);
      }
      shade[4 * k + 3] = make_float4(uvv[0][1], uvv[1][1], uvv[2][1], 0.f);
      int32_t mat = me.tri_material ? me.tri_material[tr.t] : me.material;
      if (mat >= d->n_materials) mat = -1;
      meta[k] = make_int4((int)src, mat, PRIM_TRI, (int)pack_color(me.color));
    }
  }
  std::vector<PlaneD> planes(std::max(1, d->n_planes));
  const int plane_base = (int)n_prims;
  for (int i = 0; i < d->n_planes; ++i) {
    const mrt_plane& p = d->planes[i];
    V3 n = unitv(v3(p.normal));
    planes[i].pn = make_float4((float)p.point[0], (float)p.point[1], (float)p.point[2], 0.f);
    planes[i].nn = make_float4((float)n.x, (float)n.y, (float)n.z, 0.f);
    const int mat = p.material < d->n_materials ? p.material : -1;
    planes[i].meta = make_int4(plane_base + i, mat, 0, (int)pack_color(p.color));
  }
  std::vector<LightD> lights(std::max(1, d->n_lights));
  std::vector<int> point_lights;
  for (int i = 0; i < d->n_lights; ++i) {
    const mrt_light& L = d->lights[i];
    LightD& o = lights[i];
    V3 p = L.type == MRT_LIGHT_DIRECTIONAL ? unitv(v3(L.position)) : v3(L.position);
    put3(o.pos, p);
    double br = L.brightness;
    if (L.type == MRT_LIGHT_POINT && br < 0) br = 0;
    o.brightness = (float)br;
    for (int k = 0; k < 3; ++k) o.color[k] = (float)L.color[k];
    o.radius = L.radius;
    o.type = L.type;
    o.shadow_sample = L.shadow_sample;
    if (L.type == MRT_LIGHT_POINT) point_lights.push_back(i);
  }

  CK(c->nodes.upload(bvh.nodes.data(), bvh.nodes.size(), st));
  CK(c->wnodes.upload(bvh.wnodes.data(), bvh.wnodes.size(), st));
  CK(c->geom.upload(geom.data(), geom.size(), st));
  CK(c->meta.upload(meta.data(), meta.size(), st));
  CK(c->shade.upload(shade.data(), shade.size(), st));
  CK(c->planes.upload(planes.data(), planes.size(), st));
  CK(c->mats.upload(mats.data(), mats.size(), st));
  CK(c->lights.upload(lights.data(), lights.size(), st));
  // textures: RGBA8 images back to back, per-material slots
  {
    std::vector<TexD> texs(std::max(1, d->n_textures));
    std::vector<uchar4> texels;
    for (int i = 0; i < d->n_textures; ++i) {
      const mrt_texture& t = d->textures[i];
      TexD& o = texs[i];
      o = TexD{};
      o.type = t.type;
      o.scale = (float)t.checker_scale;
      for (int k = 0; k < 3; ++k) {
        o.c1[k] = (float)(t.c1[k] / 255.0);
        o.c2[k] = (float)(t.c2[k] / 255.0);
      }
      if (t.rgba && t.width && t.height) {
        o.w = (int)t.width;
        o.h = (int)t.height;
        o.offset = (uint32_t)texels.size();
        const size_t n = (size_t)t.width * t.height;
        texels.resize(texels.size() + n);
        std::memcpy(texels.data() + o.offset, t.rgba, 4 * n);
      }
    }
    if (texels.empty()) texels.push_back(uchar4{0, 0, 0, 0});
    std::vector<MatTexD> mt(std::max(1, d->n_materials));
    bool any = false;
    for (int i = 0; i < d->n_materials; ++i) {
      const mrt_material& m = d->materials[i];
      const int32_t* tx = &m.color_tex;
      MatTexD& o = mt[i];
      o = MatTexD{};
      for (int k = 0; k < TS_COUNT; ++k) {
        o.tex[k] = tx[k];
        o.any |= tx[k] != 0;
      }
      o.normal_intensity = (float)m.normal_intensity;
      o.uv_scale = (float)m.scale;
      if (o.tex[TS_COLOR]) {
        const TexD& t = texs[o.tex[TS_COLOR] - 1];
        if (t.type == MRT_TEX_IMAGE && t.w > 0)
          for (size_t q = 0; q < (size_t)t.w * t.h && !o.alpha; ++q) o.alpha = texels[t.offset + q].w < 255;
      }
      any = any || o.any;
    }
    CK(c->texs.upload(texs.data(), texs.size(), st));
    CK(c->texels.upload(texels.data(), texels.size(), st));
    CK(c->mat_tex.upload(mt.data(), mt.size(), st));
    v.texs = c->texs.p;
    v.texels = c->texels.p;
    v.mat_tex = c->mat_tex.p;
    v.has_textures = any ? 1 : 0;
  }
  CK(c->point_lights.upload(point_lights.data(), point_lights.size(), st));
  c->n_point_lights = (int)point_lights.size();
  v.nodes = c->nodes.p;
  v.geom = c->geom.p;
  v.meta = c->meta.p;
  v.shade = c->shade.p;
  v.planes = c->planes.p;
  v.mats = c->mats.p;
  v.lights = c->lights.p;
  v.n_nodes = (int)bvh.nodes.size();
  v.wnodes = bvh.wnodes.empty() ? nullptr : c->wnodes.p;
  v.n_wnodes = (int)bvh.wnodes.size();
  v.n_prims = (int)n_prims;
  v.n_planes = d->n_planes;
  v.n_mats = d->n_materials;
  v.n_lights = d->n_lights;
  v.has_bvh = n_prims > 0;
  v.has_quadrics = (d->n_cylinders + d->n_cones + d->n_hyperboloids) > 0;
  if (v.wnodes && (v.has_quadrics || v.has_textures))   // only the SceneView kernels traverse it
    return set_err(MRT_ERR_INVALID, "wide BVH built for a scene with quadrics or textures");
  v.root_leaf = bvh.root_leaf;
  v.left_first = ref_tree ? 1 : 0;
  v.ref_boxes = nullptr;
  c->ref_boxes.release();
  if (ref_tree && !dboxes.empty()) {
    CK(c->ref_boxes.upload(dboxes.data(), dboxes.size(), st));
    v.ref_boxes = c->ref_boxes.p;
  }
  set_viewport(v, d->camera, c->W, c->H);

  // sky and importance-sampling tables
  const mrt_ambient& a = d->ambient;
  const bool has_tex = a.hdr_rgbe && a.hdr_width > 0 && a.hdr_height > 0;
  set_ambient(v, a, has_tex);
  if (has_tex) {
    const int W = a.hdr_width, H = a.hdr_height;
    const size_t n = (size_t)W * H;
    std::vector<uint32_t> px(n);
    std::memcpy(px.data(), a.hdr_rgbe, n * 4);
    CK(c->rgbe.upload(px.data(), n, st));
    v.rgbe = c->rgbe.p;
    v.env_w = W;
    v.env_h = H;
    if (H >= 2 && W >= 2) {
      DevBuf<double> gray, raw, rowcdf, scal, cdfh, prob;
      CK(gray.alloc(n));
      CK(raw.alloc(H));
      CK(rowcdf.alloc(n));
      CK(scal.alloc(8));
      CK(cdfh.alloc(H));
      CK(c->pdf_joint.alloc(n));
      CK(c->cdf_m.alloc(H));
      CK(c->cdf_c.alloc(n));
      const size_t no = (size_t)(H - 1) * W;
      CK(prob.alloc(no));
      EnvBuild E{};
      E.rgbe = c->rgbe.p;
      E.W = W;
      E.H = H;
      E.exposure_zero = a.hdr_exposure == 0;
      E.exposure_scale = (double)powf(2.0f, a.hdr_exposure);
      E.gray = gray.p;
      E.raw = raw.p;
      E.row_cdf = rowcdf.p;
      E.scal = scal.p;
      E.cdf_h = cdfh.p;
      E.pdf_joint = c->pdf_joint.p;
      E.cdf_m_inv = c->cdf_m.p;
      E.cdf_c_inv = c->cdf_c.p;
      E.out_prob = prob.p;
      CK(launch_env_tables(E, st));
      std::vector<double> hp(no);
      std::vector<float> t_pdf(n), t_cm(H), t_cc(n);
      CK(cudaMemcpyAsync(hp.data(), prob.p, no * sizeof(double), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(t_pdf.data(), c->pdf_joint.p, n * sizeof(float), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(t_cm.data(), c->cdf_m.p, H * sizeof(float), cudaMemcpyDeviceToHost, st));
      CK(cudaMemcpyAsync(t_cc.data(), c->cdf_c.p, n * sizeof(float), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      std::vector<float2> al;
      build_alias(hp, al);
      std::vector<float4> r0, r1;
      env_records(a, t_pdf, t_cm, t_cc, r0, r1);
      CK(c->alias.upload(al.data(), al.size(), st));
      CK(c->env_rec0.upload(r0.data(), r0.size(), st));
      CK(c->env_rec1.upload(r1.data(), r1.size(), st));
      CK(cudaStreamSynchronize(st));
      gray.release(); raw.release(); rowcdf.release(); scal.release(); cdfh.release(); prob.release();
      v.alias = c->alias.p;
      v.env_rec0 = c->env_rec0.p;
      v.env_rec1 = c->env_rec1.p;
      v.n_env_outcomes = (int)no;
      v.pdf_joint = c->pdf_joint.p;
      v.cdf_m_inv = c->cdf_m.p;
      v.cdf_c_inv = c->cdf_c.p;
      v.env_nee = 1;
    }
  } else {
    c->rgbe.release();
  }

  // photon map
  c->caustic = d->caustic;
  c->view = v;
  c->n_photons = 0;
  if (d->caustic.enable) {
    if (d->caustic.knn <= 0 || d->caustic.knn > 32)
      return set_err(MRT_ERR_INVALID, "caustic k=%d outside [1,32]", d->caustic.knn);
    c->photons_per_light = d->caustic.photons_per_light;
    c->view.knn = d->caustic.knn;
    c->view.caustic_radius2 = (float)d->caustic.radius;
    c->view.inv_norm = (float)(1.0 / d->caustic.norm_factor);
    c->view.caustic_mode = d->caustic.mode;
    c->view.fixed_radius2 = (float)d->caustic.radius;
    if (d->caustic.mode == 1 && d->caustic.passes > 1 &&
        (d->caustic.spp_per_pass < 0 || !(d->caustic.shrink > 0.0 && d->caustic.shrink <= 1.0)))
      return set_err(MRT_ERR_INVALID, "progressive caustics need spp_per_pass >= 0 and shrink in (0, 1]");
    c->photon_pass = 0;
    int rc2 = emit_photons(c, 0);
    if (rc2) return rc2;
  }
  CK(cudaStreamSynchronize(st));
  c->scene_bytes = c->nodes.bytes() + c->wnodes.bytes() + c->geom.bytes() + c->meta.bytes() + c->shade.bytes() +
                   c->planes.bytes() + c->mats.bytes() + c->lights.bytes() + c->rgbe.bytes() +
                   c->pdf_joint.bytes() + c->cdf_m.bytes() + c->cdf_c.bytes() + c->alias.bytes() +
                   c->env_rec0.bytes() + c->env_rec1.bytes() + c->ph_pos.bytes() + c->ph_pow.bytes() + c->ph_nodes.bytes();
  c->has_scene = true;
  return MRT_OK;
}

extern "C" int mrt_set_camera(mrt_ctx* c, const mrt_camera* cam, double ior_all, double ambient_ratio) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!cam) return set_err(MRT_ERR_INVALID, "null camera");
  set_viewport(c->view, *cam, c->W, c->H);
  c->view.ior_all = (float)ior_all;
  (void)ambient_ratio;
  return MRT_OK;
}

// ---------------------------------------------------------------- render

// Progressive photon mapping (caustic mode 1, the configuration's extension
// of the reference's single kNN pass): sample s renders with photon pass
// min(s / spp_per_pass, passes - 1); pass q is emitted from its own streams
// and gathered within radius * shrink^(2q) (radius is compared against
// squared distances, so the gather radius shrinks by `shrink` per pass).
static int pass_of(const mrt_ctx* c, int64_t sample) {
  const mrt_caustic& k = c->caustic;
  if (!k.enable || k.mode != 1 || k.passes <= 1 || k.spp_per_pass <= 0) return 0;
  return (int)std::min<int64_t>(sample / k.spp_per_pass, k.passes - 1);
}

static int ensure_photon_pass(mrt_ctx* c, int q) {
  if (q == c->photon_pass) return MRT_OK;
  const double r2 = c->caustic.radius * std::pow(c->caustic.shrink, 2.0 * q);
  c->view.fixed_radius2 = (float)r2;
  const int rc = emit_photons(c, (uint32_t)q);
  if (rc) return rc;
  c->photon_pass = q;
  return MRT_OK;
}

static int read_status(mrt_ctx* c, int* out) {
  int s = 0;
  CK(cudaMemcpyAsync(&s, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  *out = s;
  return MRT_OK;
}


extern "C" int mrt_render(mrt_ctx* c, const mrt_render_params* p, mrt_render_stats* stats) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!p) return set_err(MRT_ERR_INVALID, "null params");
  if (!c->has_scene) return set_err(MRT_ERR_INVALID, "no scene: call mrt_scene_build first");
  if (p->spp < 0 || p->sample_base < 0) return set_err(MRT_ERR_INVALID, "negative spp / sample_base");
  if (p->render_mode < 0 || p->render_mode > 2) return set_err(MRT_ERR_INVALID, "render_mode %d", p->render_mode);
  if (p->form < 0 || p->form > 3) return set_err(MRT_ERR_INVALID, "form %d", p->form);
  if (p->offset && p->spp != 1) return set_err(MRT_ERR_INVALID, "explicit offset needs spp == 1");
  if (p->block_size && (p->block_size % 32 || p->block_size > 256))
    return set_err(MRT_ERR_INVALID, "block_size %d", p->block_size);
  if (p->env_sampler < 0 || p->env_sampler > 1) return set_err(MRT_ERR_INVALID, "env_sampler %d", p->env_sampler);
  if (p->render_mode == 0 && p->spp > 0 && pass_of(c, (int64_t)p->sample_base + p->spp - 1) > 0) {
    const int q0 = pass_of(c, p->sample_base), q1 = pass_of(c, (int64_t)p->sample_base + p->spp - 1);
    if (q0 != q1) {   // one call per photon pass
      mrt_render_stats total{};
      int64_t s = p->sample_base;
      const int64_t end = (int64_t)p->sample_base + p->spp;
      while (s < end) {
        const int q = pass_of(c, s);
        const int64_t seg_end = q == c->caustic.passes - 1
                                    ? end : std::min<int64_t>(end, (int64_t)(q + 1) * c->caustic.spp_per_pass);
        mrt_render_params sub = *p;
        sub.sample_base = (int32_t)s;
        sub.spp = (int32_t)(seg_end - s);
        mrt_render_stats st{};
        rc = mrt_render(c, &sub, &st);
        if (rc) return rc;
        total.ms += st.ms;
        total.paths += st.paths;
        total.segments += st.segments;
        total.shadow_rays += st.shadow_rays;
        total.kernel_launches += st.kernel_launches;
        total.status |= st.status;
        s = seg_end;
      }
      if (stats) *stats = total;
      return MRT_OK;
    }
  }
  if (p->render_mode == 0 && p->spp > 0) {
    rc = ensure_photon_pass(c, pass_of(c, p->sample_base));
    if (rc) return rc;
  }
  SceneView v = c->view;
  v.env_lookup = p->env_sampler;
  const uint64_t npix = (uint64_t)c->W * c->H;
  LaunchParams L{};
  L.seed = p->seed;
  L.max_bounces = p->max_bounces > 0 ? p->max_bounces : v.max_bounces;
  L.jitter = p->jitter;
  L.render_mode = p->render_mode;
  if (p->offset) { L.has_offset = 1; L.ox = (float)p->offset[0]; L.oy = (float)p->offset[1]; }
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(c->counters.p, 0, c->counters.bytes(), c->stream));
  if (p->render_mode == 1) CK(cudaMemsetAsync(c->depth.p, 0xff, c->depth.bytes(), c->stream));
  int launches = 0;
  CK(cudaEventRecord(c->ev0, c->stream));
  int form = p->form;
  const bool tuned = form == MRT_FORM_AUTO;
  if (tuned) form = c->auto_form;
  const int block_size = p->block_size ? p->block_size : (tuned ? c->auto_block : 0);
  const int queue_capacity = p->queue_capacity ? p->queue_capacity : (tuned ? c->auto_capacity : 0);
  const int sort_threshold = p->sort_threshold ? p->sort_threshold : (tuned ? c->auto_sort : 0);
  if (form == MRT_FORM_WAVEFRONT && p->render_mode == 0) {
    L.sample_base = (uint32_t)p->sample_base;
    if (!c->wf) c->wf = wf_create();
    const char* err = "";
    unsigned nl = 0;
    int r2 = wf_render(c->wf, v, L, p->spp, queue_capacity, sort_threshold,
                       p->use_graph || tuned ? 1 : 0, c->accum.p, c->status.p, c->stream, &nl, &err);
    if (r2) return set_err(r2, "wavefront: %s", err);
    launches += (int)nl;
  } else {
    // chunks of spp so a single launch stays well under a second
    const uint64_t max_paths = 1ull << 26;
    int spp_chunk = (int)std::max<uint64_t>(1, max_paths / std::max<uint64_t>(npix, 1));
    // the persistent, regenerating megakernel for path tracing; the plain
    // one-path-per-thread launch for the debug modes and when counting
    const bool regen = p->render_mode == 0 && form != MRT_FORM_MEGAKERNEL_PLAIN;
    for (int s = 0; s < p->spp; s += spp_chunk) {
      int k = std::min(spp_chunk, p->spp - s);
      L.sample_base = (uint32_t)(p->sample_base + s);
      L.n_paths = npix * (uint64_t)k;
      if (regen)
        CK(launch_megakernel_regen(v, L, c->accum.p, c->status.p, c->counters.p + 7, block_size,
                                   0, c->stream));
      else
        CK(launch_megakernel(v, L, c->accum.p, c->depth.p, c->status.p, stats ? c->counters.p : nullptr,
                             block_size, c->stream));
      launches++;
    }
  }
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  int status = 0;
  rc = read_status(c, &status);
  if (rc) return rc;
  if (p->render_mode != 1) c->accum_spp += p->spp;
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    unsigned long long cnt[8] = {};
    CK(cudaMemcpy(cnt, c->counters.p, sizeof(cnt), cudaMemcpyDeviceToHost));
    stats->ms = ms;
    stats->paths = npix * (uint64_t)p->spp;
    stats->segments = cnt[0];
    stats->shadow_rays = cnt[1];
    stats->kernel_launches = launches;
    stats->status = status;
  }
  if (status & ST_STACK) return set_err(MRT_ERR_STACK, "traversal stack overflow (status 0x%x)", status);
  if (status & ST_BUDGET) return set_err(MRT_ERR_BUDGET, "traversal iteration budget exhausted (status 0x%x)", status);
  if (status & ST_QUEUE) return set_err(MRT_ERR_QUEUE_OVERFLOW, "queue overflow (status 0x%x)", status);
  if (status & ST_ABORT) return set_err(MRT_ERR_ABORTED, "aborted (status 0x%x)", status);
  return MRT_OK;
}

extern "C" int mrt_render_batch(mrt_ctx** ctxs, const mrt_render_params* params, int32_t n,
                                mrt_render_stats* stats) {
  if (!ctxs || !params || n <= 0) return set_err(MRT_ERR_INVALID, "empty batch");
  for (int i = 0; i < n; ++i) {
    if (!ctxs[i]) return set_err(MRT_ERR_INVALID, "batch entry %d: null context", i);
    if (!ctxs[i]->has_scene) return set_err(MRT_ERR_INVALID, "batch entry %d: no scene", i);
    if (ctxs[i]->device != ctxs[0]->device)
      return set_err(MRT_ERR_INVALID, "batch entry %d is on device %d, not %d", i, ctxs[i]->device,
                     ctxs[0]->device);
    if (params[i].spp < 0 || params[i].sample_base < 0 || params[i].offset || params[i].render_mode != 0)
      return set_err(MRT_ERR_INVALID, "batch entry %d: spp / sample_base / offset / render_mode", i);
    if (params[i].form < 0 || params[i].form > 3) return set_err(MRT_ERR_INVALID, "batch entry %d: form", i);
    for (int j = 0; j < i; ++j)
      if (ctxs[j] == ctxs[i]) return set_err(MRT_ERR_INVALID, "batch entry %d repeats entry %d", i, j);
  }
  mrt_ctx* c0 = ctxs[0];
  int rc = check_ctx(c0);
  if (rc) return rc;
  if (params[0].block_size && (params[0].block_size % 32 || params[0].block_size > 256))
    return set_err(MRT_ERR_INVALID, "block_size %d", params[0].block_size);
  // each scene's form: its own, or its tuned choice (FORM_AUTO); textured
  // scenes render with the megakernel
  std::vector<int> form(n);
  std::vector<double> cost(n);
  for (int i = 0; i < n; ++i) {
    const mrt_ctx* c = ctxs[i];
    form[i] = params[i].form == MRT_FORM_AUTO ? c->auto_form : params[i].form;
    const double paths = (double)c->W * c->H * params[i].spp;
    const int depth = params[i].max_bounces > 0 ? params[i].max_bounces : c->view.max_bounces;
    cost[i] = paths * depth * std::log2(2.0 + c->view.n_prims);
  }
  cudaStream_t st = c0->stream;
  // other contexts' streams may still be writing their accumulators
  for (int i = 0; i < n; ++i)
    if (ctxs[i]->stream != st) CK(cudaStreamSynchronize(ctxs[i]->stream));
  for (int i = 0; i < n; ++i) CK(cudaMemsetAsync(ctxs[i]->status.p, 0, sizeof(int), st));
  // megakernel scenes: one persistent launch per view type (the scenes of
  // a launch share its kernel instantiation), longest first within it;
  // device arrays written before anything is launched
  struct Job { int kind; int scene; double cost; size_t m; uint64_t paths; };
  std::vector<Job> jobs;
  for (int kind = 0; kind < 3; ++kind) {
    std::vector<int> order;
    for (int i = 0; i < n; ++i) {
      const SceneView& v = ctxs[i]->view;
      const int k = v.has_textures ? 2 : (v.has_quadrics ? 1 : 0);
      if (form[i] != MRT_FORM_WAVEFRONT && k == kind && params[i].spp > 0) order.push_back(i);
    }
    if (order.empty()) continue;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    const size_t m = order.size();
    std::vector<SceneView> views(m);
    std::vector<BatchItem> items(m);
    uint64_t sub = 0;
    double group_cost = 0;
    for (size_t k = 0; k < m; ++k) {
      const int i = order[k];
      views[k] = ctxs[i]->view;
      views[k].env_lookup = params[i].env_sampler;
      BatchItem& it = items[k];
      it.start = sub;
      it.paths = (uint64_t)ctxs[i]->W * ctxs[i]->H * (uint64_t)params[i].spp;
      it.seed = params[i].seed;
      it.sample_base = (uint32_t)params[i].sample_base;
      it.view = (int)k;
      it.max_bounces = params[i].max_bounces > 0 ? params[i].max_bounces : ctxs[i]->view.max_bounces;
      it.jitter = params[i].jitter;
      it.accum = ctxs[i]->accum.p;
      sub += it.paths;
      group_cost += cost[i];
    }
    DevBuf<SceneView>& dv = c0->batch_views[kind];
    DevBuf<BatchItem>& di = c0->batch_items[kind];
    if (dv.n < m) CK(dv.alloc(m));
    if (di.n < m) CK(di.alloc(m));
    CK(cudaMemcpyAsync(dv.p, views.data(), sizeof(SceneView) * m, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(di.p, items.data(), sizeof(BatchItem) * m, cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    jobs.push_back({kind, -1, group_cost, m, sub});
  }
  for (int i = 0; i < n; ++i)
    if (form[i] == MRT_FORM_WAVEFRONT && params[i].spp > 0) jobs.push_back({-1, i, cost[i], 0, 0});
  // jobs (megakernel groups, wavefront scenes) on kBatchStreams streams,
  // longest first onto the least-loaded stream, forked from and joined back
  // into the first context's stream
  for (int k = 0; k < kBatchStreams; ++k) {
    if (!c0->batch_stream[k]) CK(cudaStreamCreateWithFlags(&c0->batch_stream[k], cudaStreamNonBlocking));
    if (!c0->batch_event[k]) CK(cudaEventCreateWithFlags(&c0->batch_event[k], cudaEventDisableTiming));
  }
  std::sort(jobs.begin(), jobs.end(), [](const Job& a, const Job& b) { return a.cost > b.cost; });
  std::vector<double> load(kBatchStreams, 0.0);
  unsigned launches = 0;
  uint64_t total = 0;
  CK(cudaEventRecord(c0->ev0, st));
  for (int k = 0; k < kBatchStreams; ++k) CK(cudaStreamWaitEvent(c0->batch_stream[k], c0->ev0, 0));
  for (const Job& j : jobs) {
    const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    load[k] += j.cost;
    cudaStream_t sk = c0->batch_stream[k];
    if (j.kind >= 0) {
      // each group its own work counter: groups may run at the same time
      CK(launch_megakernel_batch(c0->batch_views[j.kind].p, c0->batch_items[j.kind].p, (int)j.m, j.paths,
                                 c0->status.p, c0->counters.p + 5 + j.kind, params[0].block_size, j.kind, sk));
      launches++;
      total += j.paths;
      continue;
    }
    mrt_ctx* c = ctxs[j.scene];
    const mrt_render_params& p = params[j.scene];
    const bool tuned = p.form == MRT_FORM_AUTO;
    SceneView v = c->view;
    v.env_lookup = p.env_sampler;
    LaunchParams L{};
    L.seed = p.seed;
    L.max_bounces = p.max_bounces > 0 ? p.max_bounces : v.max_bounces;
    L.jitter = p.jitter;
    L.sample_base = (uint32_t)p.sample_base;
    if (!c->wf) c->wf = wf_create();
    const char* err = "";
    unsigned nl = 0;
    const int r2 = wf_render(c->wf, v, L, p.spp, p.queue_capacity ? p.queue_capacity : (tuned ? c->auto_capacity : 0),
                             p.sort_threshold ? p.sort_threshold : (tuned ? c->auto_sort : 0), 1, c->accum.p,
                             c->status.p, sk, &nl, &err);
    if (r2) {
      for (int q = 0; q < kBatchStreams; ++q) cudaStreamSynchronize(c0->batch_stream[q]);
      return set_err(r2, "batch entry %d, wavefront: %s", j.scene, err);
    }
    launches += nl;
    total += (uint64_t)c->W * c->H * (uint64_t)p.spp;
  }
  for (int k = 0; k < kBatchStreams; ++k) {
    CK(cudaEventRecord(c0->batch_event[k], c0->batch_stream[k]));
    CK(cudaStreamWaitEvent(st, c0->batch_event[k], 0));
  }
  CK(cudaEventRecord(c0->ev1, st));
  CK(cudaEventSynchronize(c0->ev1));
  int status = 0;
  for (int i = 0; i < n; ++i) {
    int s = 0;
    rc = read_status(ctxs[i], &s);
    if (rc) return rc;
    status |= s;
  }
  for (int i = 0; i < n; ++i) ctxs[i]->accum_spp += params[i].spp;
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c0->ev0, c0->ev1);
    std::memset(stats, 0, sizeof(*stats));
    stats->ms = ms;
    stats->paths = total;
    stats->kernel_launches = launches;
    stats->status = status;
  }
  if (status & ST_STACK) return set_err(MRT_ERR_STACK, "traversal stack overflow (status 0x%x)", status);
  if (status & ST_BUDGET) return set_err(MRT_ERR_BUDGET, "traversal budget exhausted (status 0x%x)", status);
  if (status & ST_QUEUE) return set_err(MRT_ERR_QUEUE_OVERFLOW, "queue overflow (status 0x%x)", status);
  return MRT_OK;
}

extern "C" int mrt_tune(mrt_ctx* c, int32_t spp, uint64_t seed, mrt_tune_result* out) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!out) return set_err(MRT_ERR_INVALID, "null result");
  if (!c->has_scene) return set_err(MRT_ERR_INVALID, "no scene");
  if (spp <= 0) return set_err(MRT_ERR_INVALID, "spp %d", spp);
  std::memset(out, 0, sizeof(*out));
  auto add = [&](int form, int block, int cap, int sort) {
    if (out->n < MRT_TUNE_MAX) out->entry[out->n++] = mrt_tune_entry{form, block, cap, sort, 0.0};
  };
  for (int b : {64, 128, 256}) add(MRT_FORM_MEGAKERNEL, b, 0, 0);
  for (int cap : {1 << 21, 1 << 23, 1 << 25})
      for (int sort : {1 << 30, 1 << 16}) add(MRT_FORM_WAVEFRONT, 0, cap, sort);
  int best = -1;
  for (int i = 0; i < out->n; ++i) {
    mrt_tune_entry& t = out->entry[i];
    mrt_render_params p{};
    p.spp = spp;
    p.seed = seed;
    p.form = t.form;
    p.block_size = t.block_size;
    p.queue_capacity = t.queue_capacity;
    p.sort_threshold = t.sort_threshold;
    p.use_graph = 1;
    mrt_render_stats st{};
    if (mrt_render(c, &p, &st) != MRT_OK) continue;           // warm-up / graph capture
    if (mrt_render(c, &p, &st) != MRT_OK || st.ms <= 0) continue;
    t.mpaths_s = (double)st.paths / st.ms / 1e3;
    if (best < 0 || t.mpaths_s > out->entry[best].mpaths_s) best = i;
  }
  mrt_clear(c);
  if (best < 0) return set_err(MRT_ERR_CUDA, "no candidate rendered: %s", g_err.c_str());
  out->best = best;
  c->auto_form = out->entry[best].form;
  c->auto_block = out->entry[best].block_size;
  c->auto_capacity = out->entry[best].queue_capacity;
  c->auto_sort = out->entry[best].sort_threshold;
  return MRT_OK;
}

extern "C" int mrt_clear(mrt_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  CK(cudaMemsetAsync(c->accum.p, 0, c->accum.bytes(), c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->accum_spp = 0;
  return MRT_OK;
}

// The accumulator as rgb floats in the context's pinned host buffer: one
// conversion kernel into the context's device buffer, one copy; both
// buffers are allocated by mrt_create (the checks below only guard).
static int fetch_rgb(mrt_ctx* c) {
  const size_t n3 = (size_t)c->W * c->H * 3;
  if (c->rgb_dev.n != n3) CK(c->rgb_dev.alloc(n3));
  if (c->rgb_host_n != n3) {
    if (c->rgb_host) cudaFreeHost(c->rgb_host);
    c->rgb_host = nullptr;
    c->rgb_host_n = 0;
    CK(cudaMallocHost(&c->rgb_host, n3 * sizeof(float)));
    c->rgb_host_n = n3;
  }
  CK(launch_accum_to_rgb(c->accum.p, c->rgb_dev.p, (int)(n3 / 3), c->stream));
  CK(cudaMemcpyAsync(c->rgb_host, c->rgb_dev.p, n3 * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return MRT_OK;
}

// f(begin, end) over [0, n) on up to 16 host threads (one for small n).
template <class F>
static void host_parallel(size_t n, F&& f) {
  const unsigned t = std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
  if (t == 1 || n < (size_t)1 << 20) {
    f((size_t)0, n);
    return;
  }
  std::vector<std::thread> th;
  const size_t chunk = (n + t - 1) / t;
  for (unsigned i = 0; i < t; ++i) {
    const size_t a = i * chunk, b = std::min(n, a + chunk);
    if (a < b) th.emplace_back([&f, a, b] { f(a, b); });
  }
  for (auto& x : th) x.join();
}

extern "C" int mrt_read_accum(mrt_ctx* c, float* rgb, int32_t* spp) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!rgb) return set_err(MRT_ERR_INVALID, "null output");
  if ((rc = fetch_rgb(c))) return rc;
  const float* src = c->rgb_host;
  host_parallel(c->rgb_host_n, [&](size_t a, size_t b) { std::memcpy(rgb + a, src + a, (b - a) * sizeof(float)); });
  if (spp) *spp = c->accum_spp;
  return MRT_OK;
}

extern "C" int mrt_accumulate_double(mrt_ctx* c, double* float_render) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!float_render) return set_err(MRT_ERR_INVALID, "null output");
  if ((rc = fetch_rgb(c))) return rc;
  const float* src = c->rgb_host;
  host_parallel(c->rgb_host_n, [&](size_t a, size_t b) {
    for (size_t i = a; i < b; ++i) float_render[i] += src[i];
  });
  return mrt_clear(c);
}

namespace {
void put_i32(unsigned char* p, int32_t v) {
  for (int k = 0; k < 4; ++k) p[k] = (unsigned char)(((uint32_t)v >> (8 * k)) & 0xff);
}
int32_t get_i32(const unsigned char* p) {
  uint32_t v = 0;
  for (int k = 0; k < 4; ++k) v |= (uint32_t)p[k] << (8 * k);
  return (int32_t)v;
}
}  // namespace

extern "C" int mrt_render_state_save(mrt_ctx* c, const char* path) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!path) return set_err(MRT_ERR_INVALID, "null path");
  const size_t n = (size_t)c->W * c->H;
  std::vector<float> rgb(n * 3);
  rc = mrt_read_accum(c, rgb.data(), nullptr);
  if (rc) return rc;
  std::vector<unsigned char> buf(12 + n * 3 * sizeof(double));
  put_i32(buf.data(), c->W);
  put_i32(buf.data() + 4, c->H);
  put_i32(buf.data() + 8, c->accum_spp);
  for (size_t i = 0; i < 3 * n; ++i) {
    const double v = rgb[i];
    std::memcpy(buf.data() + 12 + 8 * i, &v, 8);   // IEEE double, little-endian hosts
  }
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_err(MRT_ERR_INVALID, "creating %s: %s", path, std::strerror(errno));
  const size_t w = std::fwrite(buf.data(), 1, buf.size(), f);
  const int closed = std::fclose(f);
  if (w != buf.size() || closed != 0) return set_err(MRT_ERR_INVALID, "writing %s failed", path);
  return MRT_OK;
}

extern "C" int mrt_render_state_load(mrt_ctx* c, const char* path) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!path) return set_err(MRT_ERR_INVALID, "null path");
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_err(MRT_ERR_INVALID, "opening %s: %s", path, std::strerror(errno));
  std::vector<unsigned char> buf;
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  std::fclose(f);
  if (buf.size() < 12) return set_err(MRT_ERR_INVALID, "%s: %zu bytes, no header", path, buf.size());
  const int32_t w = get_i32(buf.data()), h = get_i32(buf.data() + 4), sample = get_i32(buf.data() + 8);
  if (w != c->W || h != c->H)
    return set_err(MRT_ERR_INVALID, "%s holds a %dx%d render, the context is %dx%d", path, w, h, c->W, c->H);
  const size_t n = (size_t)c->W * c->H;
  if (buf.size() - 12 != n * 3 * sizeof(double) || sample < 0)
    return set_err(MRT_ERR_INVALID, "%s: %zu data bytes for %zu pixels, sample %d", path, buf.size() - 12, n,
                   sample);
  std::vector<float4> acc(n);
  for (size_t i = 0; i < n; ++i) {
    double v[3];
    std::memcpy(v, buf.data() + 12 + 24 * i, 24);
    acc[i] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)sample);
  }
  CK(cudaMemcpyAsync(c->accum.p, acc.data(), n * sizeof(float4), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->accum_spp = sample;
  return MRT_OK;
}

extern "C" int mrt_read_depth(mrt_ctx* c, int32_t* depth) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!depth) return set_err(MRT_ERR_INVALID, "null output");
  CK(cudaMemcpyAsync(depth, c->depth.p, c->depth.bytes(), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return MRT_OK;
}

extern "C" int mrt_trace_first_hit(mrt_ctx* c, const mrt_ray* rays, int64_t n, mrt_hit* hits) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (n < 0 || (n && (!rays || !hits))) return set_err(MRT_ERR_INVALID, "bad ray buffer");
  if (!c->has_scene) return set_err(MRT_ERR_INVALID, "no scene");
  if (n == 0) return MRT_OK;
  static_assert(sizeof(HitOut) == sizeof(mrt_hit), "HitOut must mirror mrt_hit");
  double* dr = nullptr;
  HitOut* dh = nullptr;
  CK(cudaMallocAsync(&dr, sizeof(mrt_ray) * n, c->stream));
  CK(cudaMallocAsync(&dh, sizeof(HitOut) * n, c->stream));
  CK(cudaMemcpyAsync(dr, rays, sizeof(mrt_ray) * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
  CK(launch_first_hit(c->view, dr, n, dh, c->status.p, c->stream));
  CK(cudaMemcpyAsync(hits, dh, sizeof(HitOut) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaFreeAsync(dr, c->stream));
  CK(cudaFreeAsync(dh, c->stream));
  int status = 0;
  rc = read_status(c, &status);
  if (rc) return rc;
  if (status) return set_err(status & ST_STACK ? MRT_ERR_STACK : MRT_ERR_BUDGET, "traversal status 0x%x", status);
  return MRT_OK;
}

extern "C" int mrt_trace_paths(mrt_ctx* c, const mrt_render_params* p, const int32_t* pixel,
                               const int32_t* sample, int32_t n, float* events, float* rgb) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!p || n < 0 || (n && (!pixel || !sample || !events || !rgb)))
    return set_err(MRT_ERR_INVALID, "bad arguments");
  if (!c->has_scene) return set_err(MRT_ERR_INVALID, "no scene");
  const int64_t npix = (int64_t)c->W * c->H;
  for (int i = 0; i < n; ++i)
    if (pixel[i] < 0 || pixel[i] >= npix || sample[i] < 0)
      return set_err(MRT_ERR_INVALID, "path %d: pixel %d / sample %d out of range", i, pixel[i], sample[i]);
  if (n == 0) return MRT_OK;
  SceneView v = c->view;
  v.env_lookup = p->env_sampler;
  LaunchParams L{};
  L.seed = p->seed;
  L.max_bounces = p->max_bounces > 0 ? p->max_bounces : v.max_bounces;
  L.jitter = p->jitter;
  const size_t ev_floats = (size_t)n * 16 * 20;
  int *dp = nullptr, *ds = nullptr;
  float *dev = nullptr, *drgb = nullptr;
  CK(cudaMallocAsync(&dp, sizeof(int) * n, c->stream));
  CK(cudaMallocAsync(&ds, sizeof(int) * n, c->stream));
  CK(cudaMallocAsync(&dev, sizeof(float) * ev_floats, c->stream));
  CK(cudaMallocAsync(&drgb, sizeof(float) * 3 * n, c->stream));
  CK(cudaMemcpyAsync(dp, pixel, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(ds, sample, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
  CK(launch_path_events(v, L, dp, ds, n, dev, drgb, c->status.p, c->stream));
  CK(cudaMemcpyAsync(events, dev, sizeof(float) * ev_floats, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(rgb, drgb, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaFreeAsync(dp, c->stream));
  CK(cudaFreeAsync(ds, c->stream));
  CK(cudaFreeAsync(dev, c->stream));
  CK(cudaFreeAsync(drgb, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return MRT_OK;
}

extern "C" int mrt_read_env_tables(mrt_ctx* c, float* pdf_joint, float* cdf_m, float* cdf_c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->view.env_nee) return set_err(MRT_ERR_INVALID, "scene has no HDRI tables");
  if (pdf_joint) CK(cudaMemcpy(pdf_joint, c->pdf_joint.p, c->pdf_joint.bytes(), cudaMemcpyDeviceToHost));
  if (cdf_m) CK(cudaMemcpy(cdf_m, c->cdf_m.p, c->cdf_m.bytes(), cudaMemcpyDeviceToHost));
  if (cdf_c) CK(cudaMemcpy(cdf_c, c->cdf_c.p, c->cdf_c.bytes(), cudaMemcpyDeviceToHost));
  return MRT_OK;
}

extern "C" int mrt_env_sample(mrt_ctx* c, int64_t n, uint64_t seed, int32_t sampler, int32_t* outcome,
                              float* out4) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->view.env_nee) return set_err(MRT_ERR_INVALID, "scene has no HDRI tables");
  if (n < 0 || (n && (!out4 || !outcome))) return set_err(MRT_ERR_INVALID, "bad output buffer");
  if (sampler < 0 || sampler > 1) return set_err(MRT_ERR_INVALID, "sampler %d", sampler);
  if (n == 0) return MRT_OK;
  SceneView v = c->view;
  v.env_lookup = sampler;
  float4* d = nullptr;
  int* dk = nullptr;
  CK(cudaMallocAsync(&d, sizeof(float4) * n, c->stream));
  CK(cudaMallocAsync(&dk, sizeof(int) * n, c->stream));
  CK(launch_env_sample(v, n, seed, dk, d, c->stream));
  CK(cudaMemcpyAsync(out4, d, sizeof(float4) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(outcome, dk, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaFreeAsync(d, c->stream));
  CK(cudaFreeAsync(dk, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return MRT_OK;
}

extern "C" int64_t mrt_photon_count(mrt_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  return c->n_photons;
}

extern "C" int mrt_read_photons(mrt_ctx* c, float* pos4, float* pow4, int64_t cap) {
  int rc = check_ctx(c);
  if (rc) return rc;
  const int64_t n = std::min<int64_t>(cap, c->n_photons);
  if (n <= 0) return MRT_OK;
  if (pos4) CK(cudaMemcpy(pos4, c->ph_pos.p, sizeof(float4) * n, cudaMemcpyDeviceToHost));
  if (pow4) CK(cudaMemcpy(pow4, c->ph_pow.p, sizeof(float4) * n, cudaMemcpyDeviceToHost));
  return MRT_OK;
}

extern "C" int mrt_set_photons(mrt_ctx* c, const double* pos3, const double* pow3, int64_t n) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (n < 0 || (n && (!pos3 || !pow3))) return set_err(MRT_ERR_INVALID, "bad photon buffers");
  if (!c->caustic.enable) return set_err(MRT_ERR_INVALID, "scene has caustics disabled");
  std::vector<float4> a(std::max<int64_t>(n, 1)), b(std::max<int64_t>(n, 1));
  for (int64_t i = 0; i < n; ++i) {
    a[i] = make_float4((float)pos3[3 * i], (float)pos3[3 * i + 1], (float)pos3[3 * i + 2], 0.f);
    b[i] = make_float4((float)pow3[3 * i], (float)pow3[3 * i + 1], (float)pow3[3 * i + 2], 0.f);
  }
  CK(c->ph_pos_raw.upload(a.data(), a.size(), c->stream));
  CK(c->ph_pow_raw.upload(b.data(), b.size(), c->stream));
  c->n_photons = n;
  rc = build_photon_map(c);
  if (rc) return rc;
  c->view.caustic = 1;
  return MRT_OK;
}

extern "C" int mrt_caustic_query(mrt_ctx* c, const double* pts3, int64_t n, int32_t k, double* rgb) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (n < 0 || (n && (!pts3 || !rgb))) return set_err(MRT_ERR_INVALID, "bad query buffers");
  if (k <= 0 || k > 32) return set_err(MRT_ERR_INVALID, "k=%d outside [1,32]", k);
  if (n == 0) return MRT_OK;
  SceneView v = c->view;
  v.knn = k;
  double *dp = nullptr, *dout = nullptr;
  CK(cudaMallocAsync(&dp, sizeof(double) * 3 * n, c->stream));
  CK(cudaMallocAsync(&dout, sizeof(double) * 3 * n, c->stream));
  CK(cudaMemcpyAsync(dp, pts3, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  CausticQuery Q{dp, n, dout};
  CK(launch_caustic_query(v, Q, c->stream));
  CK(cudaMemcpyAsync(rgb, dout, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaFreeAsync(dp, c->stream));
  CK(cudaFreeAsync(dout, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return MRT_OK;
}

// ------------------------------------------------- differentiable rendering

namespace {

// Direction and radiance texel of every (row index iv, column index iu) the
// inverse-CDF tables can return: v = iv / (H-1), u = iu / (W-1) as floats,
// then calc_inverse_transform_sampling_dir (get_dir.c:29-41) and the texel
// get_background_color reads for that direction (background.c:15-70), with
// the same double-precision libm calls as env_records.
void env_grid(int W, int H, std::vector<float4>& grid) {
  grid.assign((size_t)W * H, make_float4(0.f, 1.f, 0.f, 0.f));
  auto work = [&](int y0, int y1) {
    for (int iv = y0; iv < y1; ++iv) {
      const double v = (double)(float)((double)iv / (double)(H - 1));
      const float theta = (float)((v - 0.5) * kPiD);
      const double th = (double)theta;
      for (int iu = 0; iu < W; ++iu) {
        const double u = (double)(float)((double)iu / (double)(W - 1));
        const float phi = (float)((0.5 - u) * 2 * kPiD);
        const double ph = (double)phi;
        const V3 dir = {std::cos(th) * std::cos(ph), std::sin(th), std::cos(th) * std::sin(ph)};
        const V3 un = unitv(dir);
        const double vv = 0.5 + std::asin(un.y) / kPiD;
        const double uu = 0.5 - std::atan2(un.z, un.x) / (2.0 * kPiD);
        int x = (int)(uu * (W - 1)), yy = (int)(vv * (H - 1));
        x = std::min(std::max(x, 0), W - 1);
        yy = std::min(std::max(yy, 0), H - 1);
        grid[(size_t)iv * W + iu] =
            make_float4((float)dir.x, (float)dir.y, (float)dir.z, int_bits_as_float(yy * W + x));
      }
    }
  };
  const int nt = std::max(1, std::min((int)std::thread::hardware_concurrency(), 32));
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) pool.emplace_back(work, H * t / nt, H * (t + 1) / nt);
  for (auto& th : pool) th.join();
}

int64_t diff_count(const mrt_ctx* c, int64_t counts[4]) {
  const int64_t M = c->view.n_mats;
  const int64_t T = c->view.has_env ? (int64_t)c->view.env_w * c->view.env_h : 0;
  const int64_t k[4] = {3 * M, M, M, 3 * T};
  if (counts)
    for (int i = 0; i < 4; ++i) counts[i] = k[i];
  return k[0] + k[1] + k[2] + k[3];
}

int diff_check(mrt_ctx* c, const float* theta, const mrt_render_params* p) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->has_scene) return set_err(MRT_ERR_INVALID, "no scene: call mrt_scene_build first");
  if (!theta || !p) return set_err(MRT_ERR_INVALID, "null theta / params");
  if (p->spp <= 0 || p->sample_base < 0) return set_err(MRT_ERR_INVALID, "spp must be > 0, sample_base >= 0");
  const int mb = p->max_bounces > 0 ? p->max_bounces : c->view.max_bounces;
  if (mb < 1 || mb > kMaxTape)
    return set_err(MRT_ERR_INVALID, "differentiable paths take 1..%d bounces, not %d", kMaxTape, mb);
  if (c->view.n_mats > kDiffMaxMats)
    return set_err(MRT_ERR_INVALID, "%d materials: the adjoint handles at most %d", c->view.n_mats,
                   kDiffMaxMats);
  if (c->view.has_env && c->view.env_inv_gamma != 1.0f)
    return set_err(MRT_ERR_INVALID, "a differentiable sky needs a linear HDR (gamma 1)");
  if (c->view.has_textures)
    return set_err(MRT_ERR_INVALID, "textured materials are not differentiable (their texels are not parameters)");
  return MRT_OK;
}

// Upload theta and rebuild the materials, sky tables and NEE records from
// it; v receives the scene view the forward and the replay trace.
int diff_prepare(mrt_ctx* c, const float* theta, SceneView& v) {
  cudaStream_t st = c->stream;
  if (!c->diff) c->diff = new DiffState();
  DiffState& D = *c->diff;
  int64_t counts[4];
  const int64_t n = diff_count(c, counts);
  const int M = c->view.n_mats;
  const int W = c->view.has_env ? c->view.env_w : 0, H = c->view.has_env ? c->view.env_h : 0;
  const size_t npix = (size_t)c->W * c->H;
  if (D.theta.n != (size_t)std::max<int64_t>(n, 1) || D.M != M || D.EW != W || D.EH != H) {
    D.release();
    D.M = M; D.EW = W; D.EH = H;
    D.tables = c->view.env_nee && W >= 2 && H >= 2;
    CK(D.theta.alloc(std::max<int64_t>(n, 1)));
    CK(D.grad.alloc(n + 1));   // + d loss / d column average
    CK(D.gq.alloc(n + 1));
    CK(D.wmax.alloc(1));
    CK(D.img.alloc(3 * npix));
    CK(D.dimg.alloc(3 * npix));
    CK(D.accum_fx.alloc(3 * npix));
    CK(D.mats.alloc(std::max(M, 1)));
    if (D.tables) {
      const size_t t = (size_t)W * H, no = (size_t)(H - 1) * W;
      std::vector<float4> grid;
      env_grid(W, H, grid);
      CK(D.grid.upload(grid.data(), grid.size(), st));
      CK(D.rec0.alloc(no)); CK(D.rec1.alloc(no)); CK(D.aux.alloc(no));
      CK(D.pdf.alloc(t)); CK(D.cm.alloc(H)); CK(D.cc.alloc(t));
      CK(D.gray.alloc(t)); CK(D.raw.alloc(H)); CK(D.rowcdf.alloc(t)); CK(D.scal.alloc(8)); CK(D.cdfh.alloc(H));
    }
  }
  if (n) CK(cudaMemcpyAsync(D.theta.p, theta, sizeof(float) * n, cudaMemcpyDefault, st));
  CK(launch_diff_mats(c->mats.p, D.theta.p, M, D.mats.p, st));
  v = c->view;
  v.mats = D.mats.p;
  const float* sky = D.theta.p + 5 * (size_t)M;
  if (c->view.has_env) v.sky_rgb = sky;
  if (D.tables) {
    EnvBuild E{};
    E.rgb = sky;
    E.W = W;
    E.H = H;
    E.exposure_zero = 1;
    E.gray = D.gray.p; E.raw = D.raw.p; E.row_cdf = D.rowcdf.p; E.scal = D.scal.p; E.cdf_h = D.cdfh.p;
    E.pdf_joint = D.pdf.p; E.cdf_m_inv = D.cm.p; E.cdf_c_inv = D.cc.p;
    E.out_prob = nullptr;
    CK(launch_env_tables(E, st));
    DiffEnvRecords R{D.cm.p, D.cc.p, D.pdf.p, D.grid.p, sky, W, H, D.rec0.p, D.rec1.p, D.aux.p};
    CK(launch_diff_env_records(R, st));
    v.env_rec0 = D.rec0.p;
    v.env_rec1 = D.rec1.p;
    v.pdf_joint = D.pdf.p;
    v.cdf_m_inv = D.cm.p;
    v.cdf_c_inv = D.cc.p;
    v.alias = nullptr;
    v.env_lookup = 1;
  }
  return MRT_OK;
}

int diff_finish(mrt_ctx* c, mrt_render_stats* stats, uint64_t paths, int launches) {
  CK(cudaEventRecord(c->ev1, c->stream));
  CK(cudaEventSynchronize(c->ev1));
  int status = 0;
  int rc = read_status(c, &status);
  if (rc) return rc;
  if (stats) {
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    *stats = mrt_render_stats{};
    stats->ms = ms;
    stats->paths = paths;
    stats->kernel_launches = (uint32_t)launches;
    stats->status = status;
  }
  if (status & ST_STACK) return set_err(MRT_ERR_STACK, "traversal stack overflow (status 0x%x)", status);
  if (status & ST_BUDGET) return set_err(MRT_ERR_BUDGET, "traversal iteration budget exhausted (status 0x%x)", status);
  if (status) return set_err(MRT_ERR_ABORTED, "device status 0x%x", status);
  return MRT_OK;
}

}  // namespace

extern "C" int64_t mrt_diff_layout(mrt_ctx* c, int64_t counts[4]) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->has_scene) return set_err(MRT_ERR_INVALID, "no scene: call mrt_scene_build first");
  return diff_count(c, counts);
}

extern "C" int mrt_diff_get_params(mrt_ctx* c, float* theta) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->has_scene) return set_err(MRT_ERR_INVALID, "no scene: call mrt_scene_build first");
  if (!theta) return set_err(MRT_ERR_INVALID, "null theta");
  int64_t counts[4];
  diff_count(c, counts);
  const int M = c->view.n_mats;
  std::vector<MaterialD> mats(std::max(M, 1));
  if (M) CK(cudaMemcpy(mats.data(), c->mats.p, sizeof(MaterialD) * M, cudaMemcpyDeviceToHost));
  std::vector<float> h((size_t)5 * M);
  for (int m = 0; m < M; ++m) {
    for (int k = 0; k < 3; ++k) h[3 * m + k] = mats[m].color[k];
    h[3 * M + m] = mats[m].roughness;
    h[4 * M + m] = mats[m].emission_strength;
  }
  if (M) CK(cudaMemcpyAsync(theta, h.data(), sizeof(float) * h.size(), cudaMemcpyDefault, c->stream));
  if (counts[3]) {
    float* d = nullptr;
    CK(cudaMallocAsync(&d, sizeof(float) * counts[3], c->stream));
    cudaError_t e = launch_diff_sky_init(c->view, d, c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(theta + 5 * (size_t)M, d, sizeof(float) * counts[3], cudaMemcpyDefault, c->stream);
    cudaFreeAsync(d, c->stream);
    CK(e);
  }
  CK(cudaStreamSynchronize(c->stream));
  return MRT_OK;
}

extern "C" int mrt_forward(mrt_ctx* c, const float* theta, const mrt_render_params* p, float* image,
                           mrt_render_stats* stats) {
  int rc = diff_check(c, theta, p);
  if (rc) return rc;
  if (!image) return set_err(MRT_ERR_INVALID, "null image");
  CK(cudaEventRecord(c->ev0, c->stream));
  SceneView v;
  rc = diff_prepare(c, theta, v);
  if (rc) return rc;
  DiffState& D = *c->diff;
  const uint64_t npix = (uint64_t)c->W * c->H;
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
  CK(cudaMemsetAsync(D.accum_fx.p, 0, D.accum_fx.bytes(), c->stream));
  LaunchParams L{};
  L.seed = p->seed;
  L.max_bounces = p->max_bounces > 0 ? p->max_bounces : v.max_bounces;
  L.jitter = p->jitter;
  L.accum_fx = D.accum_fx.p;        // order-independent sums: the same image on every run
  const int spp_chunk = (int)std::max<uint64_t>(1, (1ull << 26) / std::max<uint64_t>(npix, 1));
  int launches = 0;
  for (int s = 0; s < p->spp; s += spp_chunk) {
    const int k = std::min(spp_chunk, p->spp - s);
    L.sample_base = (uint32_t)(p->sample_base + s);
    L.n_paths = npix * (uint64_t)k;
    CK(launch_megakernel_regen(v, L, nullptr, c->status.p, c->counters.p + 7, 0, 0, c->stream));
    launches++;
  }
  CK(launch_diff_image(D.accum_fx.p, D.img.p, (int)npix, p->spp, c->stream));
  CK(cudaMemcpyAsync(image, D.img.p, sizeof(float) * 3 * npix, cudaMemcpyDefault, c->stream));
  return diff_finish(c, stats, npix * (uint64_t)p->spp, launches + 1);
}

extern "C" int mrt_backward(mrt_ctx* c, const float* theta, const mrt_render_params* p,
                            const float* grad_image, float* grad_theta, mrt_render_stats* stats) {
  int rc = diff_check(c, theta, p);
  if (rc) return rc;
  if (!grad_image || !grad_theta) return set_err(MRT_ERR_INVALID, "null grad_image / grad_theta");
  CK(cudaEventRecord(c->ev0, c->stream));
  SceneView v;
  rc = diff_prepare(c, theta, v);
  if (rc) return rc;
  DiffState& D = *c->diff;
  int64_t counts[4];
  const int64_t n = diff_count(c, counts);
  const uint64_t npix = (uint64_t)c->W * c->H;
  CK(cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
  CK(cudaMemcpyAsync(D.dimg.p, grad_image, sizeof(float) * 3 * npix, cudaMemcpyDefault, c->stream));
  CK(cudaMemsetAsync(D.gq.p, 0, D.gq.bytes(), c->stream));
  // fixed-point scale of the gradient sums: 2^36 / max |d loss / d image|
  // (rounded to a power of two), so a single path's contribution, which is
  // d loss / d image / spp times factors of order 1 to 1e3, keeps about 30
  // significant bits, and sums stay below 2^63 up to 2^27 max |d loss / d image|
  CK(cudaMemsetAsync(D.wmax.p, 0, sizeof(float), c->stream));
  CK(launch_abs_max(D.dimg.p, 3 * npix, D.wmax.p, c->stream));
  float wmax = 0.f;
  CK(cudaMemcpyAsync(&wmax, D.wmax.p, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int wexp = wmax > 0.f ? (int)std::ceil(std::log2((double)wmax)) : 0;
  AdjointArgs A{};
  A.n_paths = npix * (uint64_t)p->spp;
  A.seed = p->seed;
  A.sample_base = (uint32_t)p->sample_base;
  A.max_bounces = p->max_bounces > 0 ? p->max_bounces : v.max_bounces;
  A.jitter = p->jitter;
  A.n_mats = D.M;
  A.n_texels = D.tables ? D.EW * D.EH : 0;
  A.inv_spp = 1.0f / (float)p->spp;
  A.pdf_dgray = 255.0f;
  A.col = D.tables ? D.scal.p : nullptr;
  A.dimg = D.dimg.p;
  A.env_aux = D.tables ? D.aux.p : nullptr;
  A.q_mats = D.gq.p;
  A.q_sky = D.gq.p + 5 * (size_t)D.M;
  A.q_col = D.gq.p + n;
  A.q_scale = std::ldexp(1.0, std::max(-60, std::min(100, 36 - wexp)));
  // samples per chunk: the tape (80 B per bounce) stays within a budget of
  // device memory, at most 16 GiB or a quarter of what is free
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  const size_t have = D.tape.bytes() + D.state.bytes();
  const size_t budget = std::min<size_t>(16ull << 30, (free_b + have) / 4);
  const size_t per_sample = npix * ((size_t)A.max_bounces * sizeof(TapeEntry) + 4 * sizeof(float4));
  const int spp_chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)p->spp, budget / per_sample));
  const size_t paths_chunk = npix * (size_t)spp_chunk;
  if (D.tape.n < paths_chunk * A.max_bounces) CK(D.tape.alloc(paths_chunk * A.max_bounces));
  if (D.state.n < 4 * paths_chunk) CK(D.state.alloc(4 * paths_chunk));
  int launches = 0;
  for (int s0 = 0; s0 < p->spp; s0 += spp_chunk) {
    const int k = std::min(spp_chunk, p->spp - s0);
    AdjointArgs Ac = A;
    Ac.n_paths = npix * (uint64_t)k;
    Ac.sample_base = (uint32_t)(p->sample_base + s0);
    CK(launch_adjoint_chunk(v, Ac, D.tape.p, D.state.p, c->counters.p + 7, c->status.p, c->stream));
    launches += 1 + A.max_bounces;
  }
  CK(launch_diff_grad_out(A, D.grad.p, D.grad.p + 5 * (size_t)D.M, 5 * (int64_t)D.M, c->stream));
  if (n) CK(cudaMemcpyAsync(grad_theta, D.grad.p, sizeof(float) * n, cudaMemcpyDefault, c->stream));
  return diff_finish(c, stats, A.n_paths, launches + 2);   // + abs max, fixed point -> float
}

// ------------------------------------------------------------ multi-GPU

extern "C" int mrt_comm_unique_id(unsigned char* id) {
  if (!id) return set_err(MRT_ERR_INVALID, "null id buffer");
  const char* err = nullptr;
  if (!nccl_unique_id(id, &err)) return set_err(MRT_ERR_CUDA, "ncclGetUniqueId: %s", err);
  return MRT_OK;
}

extern "C" int mrt_comm_init(mrt_ctx* c, const unsigned char* id, int32_t rank, int32_t world) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!id || world < 1 || rank < 0 || rank >= world)
    return set_err(MRT_ERR_INVALID, "mrt_comm_init: rank %d of world %d", rank, world);
  if (c->comm) return set_err(MRT_ERR_INVALID, "mrt_comm_init: the context already has a communicator");
  if (c->comm_count.n != 1) CK(c->comm_count.alloc(1));
  const char* err = nullptr;
  void* comm = nullptr;
  if (!nccl_comm_init(&comm, id, rank, world, &err)) return set_err(MRT_ERR_CUDA, "ncclCommInitRank: %s", err);
  c->comm = comm;
  c->comm_rank = rank;
  c->comm_world = world;
  return MRT_OK;
}

extern "C" int mrt_reduce_frame(mrt_ctx* c, int32_t root) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!c->comm) return set_err(MRT_ERR_INVALID, "mrt_reduce_frame: no communicator (mrt_comm_init)");
  if (root < 0 || root >= c->comm_world) return set_err(MRT_ERR_INVALID, "mrt_reduce_frame: root %d", root);
  const long long mine = c->accum_spp;
  CK(cudaMemcpyAsync(c->comm_count.p, &mine, sizeof(long long), cudaMemcpyHostToDevice, c->stream));
  const char* err = nullptr;
  if (!nccl_reduce_frame(c->comm, reinterpret_cast<float*>(c->accum.p), c->accum.n * 4, c->comm_count.p, root,
                         c->stream, &err))
    return set_err(MRT_ERR_CUDA, "mrt_reduce_frame: %s", err);
  long long total = 0;
  CK(cudaMemcpyAsync(&total, c->comm_count.p, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (c->comm_rank == root) c->accum_spp = (int)total;
  return MRT_OK;
}

extern "C" int mrt_comm_destroy(mrt_ctx* c) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (c->stream) CK(cudaStreamSynchronize(c->stream));
  nccl_comm_destroy(c->comm);
  c->comm = nullptr;
  c->comm_rank = 0;
  c->comm_world = 1;
  return MRT_OK;
}

extern "C" void mrt_shard_samples(int64_t total, int32_t world, int32_t rank, int64_t* first, int64_t* count) {
  if (world < 1 || rank < 0 || rank >= world || total < 0) {
    if (first) *first = 0;
    if (count) *count = 0;
    return;
  }
  const int64_t base = total / world, extra = total % world;
  if (first) *first = rank * base + std::min<int64_t>(rank, extra);
  if (count) *count = base + (rank < extra ? 1 : 0);
}

extern "C" int mrt_set_bvh_options(mrt_ctx* c, const mrt_bvh_options* o) {
  int rc = check_ctx(c);
  if (rc) return rc;
  if (!o || (o->mode != MRT_BVH_SAH && o->mode != MRT_BVH_REFERENCE && o->mode != MRT_BVH_WIDE) ||
      o->n_prims < 0)
    return set_err(MRT_ERR_INVALID, "mrt_set_bvh_options: mode %d", o ? o->mode : -1);
  c->bvh_mode = o->mode;
  c->bvh_list.assign(o->order ? o->order : nullptr, o->order ? o->order + o->n_prims : nullptr);
  c->bvh_pos.assign(o->positions ? o->positions : nullptr, o->positions ? o->positions + 3 * o->n_prims : nullptr);
  return MRT_OK;
}

// Host-only build of the binary SAH (default) or 8-wide tree over n boxes
// (min xyz, max xyz per box, double) followed by the structural check of the
// wide tree; stats[0..3] = nodes, depth, leaves, wide (1) or binary (0).
extern "C" int mrt_bvh_build_check(const double* boxes, int64_t n, int32_t mode, int64_t* stats) {
  if (!boxes || n <= 0 || n >= (int64_t)1 << 28 || (mode != MRT_BVH_SAH && mode != MRT_BVH_WIDE))
    return set_err(MRT_ERR_INVALID, "mrt_bvh_build_check: bad arguments");
  std::vector<PrimBox> prims((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    for (int k = 0; k < 6; ++k)
      if (!std::isfinite(boxes[6 * i + k])) return set_err(MRT_ERR_INVALID, "mrt_bvh_build_check: box %lld", (long long)i);
    prim_box_from_double(prims[(size_t)i], boxes + 6 * i, boxes + 6 * i + 3);
  }
  BvhResult bvh;
  std::string err;
  bool wide = false;
  if (mode == MRT_BVH_WIDE && build_bvh_wide(prims, bvh, err)) {
    wide = true;
    if (!check_bvh_wide(bvh, prims, err)) return set_err(MRT_ERR_INVALID, "BVH: %s", err.c_str());
  } else {
    err.clear();
    if (!build_bvh(prims, bvh, err)) return set_err(MRT_ERR_INVALID, "BVH: %s", err.c_str());
  }
  if (stats) {
    stats[0] = wide ? (int64_t)bvh.wnodes.size() : (int64_t)bvh.nodes.size();
    stats[1] = bvh.max_depth;
    stats[2] = bvh.leaves;
    stats[3] = wide ? 1 : 0;
  }
  return MRT_OK;
}

extern "C" int64_t mrt_read_bvh_leaves(mrt_ctx* c, int32_t* flat, int64_t cap) {
  if (!c || !c->has_scene) return set_err(MRT_ERR_INVALID, "mrt_read_bvh_leaves: no scene");
  const int64_t n = (int64_t)c->leaf_order.size();
  if (flat)
    for (int64_t i = 0; i < std::min(n, cap); ++i) flat[i] = (int32_t)c->leaf_order[i];
  return n;
}
