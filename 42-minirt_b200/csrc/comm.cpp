// comm.cpp — NCCL for multi-GPU sample sharding, loaded at run time.
//
// One process per GPU renders its own contiguous range of samples on a
// replicated scene; one sum-reduce of the W*H float4 accumulators (and of the
// sample counts) gives the frame of the whole job on the root rank. This is
// the role of the reference's render farm, where clients render samples and
// the server adds their float_render buffers (src/network/handle_client.c:
// 67-75), over NVLink / NVSwitch instead of TCP.
//
// libnccl.so.2 is opened with dlopen on the first mrt_comm_* call, so the
// library loads and runs single-GPU without NCCL present.
#include "comm.h"

#include <dlfcn.h>
#include <nccl.h>

#include <mutex>

namespace mrt {
namespace {

struct NcclApi {
  bool tried = false;
  void* handle = nullptr;
  decltype(&ncclGetUniqueId) get_unique_id = nullptr;
  decltype(&ncclCommInitRank) comm_init_rank = nullptr;
  decltype(&ncclCommDestroy) comm_destroy = nullptr;
  decltype(&ncclReduce) reduce = nullptr;
  decltype(&ncclAllReduce) all_reduce = nullptr;
  decltype(&ncclGroupStart) group_start = nullptr;
  decltype(&ncclGroupEnd) group_end = nullptr;
  decltype(&ncclGetErrorString) error_string = nullptr;
};

NcclApi g_nccl;
std::mutex g_nccl_mu;

const char* nccl_err(ncclResult_t r) {
  return g_nccl.error_string ? g_nccl.error_string(r) : "NCCL error";
}

}  // namespace

bool nccl_load(const char** err) {
  std::lock_guard<std::mutex> lk(g_nccl_mu);
  if (g_nccl.tried) {
    if (!g_nccl.handle) *err = "libnccl.so.2 could not be loaded";
    return g_nccl.handle != nullptr;
  }
  g_nccl.tried = true;
  void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
  if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
  if (!h) {
    *err = "libnccl.so.2 could not be loaded";
    return false;
  }
  NcclApi a;
  a.tried = true;
  a.handle = h;
#define SYM(field, name) a.field = reinterpret_cast<decltype(a.field)>(dlsym(h, name))
  SYM(get_unique_id, "ncclGetUniqueId");
  SYM(comm_init_rank, "ncclCommInitRank");
  SYM(comm_destroy, "ncclCommDestroy");
  SYM(reduce, "ncclReduce");
  SYM(all_reduce, "ncclAllReduce");
  SYM(group_start, "ncclGroupStart");
  SYM(group_end, "ncclGroupEnd");
  SYM(error_string, "ncclGetErrorString");
#undef SYM
  if (!a.get_unique_id || !a.comm_init_rank || !a.comm_destroy || !a.reduce || !a.all_reduce ||
      !a.group_start || !a.group_end) {
    dlclose(h);
    *err = "libnccl.so.2 lacks an entry point";
    return false;
  }
  g_nccl = a;
  return true;
}

bool nccl_unique_id(unsigned char* id, const char** err) {
  if (!nccl_load(err)) return false;
  static_assert(sizeof(ncclUniqueId) == kCommIdBytes, "ncclUniqueId size");
  ncclUniqueId u;
  const ncclResult_t r = g_nccl.get_unique_id(&u);
  if (r != ncclSuccess) {
    *err = nccl_err(r);
    return false;
  }
  std::memcpy(id, u.internal, kCommIdBytes);
  return true;
}

bool nccl_comm_init(void** comm, const unsigned char* id, int rank, int world, const char** err) {
  if (!nccl_load(err)) return false;
  ncclUniqueId u;
  std::memcpy(u.internal, id, kCommIdBytes);
  ncclComm_t c = nullptr;
  const ncclResult_t r = g_nccl.comm_init_rank(&c, world, u, rank);
  if (r != ncclSuccess) {
    *err = nccl_err(r);
    return false;
  }
  *comm = c;
  return true;
}

bool nccl_reduce_frame(void* comm, float* frame, size_t n_floats, long long* count_dev, int root,
                       cudaStream_t st, const char** err) {
  ncclComm_t c = static_cast<ncclComm_t>(comm);
  ncclResult_t r = g_nccl.group_start();
  if (r == ncclSuccess) r = g_nccl.reduce(frame, frame, n_floats, ncclFloat32, ncclSum, root, c, st);
  if (r == ncclSuccess) r = g_nccl.all_reduce(count_dev, count_dev, 1, ncclInt64, ncclSum, c, st);
  const ncclResult_t r2 = g_nccl.group_end();
  if (r == ncclSuccess) r = r2;
  if (r != ncclSuccess) {
    *err = nccl_err(r);
    return false;
  }
  return true;
}

void nccl_comm_destroy(void* comm) {
  if (comm && g_nccl.comm_destroy) g_nccl.comm_destroy(static_cast<ncclComm_t>(comm));
}

}  // namespace mrt
