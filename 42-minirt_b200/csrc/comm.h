// comm.h — run-time loaded NCCL for the multi-GPU entry points (comm.cpp).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>

namespace mrt {

constexpr int kCommIdBytes = 128;

bool nccl_load(const char** err);
bool nccl_unique_id(unsigned char* id, const char** err);
bool nccl_comm_init(void** comm, const unsigned char* id, int rank, int world, const char** err);
// Sum of every rank's frame into root's (in place there) and of the per-rank
// sample counts into every rank's count_dev, on stream st.
bool nccl_reduce_frame(void* comm, float* frame, size_t n_floats, long long* count_dev, int root,
                       cudaStream_t st, const char** err);
void nccl_comm_destroy(void* comm);

}  // namespace mrt
