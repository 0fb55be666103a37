// device_common.cuh — float3 helpers and the per-path counter-based RNG.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "mrt_internal.h"

namespace mrt {

#define MRT_PI_D 3.1415926535897   // PI_D of the reference (minirt.h:21)

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float len2(float3 a) { return dot(a, a); }
// vec3_unit (vec3_utils.c:21): zero vector stays zero.
__device__ __forceinline__ float3 unit(float3 a) {
  float l2 = dot(a, a);
  if (l2 > 0.0f) return a * rsqrtf(l2);
  return f3(0.f, 0.f, 0.f);
}
__device__ __forceinline__ float3 ld3(const float* p) { return f3(p[0], p[1], p[2]); }

// ---------------------------------------------------------------- RNG
// Same generator as the oracle (oracle/mrt_oracle.c ro_path_seed /
// ro_pcg_float): splitmix64-derived PCG32 state per (seed, pixel, sample),
// XSH-RR output, 24-bit floats.
__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t path_seed(uint64_t seed, uint32_t pixel, uint32_t sample) {
  return splitmix64(seed ^ splitmix64(((uint64_t)sample << 32) | pixel));
}

struct Rng {
  uint64_t s;
  __device__ __forceinline__ float next() {
    uint64_t old = s;
    s = old * 6364136223846793005ULL + 1442695040888963407ULL;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    uint32_t out = __funnelshift_r(xs, xs, rot);
    return (float)(out >> 8) * (1.0f / 16777216.0f);
  }
};

__device__ __forceinline__ uint32_t pack_rgb8(const uint8_t* c) {
  return (uint32_t)c[0] | ((uint32_t)c[1] << 8) | ((uint32_t)c[2] << 16);
}
__device__ __forceinline__ float3 unpack_rgb8(uint32_t c) {
  return f3((c & 255u) / 255.0f, ((c >> 8) & 255u) / 255.0f, ((c >> 16) & 255u) / 255.0f);
}

}  // namespace mrt
