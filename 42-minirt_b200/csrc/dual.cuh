// dual.cuh — forward-mode dual numbers with N derivative slots.
//
// The adjoint evaluates one bounce at a time in dual arithmetic to get the
// local Jacobian of the bounce's outputs (next direction, hit point, power
// multipliers, radiance terms) with respect to its inputs (incoming origin
// and direction, the material roughness); the path-level gradient is then
// accumulated in reverse order. Comparisons use the value part.
#pragma once
#include <cuda_runtime.h>

namespace mrt {

template <int N>
struct Dual {
  float v;
  float g[N];
  __device__ __forceinline__ Dual() {}
  __device__ __forceinline__ Dual(float x) : v(x) {
#pragma unroll
    for (int i = 0; i < N; ++i) g[i] = 0.f;
  }
  __device__ __forceinline__ static Dual seed(float x, int slot) {
    Dual r(x);
    r.g[slot] = 1.f;
    return r;
  }
};

#define MRT_DUAL_BIN(OP, VAL, GRAD)                                                   \
  template <int N>                                                                   \
  __device__ __forceinline__ Dual<N> operator OP(const Dual<N>& a, const Dual<N>& b) { \
    Dual<N> r;                                                                       \
    r.v = VAL;                                                                       \
    _Pragma("unroll") for (int i = 0; i < N; ++i) r.g[i] = GRAD;                    \
    return r;                                                                        \
  }
MRT_DUAL_BIN(+, a.v + b.v, a.g[i] + b.g[i])
MRT_DUAL_BIN(-, a.v - b.v, a.g[i] - b.g[i])
MRT_DUAL_BIN(*, a.v * b.v, a.g[i] * b.v + a.v * b.g[i])
#undef MRT_DUAL_BIN

template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
  Dual<N> r;
  const float inv = 1.0f / b.v;
  r.v = a.v * inv;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = (a.g[i] - r.v * b.g[i]) * inv;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
  Dual<N> r;
  r.v = -a.v;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = -a.g[i];
  return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, float b) { return a + Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator+(float a, const Dual<N>& b) { return Dual<N>(a) + b; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, float b) { return a - Dual<N>(b); }
template <int N> __device__ __forceinline__ Dual<N> operator-(float a, const Dual<N>& b) { return Dual<N>(a) - b; }
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, float b) {
  Dual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = a.g[i] * b;
  return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(float a, const Dual<N>& b) { return b * a; }
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, float b) { return a * (1.0f / b); }
template <int N> __device__ __forceinline__ Dual<N> operator/(float a, const Dual<N>& b) { return Dual<N>(a) / b; }

template <int N>
__device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& a) {
  Dual<N> r;
  r.v = sqrtf(fmaxf(a.v, 0.f));
  const float k = r.v > 0.f ? 0.5f / r.v : 0.f;
#pragma unroll
  for (int i = 0; i < N; ++i) r.g[i] = a.g[i] * k;
  return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dabs(const Dual<N>& a) { return a.v < 0.f ? -a : a; }
template <int N>
__device__ __forceinline__ Dual<N> dmin(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v ? a : b; }
template <int N>
__device__ __forceinline__ Dual<N> dpow5(const Dual<N>& x) {
  Dual<N> x2 = x * x;
  return x2 * x2 * x;
}

template <class T>
struct V3T {
  T x, y, z;
};
template <class T> __device__ __forceinline__ V3T<T> operator+(const V3T<T>& a, const V3T<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> __device__ __forceinline__ V3T<T> operator-(const V3T<T>& a, const V3T<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T, class S> __device__ __forceinline__ V3T<T> operator*(const V3T<T>& a, const S& s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> __device__ __forceinline__ V3T<T> operator-(const V3T<T>& a) { return {-a.x, -a.y, -a.z}; }
template <class T> __device__ __forceinline__ T vdot(const V3T<T>& a, const V3T<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T>
__device__ __forceinline__ V3T<T> vcross(const V3T<T>& a, const V3T<T>& b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

}  // namespace mrt
