// Shared device helpers: complex arithmetic on double2 / float2 and the
// precision traits the kernels are templated on.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace pspw {

template <typename R>
struct Cx;
template <>
struct Cx<double> {
  using T = double2;
};
template <>
struct Cx<float> {
  using T = float2;
};
template <typename R>
using cx = typename Cx<R>::T;

template <typename T>
__host__ __device__ __forceinline__ T mk(decltype(T::x) re, decltype(T::x) im) {
  T r;
  r.x = re;
  r.y = im;
  return r;
}

__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) {
  return make_double2(s * a.x, s * a.y);
}
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) {
  return make_float2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) {
  return make_float2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) {
  return make_float2(s * a.x, s * a.y);
}

// a * b
template <typename T>
__device__ __forceinline__ T cmul(T a, T b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
template <typename T>
__device__ __forceinline__ T cmulc(T a, T b) {
  return mk<T>(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// acc += a * b
template <typename T>
__device__ __forceinline__ void cfma(T &acc, T a, T b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a) * b
template <typename T>
__device__ __forceinline__ void cfmac(T &acc, T a, T b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
}

template <typename T>
__device__ __forceinline__ T czero() {
  return mk<T>(0, 0);
}

// complex value converted between precisions
template <typename T, typename S>
__device__ __forceinline__ T ccast(S v) {
  return mk<T>((decltype(T::x))v.x, (decltype(T::x))v.y);
}

}  // namespace pspw
