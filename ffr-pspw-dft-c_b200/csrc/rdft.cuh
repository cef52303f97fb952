// Small DFTs held entirely in registers, with compile-time size and sign.
//
// RDft<N, S>::run(v) replaces v[k] by sum_n v[n] exp(S*2*pi*i*n*k/N).  Sizes
// 2, 3, 4, 5 have closed-form butterflies, 7 a direct sum with constant
// twiddles; every other size N = A*B is split by Cooley-Tukey with input
// index n = b + B*a and output index k = ka + A*kb:
//   X[ka + A*kb] = sum_b w_B^{b*kb} w_N^{b*ka} sum_a w_A^{a*ka} x[b + B*a].
// All loops unroll and every twiddle is a compile-time constant
// (twiddles.cuh), so the whole transform is straight-line register code.
#pragma once

#include "common.cuh"
#include "twiddles.cuh"

namespace pspw {

template <typename T>
__device__ __forceinline__ T rmul(T a, double c, double s) {
  using R = decltype(T::x);
  const R cr = (R)c, sr = (R)s;
  return mk<T>(a.x * cr - a.y * sr, a.x * sr + a.y * cr);
}

// multiply by S*i
template <int S, typename T>
__device__ __forceinline__ T mul_i(T a) {
  return S > 0 ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

template <int N>
struct SplitOf {
  static constexpr int A = (N % 4 == 0 && N != 4) ? 4
                           : (N % 2 == 0)         ? 2
                           : (N % 3 == 0)         ? 3
                           : (N % 5 == 0)         ? 5
                                                  : 7;
  static constexpr int B = N / A;
};

template <int N, int S>
struct RDft {
  template <typename T>
  __device__ __forceinline__ static void run(T *v) {
    constexpr int A = SplitOf<N>::A, B = SplitOf<N>::B;
    T t[N];
#pragma unroll
    for (int b = 0; b < B; b++) {
      T u[A];
#pragma unroll
      for (int a = 0; a < A; a++) u[a] = v[b + B * a];
      RDft<A, S>::run(u);
#pragma unroll
      for (int ka = 0; ka < A; ka++)
        t[b * A + ka] = (b * ka == 0) ? u[ka]
                                      : rmul(u[ka], tw_cos(N, b * ka), S * tw_sin(N, b * ka));
    }
#pragma unroll
    for (int ka = 0; ka < A; ka++) {
      T w[B];
#pragma unroll
      for (int b = 0; b < B; b++) w[b] = t[b * A + ka];
      RDft<B, S>::run(w);
#pragma unroll
      for (int kb = 0; kb < B; kb++) v[ka + A * kb] = w[kb];
    }
  }
};

template <int S>
struct RDft<1, S> {
  template <typename T>
  __device__ __forceinline__ static void run(T *) {}
};

template <int S>
struct RDft<2, S> {
  template <typename T>
  __device__ __forceinline__ static void run(T *v) {
    const T a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  }
};

template <int S>
struct RDft<4, S> {
  template <typename T>
  __device__ __forceinline__ static void run(T *v) {
    const T t0 = v[0] + v[2], t1 = v[0] - v[2];
    const T t2 = v[1] + v[3], t3 = mul_i<S>(v[1] - v[3]);
    v[0] = t0 + t2;
    v[2] = t0 - t2;
    v[1] = t1 + t3;
    v[3] = t1 - t3;
  }
};

template <int S>
struct RDft<3, S> {
  template <typename T>
  __device__ __forceinline__ static void run(T *v) {
    using R = decltype(T::x);
    const R h = (R)0.8660254037844386;  // sin(2 pi / 3)
    const T s = v[1] + v[2], d = v[1] - v[2];
    const T m = mk<T>(v[0].x - (R)0.5 * s.x, v[0].y - (R)0.5 * s.y);
    const T q = mul_i<S>(mk<T>(h * d.x, h * d.y));
    v[0] = v[0] + s;
    v[1] = m + q;
    v[2] = m - q;
  }
};

template <int S>
struct RDft<5, S> {
  template <typename T>
  __device__ __forceinline__ static void run(T *v) {
    using R = decltype(T::x);
    const R c1 = (R)tw_cos(5, 1), c2 = (R)tw_cos(5, 2);
    const R s1 = (R)tw_sin(5, 1), s2 = (R)tw_sin(5, 2);
    const T a1 = v[1] + v[4], b1 = v[1] - v[4];
    const T a2 = v[2] + v[3], b2 = v[2] - v[3];
    const T m1 = mk<T>(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    const T m2 = mk<T>(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    const T n1 = mul_i<S>(mk<T>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    const T n2 = mul_i<S>(mk<T>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    v[0] = v[0] + a1 + a2;
    v[1] = m1 + n1;
    v[4] = m1 - n1;
    v[2] = m2 + n2;
    v[3] = m2 - n2;
  }
};

template <int S>
struct RDft<7, S> {
  template <typename T>
  __device__ __forceinline__ static void run(T *v) {
    T o[7];
#pragma unroll
    for (int k = 0; k < 7; k++) {
      T acc = v[0];
#pragma unroll
      for (int n = 1; n < 7; n++) acc = acc + rmul(v[n], tw_cos(7, n * k), S * tw_sin(7, n * k));
      o[k] = acc;
    }
#pragma unroll
    for (int k = 0; k < 7; k++) v[k] = o[k];
  }
};

}  // namespace pspw
