// Batched 1D FFTs of lines held in shared memory, the building block of the
// 3D transforms in the H*psi passes.
//
// Algorithm: self-sorting mixed-radix Stockham (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC 2008).
// A stage of radix R with Ns = product of the radices already applied maps
// butterfly j (0 <= j < n/R) of each line: read elements j + r*n/R, multiply
// by exp(sign*2*pi*i*r*(j mod Ns)/(Ns*R)), R-point DFT, write elements
// (j - j mod Ns)*R + (j mod Ns) + r*Ns.  Every stage reads one buffer and
// writes the other, so a transform of nf stages ping-pongs nf times; the
// function returns the buffer holding the result.  All threads of the block
// take part; the caller synchronises before the first stage.
//
// Twiddles come from a per-length table w[t] = exp(+2 pi i t / n) computed in
// FP64 on the host (FP32 kernels read its rounded copy); sign = -1 uses the
// conjugates.  Radices 2, 3, 4, 5 have dedicated butterflies; any other
// prime up to 64 uses a direct DFT.
#pragma once

#include "common.cuh"
#include "engine.h"

namespace pspw {

struct FftArg {
  int n, nf;
  int rad[kMaxStages];
};

template <typename T>
__device__ __forceinline__ T tw_at(const T *__restrict__ w, int t, int sign) {
  T v = w[t];
  if (sign < 0) v.y = -v.y;
  return v;
}

// multiply by sign*i
template <typename T>
__device__ __forceinline__ T mul_si(T a, int sign) {
  return sign > 0 ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

template <typename T, int R>
struct Dft;

template <typename T>
struct Dft<T, 2> {
  __device__ __forceinline__ static void run(T *v, int) {
    T a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  }
};

template <typename T>
struct Dft<T, 4> {
  __device__ __forceinline__ static void run(T *v, int sign) {
    T t0 = v[0] + v[2], t1 = v[0] - v[2];
    T t2 = v[1] + v[3], t3 = mul_si(v[1] - v[3], sign);
    v[0] = t0 + t2;
    v[2] = t0 - t2;
    v[1] = t1 + t3;
    v[3] = t1 - t3;
  }
};

template <typename T>
struct Dft<T, 3> {
  __device__ __forceinline__ static void run(T *v, int sign) {
    using R = decltype(T::x);
    const R h = (R)0.86602540378443864676;  // sqrt(3)/2
    T s = v[1] + v[2], d = v[1] - v[2];
    T m = mk<T>(v[0].x - (R)0.5 * s.x, v[0].y - (R)0.5 * s.y);
    T q = mul_si(mk<T>(h * d.x, h * d.y), sign);
    v[0] = v[0] + s;
    v[1] = m + q;
    v[2] = m - q;
  }
};

template <typename T>
struct Dft<T, 5> {
  __device__ __forceinline__ static void run(T *v, int sign) {
    using R = decltype(T::x);
    const R c1 = (R)0.30901699437494742410;   // cos(2 pi/5)
    const R c2 = (R)-0.80901699437494742410;  // cos(4 pi/5)
    const R s1 = (R)0.95105651629515357212;   // sin(2 pi/5)
    const R s2 = (R)0.58778525229247312917;   // sin(4 pi/5)
    T a1 = v[1] + v[4], b1 = v[1] - v[4];
    T a2 = v[2] + v[3], b2 = v[2] - v[3];
    T m1 = mk<T>(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    T m2 = mk<T>(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    T n1 = mul_si(mk<T>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y), sign);
    T n2 = mul_si(mk<T>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y), sign);
    v[0] = v[0] + a1 + a2;
    v[1] = m1 + n1;
    v[4] = m1 - n1;
    v[2] = m2 + n2;
    v[3] = m2 - n2;
  }
};

template <typename T, int R>
__device__ __forceinline__ void stage_fixed(const T *__restrict__ a, T *__restrict__ b, int nl,
                                            int ls, int n, int Ns, const T *__restrict__ w,
                                            int sign) {
  const int nb = n / R;
  const int total = nl * nb;
  const int tmul = n / (Ns * R);
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int line = t / nb;
    const int j = t - line * nb;
    const int jm = j % Ns;
    const T *src = a + line * ls + j;
    T v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = src[r * nb];
    if (Ns > 1) {
      const int step = jm * tmul;
#pragma unroll
      for (int r = 1; r < R; r++) v[r] = cmul(v[r], tw_at(w, r * step, sign));
    }
    Dft<T, R>::run(v, sign);
    T *dst = b + line * ls + (j - jm) * R + jm;
#pragma unroll
    for (int r = 0; r < R; r++) dst[r * Ns] = v[r];
  }
}

constexpr int kMaxGenericRadix = 64;

template <typename T>
__device__ void stage_generic(const T *__restrict__ a, T *__restrict__ b, int nl, int ls, int n,
                              int Ns, int R, const T *__restrict__ w, int sign) {
  const int nb = n / R;
  const int total = nl * nb;
  const int tmul = n / (Ns * R);
  const int wr = n / R;  // w[k*wr] = exp(2 pi i k / R)
  for (int t = threadIdx.x; t < total; t += blockDim.x) {
    const int line = t / nb;
    const int j = t - line * nb;
    const int jm = j % Ns;
    const T *src = a + line * ls + j;
    T v[kMaxGenericRadix];
    const int step = jm * tmul;
    for (int r = 0; r < R; r++) v[r] = cmul(src[r * nb], tw_at(w, r * step, sign));
    T *dst = b + line * ls + (j - jm) * R + jm;
    for (int k = 0; k < R; k++) {
      T acc = czero<T>();
      for (int r = 0; r < R; r++) acc = acc + cmul(v[r], tw_at(w, ((r * k) % R) * wr, sign));
      dst[k * Ns] = acc;
    }
  }
}

// Transform nl lines (line stride ls) held in `a`; `b` is scratch of the same
// shape.  Returns the buffer with the result; ends with a barrier.
template <typename T>
__device__ T *fft_lines(T *a, T *b, int nl, int ls, const FftArg &p, const T *__restrict__ w,
                        int sign) {
  int Ns = 1;
  for (int s = 0; s < p.nf; s++) {
    const int R = p.rad[s];
    switch (R) {
      case 4:
        stage_fixed<T, 4>(a, b, nl, ls, p.n, Ns, w, sign);
        break;
      case 2:
        stage_fixed<T, 2>(a, b, nl, ls, p.n, Ns, w, sign);
        break;
      case 3:
        stage_fixed<T, 3>(a, b, nl, ls, p.n, Ns, w, sign);
        break;
      case 5:
        stage_fixed<T, 5>(a, b, nl, ls, p.n, Ns, w, sign);
        break;
      default:
        stage_generic<T>(a, b, nl, ls, p.n, Ns, R, w, sign);
        break;
    }
    __syncthreads();
    T *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}

}  // namespace pspw
