// Small dense Hermitian eigensolver on the device (n <= kHeevMax), for the
// Rayleigh-Ritz step of the Chebyshev-filtered SCF loop (the eig_zheevd call
// of ChebySCFLoop.cpp:299 on the (NX+2) x (NX+2) subspace matrix) and for
// the eigenvalues of tridiagonal Lanczos matrices (ChebySCFLoop.cpp:186-190).
//
// The library eigensolver spends most of its time on launch and host
// synchronisation overhead at this size; here the whole problem lives in one
// block's shared memory for the O(n^3) part, and four launches do the rest:
//
//  1 k_hetrd      one block of 640 threads.  Householder reduction to real
//                 symmetric tridiagonal form T = Q^H A Q (Golub & Van Loan,
//                 Matrix Computations, 4th ed., Alg. 8.3.1, with the complex
//                 reflector choice that leaves the off-diagonal real).  The
//                 lower triangle is held packed row by row in shared memory
//                 (n (n+1)/2 complex, 181 KB at n = 150); trailing rows
//                 belong to groups of four threads, and a steering warp
//                 forms the next step's reflector one column ahead (see the
//                 kernel).  All reductions are fixed-order trees, so results
//                 are bitwise repeatable.
//  2 k_tri_bisect eigenvalues of T by bisection on Sturm counts, one warp per
//                 eigenvalue: the 32 lanes evaluate the count at 32 interior
//                 points of the current interval (5 bits per round).  The
//                 count uses the characteristic-polynomial recurrence
//                 p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2} with exact
//                 power-of-two rescaling, which needs no division.
//  3 k_tri_invit  eigenvectors of T, one block per cluster of eigenvalues
//                 closer than 1e-3 ||T|| (the clustering threshold of
//                 LAPACK's dstein).  An isolated eigenvalue takes one twisted
//                 factorisation (tri_vec_twisted).  A cluster takes inverse
//                 iteration: every member's (T - lambda I) is factored once
//                 (LU with partial pivoting, small pivots raised to
//                 eps ||T||), three solves with block Gram-Schmidt (twice)
//                 between them, then a Rayleigh-Ritz step inside the cluster
//                 (parallel Jacobi in one warp) unless its eigenvalues are
//                 equal to rounding.
//  4 k_back_tr    eigenvectors of A = Q Z, one warp per vector, reflectors
//                 applied from the last to the first.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "common.cuh"
#include "engine.h"
#include "heev.h"

namespace pspw {
namespace {

constexpr int kT1 = 1024;      // threads of the Cholesky block
constexpr double kEps = 2.220446049250313e-16;
constexpr int kInvitThreads = 128;
constexpr int kInvitIters = 3;
constexpr int kRRMax = 32;     // largest cluster with a Rayleigh-Ritz step
constexpr int kZs = 16;        // largest cluster whose vectors stay in shared memory
constexpr int kCB = 8;         // panel width of the blocked Cholesky

__device__ __forceinline__ int lp(int i, int j) { return i * (i + 1) / 2 + j; }  // j <= i

__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

// sum over the block of one value per thread; every thread gets the same
// bits (warp xor tree, then every thread adds the warp sums in order)
__device__ double block_sum(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < nw; i++) s += red[i];
  return s;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// two warp sums with their shuffles interleaved (one tree's latency)
__device__ __forceinline__ void warp_sum2(double &a, double &b) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_xor_sync(0xffffffffu, a, o), y = __shfl_xor_sync(0xffffffffu, b, o);
    a += x;
    b += y;
  }
}

// ---------------------------------------------------------------- 1 reduction
// A: n x n column-major (lda), only the upper triangle is read (as zheevd
// 'U').  Out: d[n], e[n-1], reflectors V (column k holds v_k on rows
// k+1..n-1, v_k(k+1) = 1), tau[n-1]; H_k = I - tau_k v_k v_k^H, Q = H_0 ...
constexpr int kTR = 640;                      // threads of the reduction block
constexpr int kTRW = kTR / 32;                // its warps; the last one steers
constexpr int kSteer = kTRW - 1;
constexpr int kGrp = 4;                       // threads per trailing row (product)
constexpr int kUpd = 8;                       // threads per pair of rows (update)
constexpr int kColsL = (kHeevMax + 31) / 32;  // column entries per lane
static_assert(kSteer * 32 / kGrp >= kHeevMax, "one row group per trailing row");
static_assert(kSteer * 32 / kUpd >= (kHeevMax - 1) / 2 + 1, "one update group per pair of rows");

__device__ __forceinline__ double2 cfma_(double2 a, double2 b, double2 c) {  // c + a b
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
  return c;
}

__device__ __forceinline__ double2 cfmac_(double2 a, double2 b, double2 c) {  // c + conj(a) b
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(-a.y, b.x, c.y);
  return c;
}

// a - (v_i conj(w_j) + w_i conj(v_j)): one element of the rank-2 update
__device__ __forceinline__ double2 her2_(double2 a, double2 vi, double2 wi, double2 vj,
                                         double2 wj) {
  a.x -= vi.x * wj.x + vi.y * wj.y + wi.x * vj.x + wi.y * vj.y;
  a.y -= vi.y * wj.x - vi.x * wj.y + wi.y * vj.x - wi.x * vj.y;
  return a;
}

// The steering warp's part of a step: column c of the trailing matrix,
// updated with the reflector of step c - 1 when `upd` (v, w of that step),
// gives d[c] and, for c < n - 1, the reflector of step c: e[c], tau[c],
// column c of V and its copy vn in shared memory, t and the reflect flag.
__device__ void hetrd_steer(const double2 *L, int n, int c, bool upd, const double2 *v,
                            const double2 *w, double2 *vn, double *d, double *e, double2 *V,
                            double2 *tau, double isa, double2 *s_t, int *s_refl) {
  const int lane = threadIdx.x & 31;
  double2 a[kColsL];
  const double2 vc = upd ? v[c] : make_double2(0.0, 0.0), wc = upd ? w[c] : vc;
  double part = 0.0;
#pragma unroll
  for (int q = 0; q < kColsL; q++) {
    const int i = c + lane + 32 * q;
    a[q] = make_double2(0.0, 0.0);
    if (i < n) {
      double2 x = L[lp(i, c)];
      if (upd) x = her2_(x, v[i], w[i], vc, wc);
      if (i == c) x.y = 0.0;
      a[q] = x;
      if (i >= c + 2) part += x.x * x.x + x.y * x.y;
    }
  }
  if (lane == 0) d[c] = a[0].x * isa;
  if (c >= n - 1) return;  // the last diagonal entry
  const double xn2 = warp_sum(part);
  double2 alpha;
  alpha.x = __shfl_sync(0xffffffffu, a[0].x, 1);  // row c + 1
  alpha.y = __shfl_sync(0xffffffffu, a[0].y, 1);
  // H^H (alpha, x) = (beta, 0), beta real (every lane the same values)
  double beta;
  double2 t, sc = make_double2(0.0, 0.0);
  if (xn2 == 0.0 && alpha.y == 0.0) {
    beta = alpha.x;
    t = make_double2(0.0, 0.0);
  } else {
    beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x);
    const double2 den = make_double2(alpha.x - beta, alpha.y);  // 1 / (alpha - beta)
    const double dd = den.x * den.x + den.y * den.y;
    const double ib = 1.0 / beta, idd = 1.0 / dd;
    t = make_double2((beta - alpha.x) * ib, -alpha.y * ib);
    sc = make_double2(den.x * idd, -den.y * idd);
  }
  const bool reflect = t.x != 0.0 || t.y != 0.0;
#pragma unroll
  for (int q = 0; q < kColsL; q++) {
    const int i = c + lane + 32 * q;
    if (i > c && i < n) {
      const double2 vi = i == c + 1 ? make_double2(1.0, 0.0)
                                    : (reflect ? cmul(a[q], sc) : make_double2(0.0, 0.0));
      vn[i] = vi;
      V[(size_t)c * n + i] = vi;
    }
  }
  if (lane == 0) {
    e[c] = beta * isa;
    tau[c] = t;
    *s_t = t;
    *s_refl = reflect;
  }
}

// Householder reduction, one block of kTR threads.  Step k applies
// H_k = I - t v v^H to the trailing matrix A22 (rows and columns k+1..n-1):
// y = t A22 v, w = y - (1/2) t (y^H v) v, A22 -= v w^H + w v^H.
//  - row groups: warps 0..kSteer-1 hold one trailing row i per group of
//    kGrp threads (sub s takes the columns = s mod kGrp); the row's
//    Hermitian product reads its stored part L(i, k+1..i) along the row and
//    the part above the diagonal as conj(L(j, i)) down column i, so every
//    sum is private to the group (two shuffles combine the subs);
//  - the steering warp updates column k+1 alone, while the groups update
//    the rest, and forms the next step's reflector from it (look-ahead):
//    three barriers per step, and one warp evaluates the reflector.
// All sums run in a fixed order, so results are bitwise repeatable.
__global__ void __launch_bounds__(kTR, 1)
    k_hetrd(const double2 *__restrict__ A, int lda, int n, double *__restrict__ d,
            double *__restrict__ e, double2 *__restrict__ V, double2 *__restrict__ tau) {
  extern __shared__ double2 L[];  // packed lower triangle, row-major
  __shared__ double2 vbuf[2][kHeevMax], w[kHeevMax], s_t[2];
  __shared__ double red[kTRW][2];
  __shared__ int s_refl[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = tid / kGrp, sub = tid % kGrp;
  // the largest |A(i,j)| sets a power-of-two scale (exact), so the sums of
  // squares of the reflectors neither overflow nor underflow
  double amax = 0.0;
  for (int i = warp; i < n; i += kTRW)
    for (int j = lane; j <= i; j += 32) {
      const double2 a = A[j + (size_t)i * lda];
      amax = fmax(amax, fmax(fabs(a.x), fabs(a.y)));
    }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if (lane == 0) red[warp][0] = amax;
  __syncthreads();
  amax = 0.0;
  for (int q = 0; q < kTRW; q++) amax = fmax(amax, red[q][0]);
  const double sa = amax > 0.0 ? ldexp(1.0, -ilogb(amax)) : 1.0, isa = 1.0 / sa;
  for (int i = warp; i < n; i += kTRW)
    for (int j = lane; j <= i; j += 32) {
      const double2 a = A[j + (size_t)i * lda];
      L[lp(i, j)] = make_double2(a.x * sa, -a.y * sa);
    }
  __syncthreads();
  if (warp == kSteer)
    hetrd_steer(L, n, 0, false, nullptr, nullptr, vbuf[0], d, e, V, tau, isa, &s_t[0],
                &s_refl[0]);
  __syncthreads();
  for (int k = 0; k < n - 1; k++) {
    const int k1 = k + 1, m = n - k1, par = k & 1;
    const double2 *v = vbuf[par];
    if (s_refl[par]) {  // uniform
      const double2 t = s_t[par];
      const int i = k1 + g;
      const bool row = warp != kSteer && g < m;
      // warps with trailing rows (uniform per warp)
      const bool wrows = warp != kSteer && warp * (32 / kGrp) < m;
      // y_i = t (A22 v)_i
      double2 acc0 = make_double2(0.0, 0.0), acc1 = acc0, vi = acc0;
      if (row) {
        vi = v[i];
        const double2 *Li = L + lp(i, 0);
        int j = k1 + sub;
        for (; j + kGrp <= i; j += 2 * kGrp) {
          acc0 = cfma_(Li[j], v[j], acc0);
          acc1 = cfma_(Li[j + kGrp], v[j + kGrp], acc1);
        }
        if (j <= i) acc0 = cfma_(Li[j], v[j], acc0);
        j = i + 1 + sub;
        int pj = lp(j, i);
        for (; j + kGrp < n; j += 2 * kGrp) {
          acc0 = cfmac_(L[pj], v[j], acc0);
          const int pj1 = pj + kGrp * j + kGrp * (kGrp + 1) / 2;  // lp(j + kGrp, i)
          acc1 = cfmac_(L[pj1], v[j + kGrp], acc1);
          pj = pj1 + kGrp * (j + kGrp) + kGrp * (kGrp + 1) / 2;
        }
        if (j < n) acc0 = cfmac_(L[pj], v[j], acc0);
      }
      double2 y = make_double2(0.0, 0.0);
      if (wrows) {
        double2 acc = make_double2(acc0.x + acc1.x, acc0.y + acc1.y);
#pragma unroll
        for (int o = 1; o < kGrp; o <<= 1) {
          const double x = __shfl_xor_sync(0xffffffffu, acc.x, o),
                       z = __shfl_xor_sync(0xffffffffu, acc.y, o);
          acc.x += x;
          acc.y += z;
        }
        y = cmul(t, acc);
        double pr = 0.0, pim = 0.0;
        if (row && sub == 0) {
          pr = y.x * vi.x + y.y * vi.y;
          pim = y.x * vi.y - y.y * vi.x;
        }
        warp_sum2(pr, pim);
        if (lane == 0) {
          red[warp][0] = pr;
          red[warp][1] = pim;
        }
      }
      __syncthreads();
      double2 wi = make_double2(0.0, 0.0);
      if (wrows) {
        // al = -(1/2) t (y^H v): the same tree over the warp sums in every
        // warp (warps without rows count zero)
        const int nwr = min(kSteer, (m + 32 / kGrp - 1) / (32 / kGrp));
        double yr = lane < nwr ? red[lane][0] : 0.0, yi = lane < nwr ? red[lane][1] : 0.0;
        warp_sum2(yr, yi);
        const double2 al = cmul(make_double2(-0.5 * t.x, -0.5 * t.y), make_double2(yr, yi));
        wi = y + cmul(al, vi);
        if (row && sub == 0) w[i] = wi;
      }
      __syncthreads();
      // A22 -= v w^H + w v^H on rows k+2.., columns k+2..i (column k+1 is
      // the steering warp's).  The rows go in pairs (k+2+p, n-1-p), whose
      // lengths add up to m, to groups of kUpd threads, so every group has
      // the same work; one row per group would leave the longest row's
      // group alone on the critical path while the others wait at the
      // barrier.  Each element gets the same update as in any order.
      if (warp != kSteer) {
        const int p = tid / kUpd, su = tid % kUpd;
        const int r1 = k1 + 1 + p, r2 = n - 1 - p;
        if (r1 <= r2) {
          const int len1 = r1 - k1, len = r1 == r2 ? len1 : m;  // elements of the pair
          const double2 v1 = v[r1], w1 = w[r1], v2 = v[r2], w2 = w[r2];
          for (int e = su; e < len; e += kUpd) {
            const bool first = e < len1;
            const int r = first ? r1 : r2, j = k1 + 1 + (first ? e : e - len1);
            double2 *a = L + lp(r, j);
            double2 x = her2_(*a, first ? v1 : v2, first ? w1 : w2, v[j], w[j]);
            if (j == r) x.y = 0.0;
            *a = x;
          }
        }
      }
    }
    if (warp == kSteer)
      hetrd_steer(L, n, k1, s_refl[par] != 0, v, w, vbuf[par ^ 1], d, e, V, tau, isa,
                  &s_t[par ^ 1], &s_refl[par ^ 1]);
    __syncthreads();
  }
}

// ---------------------------------------------------------------- 2 bisection
// number of eigenvalues of T below x (e2 = squared off-diagonal)
__device__ int sturm_below(const double *d, const double *e2, int n, double x) {
  double pm = 1.0, p = d[0] - x;
  int s = p < 0.0 || p == 0.0 ? -1 : 1;
  int cnt = s < 0;
  int i = 1;
  // two steps per rescale check: with ||T|| in [1, 2) a step changes |p| by
  // at most a factor of 16, far inside the 2^200 margins
  for (; i + 1 < n; i += 2) {
    const double p1 = fma(d[i] - x, p, -e2[i - 1] * pm);
    const int s1 = p1 == 0.0 ? -s : (p1 < 0.0 ? -1 : 1);
    const double p2 = fma(d[i + 1] - x, p1, -e2[i] * p);
    const int s2 = p2 == 0.0 ? -s1 : (p2 < 0.0 ? -1 : 1);
    cnt += (s1 != s) + (s2 != s1);
    s = s2;
    pm = p1;
    p = p2;
    const double ap = fabs(p) + fabs(pm);
    if (ap > 0x1p+200) {
      p *= 0x1p-200;
      pm *= 0x1p-200;
    } else if (ap < 0x1p-200 && ap != 0.0) {
      p *= 0x1p+200;
      pm *= 0x1p+200;
    }
  }
  for (; i < n; i++) {
    const double pn = fma(d[i] - x, p, -e2[i - 1] * pm);
    const int sn = pn == 0.0 ? -s : (pn < 0.0 ? -1 : 1);
    cnt += sn != s;
    s = sn;
    pm = p;
    p = pn;
  }
  return cnt;
}

// Gershgorin interval and ||T||_inf of the tridiagonal (every thread of the
// calling warp gets the same values)
__device__ void tri_bounds(const double *d, const double *e, int n, double *lo, double *hi,
                           double *tn) {
  double a = INFINITY, b = -INFINITY, c = 0.0;
  for (int i = threadIdx.x & 31; i < n; i += 32) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
    a = fmin(a, d[i] - r);
    b = fmax(b, d[i] + r);
    c = fmax(c, fabs(d[i]) + r);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a = fmin(a, __shfl_xor_sync(0xffffffffu, a, o));
    b = fmax(b, __shfl_xor_sync(0xffffffffu, b, o));
    c = fmax(c, __shfl_xor_sync(0xffffffffu, c, o));
  }
  *lo = a;
  *hi = b;
  *tn = c;
}

// one warp per eigenvalue index (ascending); d, e: device, n <= max shared
__global__ void __launch_bounds__(128) k_tri_bisect(const double *__restrict__ dg,
                                                    const double *__restrict__ eg, int n,
                                                    double *__restrict__ lam) {
  extern __shared__ double sh[];
  double *d = sh, *e = sh + n, *e2 = sh + 2 * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] = dg[i];
    e[i] = i + 1 < n ? eg[i] : 0.0;
  }
  __syncthreads();
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  double lo, hi, tn;
  if (threadIdx.x < 32) tri_bounds(d, e, n, &lo, &hi, &tn);
  __shared__ double s_tn;
  if (threadIdx.x == 0) s_tn = tn;
  __syncthreads();
  tn = s_tn;
  if (tn == 0.0) {  // T = 0
    if (j < n && lane == 0) lam[j] = 0.0;
    return;
  }
  // T scaled by a power of two to ||T|| in [1, 2) (exact), so the Sturm
  // recurrence neither overflows nor underflows for matrices of any scale
  const double sc = ldexp(1.0, -ilogb(tn));
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    d[i] *= sc;
    e[i] *= sc;
    e2[i] = e[i] * e[i];
  }
  __syncthreads();
  if (j >= n) return;  // whole warp
  tri_bounds(d, e, n, &lo, &hi, &tn);
  const double pad = 2.0 * kEps * tn;
  lo -= pad;
  hi += pad;
  for (int it = 0; it < 20; it++) {
    if (hi - lo <= fmax(2.0 * kEps * fmax(fabs(lo), fabs(hi)), kEps * tn)) break;
    const double x = lo + (hi - lo) * ((double)(lane + 1) * (1.0 / 33.0));
    const unsigned above = __ballot_sync(0xffffffffu, sturm_below(d, e2, n, x) > j);
    const double xs = __shfl_sync(0xffffffffu, x, above ? __ffs(above) - 1 : 31);
    if (above) {
      const int f = __ffs(above) - 1;
      const double xl = __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0);
      if (f > 0) lo = xl;
      hi = xs;
    } else {
      lo = xs;
    }
  }
  if (lane == 0) lam[j] = 0.5 * (lo + hi) / sc;
}

// ---------------------------------------------------------------- 3 vectors of T
// LU of (T - s I) with row interchanges: u0 (pivots, stored inverted), u1,
// u2 (the two super-diagonals), ml (multipliers), pv (interchange flags)
struct TriLU {
  double u0[kHeevMax], u1[kHeevMax], u2[kHeevMax], ml[kHeevMax];
  unsigned char pv[kHeevMax];
};

__device__ void tri_factor(const double *d, const double *e, int n, double s, double floor_,
                           TriLU &f) {
  double c0 = d[0] - s, c1 = n > 1 ? e[0] : 0.0, c2 = 0.0;
  for (int i = 0; i < n - 1; i++) {
    const double s0 = e[i], s1 = d[i + 1] - s, s2 = i + 2 < n ? e[i + 1] : 0.0;
    if (fabs(c0) >= fabs(s0)) {
      if (fabs(c0) < floor_) c0 = c0 >= 0.0 ? floor_ : -floor_;
      const double r = 1.0 / c0, m = s0 * r;
      f.u0[i] = r;
      f.u1[i] = c1;
      f.u2[i] = c2;
      f.ml[i] = m;
      f.pv[i] = 0;
      c0 = s1 - m * c1;
      c1 = s2 - m * c2;
    } else {
      const double r = 1.0 / s0, m = c0 * r;
      f.u0[i] = r;
      f.u1[i] = s1;
      f.u2[i] = s2;
      f.ml[i] = m;
      f.pv[i] = 1;
      c0 = c1 - m * s1;
      c1 = c2 - m * s2;
    }
    c2 = 0.0;
  }
  if (fabs(c0) < floor_) c0 = c0 >= 0.0 ? floor_ : -floor_;
  f.u0[n - 1] = 1.0 / c0;
}

// z <- (T - s I)^-1 z, scaled to avoid overflow.  The recurrences carry
// their last values in registers; loads of z and of the factors do not
// depend on them.
__device__ void tri_solve(const TriLU &f, int n, double *z) {
  double zi = z[0];
  for (int i = 0; i < n - 1; i++) {
    double zn = z[i + 1];
    if (f.pv[i]) {
      const double t = zi;
      zi = zn;
      zn = t;
    }
    z[i] = zi;
    zi = fma(-f.ml[i], zi, zn);
  }
  z[n - 1] = zi;
  double scale = 1.0, z1 = 0.0, z2 = 0.0;  // z[i + 1], z[i + 2]
  for (int i = n - 1; i >= 0; i--) {
    double s = z[i] * scale;
    s = fma(-f.u1[i], z1, s);
    s = fma(-f.u2[i], z2, s);
    s *= f.u0[i];
    z[i] = s;
    z2 = z1;
    z1 = s;
    if (fabs(s) > 0x1p+600) {  // rescale what is done; the rest of the
      for (int r = i; r < n; r++) z[r] *= 0x1p-600;  // right-hand side follows
      scale *= 0x1p-600;
      z1 *= 0x1p-600;
      z2 *= 0x1p-600;
    }
  }
}

__device__ __forceinline__ double start_value(int i, int col) {
  uint32_t h = (uint32_t)i * 2654435761u ^ ((uint32_t)col * 2246822519u + 0x9e3779b9u);
  h ^= h >> 15;
  h *= 2246822519u;
  h ^= h >> 13;
  return (double)(h & 0xffffu) * (1.0 / 65536.0) - 0.5 + 1e-3;
}

// Eigenvector of an isolated eigenvalue s of T (d, e: scaled to ||T|| in
// [1, 2), shared memory) from its twisted factorisation (Parlett & Dhillon,
// "Fernando's solution to Wilkinson's problem", Linear Algebra Appl. 267,
// 1997; Dhillon & Parlett, LAPACK's dlar1v): T - s I = L D L^T from the top
// and U R U^T from the bottom, run at the same time by two warps,
//   D_0 = d_0 - s,      l_i = e_i / D_i,      D_{i+1} = d_{i+1} - s - l_i e_i
//   R_{n-1} = d_{n-1} - s, u_i = e_i / R_{i+1}, R_i = d_i - s - u_i e_i,
// pivots below `floor_` raised to it; the twist r minimises
// |gamma_r| = |D_r + R_r - (d_r - s)|, and z solves N_r^T z = e_r:
// z_r = 1, z_i = -l_i z_{i+1} above r, z_{i+1} = -u_i z_i below, then z is
// normalised.  One pass replaces inverse iteration for eigenvalues further
// than the clustering gap from their neighbours.  wk: 4 n doubles.
__device__ void tri_vec_twisted(const double *d, const double *e, int n, double s, double floor_,
                                double *z, double *wk, double *red) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  double *D = wk, *l = wk + n, *R = wk + 2 * n, *u = wk + 3 * n;
  if (lane == 0 && warp == 0) {
    double p = d[0] - s;
    for (int i = 0; i + 1 < n; i++) {
      if (fabs(p) < floor_) p = p >= 0.0 ? floor_ : -floor_;
      D[i] = p;
      const double li = e[i] / p;
      l[i] = li;
      p = (d[i + 1] - s) - li * e[i];
    }
    if (fabs(p) < floor_) p = p >= 0.0 ? floor_ : -floor_;
    D[n - 1] = p;
  } else if (lane == 0 && warp == 1) {
    double p = d[n - 1] - s;
    for (int i = n - 2; i >= 0; i--) {
      if (fabs(p) < floor_) p = p >= 0.0 ? floor_ : -floor_;
      R[i + 1] = p;
      const double ui = e[i] / p;
      u[i] = ui;
      p = (d[i] - s) - ui * e[i];
    }
    if (fabs(p) < floor_) p = p >= 0.0 ? floor_ : -floor_;
    R[0] = p;
  }
  __syncthreads();
  // twist index: the smallest |gamma_r|, ties to the smaller r
  double best = INFINITY;
  int br = 0;
  for (int r = tid; r < n; r += blockDim.x) {
    const double g = fabs(D[r] + R[r] - (d[r] - s));
    if (g < best) {
      best = g;
      br = r;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int orr = __shfl_xor_sync(0xffffffffu, br, o);
    if (ob < best || (ob == best && orr < br)) {
      best = ob;
      br = orr;
    }
  }
  __shared__ int s_r[kInvitThreads / 32];
  if (lane == 0) {
    red[warp] = best;
    s_r[warp] = br;
  }
  __syncthreads();
  int r = s_r[0];
  best = red[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); w++)
    if (red[w] < best || (red[w] == best && s_r[w] < r)) {
      best = red[w];
      r = s_r[w];
    }
  if (lane == 0 && warp == 0) {
    double zi = 1.0;
    z[r] = 1.0;
    for (int i = r - 1; i >= 0; i--) {
      zi = -l[i] * zi;
      z[i] = zi;
    }
  } else if (lane == 0 && warp == 1) {
    double zi = 1.0;
    for (int i = r; i + 1 < n; i++) {
      zi = -u[i] * zi;
      z[i + 1] = zi;
    }
  }
  __syncthreads();
  double p = 0.0;
  for (int i = tid; i < n; i += blockDim.x) p += z[i] * z[i];
  const double inv = 1.0 / sqrt(block_sum(p, red));
  for (int i = tid; i < n; i += blockDim.x) z[i] *= inv;
}

// inverse iteration, Gram-Schmidt and Rayleigh-Ritz for the cluster of
// c eigenvalues lam[j..j+c-1]; zc: the cluster's columns (ld n)
__device__ void invit_cluster(const double *__restrict__ dg, const double *__restrict__ eg,
                              const double *__restrict__ lam, int n, int j, int c, double tn,
                              double *zc, double *d, double *e, double *red, double *S, double *U,
                              double *coef, double *wk) {
  const int tid = threadIdx.x;
  // T and the shifts scaled by a power of two to ||T|| in [1, 2) (exact),
  // so the solves' growth (up to 1/eps) cannot overflow for any scale of T
  const double sc = ldexp(1.0, -ilogb(tn));
  for (int i = tid; i < n; i += blockDim.x) {
    d[i] = dg[i] * sc;
    e[i] = i + 1 < n ? eg[i] * sc : 0.0;
  }
  tn *= sc;
  const double floor_ = kEps * tn;
  if (c == 1) {  // an isolated eigenvalue: one twisted factorisation
    __syncthreads();
    tri_vec_twisted(d, e, n, lam[j] * sc, floor_, zc, wk, red);
    return;
  }
  for (int m = tid; m < c; m += blockDim.x)
    for (int i = 0; i < n; i++) zc[(size_t)m * n + i] = start_value(i, j + m);
  __syncthreads();
  // each member's factorisation lives in the thread's own (local,
  // L1-cached) memory; members beyond the block size
  // (clusters larger than the block) are factored again for every solve
  TriLU f;
  if (tid < c) tri_factor(d, e, n, lam[j + tid] * sc, floor_, f);
  for (int it = 0; it < kInvitIters; it++) {
    for (int m = tid; m < c; m += blockDim.x) {
      if (m != tid) tri_factor(d, e, n, lam[j + m] * sc, floor_, f);
      tri_solve(f, n, zc + (size_t)m * n);
      if (m != tid && tid < c) tri_factor(d, e, n, lam[j + tid] * sc, floor_, f);
    }
    __syncthreads();
    // block Gram-Schmidt, twice per column, in column order
    for (int m = 0; m < c; m++) {
      double *zm = zc + (size_t)m * n;
      for (int pass = 0; pass < 2; pass++) {
        for (int q = 0; q < m; q++) {
          double p = 0.0;
          for (int i = tid; i < n; i += blockDim.x) p += zc[(size_t)q * n + i] * zm[i];
          const double s = block_sum(p, red);
          if (tid == 0) coef[q] = s;
        }
        __syncthreads();
        for (int i = tid; i < n; i += blockDim.x) {
          double v = zm[i];
          for (int q = 0; q < m; q++) v = fma(-coef[q], zc[(size_t)q * n + i], v);
          zm[i] = v;
        }
        __syncthreads();
      }
      double p = 0.0;
      for (int i = tid; i < n; i += blockDim.x) p += zm[i] * zm[i];
      const double nrm = sqrt(block_sum(p, red));
      const double inv = nrm > 0.0 ? 1.0 / nrm : 0.0;
      for (int i = tid; i < n; i += blockDim.x) zm[i] *= inv;
      __syncthreads();
    }
  }
  // Rayleigh-Ritz inside a cluster whose eigenvalues differ beyond rounding
  if (c > 1 && c <= kRRMax && (lam[j + c - 1] - lam[j]) * sc > 4.0 * c * floor_) {
    const int warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    for (int ab = warp; ab < c * c; ab += nw) {  // S(a, b) = z_a . T z_b
      const int a = ab % c, b = ab / c;
      const double *za = zc + (size_t)a * n, *zb = zc + (size_t)b * n;
      double p = 0.0;
      for (int i = lane; i < n; i += 32) {
        double tz = d[i] * zb[i];
        if (i > 0) tz = fma(e[i - 1], zb[i - 1], tz);
        if (i + 1 < n) tz = fma(e[i], zb[i + 1], tz);
        p = fma(za[i], tz, p);
      }
      p = warp_sum(p);
      if (lane == 0) S[a + b * kRRMax] = p;
    }
    __syncthreads();
    if (warp == 0) {
      // symmetrise, U = I, then cyclic parallel Jacobi (round-robin pairs,
      // one lane per pair; c odd gets a dummy index)
      for (int r = lane; r < c * c; r += 32) {
        const int a = r % c, b = r / c;
        U[a + b * kRRMax] = a == b ? 1.0 : 0.0;
      }
      __syncwarp();
      for (int r = lane; r < c * c; r += 32) {
        const int a = r % c, b = r / c;
        if (a < b) {
          const double s = 0.5 * (S[a + b * kRRMax] + S[b + a * kRRMax]);
          S[a + b * kRRMax] = s;
          S[b + a * kRRMax] = s;
        }
      }
      __syncwarp();
      const int cp = c + (c & 1);
      for (int sweep = 0; sweep < 30; sweep++) {
        double off = 0.0, dia = 0.0;
        for (int r = lane; r < c * c; r += 32) {
          const int a = r % c, b = r / c;
          const double v = S[a + b * kRRMax];
          if (a != b) off += v * v; else dia += v * v;
        }
        off = warp_sum(off);
        dia = warp_sum(dia);
        if (off <= 1e-30 * dia || off == 0.0) break;
        for (int round = 0; round < cp - 1; round++) {
          // pair `lane` of this round (circle method, index cp-1 fixed)
          int p = -1, q = -1;
          if (lane < cp / 2) {
            const int a = lane == 0 ? cp - 1 : (round + lane) % (cp - 1);
            const int b = (round + cp - 1 - lane) % (cp - 1);
            p = min(a, b);
            q = max(a, b);
            if (q >= c) p = q = -1;  // dummy index
          }
          double cs = 1.0, sn = 0.0;
          if (p >= 0) {
            const double app = S[p + p * kRRMax], aqq = S[q + q * kRRMax],
                         apq = S[p + q * kRRMax];
            if (apq != 0.0) {
              const double th = 0.5 * (aqq - app) / apq;
              const double tt = copysign(1.0, th) / (fabs(th) + sqrt(th * th + 1.0));
              cs = 1.0 / sqrt(tt * tt + 1.0);
              sn = tt * cs;
            }
          }
          __syncwarp();
          // columns p, q of S and U
          if (p >= 0 && sn != 0.0)
            for (int r = 0; r < c; r++) {
              const double sp = S[r + p * kRRMax], sq = S[r + q * kRRMax];
              S[r + p * kRRMax] = cs * sp - sn * sq;
              S[r + q * kRRMax] = sn * sp + cs * sq;
              const double up = U[r + p * kRRMax], uq = U[r + q * kRRMax];
              U[r + p * kRRMax] = cs * up - sn * uq;
              U[r + q * kRRMax] = sn * up + cs * uq;
            }
          __syncwarp();
          // rows p, q of S
          if (p >= 0 && sn != 0.0)
            for (int r = 0; r < c; r++) {
              const double sp = S[p + r * kRRMax], sq = S[q + r * kRRMax];
              S[p + r * kRRMax] = cs * sp - sn * sq;
              S[q + r * kRRMax] = sn * sp + cs * sq;
            }
          __syncwarp();
        }
      }
      // order the Ritz pairs ascending (selection sort of the permutation)
      if (lane == 0) {
        int perm[kRRMax];
        for (int a = 0; a < c; a++) perm[a] = a;
        for (int a = 0; a < c; a++) {
          int best = a;
          for (int b = a + 1; b < c; b++)
            if (S[perm[b] * (kRRMax + 1)] < S[perm[best] * (kRRMax + 1)]) best = b;
          const int t2 = perm[a];
          perm[a] = perm[best];
          perm[best] = t2;
        }
        for (int a = 0; a < c; a++) coef[a] = (double)perm[a];
      }
    }
    __syncthreads();
    // z' = Z U(:, perm), one row per thread
    for (int i = tid; i < n; i += blockDim.x) {
      double row[kRRMax];
      for (int a = 0; a < c; a++) row[a] = zc[(size_t)a * n + i];
      for (int a = 0; a < c; a++) {
        const int pa = (int)coef[a];
        double s = 0.0;
        for (int b = 0; b < c; b++) s = fma(row[b], U[b + pa * kRRMax], s);
        zc[(size_t)a * n + i] = s;
      }
    }
  }
}

// One block per eigenvalue index j; the block of a cluster's first index
// computes the cluster's vectors into columns of Z (n x n, column-major),
// in shared memory for clusters of up to kZs members (the common case),
// else in place in Z.
__global__ void __launch_bounds__(kInvitThreads)
    k_tri_invit(const double *__restrict__ dg, const double *__restrict__ eg,
                const double *__restrict__ lam, int n, double *__restrict__ Z) {
  __shared__ double red[kInvitThreads / 32];
  __shared__ double S[kRRMax * kRRMax], U[kRRMax * kRRMax];
  __shared__ double coef[kHeevMax];
  __shared__ double d[kHeevMax], e[kHeevMax];
  const int j = blockIdx.x, tid = threadIdx.x;
  double glo, ghi, tn;
  tri_bounds(dg, eg, n, &glo, &ghi, &tn);  // every warp computes the same
  const double gaptol = 1e-3 * tn;
  if (j > 0 && !(lam[j] - lam[j - 1] > gaptol)) return;  // not a cluster's first index
  int c = 1;
  while (j + c < n && lam[j + c] - lam[j + c - 1] <= gaptol) c++;
  __shared__ double zs[kZs * kHeevMax];
  double *zc = c <= kZs ? zs : Z + (size_t)j * n;  // the cluster's c columns
  if (tn == 0.0) {  // T = 0: the unit vectors
    for (int r = tid; r < c * n; r += blockDim.x) zc[r] = (r % n) == j + r / n ? 1.0 : 0.0;
  } else {
    // an isolated eigenvalue's work space: the rows of zs after its vector
    invit_cluster(dg, eg, lam, n, j, c, tn, zc, d, e, red, S, U, coef, zs + kHeevMax);
  }
  if (c <= kZs) {
    __syncthreads();
    for (int r = tid; r < c * n; r += blockDim.x) Z[(size_t)j * n + r] = zs[r];
  }
}

// ---------------------------------------------------------------- 4 back-transform
// column j of A <- Q z_j, one warp per column, kBTWarps columns per block;
// lane l holds rows l, l+32, ...  Each warp reads the reflectors straight
// from global memory (coalesced, L2-resident), the next one loaded into
// registers while the current one is applied.
constexpr int kBTWarps = 2;
__global__ void __launch_bounds__(32 * kBTWarps) k_back_tr(const double2 *__restrict__ V,
                                                            const double2 *__restrict__ tau,
                                                            const double *__restrict__ Z, int n,
                                                            double2 *__restrict__ A, int lda) {
  constexpr int R = (kHeevMax + 31) / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * kBTWarps + warp;
  if (j >= n) return;  // whole warp
  double2 y[R], vn[R];
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = lane + 32 * r;
    y[r] = make_double2(i < n ? Z[(size_t)j * n + i] : 0.0, 0.0);
  }
  // v_k holds rows > k (rows <= k read as zero); applied from k = n-2 down
  auto load = [&](int k, double2 *v) {
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int i = lane + 32 * r;
      v[r] = (k >= 0 && i > k && i < n) ? V[(size_t)k * n + i] : make_double2(0.0, 0.0);
    }
  };
  load(n - 2, vn);
  double2 tn = n >= 2 ? tau[n - 2] : make_double2(0.0, 0.0);
  for (int k = n - 2; k >= 0; k--) {
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = vn[r];
    const double2 t = tn;
    load(k - 1, vn);
    tn = k >= 1 ? tau[k - 1] : make_double2(0.0, 0.0);
    if (t.x == 0.0 && t.y == 0.0) continue;  // uniform
    double sr = 0.0, si = 0.0;  // s = v^H y
#pragma unroll
    for (int r = 0; r < R; r++) {
      sr += v[r].x * y[r].x + v[r].y * y[r].y;
      si += v[r].x * y[r].y - v[r].y * y[r].x;
    }
    warp_sum2(sr, si);
    const double2 tsum = cmul(t, make_double2(sr, si));
#pragma unroll
    for (int r = 0; r < R; r++) y[r] = y[r] - cmul(v[r], tsum);
  }
#pragma unroll
  for (int r = 0; r < R; r++) {
    const int i = lane + 32 * r;
    if (i < n) A[(size_t)j * lda + i] = y[r];
  }
}

// ---------------------------------------------------------------- Cholesky
// G = U^H U (upper U), one block, for the CholeskyQR passes of the span
// orthonormalisation: G (n x n, ldg, upper triangle read) -> the lower factor
// L = U^H packed row-major into Lg, stat[0] = 0 or k + 1 when the k-th pivot
// is not positive, stat[1] = max |U_kk| / min |U_kk|.  Works on L packed in
// shared memory; k_tri_inv then forms U^-1 on many blocks.
__global__ void __launch_bounds__(kT1, 1)
    k_chol_inv(const double2 *__restrict__ G, int ldg, int n, double2 *__restrict__ Lg,
               double *__restrict__ stat) {
  extern __shared__ double2 L[];
  __shared__ int s_failed;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int i = warp; i < n; i += nw)
    for (int j = lane; j <= i; j += 32) L[lp(i, j)] = cconj(G[j + (size_t)i * ldg]);
  if (tid == 0) s_failed = 0;
  __syncthreads();
  // blocked right-looking Cholesky with panels of kCB columns: warp 0
  // factors the panel's kCB x kCB diagonal block (warp-synchronous steps),
  // one thread per row solves the rows below it against that block, and
  // every warp applies the panel's rank-kCB update to the trailing triangle:
  // three barriers per panel
  __shared__ double s_idk[kCB];
  double dmax = 0.0, dmin = INFINITY;  // kept by thread 0
  for (int k0 = 0; k0 < n; k0 += kCB) {
    const int k1 = min(n, k0 + kCB);
    if (warp == 0) {
      for (int k = k0; k < k1; k++) {
        const double akk = L[lp(k, k)].x;
        if (!(akk > 0.0)) {
          if (lane == 0) s_failed = k + 1;
          break;  // warp-uniform
        }
        const double dk = sqrt(akk), idk = 1.0 / dk;
        dmax = fmax(dmax, dk);
        dmin = fmin(dmin, dk);
        __syncwarp();
        if (lane == 0) {
          L[lp(k, k)] = make_double2(dk, 0.0);
          s_idk[k - k0] = idk;
        }
        if (lane < k1 - k - 1) {
          const int i = k + 1 + lane;
          const double2 a = L[lp(i, k)];
          L[lp(i, k)] = make_double2(a.x * idk, a.y * idk);
        }
        __syncwarp();
        // the block's later columns, one element per lane (at most 28):
        // L(i, j) -= L(i, k) conj(L(j, k)), k < j <= i < k1
        const int d = k1 - k - 1;
        if (lane < d * (d + 1) / 2) {
          int jj = 0, rem = lane;
          while (rem >= d - jj) {
            rem -= d - jj;
            jj++;
          }
          const int j = k + 1 + jj, i = j + rem;
          const double2 lik = L[lp(i, k)], ljk = L[lp(j, k)];
          double2 a = L[lp(i, j)];
          a.x -= lik.x * ljk.x + lik.y * ljk.y;
          a.y -= lik.y * ljk.x - lik.x * ljk.y;
          if (i == j) a.y = 0.0;
          L[lp(i, j)] = a;
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (s_failed) break;  // uniform
    const int kb = k1 - k0;
    // rows below the block: L(i, k) = (A(i, k) - sum_{p<k} L(i, p) conj(L(k, p))) / L(k, k)
    for (int i = k1 + tid; i < n; i += blockDim.x) {
      double2 r[kCB];
      const int ri = lp(i, 0) + k0;
#pragma unroll
      for (int q = 0; q < kCB; q++) r[q] = q < kb ? L[ri + q] : make_double2(0.0, 0.0);
#pragma unroll
      for (int q = 0; q < kCB; q++) {
        if (q < kb) {
          double2 a = r[q];
          const int rq = lp(k0 + q, 0) + k0;
#pragma unroll
          for (int p2 = 0; p2 < q; p2++) {
            const double2 lq = L[rq + p2];
            a.x -= r[p2].x * lq.x + r[p2].y * lq.y;
            a.y -= r[p2].y * lq.x - r[p2].x * lq.y;
          }
          const double id = s_idk[q];
          r[q] = make_double2(a.x * id, a.y * id);
        }
      }
#pragma unroll
      for (int q = 0; q < kCB; q++)
        if (q < kb) L[ri + q] = r[q];
    }
    __syncthreads();
    // trailing triangle: rows i >= k1 (warp per row), columns k1..i (lanes)
    for (int i = k1 + warp; i < n; i += nw) {
      double2 li[kCB];
      const int ri = lp(i, 0);
#pragma unroll
      for (int q = 0; q < kCB; q++) li[q] = q < kb ? L[ri + k0 + q] : make_double2(0.0, 0.0);
      for (int j = k1 + lane; j <= i; j += 32) {
        const int rj = lp(j, 0) + k0;
        double2 a = L[ri + j];
#pragma unroll
        for (int q = 0; q < kCB; q++) {
          if (q < kb) {
            const double2 lj = L[rj + q];
            a.x -= li[q].x * lj.x + li[q].y * lj.y;
            a.y -= li[q].y * lj.x - li[q].x * lj.y;
          }
        }
        if (j == i) a.y = 0.0;
        L[ri + j] = a;
      }
    }
    __syncthreads();
  }
  if (s_failed) {
    if (tid == 0) {
      stat[0] = (double)s_failed;
      stat[1] = INFINITY;
    }
    return;
  }
  // the factor goes to global memory for the triangular inverse
  const int np = n * (n + 1) / 2;
  for (int e = tid; e < np; e += blockDim.x) Lg[e] = L[e];
  if (tid == 0) {
    stat[0] = 0.0;
    stat[1] = dmax / dmin;
  }
}

// Uinv = (L^-1)^H from the packed factor Lg, kInvWarps columns per block,
// one warp per column: block b stages the packed rows j0..n-1 of L (j0 its
// first column) in shared memory, then warp w forms column j = j0 + w of
// M = L^-1 by forward substitution: lane l keeps the running sums
// s_i = sum_{k=j}^{i-1} L(i, k) M(k, j) of rows i = l (mod 32) in registers,
// M(k, j) = -(1 / L(k, k)) s_k is broadcast from its owner and added into
// the rows below.  Uinv(r, c) = conj(M(c, r)) for r <= c, 0 below.  Nothing
// is written when the factorisation failed (stat[0] != 0).
constexpr int kInvWarps = 4;
__global__ void __launch_bounds__(32 * kInvWarps) k_tri_inv(const double2 *__restrict__ Lg, int n,
                                                           double2 *__restrict__ Uinv, int ldu,
                                                           const double *__restrict__ stat) {
  extern __shared__ double2 Ls[];  // packed rows j0..n-1
  __shared__ double dinv[kHeevMax];
  if (stat[0] != 0.0) return;  // uniform
  const int j0 = blockIdx.x * kInvWarps, tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int base = lp(j0, 0), np = n * (n + 1) / 2;
  for (int e = tid; e < np - base; e += blockDim.x) Ls[e] = Lg[base + e];
  __syncthreads();
  for (int i = j0 + tid; i < n; i += blockDim.x) dinv[i] = 1.0 / Ls[lp(i, i) - base].x;
  __syncthreads();
  const int j = j0 + warp;
  if (j >= n) return;  // whole warp
  double2 sacc[kColsL];
  int ro[kColsL];  // lp(i, 0) - base of the lane's rows
#pragma unroll
  for (int q = 0; q < kColsL; q++) {
    const int i = lane + 32 * q;
    sacc[q] = make_double2(0.0, 0.0);
    ro[q] = i * (i + 1) / 2 - base;
  }
  for (int r = lane; r < n; r += 32)
    if (r > j) Uinv[(size_t)j * ldu + r] = make_double2(0.0, 0.0);
  // k in blocks of 32: the owner of row k is lane k % 32, slot kb
#pragma unroll
  for (int kb = 0; kb < kColsL; kb++) {
    const int ka = max(j, 32 * kb), kz = min(n, 32 * kb + 32);
    for (int k = ka; k < kz; k++) {
      const int kl = k & 31;
      const double sx = __shfl_sync(0xffffffffu, sacc[kb].x, kl),
                   sy = __shfl_sync(0xffffffffu, sacc[kb].y, kl);
      const double di = dinv[k];
      const double2 mk = k == j ? make_double2(di, 0.0) : make_double2(-di * sx, -di * sy);
      if (lane == 0) Uinv[(size_t)k * ldu + j] = cconj(mk);
      if (lane > kl && lane + 32 * kb < n) sacc[kb] = cfma_(Ls[ro[kb] + k], mk, sacc[kb]);
#pragma unroll
      for (int q = kb + 1; q < kColsL; q++)
        if (lane + 32 * q < n) sacc[q] = cfma_(Ls[ro[q] + k], mk, sacc[q]);
    }
  }
}

}  // namespace

size_t heev_small_workspace(int n) {
  const size_t nn = (size_t)n * n;
  return sizeof(double2) * (nn + n) + sizeof(double) * (nn + 2 * (size_t)n) + 6 * 256;
}

int dev_heev_small(pspw_cell *c, double2 *A, int lda, double *w, int n, void *work) {
  if (n < 1 || n > kHeevMax || lda < n)
    return fail(PSPW_ERR_ARG, "heev_small: n must be in 1.." + std::to_string(kHeevMax));
  cudaStream_t st = c->stream;
  const size_t nn = (size_t)n * n;
  char *p = static_cast<char *>(work);
  auto take = [&](size_t bytes) {
    void *q = p;
    p += (bytes + 255) / 256 * 256;
    return q;
  };
  double2 *V = static_cast<double2 *>(take(sizeof(double2) * nn));
  double2 *tau = static_cast<double2 *>(take(sizeof(double2) * n));
  double *d = static_cast<double *>(take(sizeof(double) * n));
  double *e = static_cast<double *>(take(sizeof(double) * n));
  double *Z = static_cast<double *>(take(sizeof(double) * nn));
  const int smem1 = (int)(sizeof(double2) * ((size_t)n * (n + 1) / 2));
  {
    const int rc = smem_allow_max(k_hetrd);
    if (rc) return rc;
  }
  k_hetrd<<<1, kTR, smem1, st>>>(A, lda, n, d, e, V, tau);
  const int wpb = 4;
  k_tri_bisect<<<(n + wpb - 1) / wpb, 32 * wpb, sizeof(double) * 3 * n, st>>>(d, e, n, w);
  k_tri_invit<<<n, kInvitThreads, 0, st>>>(d, e, w, n, Z);
  k_back_tr<<<(n + kBTWarps - 1) / kBTWarps, 32 * kBTWarps, 0, st>>>(V, tau, Z, n, A, lda);
  c->kernel_launches += 4;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int dev_chol_inv_upper(pspw_cell *c, const double2 *G, int ldg, int n, double2 *Uinv, int ldu,
                       double *stat) {
  if (n < 1 || n > kHeevMax || ldg < n || ldu < n)
    return fail(PSPW_ERR_ARG, "chol_inv_upper: n must be in 1.." + std::to_string(kHeevMax));
  const int np = n * (n + 1) / 2;
  const int smem = (int)(sizeof(double2) * (size_t)np);
  double2 *Lg = nullptr;
  int rc;
  if ((rc = ws_reserve(c, kWsChol, sizeof(double2) * (size_t)np, (void **)&Lg))) return rc;
  if ((rc = smem_allow_max(k_chol_inv)) || (rc = smem_allow_max(k_tri_inv))) return rc;
  k_chol_inv<<<1, kT1, smem, c->stream>>>(G, ldg, n, Lg, stat);
  k_tri_inv<<<(n + kInvWarps - 1) / kInvWarps, 32 * kInvWarps, smem, c->stream>>>(Lg, n, Uinv,
                                                                               ldu, stat);
  c->kernel_launches += 2;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int dev_tri_eigvals(pspw_cell *c, const double *d, const double *e, int n, double *w) {
  if (n < 1 || n > kTriEigMax) return fail(PSPW_ERR_ARG, "tri_eigvals: bad size");
  const int wpb = 4;
  const size_t smem = sizeof(double) * 3 * (size_t)n;
  if (smem > 48 * 1024) {
    const int rc = smem_allow_max(k_tri_bisect);
    if (rc) return rc;
  }
  k_tri_bisect<<<(n + wpb - 1) / wpb, 32 * wpb, smem, c->stream>>>(d, e, n, w);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

}  // namespace pspw
