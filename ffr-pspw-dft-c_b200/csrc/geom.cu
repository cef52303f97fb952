// One system set up from the reference's own inputs, with the heavy set-up
// arrays built on the device:
//   INPUT and FHI98 files          ReadInputFile.cpp, ReadPseudopotentials.cpp
//   grid, sphere, G order, N123    Setup.cpp:10-130, GVectorsGen*.cpp,
//                                  GkVectorsGen.cpp (host: basis.cpp; the heap
//                                  sort is sequential by definition)
//   occupations                    InitOcc.cpp
//   EI tables                      PhaseFactor.cpp:23-64 (host, O(NR x Nat))
//   EIGR                           PhaseFactor.cpp:66-78        device
//   SFAC                           StructureFactor.cpp:5-29     device
//   VPS, RHOPS, ESELF              FormFactor.cpp:5-73          device (ESELF host)
//   PKG_A, WNL                     NLFormFactor.cpp:5-133       device (WNL host)
//   starting density               FormFactorAtomic.cpp + ChebySCFLoop.cpp:157-168
//   ESR                            EwaldEnergy.cpp:5-120        device
// The radial integrals are evaluated once per distinct |G| (the reference
// evaluates FormFactorAtomic and NLFormFactor once per G; the value only
// depends on |G|), one thread per (shell, channel), summing Simpson's rule
// in the reference's order (simpson.cpp, dsum.cpp) with every product and sum
// rounded separately (no contraction into FMA), so the only differences from
// the reference are the last-bit differences of the device sin/cos/exp/erf.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "basis.h"
#include "common.cuh"
#include "engine.h"
#include "input.h"
#include "scf.h"

struct pspw_system {
  int device = 0;
  pspw::InputData in;
  int nr[3] = {0, 0, 0};
  int nnr = 0, ngw = 0, ngwx = 0, ngx = 0, ng = 0, nx = 0, nlmax = 0, nax = 0, nsp = 0;
  double alat = 0, omega = 0, tpiba = 0, tpiba2 = 0, gcut = 0, gcutw = 0, nel = 0, esr = 0,
         eself = 0, wkpt = 1.0;
  std::vector<int> na, lm_end;
  std::vector<unsigned> n123;
  std::vector<double> xkg;
  std::vector<int> igk, n1, n2, n3, in1, in2, in3;
  std::vector<double> g, gg;
  std::vector<double> focc, wnl;
  double2 *d_eigr = nullptr, *d_sfac = nullptr;
  double *d_vps = nullptr, *d_rhops = nullptr, *d_pkg_a = nullptr, *d_rho_start = nullptr;
  pspw_cell *cell = nullptr;
  pspw_scf *scf = nullptr;
  cudaStream_t st = nullptr;
  // set-up phase times (ms): host input + basis, phase/structure factors,
  // local form factors, nonlocal form factors, cell + SCF handles, starting
  // density, Ewald sum, total
  double ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

namespace pspw {
namespace {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
  // (a.x b.x - a.y b.y, a.x b.y + a.y b.x), each product and sum rounded
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

// Simpson's rule of simpson.cpp:5-16 over n (odd) samples spaced h, fed one
// sample at a time in index order: 4 sum(odd) + 2 sum(even interior) + first +
// last, each partial sum running from its first element as dsum.cpp does.
struct SimpsonAcc {
  double s1 = 0.0, s2 = 0.0, f0 = 0.0, fl = 0.0;
  __device__ __forceinline__ void add(int i, int n, double v) {
    if (i == 0) {
      f0 = v;
    } else if (i == n - 1) {
      fl = v;
    } else if (i & 1) {
      s1 = i == 1 ? v : __dadd_rn(s1, v);
    } else {
      s2 = i == 2 ? v : __dadd_rn(s2, v);
    }
  }
  __device__ __forceinline__ double result(double h) const {
    const double simps = __dadd_rn(
        __dadd_rn(__dadd_rn(__dmul_rn(4.0, s1), __dmul_rn(2.0, s2)), f0), fl);
    return __ddiv_rn(__dmul_rn(simps, h), 3.0);
  }
};

double simpson_host(int n, const double *f, double h) {
  const int m = (n - 1) / 2;
  double s1 = f[1];
  for (int i = 1; i < m; i++) s1 = s1 + f[1 + 2 * i];
  double s2 = f[2];
  for (int i = 1; i < m - 1; i++) s2 = s2 + f[2 + 2 * i];
  const double simps = 4.0 * s1 + 2.0 * s2 + f[0] + f[n - 1];
  return simps * h / 3.0;
}

// ---------------------------------------------------------------- kernels
// EIGR(ig, a, s) = EI1 EI2 EI3 at the Miller indices of wavefunction G ig
// (PhaseFactor.cpp:66-78); zero for ig >= ngw.
__global__ void k_eigr(const double2 *__restrict__ ei1, const double2 *__restrict__ ei2,
                       const double2 *__restrict__ ei3, int3 len, int3 zero,
                       const int3 *__restrict__ mill, int ngw, int ngwx, int nsa, double2 *eigr) {
  const long long n = (long long)ngwx * nsa;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int ig = (int)(i % ngwx), sa = (int)(i / ngwx);
    double2 r = make_double2(0.0, 0.0);
    if (ig < ngw) {
      const int3 m = mill[ig];
      const double2 a = ei1[(size_t)sa * len.x + zero.x - 1 + m.x];
      const double2 b = ei2[(size_t)sa * len.y + zero.y - 1 + m.y];
      const double2 c = ei3[(size_t)sa * len.z + zero.z - 1 + m.z];
      r = cmul_rn(cmul_rn(a, b), c);
    }
    eigr[i] = r;
  }
}

// SFAC(is, ig) = sum_a EI1 EI2 EI3 (StructureFactor.cpp:17-27)
__global__ void k_sfac(const double2 *__restrict__ ei1, const double2 *__restrict__ ei2,
                       const double2 *__restrict__ ei3, int3 len, int3 zero,
                       const int3 *__restrict__ mill, const int *__restrict__ na, int ng, int nsp,
                       int nax, double2 *sfac) {
  const long long n = (long long)ng * nsp;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(i % nsp), ig = (int)(i / nsp);
    const int3 m = mill[ig];
    double2 sf = make_double2(0.0, 0.0);
    for (int a = 0; a < na[s]; a++) {
      const size_t sa = (size_t)s * nax + a;
      const double2 p = cmul_rn(cmul_rn(ei1[sa * len.x + zero.x - 1 + m.x],
                                        ei2[sa * len.y + zero.y - 1 + m.y]),
                                ei3[sa * len.z + zero.z - 1 + m.z]);
      sf = make_double2(__dadd_rn(sf.x, p.x), __dadd_rn(sf.y, p.y));
    }
    sfac[i] = sf;
  }
}

enum RadialMode {
  kRadLocal = 0,  // FormFactor.cpp:58-66: vloc sin(x)/x r^3, x = (r |G|) TPIBA
  kRadAtom = 1,   // FormFactorAtomic.cpp:148-151: f sin(x)/x, x = (r |G|) TPIBA
  kRadS = 2,      // NLFormFactor.cpp:47-59: j0, x = (|G| TPIBA) r
  kRadP = 3,      // NLFormFactor.cpp:62-71: j1
  kRadD = 4,      // NLFormFactor.cpp:76-92: j2
};

// q[k] = Simpson integral of the mode's integrand at |G|^2 = shell[k]
template <int MODE>
__global__ void k_radial(const double *__restrict__ r, const double *__restrict__ f, int mmax,
                         double h, double tpiba, const double *__restrict__ shell, int nshell,
                         double *q) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nshell) return;
  const double gabs = sqrt(shell[k]);
  SimpsonAcc acc;
  if ((MODE == kRadP || MODE == kRadD) && gabs < 1.0e-4) {
    q[k] = 0.0;
    return;
  }
  const double arg_nl = __dmul_rn(gabs, tpiba);
  for (int ir = 0; ir < mmax; ir++) {
    const double rr = __ldg(r + ir), fr = __ldg(f + ir);
    double v;
    if (MODE == kRadLocal || MODE == kRadAtom) {
      const double x = __dmul_rn(__dmul_rn(rr, gabs), tpiba);
      v = __ddiv_rn(__dmul_rn(fr, sin(x)), x);
      if (MODE == kRadLocal) v = __dmul_rn(v, __dmul_rn(__dmul_rn(rr, rr), rr));
    } else if (MODE == kRadS) {
      if (gabs < 1.0e-4) {
        v = fr;
      } else {
        const double x = __dmul_rn(arg_nl, rr);
        v = __dmul_rn(__ddiv_rn(sin(x), x), fr);
      }
    } else if (MODE == kRadP) {
      const double x = __dmul_rn(arg_nl, rr);
      const double fac = __ddiv_rn(__dsub_rn(__ddiv_rn(sin(x), x), cos(x)), x);
      v = __dmul_rn(fac, fr);
    } else {
      const double x = __dmul_rn(arg_nl, rr);
      const double t1 = __dmul_rn(__dsub_rn(__ddiv_rn(3.0, __dmul_rn(x, x)), 1.0), sin(x));
      const double t2 = __dmul_rn(__ddiv_rn(3.0, x), cos(x));
      v = __dmul_rn(__ddiv_rn(__dsub_rn(t1, t2), x), fr);
    }
    acc.add(ir, mmax, v);
  }
  q[k] = acc.result(h);
}

// VPS and RHOPS of species s over the density sphere (FormFactor.cpp:28-70):
// VPS(s, 0) = q0 FPIBOM, VPS(s, ig) = q[shell(ig)] FPIBOM,
// RHOPS(s, ig) = (-ZV/OMEGA) exp(-facc G(ig)), RHOPS(s, 0) = 0.
__global__ void k_local_ff(const double *__restrict__ q, double q0, const int *__restrict__ shell_of,
                           const double *__restrict__ g, int ng, int nsp, int s, double fpibom,
                           double zv_om, double facc, double *vps, double *rhops) {
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ng; ig += gridDim.x * blockDim.x) {
    const size_t o = (size_t)ig * nsp + s;
    if (ig == 0) {
      vps[o] = __dmul_rn(q0, fpibom);
      rhops[o] = 0.0;
    } else {
      vps[o] = __dmul_rn(q[shell_of[ig]], fpibom);
      rhops[o] = __dmul_rn(zv_om, exp(__dmul_rn(-facc, g[ig])));
    }
  }
}

// PKG_A(m_l + j, ig, s) of one channel of species s (NLFormFactor.cpp:55-114)
__global__ void k_pkg(const double *__restrict__ q, const int *__restrict__ shell_of,
                      const double *__restrict__ xkg, const double3 *__restrict__ ggk, int ngw,
                      int ngwx, int nlmax, int s, int l, int ml, double sqrt3, double *pkg_a) {
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ngw; ig += gridDim.x * blockDim.x) {
    const double t = sqrt(xkg[ig]);
    const double q1 = q[shell_of[ig]];
    double *o = pkg_a + ((size_t)s * ngwx + ig) * nlmax + ml;
    if (l == 1) {
      o[0] = q1;
    } else if (t < 1.0e-4) {
      for (int j = 0; j < 2 * l - 1; j++) o[j] = 0.0;
    } else if (l == 2) {
      const double3 gv = ggk[ig];
      o[0] = __ddiv_rn(__dmul_rn(q1, __dadd_rn(gv.x, 0.0)), t);
      o[1] = __ddiv_rn(__dmul_rn(q1, __dadd_rn(gv.y, 0.0)), t);
      o[2] = __ddiv_rn(__dmul_rn(q1, __dadd_rn(gv.z, 0.0)), t);
    } else {
      const double3 gv = ggk[ig];
      const double cx = __ddiv_rn(__dadd_rn(gv.x, 0.0), t);
      const double cy = __ddiv_rn(__dadd_rn(gv.y, 0.0), t);
      const double cz = __ddiv_rn(__dadd_rn(gv.z, 0.0), t);
      const double qs = __dmul_rn(q1, sqrt3);
      o[0] = __dmul_rn(__dmul_rn(q1, 0.5), __dsub_rn(__dmul_rn(3.0, __dmul_rn(cz, cz)), 1.0));
      o[1] = __dmul_rn(__dmul_rn(qs, cz), cx);
      o[2] = __dmul_rn(__dmul_rn(qs, cz), cy);
      o[3] = __dmul_rn(__dmul_rn(qs, cx), cy);
      o[4] = __dmul_rn(__ddiv_rn(qs, 2.0), __dsub_rn(__dmul_rn(cx, cx), __dmul_rn(cy, cy)));
    }
  }
}

// v(G) = sum_s SFAC(s, G) X(s, G) in species order (EvalEnergy.cpp:63-70)
__global__ void k_species_sum(const double2 *__restrict__ sfac, const double *__restrict__ x,
                              int ng, int nsp, double2 *out) {
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ng; ig += gridDim.x * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int s = 0; s < nsp; s++) {
      const double2 sf = sfac[(size_t)ig * nsp + s];
      const double v = x[(size_t)ig * nsp + s];
      re = __dadd_rn(re, __dmul_rn(sf.x, v));
      im = __dadd_rn(im, __dmul_rn(sf.y, v));
    }
    out[ig] = make_double2(re, im);
  }
}

// qat(G) = sum_s q_s(|G|) SFAC(s, G) placed on the grid point of G
// (FormFactorAtomic.cpp:139-160); where density G alias onto one grid point
// (a grid smaller than the density sphere needs), the reference's loop in G
// order leaves the last one's value, so only that one writes
__global__ void k_atomic_grid(const double *__restrict__ qa, const double *__restrict__ qa0,
                              int nshell, const int *__restrict__ shell_of,
                              const double2 *__restrict__ sfac, const int *__restrict__ gidx,
                              const unsigned char *__restrict__ last, int ng, int nsp,
                              double2 *grid) {
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ng; ig += gridDim.x * blockDim.x) {
    if (!last[ig]) continue;
    double re = 0.0, im = 0.0;
    for (int s = 0; s < nsp; s++) {
      const double q = ig == 0 ? qa0[s] : qa[(size_t)s * nshell + shell_of[ig]];
      const double2 sf = sfac[(size_t)ig * nsp + s];
      re = __dadd_rn(re, __dmul_rn(q, sf.x));
      im = __dadd_rn(im, __dmul_rn(q, sf.y));
    }
    grid[gidx[ig]] = make_double2(re, im);
  }
}

__global__ void k_real_part(const double2 *__restrict__ z, double *r, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    r[i] = z[i].x;
}

// Ewald real-space sum (EwaldEnergy.cpp:78-112): thread (a1, lattice vector)
// sums over a2 in species order; per-block partials in a fixed tree, then one
// block sums the partials in order.
constexpr int kEwBlock = 256;
__global__ void k_ewald(const double3 *__restrict__ tau, const double *__restrict__ zv,
                        const double *__restrict__ rg, const int *__restrict__ sp, int nat,
                        const double3 *__restrict__ rlat, int nrvec, double *part) {
  __shared__ double red[kEwBlock];
  const long long n = (long long)nat * nrvec;
  const long long i = blockIdx.x * (long long)kEwBlock + threadIdx.x;
  double sum = 0.0;
  if (i < n) {
    const int a1 = (int)(i / nrvec), ir = (int)(i % nrvec);
    const double3 t1 = tau[a1], rv = rlat[ir];
    const double z1 = zv[a1], g1 = rg[sp[a1]];
    for (int a2 = 0; a2 < nat; a2++) {
      const double3 t2 = make_double3(__dadd_rn(rv.x, tau[a2].x), __dadd_rn(rv.y, tau[a2].y),
                                      __dadd_rn(rv.z, tau[a2].z));
      if (t1.x == t2.x && t1.y == t2.y && t1.z == t2.z) continue;
      const double g2 = rg[sp[a2]];
      const double gkl = __ddiv_rn(1.0, sqrt(__dadd_rn(__dmul_rn(g1, g1), __dmul_rn(g2, g2))));
      const double dx = __dsub_rn(t1.x, t2.x), dy = __dsub_rn(t1.y, t2.y),
                   dz = __dsub_rn(t1.z, t2.z);
      const double e2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
      const double d = sqrt(e2);
      const double fac = __dmul_rn(__ddiv_rn(__dmul_rn(z1, zv[a2]), d), 0.5);
      const double add = __dmul_rn(__dsub_rn(1.0, erf(__dmul_rn(d, gkl))), fac);
      sum = __dadd_rn(sum, add);
    }
  }
  red[threadIdx.x] = sum;
  __syncthreads();
  for (int w = kEwBlock / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = __dadd_rn(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void k_sum_ordered(const double *__restrict__ part, int n, double *out) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s = __dadd_rn(s, part[i]);
    *out = s;
  }
}

// ---------------------------------------------------------------- host side
struct Dev {
  std::vector<void *> p;
  ~Dev() {
    for (void *q : p) cudaFree(q);
  }
  template <typename T>
  int up(T **d, const std::vector<T> &h, cudaStream_t st) {
    void *q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(1, h.size()) * sizeof(T)) != cudaSuccess)
      return fail(PSPW_ERR_OOM, "system: device memory");
    p.push_back(q);
    *d = static_cast<T *>(q);
    if (!h.empty())
      PSPW_CUDA(cudaMemcpyAsync(q, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return PSPW_OK;
  }
  template <typename T>
  int get(T **d, size_t n) {
    void *q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(1, n) * sizeof(T)) != cudaSuccess)
      return fail(PSPW_ERR_OOM, "system: device memory");
    p.push_back(q);
    *d = static_cast<T *>(q);
    return PSPW_OK;
  }
};

// distinct values of v[from..n) in first-seen order and the index of each
// element's value
void shells(const double *v, int from, int n, std::vector<double> *vals, std::vector<int> *of) {
  std::unordered_map<uint64_t, int> seen;
  of->assign(n, 0);
  vals->clear();
  for (int i = from; i < n; i++) {
    uint64_t b;
    std::memcpy(&b, &v[i], 8);
    auto it = seen.find(b);
    if (it == seen.end()) {
      it = seen.emplace(b, (int)vals->size()).first;
      vals->push_back(v[i]);
    }
    (*of)[i] = it->second;
  }
}

// atomic occupations by valence charge (FormFactorAtomic.cpp:30-125)
int atomic_occupations(double zv, double *fs, double *fp, double *fd) {
  struct Row {
    double z, s, p, d;
  };
  static const Row rows[] = {
      {1.0, 1.0, 0, 0},    {0.75, 0.75, 0, 0}, {1.25, 1.25, 0, 0}, {2.0, 2.0, 0, 0},
      {3.0, 2.0, 1.0, 0},  {4.0, 2.0, 2.0, 0}, {5.0, 2.0, 3.0, 0}, {6.0, 2.0, 4.0, 0},
      {7.0, 2.0, 5.0, 0},  {8.0, 2.0, 6.0, 0}, {9.0, 1.0, 0, 8.0}, {10.0, 2.0, 0, 8.0},
      {11.0, 1.0, 0, 10.0}, {12.0, 2.0, 0, 10.0}, {13.0, 2.0, 1.0, 10.0}, {14.0, 2.0, 2.0, 10.0},
      {15.0, 2.0, 3.0, 10.0}, {16.0, 2.0, 4.0, 10.0}, {17.0, 2.0, 5.0, 10.0},
      {18.0, 2.0, 6.0, 10.0}};
  for (const Row &r : rows)
    if (std::fabs(zv - r.z) < 1.e-4) {
      *fs = r.s;
      *fp = r.p;
      *fd = r.d;
      return PSPW_OK;
    }
  return fail(PSPW_ERR_NOT_IMPL, "starting density: valence charge above 18 (FormFactorAtomic)");
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

std::string join(const std::string &dir, const std::string &f) {
  if (f.empty() || f[0] == '/' || dir.empty()) return f;
  return dir + "/" + f;
}

int system_build(pspw_system *S, const std::string &dir) {
  using clk = std::chrono::steady_clock;
  auto t0 = clk::now();
  InputData &in = S->in;
  std::string err;
  int rc = read_input_file(join(dir, "INPUT"), &in, &err);
  if (rc) return fail(rc, err);
  for (SpeciesData &sp : in.sp) {
    if (sp.lloc > sp.lmax) return fail(PSPW_ERR_ARG, "INPUT: L_LOC larger than L_MAX (Setup.cpp)");
    if (sp.lloc < 1) return fail(PSPW_ERR_ARG, "INPUT: L_LOC < 1 (FormFactor.cpp:40-44)");
    if (sp.lmax > kMaxAM)
      return fail(PSPW_ERR_NOT_IMPL, "L_MAX > 3 is not implemented (NLFormFactor.cpp:32-37)");
    if ((rc = read_fhi_file(join(dir, sp.file), &sp, &err))) return fail(rc, err);
    if (sp.mmax < 5 || sp.mmax % 2 == 0)
      return fail(PSPW_ERR_ARG, "radial mesh size must be odd and >= 5 (simpson.cpp:7-11)");
  }
  if (in.nkpt != 1) return fail(PSPW_ERR_NOT_IMPL, "one k-point only (ChebySCFLoop.cpp:74-77)");
  if (in.xk[0] != 0.0 || in.xk[1] != 0.0 || in.xk[2] != 0.0)
    return fail(PSPW_ERR_NOT_IMPL, "the Gamma point only");
  const int nsp = in.nsp;
  S->nsp = nsp;
  S->nax = in.nax;
  S->na.resize(nsp);
  S->lm_end.resize(nsp);
  // NLMAX (Setup.cpp:12-17)
  int nlmax = 0;
  for (int s = 0; s < nsp; s++) {
    S->na[s] = in.sp[s].na;
    const int lm = in.sp[s].lmax * in.sp[s].lmax - 2 * in.sp[s].lloc + 1;
    S->lm_end[s] = lm;
    nlmax = std::max(nlmax, lm);
  }
  S->nlmax = nlmax = std::max(nlmax, 4);
  // basis (Setup.cpp:20-66, GVectorsGen, GkVectorsGen)
  pspw_basis_info info;
  const int *nrf = in.user_fft_grid ? in.nr : nullptr;
  if ((rc = pspw_basis_info_gamma(in.a, in.ecut, nrf, &info)))
    return fail(rc, "basis: bad lattice or cutoff");
  const int ngx = info.ngx, ngwx = info.ngwx;
  S->n123.assign(ngwx, 0);
  S->xkg.assign(ngwx, 0.0);
  S->igk.assign(ngwx, 0);
  for (auto *v : {&S->n1, &S->n2, &S->n3, &S->in1, &S->in2, &S->in3}) v->assign(ngx, 0);
  S->g.assign(ngx, 0.0);
  S->gg.assign((size_t)(ngx + 1) * 3, 0.0);
  if ((rc = pspw_basis_build_gamma(in.a, in.ecut, nrf, nsp, S->na.data(), in.tau.data(), &info,
                                   S->n123.data(), S->xkg.data(), S->igk.data(), S->n1.data(),
                                   S->n2.data(), S->n3.data(), S->in1.data(), S->in2.data(),
                                   S->in3.data(), S->g.data(), S->gg.data(), nullptr)))
    return fail(rc, "basis: G-vector list");
  for (int d = 0; d < 3; d++) S->nr[d] = info.nr[d];
  S->nnr = info.nr[0] * info.nr[1] * info.nr[2];
  S->ngw = info.ngw;
  S->ngwx = ngwx;
  S->ngx = ngx;
  S->ng = info.ng;
  S->alat = info.alat;
  S->omega = info.omega;
  S->tpiba = info.tpiba;
  S->tpiba2 = info.tpiba2;
  S->gcut = info.gcut;
  S->gcutw = info.gcutw;
  // electrons, states, occupations (Setup.cpp:75-87, InitOcc.cpp)
  double nel = 0.0;
  for (int s = 0; s < nsp; s++) nel = nel + in.sp[s].na * in.sp[s].zv;
  S->nel = nel;
  S->nx = in.nempty + (int)((nel + 1.0) / 2.0);
  if (in.tmetal && in.nempty > 0 && S->nx / in.nempty > 50)
    return fail(PSPW_ERR_ARG, "more empty states needed for TMETAL (Setup.cpp:92-96)");
  double w = in.wkpt[0];
  if (std::fabs(w - 1.0) > 1.e-8) w = w / w;
  S->wkpt = w;
  S->focc.assign(S->nx, 0.0);
  const int nocc = (int)std::ceil(nel / 2.0);
  if (nocc < 1 || nocc > S->nx) return fail(PSPW_ERR_ARG, "occupations: no electrons");
  S->focc[nocc - 1] = ((int)nel % 2 != 0) ? 1.0 : 2.0;
  for (int i = 0; i < nocc - 1; i++) S->focc[i] = 2.0;
  double sum_el = 0.0;
  for (int i = 0; i < S->nx; i++) sum_el = sum_el + S->focc[i] * w;
  if (std::fabs(nel - sum_el) > 1.e-5)
    return fail(PSPW_ERR_ARG, "wrong initial occupation numbers (InitOcc.cpp:30-40)");
  // ESELF (FormFactor.cpp:18-22) and WNL + radial integrands (NLFormFactor.cpp:22-45)
  const double sq2pim1 = 1.0 / std::sqrt(2.0 * M_PI);
  double eself = 0.0;
  for (int s = 0; s < nsp; s++)
    eself = eself + in.sp[s].zv * in.sp[s].zv / in.sp[s].rgauss * in.sp[s].na;
  S->eself = eself * sq2pim1;
  const double fpibo = 4.0 * M_PI / S->omega;
  S->wnl.assign((size_t)nsp * nlmax, 0.0);
  // the NL radial integrands of each projector channel, species-major
  struct Channel {
    int s, l, ml;
    std::vector<double> fun;
  };
  std::vector<Channel> chans;
  for (int s = 0; s < nsp; s++) {
    const SpeciesData &sp = in.sp[s];
    const int lloc = sp.lloc - 1;
    int ml = 0;
    for (int l = 1; l <= sp.lmax; l++) {
      if (l == sp.lloc) continue;
      std::vector<double> fun(sp.mmax), fun1(sp.mmax);
      for (int ir = 0; ir < sp.mmax; ir++) {
        const double rr = sp.r[ir], rr2 = rr * rr;
        const double dv = sp.vion[l - 1][ir] - sp.vion[lloc][ir];
        fun[ir] = dv * sp.psi[l - 1][ir] * rr2;
        fun1[ir] = dv * (sp.psi[l - 1][ir] * sp.psi[l - 1][ir]) * rr;
      }
      const double q1 = simpson_host(sp.mmax, fun1.data(), sp.clog);
      for (int j = 0; j < 2 * l - 1; j++)
        S->wnl[(size_t)(ml + j) * nsp + s] = (2.0 * l - 1.0) * fpibo / q1;
      chans.push_back(Channel{s, l, ml, fun});
      ml += 2 * l - 1;
    }
  }
  S->ms[0] = ms_since(t0);
  if (S->device < 0) return PSPW_OK;  // host set-up only

  // ---------------------------------------------------------- device
  PSPW_CUDA(cudaSetDevice(S->device));
  if (cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking) != cudaSuccess)
    return fail(PSPW_ERR_CUDA, "system: stream");
  cudaStream_t st = S->st;
  cudaEvent_t ev[8];
  for (cudaEvent_t &e : ev) PSPW_CUDA(cudaEventCreate(&e));
  struct EvFree {
    cudaEvent_t *e;
    ~EvFree() {
      for (int i = 0; i < 8; i++) cudaEventDestroy(e[i]);
    }
  } evfree{ev};
  Dev tmp;
  const int ng = S->ng, ngw = S->ngw, nsa = S->nax * nsp;
  const int gb = 148 * 8;
  PSPW_CUDA(cudaEventRecord(ev[0], st));
  // phase factors and structure factor
  PhaseTables pt;
  phase_tables(in.a, S->nr, nsp, S->na.data(), in.tau.data(), &pt);
  std::vector<double2> ei[3];
  for (int d = 0; d < 3; d++) {
    ei[d].resize(pt.ei[d].size() / 2);
    std::memcpy(ei[d].data(), pt.ei[d].data(), pt.ei[d].size() * sizeof(double));
  }
  std::vector<int3> mill_w(ngw), mill_g(ng);
  for (int ig = 0; ig < ngw; ig++) {
    const int p = S->igk[ig] - 1;
    mill_w[ig] = make_int3(S->in1[p], S->in2[p], S->in3[p]);
  }
  for (int ig = 0; ig < ng; ig++) mill_g[ig] = make_int3(S->in1[ig], S->in2[ig], S->in3[ig]);
  double2 *d_ei[3];
  int3 *d_mw, *d_mg;
  int *d_na;
  if ((rc = tmp.up(&d_ei[0], ei[0], st)) || (rc = tmp.up(&d_ei[1], ei[1], st)) ||
      (rc = tmp.up(&d_ei[2], ei[2], st)) || (rc = tmp.up(&d_mw, mill_w, st)) ||
      (rc = tmp.up(&d_mg, mill_g, st)) || (rc = tmp.up(&d_na, S->na, st)))
    return rc;
  if (cudaMalloc(&S->d_eigr, sizeof(double2) * (size_t)ngwx * std::max(nsa, 1)) != cudaSuccess ||
      cudaMalloc(&S->d_sfac, sizeof(double2) * (size_t)ng * nsp) != cudaSuccess ||
      cudaMalloc(&S->d_vps, sizeof(double) * (size_t)ng * nsp) != cudaSuccess ||
      cudaMalloc(&S->d_rhops, sizeof(double) * (size_t)ng * nsp) != cudaSuccess ||
      cudaMalloc(&S->d_pkg_a, sizeof(double) * (size_t)nlmax * ngwx * nsp) != cudaSuccess ||
      cudaMalloc(&S->d_rho_start, sizeof(double) * (size_t)S->nnr) != cudaSuccess)
    return fail(PSPW_ERR_OOM, "system: device memory");
  const int3 len = make_int3(pt.len[0], pt.len[1], pt.len[2]);
  const int3 zero = make_int3(pt.zero[0], pt.zero[1], pt.zero[2]);
  if (nsa > 0)
    k_eigr<<<gb, 256, 0, st>>>(d_ei[0], d_ei[1], d_ei[2], len, zero, d_mw, ngw, ngwx, nsa,
                               S->d_eigr);
  k_sfac<<<gb, 256, 0, st>>>(d_ei[0], d_ei[1], d_ei[2], len, zero, d_mg, d_na, ng, nsp, S->nax,
                             S->d_sfac);
  PSPW_CUDA(cudaGetLastError());
  PSPW_CUDA(cudaEventRecord(ev[1], st));
  // local form factors
  std::vector<double> gshell, wshell;
  std::vector<int> g_of, w_of;
  shells(S->g.data(), 1, ng, &gshell, &g_of);
  shells(S->xkg.data(), 0, ngw, &wshell, &w_of);
  const int ngs = std::max<int>(1, (int)gshell.size()), nws = std::max<int>(1, (int)wshell.size());
  if (gshell.empty()) gshell.push_back(0.0);
  double *d_gshell, *d_wshell, *d_g, *d_xkg, *d_q;
  int *d_gof, *d_wof;
  std::vector<double> xkg_w(S->xkg.begin(), S->xkg.begin() + ngw);
  if ((rc = tmp.up(&d_gshell, gshell, st)) || (rc = tmp.up(&d_wshell, wshell, st)) ||
      (rc = tmp.up(&d_gof, g_of, st)) || (rc = tmp.up(&d_wof, w_of, st)) ||
      (rc = tmp.up(&d_g, std::vector<double>(S->g.begin(), S->g.begin() + ng), st)) ||
      (rc = tmp.up(&d_xkg, xkg_w, st)) ||
      (rc = tmp.get(&d_q, (size_t)std::max(ngs, nws) * (nsp + 1))))
    return rc;
  std::vector<double> hq(nsp);
  const double fpibom = 4.0 * M_PI / S->omega;
  for (int s = 0; s < nsp; s++) {
    const SpeciesData &sp = in.sp[s];
    const int ll = sp.lloc - 1;
    std::vector<double> vloc(sp.mmax), f0(sp.mmax);
    for (int ir = 0; ir < sp.mmax; ir++) {
      const double rr = sp.r[ir];
      const double vv = -sp.zv / rr * std::erf(rr / sp.rgauss);
      vloc[ir] = sp.vion[ll][ir] - vv;
      f0[ir] = vloc[ir] * (rr * rr * rr);
    }
    const double q0 = simpson_host(sp.mmax, f0.data(), sp.clog);
    double *d_r, *d_f;
    if ((rc = tmp.up(&d_r, sp.r, st)) || (rc = tmp.up(&d_f, vloc, st))) return rc;
    double *q = d_q + (size_t)s * ngs;
    k_radial<kRadLocal><<<(ngs + 127) / 128, 128, 0, st>>>(d_r, d_f, sp.mmax, sp.clog, S->tpiba,
                                                           d_gshell, ngs, q);
    const double facc = 0.25 * S->tpiba2 * sp.rgauss * sp.rgauss;
    k_local_ff<<<gb, 256, 0, st>>>(q, q0, d_gof, d_g, ng, nsp, s, fpibom, -sp.zv / S->omega, facc,
                                   S->d_vps, S->d_rhops);
  }
  PSPW_CUDA(cudaGetLastError());
  PSPW_CUDA(cudaEventRecord(ev[2], st));
  // nonlocal form factors
  PSPW_CUDA(cudaMemsetAsync(S->d_pkg_a, 0, sizeof(double) * (size_t)nlmax * ngwx * nsp, st));
  std::vector<double3> ggk(ngw);
  const int ldg = ngx + 1;
  for (int ig = 0; ig < ngw; ig++) {
    const int p = S->igk[ig] - 1;
    ggk[ig] = make_double3(S->gg[p], S->gg[(size_t)ldg + p], S->gg[(size_t)2 * ldg + p]);
  }
  double3 *d_ggk;
  if ((rc = tmp.up(&d_ggk, ggk, st))) return rc;
  const double sqrt3 = std::sqrt(3.0);
  // one q column shared by the channels: stream order makes each channel's
  // k_pkg read its integrals before the next channel's k_radial writes them
  double *qn = d_q + (size_t)nsp * std::max(ngs, nws);
  for (const Channel &ch : chans) {
    const SpeciesData &sp = in.sp[ch.s];
    double *d_r, *d_f;
    if ((rc = tmp.up(&d_r, sp.r, st)) || (rc = tmp.up(&d_f, ch.fun, st))) return rc;
    const int nb = (nws + 127) / 128;
    if (ch.l == 1)
      k_radial<kRadS><<<nb, 128, 0, st>>>(d_r, d_f, sp.mmax, sp.clog, S->tpiba, d_wshell, nws, qn);
    else if (ch.l == 2)
      k_radial<kRadP><<<nb, 128, 0, st>>>(d_r, d_f, sp.mmax, sp.clog, S->tpiba, d_wshell, nws, qn);
    else
      k_radial<kRadD><<<nb, 128, 0, st>>>(d_r, d_f, sp.mmax, sp.clog, S->tpiba, d_wshell, nws, qn);
    k_pkg<<<gb, 256, 0, st>>>(qn, d_wof, d_xkg, d_ggk, ngw, ngwx, nlmax, ch.s, ch.l, ch.ml, sqrt3,
                              S->d_pkg_a);
  }
  PSPW_CUDA(cudaGetLastError());
  PSPW_CUDA(cudaEventRecord(ev[3], st));
  PSPW_CUDA(cudaStreamSynchronize(st));
  // cell and SCF handles built from the device arrays
  const auto t_cell = clk::now();
  if ((rc = cell_create(&S->cell, S->device, S->nr[0], S->nr[1], S->nr[2], ngw, ngwx,
                        S->n123.data(), S->xkg.data(), S->tpiba2, nsp, S->na.data(), S->nax,
                        S->lm_end.data(), nlmax, nullptr, nullptr, S->wnl.data(), S->d_eigr,
                        S->d_pkg_a)))
    return rc;
  if ((rc = pspw_scf_create(S->cell, ng, S->n1.data(), S->n2.data(), S->n3.data(), S->g.data(), 0,
                            nullptr, nullptr, nullptr, S->omega, S->nel, 0.0, S->eself,
                            &S->scf)))
    return rc;
  S->scf->nsp = nsp;
  cudaStream_t cst = S->cell->stream;
  k_species_sum<<<gb, 256, 0, cst>>>(S->d_sfac, S->d_vps, ng, nsp, S->scf->d_vp);
  k_species_sum<<<gb, 256, 0, cst>>>(S->d_sfac, S->d_rhops, ng, nsp, S->scf->d_rp);
  PSPW_CUDA(cudaGetLastError());
  PSPW_CUDA(cudaStreamSynchronize(cst));
  S->ms[4] = ms_since(t_cell);
  // starting density (ChebySCFLoop.cpp:157-168) on the cell stream
  PSPW_CUDA(cudaEventRecord(ev[4], cst));
  std::vector<double> qa0(nsp);
  double *d_qa, *d_qa0;
  if ((rc = tmp.get(&d_qa, (size_t)nsp * ngs)) || (rc = tmp.get(&d_qa0, nsp))) return rc;
  for (int s = 0; s < nsp; s++) {
    const SpeciesData &sp = in.sp[s];
    double fs = 2.0, fp = 0.0, fd = 0.0;
    if ((rc = atomic_occupations(sp.zv, &fs, &fp, &fd))) return rc;
    std::vector<double> fun(sp.mmax);
    for (int ir = 0; ir < sp.mmax; ir++) {
      const double p1 = sp.psi[0][ir], p2 = sp.psi[1][ir], p3 = sp.psi[2][ir];
      double v = 0.0;
      if (sp.lmax == 3)
        v = (fs * (p1 * p1) + fp * (p2 * p2) + fd * (p3 * p3)) * sp.r[ir] / S->omega;
      else if (sp.lmax == 2)
        v = (fs * (p1 * p1) + fp * (p2 * p2)) * sp.r[ir] / S->omega;
      else if (sp.lmax == 1)
        v = fs * (p1 * p1) * sp.r[ir] / S->omega;
      fun[ir] = v;
    }
    qa0[s] = simpson_host(sp.mmax, fun.data(), sp.clog);
    double *d_r, *d_f;
    if ((rc = tmp.up(&d_r, sp.r, cst)) || (rc = tmp.up(&d_f, fun, cst))) return rc;
    k_radial<kRadAtom><<<(ngs + 127) / 128, 128, 0, cst>>>(d_r, d_f, sp.mmax, sp.clog, S->tpiba,
                                                           d_gshell, ngs, d_qa + (size_t)s * ngs);
  }
  PSPW_CUDA(cudaMemcpyAsync(d_qa0, qa0.data(), sizeof(double) * nsp, cudaMemcpyHostToDevice, cst));
  PSPW_CUDA(cudaMemsetAsync(S->scf->d_grid, 0, sizeof(double2) * (size_t)S->nnr, cst));
  k_atomic_grid<<<gb, 256, 0, cst>>>(d_qa, d_qa0, ngs, d_gof, S->d_sfac, S->scf->d_gidx,
                                     S->scf->d_glast, ng, nsp,
                                     S->scf->d_grid);
  PSPW_CUDA(cudaGetLastError());
  if ((rc = grid_fft(S->cell, S->scf->d_grid, +1))) return rc;
  k_real_part<<<gb, 256, 0, cst>>>(S->scf->d_grid, S->d_rho_start, S->nnr);
  int warn = 0;
  if ((rc = normalize_rho_dev(S->scf, S->d_rho_start, S->omega, S->nel, &warn))) return rc;
  PSPW_CUDA(cudaEventRecord(ev[5], cst));
  // Ewald sum (EwaldEnergy.cpp): Wigner-Seitz-folded positions and the
  // lattice vectors within RCUT (plus the 27 nearest cells), host
  {
    double xmat[9], xmati[9];
    for (int i = 0; i < 3; i++) {
      xmat[0 * 3 + i] = in.a[i];
      xmat[1 * 3 + i] = in.a[3 + i];
      xmat[2 * 3 + i] = in.a[6 + i];
    }
    matinv3(xmat, xmati);
    const double *A1 = in.a, *A2 = in.a + 3, *A3 = in.a + 6;
    std::vector<double3> tws;
    std::vector<double> zvs;
    std::vector<int> spc;
    for (int s = 0; s < nsp; s++)
      for (int a = 0; a < S->na[s]; a++) {
        const double *tp = &in.tau[3 * ((size_t)s * S->nax + a)];
        double t1[3], tw[3];
        for (int i = 0; i < 3; i++) {
          double sumh = xmati[i] * tp[0];
          sumh = sumh + xmati[3 + i] * tp[1];
          sumh = sumh + xmati[6 + i] * tp[2];
          t1[i] = sumh - std::floor(sumh);
        }
        for (int i = 0; i < 3; i++) tw[i] = A1[i] * t1[0] + A2[i] * t1[1] + A3[i] * t1[2];
        tws.push_back(make_double3(tw[0], tw[1], tw[2]));
        zvs.push_back(in.sp[s].zv);
        spc.push_back(s);
      }
    const double rcut = 30.0, rcut2 = rcut * rcut;
    const int ncell = std::max((int)std::round(5.0 * rcut / std::pow(S->omega, 1.0 / 3.0)), 2);
    std::vector<double3> rl;
    for (int i = -ncell; i <= ncell; i++)
      for (int j = -ncell; j <= ncell; j++)
        for (int k = -ncell; k <= ncell; k++) {
          double t[3], r2 = 0.0;
          for (int c = 0; c < 3; c++) {
            t[c] = (double)i * A1[c] + (double)j * A2[c] + (double)k * A3[c];
            r2 = r2 + t[c] * t[c];
          }
          const bool nn = std::abs(i) <= 1 && std::abs(j) <= 1 && std::abs(k) <= 1;
          if (r2 <= rcut2 || nn) rl.push_back(make_double3(t[0], t[1], t[2]));
        }
    if (rl.size() > 40000) return fail(PSPW_ERR_SHAPE, "Ewald sum: more than 40000 lattice vectors");
    std::vector<double> rgs(nsp);
    for (int s = 0; s < nsp; s++) rgs[s] = in.sp[s].rgauss;
    const int nat = (int)tws.size(), nrvec = (int)rl.size();
    double3 *d_tau, *d_rl;
    double *d_zv, *d_rg, *d_part, *d_esr;
    int *d_sp;
    const long long pairs = (long long)nat * nrvec;
    const int nblk = (int)std::max<long long>(1, (pairs + kEwBlock - 1) / kEwBlock);
    if ((rc = tmp.up(&d_tau, tws, cst)) || (rc = tmp.up(&d_rl, rl, cst)) ||
        (rc = tmp.up(&d_zv, zvs, cst)) || (rc = tmp.up(&d_rg, rgs, cst)) ||
        (rc = tmp.up(&d_sp, spc, cst)) || (rc = tmp.get(&d_part, nblk)) ||
        (rc = tmp.get(&d_esr, 1)))
      return rc;
    PSPW_CUDA(cudaEventRecord(ev[6], cst));
    k_ewald<<<nblk, kEwBlock, 0, cst>>>(d_tau, d_zv, d_rg, d_sp, nat, d_rl, nrvec, d_part);
    k_sum_ordered<<<1, 32, 0, cst>>>(d_part, nblk, d_esr);
    PSPW_CUDA(cudaGetLastError());
    PSPW_CUDA(cudaEventRecord(ev[7], cst));
    PSPW_CUDA(cudaMemcpyAsync(&S->esr, d_esr, sizeof(double), cudaMemcpyDeviceToHost, cst));
    PSPW_CUDA(cudaStreamSynchronize(cst));
  }
  S->scf->esr = S->esr;
  float a = 0.f;
  cudaEventElapsedTime(&a, ev[0], ev[1]);
  S->ms[1] = a;
  cudaEventElapsedTime(&a, ev[1], ev[2]);
  S->ms[2] = a;
  cudaEventElapsedTime(&a, ev[2], ev[3]);
  S->ms[3] = a;
  cudaEventElapsedTime(&a, ev[4], ev[5]);
  S->ms[5] = a;
  cudaEventElapsedTime(&a, ev[6], ev[7]);
  S->ms[6] = a;
  return device_status(S->cell);
}

void system_free(pspw_system *S) {
  if (!S) return;
  if (S->device >= 0) cudaSetDevice(S->device);
  if (S->scf) pspw_scf_destroy(S->scf);
  if (S->cell) pspw_cell_destroy(S->cell);
  for (void *p : {(void *)S->d_eigr, (void *)S->d_sfac, (void *)S->d_vps, (void *)S->d_rhops,
                  (void *)S->d_pkg_a, (void *)S->d_rho_start})
    if (p) cudaFree(p);
  if (S->st) cudaStreamDestroy(S->st);
  delete S;
}

// glibc rand() after srand(seed), drawn from a private state (the same
// generator: random_r with a 128-byte TYPE_3 table), so the host
// application's rand() sequence is untouched.
struct GlibcRand {
  struct random_data rd;
  char state[128];
  explicit GlibcRand(unsigned seed) {
    std::memset(&rd, 0, sizeof rd);
    std::memset(state, 0, sizeof state);
    initstate_r(seed, state, sizeof state, &rd);
  }
  double next() {
    int32_t r = 0;
    random_r(&rd, &r);
    return r / 2147483647.0;
  }
};

}  // namespace
}  // namespace pspw

using namespace pspw;

extern "C" {

int pspw_system_load(const char *dir, int device, pspw_system **out) {
  if (!dir || !out) return fail(PSPW_ERR_ARG, "system_load: null argument");
  *out = nullptr;
  pspw_system *S = new pspw_system;
  S->device = device;
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = system_build(S, dir);
  S->ms[7] = ms_since(t0);  // including the release of the set-up temporaries
  if (rc) {
    system_free(S);
    return rc;
  }
  *out = S;
  return PSPW_OK;
}

int pspw_system_destroy(pspw_system *S) {
  system_free(S);
  return PSPW_OK;
}

int pspw_system_info(pspw_system *S, int *dims16, double *scal16) {
  if (!S) return fail(PSPW_ERR_ARG, "system_info: null handle");
  if (dims16) {
    const int d[16] = {S->nr[0], S->nr[1], S->nr[2], S->nnr,   S->ngw,       S->ngwx,
                       S->ng,    S->ngx,   S->nx,    S->nlmax, S->nax,       S->nsp,
                       S->in.nempty, S->in.iscf, S->in.nkpt, S->in.idiag};
    std::memcpy(dims16, d, sizeof d);
  }
  if (scal16) {
    const double v[16] = {S->tpiba, S->tpiba2, S->omega, S->alat, S->gcut, S->gcutw,
                          S->nel,   S->esr,    S->eself, S->in.ecut, S->wkpt, 0, 0, 0, 0, 0};
    std::memcpy(scal16, v, sizeof v);
  }
  return PSPW_OK;
}

int pspw_system_species(pspw_system *S, int *natoms, int *nproj) {
  if (!S || !natoms || !nproj) return fail(PSPW_ERR_ARG, "system_species: null argument");
  int na = 0, np = 0;
  for (int s = 0; s < S->nsp; s++) {
    na += S->na[s];
    np += S->na[s] * S->lm_end[s];
  }
  *natoms = na;
  *nproj = np;
  return PSPW_OK;
}

int pspw_system_params(pspw_system *S, pspw_scf_params *p) {
  if (!S || !p) return fail(PSPW_ERR_ARG, "system_params: null argument");
  const InputData &in = S->in;
  p->nx = S->nx;
  p->nempty = in.nempty;
  p->degree = in.chebypol_degree;
  p->max_scf_iter = in.max_scf_iter;
  p->conv = in.scf_conv_crit;
  p->imix = in.imix;
  p->mixdim = in.mixdim;
  p->mix_beta = in.rho_mix_fac;
  p->pulay_beta = 0.25;
  p->kerker_q0 = in.kerker_q0;
  p->idiag = in.idiag;
  p->max_diag_iter = in.user_max_diag_iter ? in.max_diag_iter : 0;
  p->filter_prec = PSPW_PREC_F64;
  p->tmetal = in.tmetal ? 1 : 0;
  p->ekt = in.ekt;
  return PSPW_OK;
}

int pspw_system_array(pspw_system *S, int which, void *host, long long nbytes) {
  if (!S || !host) return fail(PSPW_ERR_ARG, "system_array: null argument");
  if (S->device >= 0) PSPW_CUDA(cudaSetDevice(S->device));
  const void *src = nullptr;
  bool dev = false;
  size_t n = 0;
  std::vector<double> tmp;
  switch (which) {
    case PSPW_SYS_EIGR:
      src = S->d_eigr, dev = true, n = sizeof(double2) * (size_t)S->ngwx * S->nax * S->nsp;
      break;
    case PSPW_SYS_SFAC:
      src = S->d_sfac, dev = true, n = sizeof(double2) * (size_t)S->nsp * S->ng;
      break;
    case PSPW_SYS_VPS:
      src = S->d_vps, dev = true, n = sizeof(double) * (size_t)S->nsp * S->ng;
      break;
    case PSPW_SYS_RHOPS:
      src = S->d_rhops, dev = true, n = sizeof(double) * (size_t)S->nsp * S->ng;
      break;
    case PSPW_SYS_PKG_A:
      src = S->d_pkg_a, dev = true, n = sizeof(double) * (size_t)S->nlmax * S->ngwx * S->nsp;
      break;
    case PSPW_SYS_RHO_START:
      src = S->d_rho_start, dev = true, n = sizeof(double) * (size_t)S->nnr;
      break;
    case PSPW_SYS_WNL:
      src = S->wnl.data(), n = sizeof(double) * S->wnl.size();
      break;
    case PSPW_SYS_FOCC:
      src = S->focc.data(), n = sizeof(double) * S->focc.size();
      break;
    case PSPW_SYS_N123:
      src = S->n123.data(), n = sizeof(unsigned) * S->n123.size();
      break;
    case PSPW_SYS_XKG:
      src = S->xkg.data(), n = sizeof(double) * S->xkg.size();
      break;
    case PSPW_SYS_TAU:
      src = S->in.tau.data(), n = sizeof(double) * S->in.tau.size();
      break;
    case PSPW_SYS_G:
      src = S->g.data(), n = sizeof(double) * (size_t)S->ng;
      break;
    default:
      return fail(PSPW_ERR_ARG, "system_array: unknown array");
  }
  if ((long long)n != nbytes) return fail(PSPW_ERR_SHAPE, "system_array: wrong byte count");
  if (dev && !src) return fail(PSPW_ERR_ARG, "system_array: a host-only system has no device arrays");
  if (dev) {
    PSPW_CUDA(cudaMemcpy(host, src, n, cudaMemcpyDeviceToHost));
  } else if (n) {
    std::memcpy(host, src, n);
  }
  return PSPW_OK;
}

int pspw_system_cell(pspw_system *S, pspw_cell **cell) {
  if (!S || !cell) return fail(PSPW_ERR_ARG, "system_cell: null argument");
  if (!S->cell) return fail(PSPW_ERR_ARG, "system_cell: a host-only system has no cell");
  *cell = S->cell;
  return PSPW_OK;
}

int pspw_system_scf(pspw_system *S, pspw_scf **scf) {
  if (!S || !scf) return fail(PSPW_ERR_ARG, "system_scf: null argument");
  if (!S->scf) return fail(PSPW_ERR_ARG, "system_scf: a host-only system has no SCF handle");
  *scf = S->scf;
  return PSPW_OK;
}

int pspw_system_timing(pspw_system *S, double *ms8) {
  if (!S || !ms8) return fail(PSPW_ERR_ARG, "system_timing: null argument");
  std::memcpy(ms8, S->ms, sizeof S->ms);
  return PSPW_OK;
}

int pspw_system_cheby_scf(pspw_system *S, int filter_prec, const char *outdir, double *eig,
                          double *e6, int *iterations, int *converged, double *hist) {
  if (!S) return fail(PSPW_ERR_ARG, "system_cheby_scf: null argument");
  pspw_scf_params p;
  int rc = pspw_system_params(S, &p);
  if (rc) return rc;
  p.filter_prec = filter_prec;
  return pspw_system_cheby_scf_with(S, &p, outdir, eig, e6, iterations, converged, hist);
}

int pspw_system_cheby_scf_with(pspw_system *S, const pspw_scf_params *params, const char *outdir,
                               double *eig, double *e6, int *iterations, int *converged,
                               double *hist) {
  if (!S || !params || !eig || !e6 || !iterations || !converged)
    return fail(PSPW_ERR_ARG, "system_cheby_scf: null argument");
  if (!S->scf) return fail(PSPW_ERR_ARG, "system_cheby_scf: a host-only system");
  pspw_scf_params p = *params;
  if (p.nx != S->nx) return fail(PSPW_ERR_ARG, "system_cheby_scf: params.nx is not the system's NX");
  int rc = PSPW_OK;
  const int ngw = S->ngw, nx2 = S->nx + 2;
  // ChebySCFLoop.cpp:100-106 and 201-208: v0 (NGWX draws) then the random
  // start block, from rand() seeded 1 as in a fresh reference process
  GlibcRand rnd(1);
  std::vector<double> v0(2 * (size_t)S->ngwx), X(2 * (size_t)ngw * nx2, 0.0);
  for (int i = 0; i < S->ngwx; i++) {
    v0[2 * i] = rnd.next();
    v0[2 * i + 1] = rnd.next();
  }
  if (p.idiag < 0)
    for (size_t i = 0; i < (size_t)ngw * nx2; i++) {
      X[2 * i] = rnd.next();
      X[2 * i + 1] = rnd.next();
    }
  std::vector<double> rho0(S->nnr), rho1(S->nnr);
  PSPW_CUDA(cudaSetDevice(S->device));
  PSPW_CUDA(cudaMemcpy(rho0.data(), S->d_rho_start, sizeof(double) * S->nnr,
                       cudaMemcpyDeviceToHost));
  const std::string od = outdir ? outdir : "";
  if (outdir && (rc = write_3d_array(rho0.data(), S->nnr, join(od, "STARTING_RHO.dat"))))
    return fail(rc, "cannot write STARTING_RHO.dat");
  if ((rc = pspw_cheby_scf(S->scf, &p, S->focc.data(), rho0.data(), v0.data(), X.data(), eig,
                           rho1.data(), hist, iterations, converged, e6)))
    return rc;
  if (outdir && (rc = write_3d_array(rho1.data(), S->nnr, join(od, "FINAL_RHO.dat"))))
    return fail(rc, "cannot write FINAL_RHO.dat");
  return PSPW_OK;
}

int pspw_print_3d_array(const double *a, int n1, int n2, int n3, const char *path) {
  if (!a || !path || n1 < 0 || n2 < 0 || n3 < 0) return fail(PSPW_ERR_ARG, "print_3d_array: bad argument");
  const int rc = write_3d_array(a, (long long)n1 * n2 * n3, path);
  return rc ? fail(rc, std::string("cannot write ") + path) : PSPW_OK;
}

}  // extern "C"
