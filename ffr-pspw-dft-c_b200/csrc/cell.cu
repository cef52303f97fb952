// Cell set-up (the engine side of SetupArrays_ApplyHam_cuda /
// CopyRho_ApplyHam_cuda, common_pspw.h:255-257), error state, workspaces and
// the optional device timing hooks.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "nl_tc.h"
#include "fft2.cuh"
#include "fftpath.h"

namespace pspw {

static thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? PSPW_ERR_OOM : PSPW_ERR_CUDA;
}

int ws_reserve(pspw_cell *c, int slot, size_t bytes, void **out) {
  Workspace &w = c->ws[slot];
  if (w.bytes < bytes) {
    if (w.ptr) {
      PSPW_CUDA(cudaStreamSynchronize(c->stream));
      PSPW_CUDA(cudaFree(w.ptr));
      w.ptr = nullptr;
      w.bytes = 0;
    }
    size_t want = bytes + bytes / 8;  // headroom for slightly larger later calls
    PSPW_CUDA(cudaMalloc(&w.ptr, want));
    w.bytes = want;
  }
  *out = w.ptr;
  return PSPW_OK;
}

int smem_allow_max(const void *kernel) {
  static std::mutex mu;
  static std::map<std::pair<int, const void *>, bool> done;
  int dev = 0;
  PSPW_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, kernel})) return PSPW_OK;
  cudaFuncAttributes a;
  PSPW_CUDA(cudaFuncGetAttributes(&a, kernel));
  int optin = 0;
  PSPW_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  PSPW_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 optin - (int)a.sharedSizeBytes));
  done[{dev, kernel}] = true;
  return PSPW_OK;
}

int device_status(pspw_cell *c) {
  volatile int *e = c->h_err;
  if (e && *e) {
    *e = 0;
    return fail(PSPW_ERR_TIMEOUT, "a tensor-core kernel gave up waiting on its pipeline barrier");
  }
  return PSPW_OK;
}

void timing_begin(pspw_cell *c, int family, cudaEvent_t *ev) {
  *ev = nullptr;
  if (!(c->timing.mask & (1 << family))) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, c->stream);
  *ev = e;
}

void timing_end(pspw_cell *c, int family, cudaEvent_t ev) {
  if (!ev) return;
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, c->stream);
  c->timing.pending.push_back({family, {ev, e}});
}

static int drain_timing(pspw_cell *c) {
  if (c->timing.pending.empty()) return PSPW_OK;
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  for (auto &p : c->timing.pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.second.first, p.second.second);
    c->timing.ms[p.first] += ms;
    c->timing.launches[p.first] += 1;
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  c->timing.pending.clear();
  return PSPW_OK;
}

namespace {

int factor_radices(int n, int *rad, int *nf) {
  int k = 0;
  auto push = [&](int r) {
    if (k >= kMaxStages) return false;
    rad[k++] = r;
    return true;
  };
  while (n % 4 == 0) {
    if (!push(4)) return PSPW_ERR_NOT_IMPL;
    n /= 4;
  }
  while (n % 2 == 0) {
    if (!push(2)) return PSPW_ERR_NOT_IMPL;
    n /= 2;
  }
  for (int p = 3; n > 1; p += 2) {
    while (n % p == 0) {
      if (p > 64) return PSPW_ERR_NOT_IMPL;
      if (!push(p)) return PSPW_ERR_NOT_IMPL;
      n /= p;
    }
  }
  *nf = k;
  return PSPW_OK;
}

// A synchronous copy from pageable host memory returns once the data is
// staged, before its DMA has landed, and the engine's streams are
// non-blocking (not ordered after the legacy stream that copy runs on): the
// legacy stream is synchronised before any kernel may read the table.
template <typename T>
int upload(T **d, const std::vector<T> &h) {
  PSPW_CUDA(cudaMalloc((void **)d, std::max<size_t>(1, h.size()) * sizeof(T)));
  if (!h.empty()) {
    PSPW_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    PSPW_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
  }
  return PSPW_OK;
}

// exp(2 pi i t / n) with the angle reduced exactly to the first half
// quadrant (integer arithmetic) and exact values at multiples of 30 and 45
// degrees, so the table is symmetric to the last bit.
void root_of_unity(long t, long n, double *c, double *s) {
  t %= n;
  const long q = (4 * t) / n;           // quadrant
  long rem = 4 * t - q * n;             // quarter-turn fraction rem/n
  const bool flip = 2 * rem > n;
  if (flip) rem = n - rem;
  double cc, ss;
  if (rem == 0) {
    cc = 1.0;
    ss = 0.0;
  } else if (3 * rem == n) {
    cc = std::sqrt(3.0) / 2.0;
    ss = 0.5;
  } else if (2 * rem == n) {
    cc = ss = std::sqrt(0.5);
  } else {
    const double a = (M_PI / 2.0) * (double)rem / (double)n;
    cc = std::cos(a);
    ss = std::sin(a);
  }
  if (flip) std::swap(cc, ss);
  for (long k = 0; k < q; k++) {
    const double tmp = cc;
    cc = -ss;
    ss = tmp;
  }
  *c = cc + 0.0;
  *s = ss + 0.0;
}

int make_dim(FftDim &d, int n) {
  d.n = n;
  int rc = factor_radices(n, d.rad, &d.nf);
  if (rc) return fail(rc, "FFT length " + std::to_string(n) + " has a prime factor > 64");
  std::vector<double2> w64(n);
  std::vector<float2> w32(n);
  for (int t = 0; t < n; t++) {
    double c, s;
    root_of_unity(t, n, &c, &s);
    w64[t] = make_double2(c, s);
    w32[t] = make_float2((float)c, (float)s);
  }
  if ((rc = upload(&d.d_w64, w64))) return rc;
  return upload(&d.d_w32, w32);
}

}  // namespace

}  // namespace pspw

using namespace pspw;

extern "C" {

const char *pspw_error_string(int code) {
  switch (code) {
    case PSPW_OK: return "ok";
    case PSPW_ERR_ARG: return "invalid argument";
    case PSPW_ERR_SHAPE: return "inconsistent sizes";
    case PSPW_ERR_CUDA: return "CUDA error";
    case PSPW_ERR_OOM: return "device out of memory";
    case PSPW_ERR_NONFINITE: return "non-finite input";
    case PSPW_ERR_TIMEOUT: return "device wait timed out";
    case PSPW_ERR_LAPACK: return "dense factorisation failed";
    case PSPW_ERR_CHARGE: return "wrong charge density in G-space";
    case PSPW_ERR_NOT_IMPL: return "not implemented";
    default: return "unknown error";
  }
}

const char *pspw_last_error(void) { return g_last_error.c_str(); }

int pspw_version(void) { return 100; }

int pspw_cell_destroy(pspw_cell *c) {
  if (!c) return PSPW_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->stream2) cudaStreamSynchronize(c->stream2);
  if (c->stream_copy) cudaStreamSynchronize(c->stream_copy);
  Basis &B = c->basis;
  void *ptrs[] = {B.d_col_start, B.d_sg_ig, B.d_sg_z, B.d_sg_col, B.d_sg_off, B.d_col_of_xy,
                  B.d_xa_list,
                  B.d_xa_of_x, B.d_kin64, B.d_kin32, B.d_xkg64, c->proj.d_eigr64, c->proj.d_eigr32,
                  c->proj.d_pkga64, c->proj.d_pkga32, c->proj.d_patom, c->proj.d_psp,
                  c->proj.d_plm, c->proj.d_pw64, c->proj.d_pw32, c->d_veff64, c->d_veff32,
                  B.d_col_x, B.d_col_y, B.d_pinv[0], B.d_pinv[1], B.d_pinv[2], c->d_vperm64,
                  c->d_vperm32, c->proj.d_etp, c->proj.d_etb, B.d_wgrid, c->proj.d_beta64,
                  c->stick.sg_ig, c->stick.kin64, c->stick.kin32, c->stick.eigr64,
                  c->stick.eigr32, c->stick.pkga64, c->stick.pkga32, c->stick.etp,
                  c->stick.etb, c->stick.beta64};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (int i = 0; i < 3; i++) {
    if (B.dim[i].d_w64) cudaFree(B.dim[i].d_w64);
    if (B.dim[i].d_w32) cudaFree(B.dim[i].d_w32);
  }
  for (auto &w : c->ws)
    if (w.ptr) cudaFree(w.ptr);
  if (c->h_err) cudaFreeHost(c->h_err);
  for (auto &p : c->timing.pending) {
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  if (c->cusolver) cusolverDnDestroy(static_cast<cusolverDnHandle_t>(c->cusolver));
  if (c->cublas) cublasDestroy(static_cast<cublasHandle_t>(c->cublas));
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->stream2) cudaStreamDestroy(c->stream2);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->stream_copy) cudaStreamDestroy(c->stream_copy);
  for (int i = 0; i < 2; i++) {
    if (c->ev_in[i]) cudaEventDestroy(c->ev_in[i]);
    if (c->ev_out[i]) cudaEventDestroy(c->ev_out[i]);
  }
  delete c;
  return PSPW_OK;
}

int pspw_cell_create(pspw_cell **out, int device, int nr1, int nr2, int nr3, int ngw, int ngwx,
                     const unsigned int *n123, const double *xkg, double tpiba2, int nsp,
                     const int *na, int nax, const int *lm_end, int nlmax, const double *eigr,
                     const double *pkg_a, const double *wnl) {
  return pspw::cell_create(out, device, nr1, nr2, nr3, ngw, ngwx, n123, xkg, tpiba2, nsp, na, nax,
                           lm_end, nlmax, eigr, pkg_a, wnl, nullptr, nullptr);
}

}  // extern "C"

namespace pspw {
namespace {

// Projector arrays of the cell from device copies of EIGR(NGWX, NAX, NSP) and
// PKG_A(NLMAX, NGWX, NSP): the same packing as the host loop of cell_create.
__global__ void k_pack_projectors(const double2 *__restrict__ eigr, const double *__restrict__ pkga,
                                  const int *__restrict__ atom_col, int nat, int ngw, int ngwx,
                                  int nsp, int nlmax, double2 *e64, float2 *e32, double *k64,
                                  float *k32) {
  const long long ne = (long long)nat * ngw, nk = (long long)nsp * ngw * 4;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ne + nk;
       i += (long long)gridDim.x * blockDim.x) {
    if (i < ne) {
      const int ga = (int)(i / ngw), ig = (int)(i % ngw);
      const double2 v = eigr[(size_t)atom_col[ga] * ngwx + ig];
      e64[i] = v;
      e32[i] = make_float2((float)v.x, (float)v.y);
    } else {
      const long long j = i - ne;
      const int lm = (int)(j % 4), ig = (int)((j / 4) % ngw), s = (int)(j / (4LL * ngw));
      const double v = lm < nlmax ? pkga[((size_t)s * ngwx + ig) * nlmax + lm] : 0.0;
      k64[j] = v;
      k32[j] = (float)v;
    }
  }
}

}  // namespace

int cell_create(pspw_cell **out, int device, int nr1, int nr2, int nr3, int ngw, int ngwx,
                const unsigned int *n123, const double *xkg, double tpiba2, int nsp, const int *na,
                int nax, const int *lm_end, int nlmax, const double *eigr, const double *pkg_a,
                const double *wnl, const double2 *d_eigr, const double *d_pkg_a) {
  if (!out || !n123 || !xkg || !na || !lm_end) return fail(PSPW_ERR_ARG, "cell_create: null argument");
  *out = nullptr;
  if (nr1 < 1 || nr2 < 1 || nr3 < 1 || ngw < 1 || ngwx < ngw || nsp < 0 || nax < 0 || nlmax < 0)
    return fail(PSPW_ERR_ARG, "cell_create: bad sizes");
  const long long nnr_ll = (long long)nr1 * nr2 * nr3;
  if (nnr_ll > (1LL << 31) - 1) return fail(PSPW_ERR_SHAPE, "cell_create: grid too large");
  int nat = 0, nproj = 0;
  for (int s = 0; s < nsp; s++) {
    if (na[s] < 0 || na[s] > nax) return fail(PSPW_ERR_ARG, "cell_create: na > nax");
    if (lm_end[s] > 4)
      return fail(PSPW_ERR_NOT_IMPL, "lm_end > 4 is not implemented (ApplyHam_block.cpp:70-73)");
    if (lm_end[s] > nlmax) return fail(PSPW_ERR_SHAPE, "cell_create: lm_end > nlmax");
    nat += na[s];
    nproj += na[s] * std::max(0, lm_end[s]);
  }
  const bool dev_src = d_eigr && d_pkg_a;
  if (nproj > 0 && (!wnl || (!dev_src && (!eigr || !pkg_a))))
    return fail(PSPW_ERR_ARG, "cell_create: null projector arrays");
  PSPW_CUDA(cudaSetDevice(device));
  pspw_cell *c = new pspw_cell();
  c->device = device;
  c->ngwx = ngwx;
  int rc = PSPW_OK;
  auto bail = [&](int code) {
    pspw_cell_destroy(c);
    return code;
  };
  if (cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(PSPW_ERR_CUDA, "cell_create: projection stream"));
  if (cudaStreamCreateWithFlags(&c->stream_copy, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(PSPW_ERR_CUDA, "cell_create: copy stream"));
  for (int i = 0; i < 2; i++)
    if (cudaEventCreateWithFlags(&c->ev_in[i], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_out[i], cudaEventDisableTiming) != cudaSuccess)
      return bail(fail(PSPW_ERR_CUDA, "cell_create: copy events"));
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(PSPW_ERR_CUDA, "cell_create: stream"));
  Basis &B = c->basis;
  B.n1 = nr1;
  B.n2 = nr2;
  B.n3 = nr3;
  B.nnr = (int)nnr_ll;
  B.ngw = ngw;
  // ---- sticks
  std::vector<int> gi1(ngw), gi2(ngw), gi3(ngw);
  std::vector<int> col_of_xy((size_t)nr1 * nr2, -1);
  for (int ig = 0; ig < ngw; ig++) {
    const long long idx = (long long)n123[ig] - 1;
    if (idx < 0 || idx >= nnr_ll) return bail(fail(PSPW_ERR_SHAPE, "cell_create: N123 outside the grid"));
    gi1[ig] = (int)(idx % nr1);
    gi2[ig] = (int)((idx / nr1) % nr2);
    gi3[ig] = (int)(idx / ((long long)nr1 * nr2));
    col_of_xy[(size_t)gi1[ig] + (size_t)nr1 * gi2[ig]] = 0;
  }
  int ncol = 0;
  std::vector<int> col_x, col_y;
  for (int y = 0; y < nr2; y++)
    for (int x = 0; x < nr1; x++)
      if (col_of_xy[(size_t)x + (size_t)nr1 * y] == 0) {
        col_of_xy[(size_t)x + (size_t)nr1 * y] = ncol++;
        col_x.push_back(x);
        col_y.push_back(y);
      }
  std::vector<int> cnt(ncol + 1, 0);
  for (int ig = 0; ig < ngw; ig++) cnt[col_of_xy[(size_t)gi1[ig] + (size_t)nr1 * gi2[ig]] + 1]++;
  for (int k = 0; k < ncol; k++) cnt[k + 1] += cnt[k];
  std::vector<int> col_start = cnt;
  std::vector<std::pair<int, int>> entries(ngw);  // (stick, z) per G, sorted later
  std::vector<int> order(ngw);
  for (int ig = 0; ig < ngw; ig++) order[ig] = ig;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const int ca = col_of_xy[(size_t)gi1[a] + (size_t)nr1 * gi2[a]];
    const int cb = col_of_xy[(size_t)gi1[b] + (size_t)nr1 * gi2[b]];
    return ca != cb ? ca < cb : gi3[a] < gi3[b];
  });
  std::vector<int> sg_ig(ngw), sg_z(ngw), sg_col(ngw);
  std::vector<unsigned short> sg_off(ngw);
  const int tile = stick_tile(nr3);
  for (int k = 0; k < ngw; k++) {
    const int ig = order[k];
    sg_ig[k] = ig;
    sg_z[k] = gi3[ig];
    sg_col[k] = col_of_xy[(size_t)gi1[ig] + (size_t)nr1 * gi2[ig]];
    // below 2^16 on every compiled length (at most 16 x 129); the generic
    // path does not read it
    sg_off[k] = (unsigned short)std::min(65535, (sg_col[k] % tile) * (nr3 + 1) + sg_z[k]);
  }
  std::vector<int> xa_of_x(nr1, -1), xa_list;
  for (int k = 0; k < ncol; k++) xa_of_x[col_x[k]] = 0;
  for (int x = 0; x < nr1; x++)
    if (xa_of_x[x] == 0) {
      xa_of_x[x] = (int)xa_list.size();
      xa_list.push_back(x);
    }
  B.ncol = ncol;
  B.nxa = (int)xa_list.size();
  std::vector<double> kin64(ngw), xkg64(xkg, xkg + ngw);
  std::vector<int> wgrid(ngw);
  for (int ig = 0; ig < ngw; ig++) wgrid[ig] = (int)(n123[ig] - 1);
  std::vector<float> kin32(ngw);
  c->tpiba2 = tpiba2;
  for (int ig = 0; ig < ngw; ig++) {
    kin64[ig] = 0.5 * xkg[ig] * tpiba2;  // ApplyHam_block.cpp:59, same rounding order
    kin32[ig] = (float)kin64[ig];
  }
  if ((rc = upload(&B.d_col_start, col_start)) || (rc = upload(&B.d_sg_ig, sg_ig)) ||
      (rc = upload(&B.d_sg_z, sg_z)) || (rc = upload(&B.d_sg_col, sg_col)) ||
      (rc = upload(&B.d_sg_off, sg_off)) ||
      (rc = upload(&B.d_col_of_xy, col_of_xy)) || (rc = upload(&B.d_xa_list, xa_list)) ||
      (rc = upload(&B.d_xa_of_x, xa_of_x)) || (rc = upload(&B.d_kin64, kin64)) ||
      (rc = upload(&B.d_xkg64, xkg64)) || (rc = upload(&B.d_wgrid, wgrid)) ||
      (rc = upload(&B.d_kin32, kin32)))
    return bail(rc);
  const int nr[3] = {nr1, nr2, nr3};
  for (int i = 0; i < 3; i++)
    if ((rc = make_dim(B.dim[i], nr[i]))) return bail(rc);
  // register-FFT path when all three lengths split into two register DFTs
  B.fast = !std::getenv("PSPW_GENERIC_FFT") && fast_supported(nr1, nr2, nr3);
  if (B.fast) {
    if ((rc = upload(&B.d_col_x, col_x)) || (rc = upload(&B.d_col_y, col_y))) return bail(rc);
    for (int i = 0; i < 3; i++) {
      const NSplit sp = nsplit_for(nr[i]);
      std::vector<int> pinv(nr[i]);
      for (int p = 0; p < nr[i]; p++) pinv[p] = p / sp.n1 + sp.n2 * (p % sp.n1);
      if ((rc = upload(&B.d_pinv[i], pinv))) return bail(rc);
    }
    if (cudaMalloc(&c->d_vperm64, (size_t)B.nnr * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->d_vperm32, (size_t)B.nnr * sizeof(float)) != cudaSuccess)
      return bail(fail(PSPW_ERR_OOM, "cell_create: permuted V_eff"));
  }
  // ---- projectors, species-major then atom then lm (ApplyHam_block.cpp:68-117)
  Projectors &P = c->proj;
  P.nat = nat;
  P.nsp = nsp;
  P.nproj = nproj;
  P.sp_na.assign(na, na + nsp);
  P.sp_lm.assign(lm_end, lm_end + nsp);
  if (nproj > 0) {
    std::vector<double2> e64(dev_src ? 0 : (size_t)nat * ngw);
    std::vector<float2> e32(dev_src ? 0 : (size_t)nat * ngw);
    std::vector<double> k64(dev_src ? 0 : (size_t)nsp * ngw * 4, 0.0);
    std::vector<float> k32(dev_src ? 0 : (size_t)nsp * ngw * 4, 0.f);
    std::vector<int> patom, psp, plm, atom_col;
    std::vector<double> pw64;
    std::vector<float> pw32;
    int ga = 0;
    for (int s = 0; s < nsp; s++) {
      for (int a = 0; a < na[s]; a++, ga++) {
        atom_col.push_back(s * nax + a);
        for (int ig = 0; ig < ngw && !dev_src; ig++) {
          const double *src = eigr + 2 * (((size_t)s * nax + a) * ngwx);
          e64[(size_t)ga * ngw + ig] = make_double2(src[2 * ig], src[2 * ig + 1]);
          e32[(size_t)ga * ngw + ig] = make_float2((float)src[2 * ig], (float)src[2 * ig + 1]);
        }
        for (int lm = 0; lm < lm_end[s]; lm++) {
          patom.push_back(ga);
          psp.push_back(s);
          plm.push_back(lm);
          const double wv = wnl[(size_t)lm * nsp + s];  // WNL(is,lm), NSP leading
          pw64.push_back(wv);
          pw32.push_back((float)wv);
        }
      }
      for (int ig = 0; ig < ngw && !dev_src; ig++)
        for (int lm = 0; lm < std::min(4, nlmax); lm++) {
          const double v = pkg_a[((size_t)s * ngwx + ig) * nlmax + lm];  // PKG_A(lm,ig,is)
          k64[((size_t)s * ngw + ig) * 4 + lm] = v;
          k32[((size_t)s * ngw + ig) * 4 + lm] = (float)v;
        }
    }
    if (dev_src) {
      int *d_col = nullptr;
      if ((rc = upload(&d_col, atom_col))) return bail(rc);
      const size_t ne = (size_t)nat * ngw, nk = (size_t)nsp * ngw * 4;
      const bool ok = cudaMalloc(&P.d_eigr64, ne * sizeof(double2)) == cudaSuccess &&
                      cudaMalloc(&P.d_eigr32, ne * sizeof(float2)) == cudaSuccess &&
                      cudaMalloc(&P.d_pkga64, nk * sizeof(double)) == cudaSuccess &&
                      cudaMalloc(&P.d_pkga32, nk * sizeof(float)) == cudaSuccess;
      if (ok) {
        const int blocks = (int)std::min<size_t>((ne + nk + 255) / 256, 148 * 16);
        k_pack_projectors<<<blocks, 256, 0, c->stream>>>(d_eigr, d_pkg_a, d_col, nat, ngw, ngwx,
                                                         nsp, nlmax,
                                                         P.d_eigr64, P.d_eigr32, P.d_pkga64,
                                                         P.d_pkga32);
        c->kernel_launches++;
      }
      const cudaError_t e = ok ? cudaStreamSynchronize(c->stream) : cudaErrorMemoryAllocation;
      cudaFree(d_col);
      if (e != cudaSuccess) return bail(fail(ok ? PSPW_ERR_CUDA : PSPW_ERR_OOM, "cell_create: packing projectors"));
    } else if ((rc = upload(&P.d_eigr64, e64)) || (rc = upload(&P.d_eigr32, e32)) ||
               (rc = upload(&P.d_pkga64, k64)) || (rc = upload(&P.d_pkga32, k32))) {
      return bail(rc);
    }
    if ((rc = upload(&P.d_patom, patom)) || (rc = upload(&P.d_psp, psp)) ||
        (rc = upload(&P.d_plm, plm)) || (rc = upload(&P.d_pw64, pw64)) ||
        (rc = upload(&P.d_pw32, pw32)))
      return bail(rc);
  }
  if (cudaMalloc(&c->d_veff64, (size_t)B.nnr * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&c->d_veff32, (size_t)B.nnr * sizeof(float)) != cudaSuccess)
    return bail(fail(PSPW_ERR_OOM, "cell_create: V_eff"));
  if (cudaHostAlloc((void **)&c->h_err, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&c->d_err, c->h_err, 0) != cudaSuccess)
    return bail(fail(PSPW_ERR_OOM, "cell_create: error word"));
  *c->h_err = 0;
  if ((rc = pspw::nl_tc_prepare(c))) return bail(rc);
  *out = c;
  return PSPW_OK;
}

namespace {

// out[(r * ngw + k) * inner + q] = in[(r * ngw + sg_ig[k]) * inner + q]
template <typename T>
__global__ void k_gather_stick_order(const T *__restrict__ in, int rows, int ngw, int inner,
                                     const int *__restrict__ sg_ig, T *out) {
  const long long n = (long long)rows * ngw * inner;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(i % inner), k = (int)((i / inner) % ngw), r = (int)(i / ((long long)inner * ngw));
    out[i] = in[((size_t)r * ngw + sg_ig[k]) * inner + q];
  }
}

__global__ void k_iota(int *a, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

template <typename T>
int gather_copy(pspw_cell *c, const T *in, int rows, int inner, T **out) {
  if (!in || rows <= 0) return PSPW_OK;
  const int ngw = c->basis.ngw;
  const size_t n = (size_t)rows * ngw * inner;
  if (cudaMalloc(out, n * sizeof(T)) != cudaSuccess) return fail(PSPW_ERR_OOM, "stick-order copies");
  k_gather_stick_order<T><<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0,
                            c->stream>>>(in, rows, ngw, inner, c->basis.d_sg_ig, *out);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

}  // namespace

int swap_stick_order(pspw_cell *c) {
  Basis &B = c->basis;
  Projectors &P = c->proj;
  auto &S = c->stick;
  if (!S.built) {
    int rc;
    if (cudaMalloc(&S.sg_ig, sizeof(int) * (size_t)B.ngw) != cudaSuccess)
      return fail(PSPW_ERR_OOM, "stick-order copies");
    k_iota<<<(B.ngw + 255) / 256, 256, 0, c->stream>>>(S.sg_ig, B.ngw);
    c->kernel_launches++;
    if ((rc = gather_copy(c, B.d_kin64, 1, 1, &S.kin64)) ||
        (rc = gather_copy(c, B.d_kin32, 1, 1, &S.kin32)) ||
        (rc = gather_copy(c, P.d_eigr64, P.nproj > 0 ? P.nat : 0, 1, &S.eigr64)) ||
        (rc = gather_copy(c, P.d_eigr32, P.nproj > 0 ? P.nat : 0, 1, &S.eigr32)) ||
        (rc = gather_copy(c, P.d_pkga64, P.nproj > 0 ? P.nsp : 0, 4, &S.pkga64)) ||
        (rc = gather_copy(c, P.d_pkga32, P.nproj > 0 ? P.nsp : 0, 4, &S.pkga32)))
      return rc;
    if (P.d_etp && S.eigr32 && (rc = nl_tc_build_tiles(c, S.eigr32, &S.etp, &S.etb))) return rc;
    S.built = true;
  }
  std::swap(B.d_sg_ig, S.sg_ig);
  std::swap(B.d_kin64, S.kin64);
  std::swap(B.d_kin32, S.kin32);
  std::swap(P.d_eigr64, S.eigr64);
  std::swap(P.d_eigr32, S.eigr32);
  std::swap(P.d_pkga64, S.pkga64);
  std::swap(P.d_pkga32, S.pkga32);
  std::swap(P.d_etp, S.etp);
  std::swap(P.d_etb, S.etb);
  std::swap(P.d_beta64, S.beta64);
  S.active = !S.active;
  return PSPW_OK;
}

}  // namespace pspw

namespace pspw {
namespace {

// V_eff/NNR gathered into the digit-permuted order of the register-FFT path,
// each z-plane stored x-major (z, x, y): the plane kernel's fused x step
// reads, for one x position, the rows of 32 consecutive y in one coalesced
// load.
__global__ void k_veff_perm(const double *__restrict__ v, int n1, int n2, int n3, double s,
                            const int *__restrict__ px, const int *__restrict__ py,
                            const int *__restrict__ pz, double *o64, float *o32) {
  const int n = n1 * n2 * n3;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int b = i % n2, a = (i / n2) % n1, cz = i / (n1 * n2);
    const double x = v[((size_t)pz[cz] * n2 + py[b]) * n1 + px[a]] * s;
    o64[i] = x;
    o32[i] = (float)x;
  }
}

__global__ void k_veff_scale(const double *__restrict__ v, int n, double s, double *o64,
                             float *o32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = v[i] * s;
    o64[i] = x;
    o32[i] = (float)x;
  }
}

}  // namespace
}  // namespace pspw

extern "C" {

int pspw_cell_set_veff_device(pspw_cell *c, const double *d_veff, int nnr) {
  if (!c || !d_veff) return fail(PSPW_ERR_ARG, "set_veff: null argument");
  if (nnr != c->basis.nnr) return fail(PSPW_ERR_SHAPE, "nnr != NNR (ApplyHam_block.cpp:18-21)");
  PSPW_CUDA(cudaSetDevice(c->device));
  k_veff_scale<<<2 * 148, 256, 0, c->stream>>>(d_veff, nnr, 1.0 / (double)nnr, c->d_veff64,
                                                c->d_veff32);
  c->kernel_launches++;
  const Basis &B = c->basis;
  if (B.fast) {
    k_veff_perm<<<2 * 148, 256, 0, c->stream>>>(d_veff, B.n1, B.n2, B.n3, 1.0 / (double)nnr,
                                                 B.d_pinv[0], B.d_pinv[1], B.d_pinv[2],
                                                 c->d_vperm64, c->d_vperm32);
    c->kernel_launches++;
  }
  PSPW_CUDA(cudaGetLastError());
  c->veff_set = true;
  return PSPW_OK;
}

int pspw_cell_set_veff(pspw_cell *c, const double *veff, int nnr) {
  if (!c || !veff) return fail(PSPW_ERR_ARG, "set_veff: null argument");
  if (nnr != c->basis.nnr) return fail(PSPW_ERR_SHAPE, "nnr != NNR (ApplyHam_block.cpp:18-21)");
  PSPW_CUDA(cudaSetDevice(c->device));
  double *tmp = nullptr;
  int rc = ws_reserve(c, kWsVeffTmp, (size_t)nnr * sizeof(double), (void **)&tmp);
  if (rc) return rc;
  PSPW_CUDA(cudaMemcpyAsync(tmp, veff, (size_t)nnr * sizeof(double), cudaMemcpyHostToDevice,
                            c->stream));
  rc = pspw_cell_set_veff_device(c, tmp, nnr);
  if (rc) return rc;
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  return PSPW_OK;
}

int pspw_cell_get_stream(pspw_cell *c, void **stream) {
  if (!c || !stream) return fail(PSPW_ERR_ARG, "get_stream: null argument");
  *stream = (void *)c->stream;
  return PSPW_OK;
}

int pspw_cell_synchronize(pspw_cell *c) {
  if (!c) return fail(PSPW_ERR_ARG, "synchronize: null cell");
  PSPW_CUDA(cudaSetDevice(c->device));
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  return pspw::device_status(c);
}

int pspw_cell_sizes(pspw_cell *c, int *o) {
  if (!c || !o) return fail(PSPW_ERR_ARG, "sizes: null argument");
  o[0] = c->basis.n1;
  o[1] = c->basis.n2;
  o[2] = c->basis.n3;
  o[3] = c->basis.ngw;
  o[4] = c->basis.ncol;
  o[5] = c->basis.nxa;
  o[6] = c->proj.nat;
  o[7] = c->proj.nproj;
  return PSPW_OK;
}

int pspw_cell_set_band_batch(pspw_cell *c, int nbatch) {
  if (!c || nbatch < 0) return fail(PSPW_ERR_ARG, "set_band_batch: bad argument");
  c->band_batch = nbatch;
  return PSPW_OK;
}

int pspw_cell_set_nl_path(pspw_cell *c, int path) {
  if (!c || path < PSPW_NL_AUTO || path > PSPW_NL_TENSOR_CORE)
    return fail(PSPW_ERR_ARG, "set_nl_path: bad argument");
  const int keep = c->nl_path;
  c->nl_path = PSPW_NL_AUTO;
  if (path == PSPW_NL_TENSOR_CORE && !pspw::nl_tc_usable(c)) {
    c->nl_path = keep;
    return fail(PSPW_ERR_NOT_IMPL, "set_nl_path: tensor-core projector kernels need at most "
                                   "256 atoms and 4 projectors per atom in every species");
  }
  c->nl_path = path;
  return PSPW_OK;
}

int pspw_cell_set_nl_overlap(pspw_cell *c, int mode) {
  if (!c || mode < PSPW_OVERLAP_AUTO || mode > PSPW_OVERLAP_OFF)
    return fail(PSPW_ERR_ARG, "set_nl_overlap: bad argument");
  c->nl_overlap = mode;
  return PSPW_OK;
}

int pspw_cell_check_device_wait(pspw_cell *c, int complete) {
  if (!c) return fail(PSPW_ERR_ARG, "check_device_wait: null cell");
  PSPW_CUDA(cudaSetDevice(c->device));
  return pspw::nl_tc_wait_check(c, complete);
}

int pspw_timing_enable(pspw_cell *c, int mask) {
  if (!c) return fail(PSPW_ERR_ARG, "timing: null cell");
  c->timing.mask = mask;
  return PSPW_OK;
}

int pspw_timing_read(pspw_cell *c, int family, double *total_ms, long long *launches) {
  if (!c || family < 0 || family >= kNumFamilies) return fail(PSPW_ERR_ARG, "timing: bad argument");
  int rc = drain_timing(c);
  if (rc) return rc;
  if (total_ms) *total_ms = c->timing.ms[family];
  if (launches) *launches = c->timing.launches[family];
  return PSPW_OK;
}

int pspw_timing_reset(pspw_cell *c) {
  if (!c) return fail(PSPW_ERR_ARG, "timing: null cell");
  int rc = drain_timing(c);
  for (int i = 0; i < kNumFamilies; i++) {
    c->timing.ms[i] = 0;
    c->timing.launches[i] = 0;
  }
  return rc;
}

int pspw_kernel_launches(pspw_cell *c, long long *count) {
  if (!c || !count) return fail(PSPW_ERR_ARG, "kernel_launches: null argument");
  *count = c->kernel_launches;
  return PSPW_OK;
}

}  // extern "C"
