// C ABI entry points for H*psi and the Chebyshev filter.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "engine.h"

namespace pspw {
namespace {

__global__ void k_z_to_c(const double2 *__restrict__ a, int lda, float2 *__restrict__ b, int ldb,
                         int m, int n) {
  const size_t tot = (size_t)m * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot;
       i += (size_t)gridDim.x * blockDim.x) {
    const int col = (int)(i / m), row = (int)(i - (size_t)col * m);
    const double2 v = a[(size_t)col * lda + row];
    b[(size_t)col * ldb + row] = make_float2((float)v.x, (float)v.y);
  }
}

__global__ void k_c_to_z(const float2 *__restrict__ a, int lda, double2 *__restrict__ b, int ldb,
                         int m, int n) {
  const size_t tot = (size_t)m * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot;
       i += (size_t)gridDim.x * blockDim.x) {
    const int col = (int)(i / m), row = (int)(i - (size_t)col * m);
    const float2 v = a[(size_t)col * lda + row];
    b[(size_t)col * ldb + row] = make_double2((double)v.x, (double)v.y);
  }
}

template <typename T>
int copy_block(pspw_cell *c, const T *src, int lds, T *dst, int ldd, int m, int n) {
  PSPW_CUDA(cudaMemcpy2DAsync(dst, (size_t)ldd * sizeof(T), src, (size_t)lds * sizeof(T),
                              (size_t)m * sizeof(T), n, cudaMemcpyDeviceToDevice, c->stream));
  return PSPW_OK;
}

int check_cell(pspw_cell *c) {
  if (!c) return fail(PSPW_ERR_ARG, "null cell");
  PSPW_CUDA(cudaSetDevice(c->device));
  return PSPW_OK;
}

// X (ld) <-> Xs (ld ngw) between the caller's G order and the stick order
template <typename T>
__global__ void k_to_stick_order(const T *__restrict__ X, int ld, T *Xs, int ngw, int nb,
                                 const int *__restrict__ sg_ig) {
  const long long n = (long long)ngw * nb;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / ngw), k = (int)(i % ngw);
    Xs[i] = X[(size_t)b * ld + sg_ig[k]];
  }
}
template <typename T>
__global__ void k_from_stick_order(const T *__restrict__ Xs, int ldxs, T *X, int ld, int ngw,
                                   int nb, const int *__restrict__ sg_ig) {
  const long long n = (long long)ngw * nb;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(i / ngw), k = (int)(i % ngw);
    X[(size_t)b * ld + sg_ig[k]] = Xs[(size_t)b * ldxs + k];
  }
}

// The Chebyshev filter of chebyfilt.cpp:6-74 on a device block X (in place).
// Y_1 = (sigma1/e)(H X - c X); Y_d = (2 sigma_d/e)(H Y_{d-1} - c Y_{d-1})
// - sigma sigma_d Y_{d-2}; the three blocks rotate instead of being copied.
template <typename R>
int chebyfilt_dev(pspw_cell *c, void *Xv, int ld, int ngw, int nb, int degree, double lb,
                  double ub) {
  using T = cx<R>;
  if (degree < 1) return PSPW_OK;
  const double e = (ub - lb) / 2.0;
  const double cc = (ub + lb) / 2.0;
  double sigma = e / (lb - ub);
  const double sigma1 = sigma;
  T *X = static_cast<T *>(Xv);
  T *w1 = nullptr, *w2 = nullptr;
  const size_t blk = sizeof(T) * (size_t)ngw * nb;
  int rc = ws_reserve(c, 6, blk, (void **)&w1);
  if (rc) return rc;
  rc = ws_reserve(c, 7, blk, (void **)&w2);
  if (rc) return rc;
  // On the register-FFT path with the whole sphere the filter runs in the
  // stick order: the block is permuted once into it, every H*psi runs with
  // the cell's stick-order arrays swapped in (contiguous stick gathers and
  // scatters), and the result is permuted back.  The recurrence is the same
  // arithmetic on the same numbers in another order of G.
  const bool stick = c->basis.fast && ngw == c->basis.ngw;
  T *X0 = X;
  int ld0 = ld;
  if (stick) {
    T *xs = nullptr;
    if ((rc = ws_reserve(c, kWsStickX, blk, (void **)&xs))) return rc;
    const long long n = (long long)ngw * nb;
    k_to_stick_order<T><<<(unsigned)std::min<long long>((n + 255) / 256, 148 * 16), 256, 0,
                          c->stream>>>(X, ld, xs, ngw, nb, c->basis.d_sg_ig);
    c->kernel_launches++;
    PSPW_CUDA(cudaGetLastError());
    if ((rc = swap_stick_order(c))) return rc;
    X = xs;
    ld = ngw;
  }
  struct SwapBack {
    pspw_cell *c;
    bool on;
    ~SwapBack() {
      if (on) swap_stick_order(c);
    }
  } back{c, stick};
  // buffers: X (ld), w1, w2 (ld = ngw)
  T *buf[3] = {X, w1, w2};
  int lds[3] = {ld, ngw, ngw};
  // Y1 = (sigma1/e) H X + (-c sigma1/e) X
  rc = hpsi_apply<R>(c, X, ld, w1, ngw, ngw, nb, sigma1 / e, -cc * sigma1 / e, 0.0, nullptr, ngw);
  if (rc) return rc;
  int im2 = 0, im1 = 1;  // Y_{d-2} in buf[im2], Y_{d-1} in buf[im1]
  for (int d = 2; d <= degree; d++) {
    const double sigma2 = 1.0 / (2.0 / sigma1 - sigma);
    const int io = 3 - im2 - im1;
    rc = hpsi_apply<R>(c, buf[im1], lds[im1], buf[io], lds[io], ngw, nb, 2.0 * sigma2 / e,
                       -cc * 2.0 * sigma2 / e, -sigma * sigma2, buf[im2], lds[im2]);
    if (rc) return rc;
    // Y_{d-1} becomes Y_{d-2}; the slot Y_{d-2} had is reused for Y_{d+1}
    im2 = im1;
    im1 = io;
    sigma = sigma2;
  }
  if (stick) {
    back.on = false;
    if ((rc = swap_stick_order(c))) return rc;  // the cell's own order again
    const long long n = (long long)ngw * nb;
    k_from_stick_order<T><<<(unsigned)std::min<long long>((n + 255) / 256, 148 * 16), 256, 0,
                            c->stream>>>(buf[im1], lds[im1], X0, ld0, ngw, nb, c->basis.d_sg_ig);
    c->kernel_launches++;
    PSPW_CUDA(cudaGetLastError());
    return PSPW_OK;
  }
  if (im1 != 0) return copy_block<T>(c, buf[im1], lds[im1], X, ld, ngw, nb);
  return PSPW_OK;
}

}  // namespace
}  // namespace pspw

using namespace pspw;

extern "C" {

int pspw_apply_ham_block_dev(pspw_cell *c, int prec, const void *d_vin, void *d_vout, int ld,
                             int ngw, int nstates) {
  int rc = check_cell(c);
  if (rc) return rc;
  cudaEvent_t ev;
  timing_begin(c, 0, &ev);
  if (prec == PSPW_PREC_F64)
    rc = hpsi_apply<double>(c, d_vin, ld, d_vout, ld, ngw, nstates, 1.0, 0.0, 0.0, nullptr, ld);
  else if (prec == PSPW_PREC_F32)
    rc = hpsi_apply<float>(c, d_vin, ld, d_vout, ld, ngw, nstates, 1.0, 0.0, 0.0, nullptr, ld);
  else
    rc = fail(PSPW_ERR_ARG, "unknown precision");
  timing_end(c, 0, ev);
  return rc;
}

int pspw_apply_ham_block(pspw_cell *c, const double *vin, double *vout, int ngw, int nstates) {
  int rc = check_cell(c);
  if (rc) return rc;
  if (!vin || !vout) return fail(PSPW_ERR_ARG, "apply_ham_block: null buffer");
  if (nstates <= 0) return PSPW_OK;
  const size_t bytes = sizeof(double2) * (size_t)ngw * nstates;
  double2 *din = nullptr, *dout = nullptr;
  if ((rc = ws_reserve(c, 4, bytes, (void **)&din)) || (rc = ws_reserve(c, 5, bytes, (void **)&dout)))
    return rc;
  PSPW_CUDA(cudaMemcpyAsync(din, vin, bytes, cudaMemcpyHostToDevice, c->stream));
  rc = pspw_apply_ham_block_dev(c, PSPW_PREC_F64, din, dout, ngw, ngw, nstates);
  if (rc) return rc;
  PSPW_CUDA(cudaMemcpyAsync(vout, dout, bytes, cudaMemcpyDeviceToHost, c->stream));
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  return device_status(c);
}

int pspw_chebyfilt_dev(pspw_cell *c, int prec, void *d_X, int ld, int ngw, int nstates, int degree,
                       double lb, double ub) {
  int rc = check_cell(c);
  if (rc) return rc;
  if (!d_X || ld < ngw || nstates < 0) return fail(PSPW_ERR_ARG, "chebyfilt: bad block");
  if (nstates == 0) return PSPW_OK;
  if (!(ub > lb)) return fail(PSPW_ERR_ARG, "chebyfilt: need ub > lb");
  cudaEvent_t ev;
  timing_begin(c, 0, &ev);
  if (prec == PSPW_PREC_F64)
    rc = chebyfilt_dev<double>(c, d_X, ld, ngw, nstates, degree, lb, ub);
  else if (prec == PSPW_PREC_F32)
    rc = chebyfilt_dev<float>(c, d_X, ld, ngw, nstates, degree, lb, ub);
  else
    rc = fail(PSPW_ERR_ARG, "unknown precision");
  timing_end(c, 0, ev);
  return rc;
}

int pspw_chebyfilt(pspw_cell *c, double *X, int ngw, int nstates, int degree, double lb, double ub,
                   int prec) {
  int rc = check_cell(c);
  if (rc) return rc;
  if (!X) return fail(PSPW_ERR_ARG, "chebyfilt: null block");
  if (nstates <= 0) return PSPW_OK;
  if (prec != PSPW_PREC_F64 && prec != PSPW_PREC_F32)
    return fail(PSPW_ERR_ARG, "unknown precision");
  const size_t n = (size_t)ngw * nstates;
  double2 *dx = nullptr;
  float2 *fx = nullptr;
  if ((rc = ws_reserve(c, 4, n * sizeof(double2), (void **)&dx))) return rc;
  if (prec == PSPW_PREC_F32 && (rc = ws_reserve(c, 8, n * sizeof(float2), (void **)&fx)))
    return rc;
  // Bands are independent under the filter, so the block goes in two band
  // chunks: the copy stream brings chunk 1 in while the cell stream filters
  // chunk 0, and takes chunk 0 out while it filters chunk 1 (a block of fewer
  // than 32 bands goes whole).  Each chunk's copies and its filter are
  // ordered by events; the call returns after the last copy out.
  const int nchunk = nstates >= 32 ? 2 : 1;
  const int b_split = (nstates + 1) / 2;
  const int b0[2] = {0, nchunk == 2 ? b_split : nstates};
  const int nbc[2] = {nchunk == 2 ? b_split : nstates, nstates - b_split};
  cudaStream_t cs = c->stream_copy;
  double2 *hX = reinterpret_cast<double2 *>(X);
  for (int k = 0; k < nchunk; k++) {
    const size_t off = (size_t)b0[k] * ngw, bytes = sizeof(double2) * (size_t)nbc[k] * ngw;
    PSPW_CUDA(cudaMemcpyAsync(dx + off, hX + off, bytes, cudaMemcpyHostToDevice, cs));
    PSPW_CUDA(cudaEventRecord(c->ev_in[k], cs));
  }
  // every chunk's filter is enqueued before the copies out, so a copy into
  // pageable host memory (which returns only when done) still overlaps the
  // next chunk's filter
  int nready = 0;
  for (int k = 0; k < nchunk && rc == PSPW_OK; k++) {
    const size_t off = (size_t)b0[k] * ngw;
    PSPW_CUDA(cudaStreamWaitEvent(c->stream, c->ev_in[k], 0));
    if (prec == PSPW_PREC_F32) {
      k_z_to_c<<<4 * 148, 256, 0, c->stream>>>(dx + off, ngw, fx + off, ngw, ngw, nbc[k]);
      c->kernel_launches++;
      rc = pspw_chebyfilt_dev(c, PSPW_PREC_F32, fx + off, ngw, ngw, nbc[k], degree, lb, ub);
      if (rc) break;
      k_c_to_z<<<4 * 148, 256, 0, c->stream>>>(fx + off, ngw, dx + off, ngw, ngw, nbc[k]);
      c->kernel_launches++;
    } else {
      rc = pspw_chebyfilt_dev(c, PSPW_PREC_F64, dx + off, ngw, ngw, nbc[k], degree, lb, ub);
      if (rc) break;
    }
    PSPW_CUDA(cudaEventRecord(c->ev_out[k], c->stream));
    nready = k + 1;
  }
  for (int k = 0; k < nready && rc == PSPW_OK; k++) {
    const size_t off = (size_t)b0[k] * ngw, bytes = sizeof(double2) * (size_t)nbc[k] * ngw;
    PSPW_CUDA(cudaStreamWaitEvent(cs, c->ev_out[k], 0));
    PSPW_CUDA(cudaMemcpyAsync(hX + off, dx + off, bytes, cudaMemcpyDeviceToHost, cs));
  }
  // no copy may still be writing the caller's block when this returns
  PSPW_CUDA(cudaStreamSynchronize(cs));
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  if (rc) return rc;
  return device_status(c);
}

}  // extern "C"
