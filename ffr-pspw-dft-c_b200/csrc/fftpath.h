// The register-FFT local part of H*psi (fftpath.cuh), compiled per
// precision in fftpath_f32.cu / fftpath_f64.cu.
#pragma once

#include "common.cuh"
#include "engine.h"

namespace pspw {

// What the stick/plane kernels read about the basis (device pointers).
struct FastGeo {
  int ncol, nxa;
  const int *col_start, *sg_ig, *sg_z, *sg_col, *xa_list, *col_x, *col_y;
  const int *xa_of_x;  // [n1] active index of x, or -1
  // sg_ig is the identity (the block is in stick order): the kernels use k
  // itself, so the psi loads do not wait for an index load
  bool ig_iota = false;
};

// True when (n1, n2, n3) has compiled stick and plane kernels.
bool fast_supported(int n1, int n2, int n3);

// The Chebyshev recurrence applied by the last local pass:
// out = ca * (H_loc in) + cb * in + cg * xm2 when `on`.
template <typename T, typename R>
struct RecArg {
  bool on = false;
  R ca = 1, cb = 0, cg = 0;
  const T *xm2 = nullptr;
  int ldx = 0;
};

// Local part (kinetic + V_eff sandwich) of H*psi for nb bands:
// out = kin*in + FFT^-1 sandwich (or the recurrence of ra), on the cell
// stream.
template <typename R>
int local_fast(pspw_cell *c, const FastGeo &g, const cx<R> *in, int ld_in, cx<R> *out,
               int ld_out, int ngw, int nb, const ScratchPlan *plan, const RecArg<cx<R>, R> &ra);

// rho (device, natural grid order) += sum_b wband[b] |psi_b(r)|^2, with the
// scatter limited to G index < ngw_scatter.
template <typename R>
int rho_fast(pspw_cell *c, const FastGeo &g, const cx<R> *psi, int ld, int ngw_scatter, int nb,
             const double *d_wband, double *d_rho);

// The same on the generic FFT path (any grid length; hpsi.cu), FP64.
int rho_generic(pspw_cell *c, const double2 *psi, int ld, int ngw_scatter, int nb,
                const double *d_wband, double *d_rho);

}  // namespace pspw
