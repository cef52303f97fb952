// The register-FFT local part of H*psi (fftpath.cuh), compiled per
// precision in fftpath_f32.cu / fftpath_f64.cu.
#pragma once

#include "common.cuh"
#include "engine.h"

namespace pspw {

// Sticks per block of the stick kernels for a z length nz (their tile of
// sticks x (nz + 1) elements); the host's tile offsets use the same value.
__host__ __device__ constexpr int stick_tile(int nz) {
  return (2048 / nz) < 1 ? 1 : ((2048 / nz) > 32 ? 32 : (2048 / nz));
}

// What the stick/plane kernels read about the basis (device pointers).
struct FastGeo {
  int ncol, nxa;
  const int *col_start, *sg_ig, *sg_z, *sg_col, *xa_list, *col_x, *col_y;
  const int *xa_of_x;  // [n1] active index of x, or -1
  // sg_ig is the identity (the block is in stick order): the kernels use k
  // itself, so the psi loads do not wait for an index load
  bool ig_iota = false;
  // [ngw] offset of G entry k in its block's tile of the stick kernels,
  // (stick mod stick_tile(n3)) * (n3 + 1) + i3: k_sticks_inv's one 2-byte
  // load instead of the stick and z loads (39 -> 34 registers).
  // k_sticks_fwd keeps the two loads: with this one it took 40 registers
  // instead of 32 and held 6 blocks per SM instead of 8.
  const unsigned short *sg_off = nullptr;
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
