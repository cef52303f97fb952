// Device-resident SCF pieces around the eigensolver (scf.cu): full-grid FP64
// FFT, EvalEnergy, xc_PZ, NormalizeRho, KerkerPrec and the density mixers,
// with the local-potential data and the mixing history kept on the device.
#pragma once

#include <vector>

#include "engine.h"

struct pspw_scf {
  pspw_cell *cell = nullptr;
  int device = 0;  // the cell's device, so destroy needs no live cell
  int ng = 0, nsp = 0;
  double omega = 0.0, nel = 0.0, esr = 0.0, eself = 0.0;
  int *d_gidx = nullptr;    // [ng] 0-based grid index of density G ig
  // [ng] 1 where ig is the last density G on its grid point: on a grid
  // smaller than the density sphere needs, several G alias onto one point and
  // the reference's sequential scatters leave the last one's value there
  unsigned char *d_glast = nullptr;
  double2 *d_vg = nullptr;  // [ng] V_H + V_loc per density G (EvalEnergy)
  double *d_g = nullptr;    // [ng] |G|^2 in (2 pi / alat)^2 units (G[0] = 0)
  double2 *d_vp = nullptr;  // [ng] sum_s SFAC(s,ig) VPS(s,ig)
  double2 *d_rp = nullptr;  // [ng] sum_s SFAC(s,ig) RHOPS(s,ig)
  double2 *d_grid = nullptr;  // NNR complex work grid
  double *d_vxc = nullptr;    // NNR
  double *d_tmp = nullptr;    // NNR real work vector
  double *d_part = nullptr;   // reduction partials
  double *h_part = nullptr;   // pinned copy of the reduced sums
  // density mixing (PSPW_MIX_*): history columns of NNR doubles
  int mix_kind = -1, mixdim = 0;
  double mix_beta = 0.0, mix_q0 = 0.0;
  double *d_hist = nullptr;   // rho_old history
  double *d_f = nullptr;      // residual history
  double *d_gm = nullptr;     // Anderson differences (2 columns); Broyden df then u
  std::vector<double> mix_a;  // Broyden's a(MIXDIM, MIXDIM), kept between calls
};

namespace pspw {

// In-place 3D FFT of the cell's full grid (n1 fastest), FP64, on the cell
// stream.  sign +1: exp(+iGr), unscaled (fft_fftw3 inverse); sign -1:
// exp(-iGr) then x 1/NNR (fft_fftw3 forward).
int grid_fft(pspw_cell *c, double2 *grid, int sign);

// Device versions of the pieces (all vectors NNR doubles on the device).
// e6 = {ETOT, EKIN, EHT, EPSEU, ENL, EXC}.
int eval_energy_dev(pspw_scf *s, double *d_rho, double ekin, double enl, double *e6);
int xc_pz_dev(pspw_scf *s, const double *d_rho, double *d_vxc, double *exc);
int normalize_rho_dev(pspw_scf *s, double *d_rho, double omega, double nel, int *warn);
int kerker_prec_dev(pspw_scf *s, double *d_x, double beta, double q0);
int mix_dev(pspw_scf *s, int iter, double *d_rhoe, double *d);

}  // namespace pspw
