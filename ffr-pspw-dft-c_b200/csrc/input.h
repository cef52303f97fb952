// Host readers of the reference's input formats (input.cpp): the INPUT
// keyword file (ReadInputFile.cpp:5-217) and the FHI98 pseudopotential
// tables (ReadPseudopotentials.cpp:5-66), plus the Print3DArray text dump
// (Print3DArray.cpp:5-22).
#pragma once

#include <string>
#include <vector>

namespace pspw {

// The reference's radial-mesh capacity (common_pspw.h: MAXR) and angular
// momentum capacity (MAXAM).
constexpr int kMaxR = 570;
constexpr int kMaxAM = 3;

struct SpeciesData {
  std::string file;  // pseudopotential file named in INPUT (ATOMTYP)
  int na = 0, lmax = 0, lloc = 0;
  double rgauss = 1.0;  // RGAUSS default (ReadInputFile.cpp:60)
  // FHI98 table (ReadPseudopotentials.cpp): ZV, the mesh of the last channel
  // read, and per channel l = 1..lmax the wavefunction u_l(r) and V_l(r)
  double zv = 0.0;
  int mmax = 0;
  double clog = 0.0;  // log of the mesh ratio
  std::vector<double> r;
  std::vector<double> psi[kMaxAM], vion[kMaxAM];
};

struct InputData {
  // ReadInputFile.cpp:22-35 defaults (IMIX and the flags are zero-initialised
  // globals, global_variables.cpp)
  double ecut = 0.0;
  double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // A1, A2, A3
  int nsp = 0, nax = 0;
  std::vector<SpeciesData> sp;
  std::vector<double> tau;  // TAU(3, NAX, NSP), bohr after conversion
  std::string coord_type;
  int nkpt = 0;
  std::vector<double> xk, wkpt;
  int nempty = 5;
  bool tmetal = false;
  double ekt = 0.004;
  int max_scf_iter = 30;
  double scf_conv_crit = 1e-6, rho_mix_fac = 0.3, kerker_q0 = 0.5, betamax = 0.5;
  int mixdim = 4, idiag = 0, max_diag_iter = 30, iscf = 0, chebypol_degree = 10, imix = 0;
  bool user_max_diag_iter = false, diag_verbose = false, user_fft_grid = false;
  int nr[3] = {0, 0, 0};
};

// INPUT at `path`; pseudopotential names are kept as written.  Returns a
// PSPW_* status; *err names the offending line on failure.
int read_input_file(const std::string &path, InputData *in, std::string *err);
// FHI98 table of one species at `path` for channels 1..sp->lmax.
int read_fhi_file(const std::string &path, SpeciesData *sp, std::string *err);
// `%18.10f` per line, n values.
int write_3d_array(const double *a, long long n, const std::string &path);

}  // namespace pspw
