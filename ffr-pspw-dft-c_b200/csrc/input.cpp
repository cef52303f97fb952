// Readers of the reference's input formats, with the reference's parsing
// rules: keyword lines compared verbatim, values read from the following
// line (or as the next whitespace-separated token where the reference uses
// `>>`), unknown keywords rejected.  Where the reference would loop forever
// (a failed numeric token read leaves its stream failed, ReadInputFile.cpp:
// 37-41) or read past its arrays, these readers return an error instead.
#include "input.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>

#include "pspw_gpu.h"

namespace pspw {
namespace {

int bad(std::string *err, const std::string &msg, int code = PSPW_ERR_ARG) {
  if (err) *err = msg;
  return code;
}

}  // namespace

int read_input_file(const std::string &path, InputData *out, std::string *err) {
  std::ifstream f(path.c_str());
  if (!f.is_open()) return bad(err, "cannot open " + path);
  InputData d;
  std::string line, rest;
  // keyword -> reader of the value on the next line (ReadInputFile.cpp:97-186)
  auto next_line = [&]() -> const char * {
    std::getline(f, line);
    return line.c_str();
  };
  while (!f.eof()) {
    std::getline(f, line);
    if (f.fail() && !f.eof()) return bad(err, "INPUT: read error");
    const std::string key = line;
    if (key.empty()) continue;
    if (key == "ecut") {
      f >> d.ecut;
      if (f.fail()) return bad(err, "INPUT: ecut is not a number");
    } else if (key == "latvec") {
      for (int v = 0; v < 3; v++)
        std::sscanf(next_line(), "%lf %lf %lf", &d.a[3 * v], &d.a[3 * v + 1], &d.a[3 * v + 2]);
    } else if (key == "atoms") {
      // ReadInputFile.cpp:53-92: NSP; NA per species (tokens); per species
      // the file name token, a `LMAX LLOC` line, the coordinate-type token
      // and NA coordinate lines
      int nsp = 0;
      std::sscanf(next_line(), "%d", &nsp);
      if (nsp < 1 || nsp > 4096) return bad(err, "INPUT: bad number of species");
      d.nsp = nsp;
      d.sp.assign(nsp, SpeciesData());
      d.nax = 0;
      for (int is = 0; is < nsp; is++) {
        f >> d.sp[is].na;
        if (f.fail() || d.sp[is].na < 0) return bad(err, "INPUT: bad number of atoms");
        d.nax = std::max(d.nax, d.sp[is].na);
      }
      d.tau.assign((size_t)3 * d.nax * nsp, 0.0);
      for (int is = 0; is < nsp; is++) {
        f >> d.sp[is].file;
        std::getline(f, rest);
        std::sscanf(next_line(), "%d %d", &d.sp[is].lmax, &d.sp[is].lloc);
        f >> d.coord_type;
        std::getline(f, rest);
        if (f.fail()) return bad(err, "INPUT: truncated atoms block");
        for (int ia = 0; ia < d.sp[is].na; ia++) {
          double *t = &d.tau[3 * ((size_t)is * d.nax + ia)];
          std::sscanf(next_line(), "%lf %lf %lf", &t[0], &t[1], &t[2]);
        }
      }
    } else if (key == "k_points") {
      std::sscanf(next_line(), "%d", &d.nkpt);
      if (d.nkpt < 1 || d.nkpt > 100000) return bad(err, "INPUT: bad number of k-points");
      d.xk.assign(3 * (size_t)d.nkpt, 0.0);
      d.wkpt.assign(d.nkpt, 0.0);
      for (int ik = 0; ik < d.nkpt; ik++)
        std::sscanf(next_line(), "%lf %lf %lf %lf", &d.xk[3 * ik], &d.xk[3 * ik + 1],
                    &d.xk[3 * ik + 2], &d.wkpt[ik]);
    } else if (key == "rho_mix_fac") {
      std::sscanf(next_line(), "%lf", &d.rho_mix_fac);
    } else if (key == "kerker_q0") {
      std::sscanf(next_line(), "%lf", &d.kerker_q0);
    } else if (key == "nempty") {
      std::sscanf(next_line(), "%d", &d.nempty);
    } else if (key == "tmetal") {
      if (std::string(next_line()) == " .true.") d.tmetal = true;
    } else if (key == "ekt") {
      std::sscanf(next_line(), "%lf", &d.ekt);
    } else if (key == "imix") {
      std::sscanf(next_line(), "%d", &d.imix);
    } else if (key == "mixdim") {
      std::sscanf(next_line(), "%d", &d.mixdim);
    } else if (key == "max_scf_iter") {
      std::sscanf(next_line(), "%d", &d.max_scf_iter);
    } else if (key == "scf_conv_crit") {
      std::sscanf(next_line(), "%lf", &d.scf_conv_crit);
    } else if (key == "fft_grid") {
      d.user_fft_grid = true;
      std::sscanf(next_line(), "%d %d %d", &d.nr[0], &d.nr[1], &d.nr[2]);
    } else if (key == "idiag") {
      std::sscanf(next_line(), "%d", &d.idiag);
    } else if (key == "max_diag_iter") {
      std::sscanf(next_line(), "%d", &d.max_diag_iter);
      d.user_max_diag_iter = true;
    } else if (key == "iscf") {
      std::sscanf(next_line(), "%d", &d.iscf);
    } else if (key == "chebypol_degree") {
      std::sscanf(next_line(), "%d", &d.chebypol_degree);
    } else if (key == "diag_verbose") {
      if (std::string(next_line()) == " .true.") d.diag_verbose = true;
    } else {
      return bad(err, "INPUT: unknown line '" + key + "'");
    }
  }
  if (d.nsp < 1) return bad(err, "INPUT: no atoms block");
  if (d.nkpt < 1) return bad(err, "INPUT: no k_points block");
  // coordinate conversion (ReadInputFile.cpp:190-214), by the coordinate
  // type of the last species.  "crystal" updates x, y, z in place one after
  // the other, so y and z see the already converted x (and z the new y), as
  // the reference does.
  for (int is = 0; is < d.nsp; is++)
    for (int ia = 0; ia < d.sp[is].na; ia++) {
      double *t = &d.tau[3 * ((size_t)is * d.nax + ia)];
      if (d.coord_type == "angstrom") {
        for (int i = 0; i < 3; i++) t[i] = t[i] / 0.529;
      } else if (d.coord_type == "crystal") {
        const double *A1 = d.a, *A2 = d.a + 3, *A3 = d.a + 6;
        t[0] = t[0] * A1[0] + t[1] * A2[0] + t[2] * A3[0];
        t[1] = t[0] * A1[1] + t[1] * A2[1] + t[2] * A3[1];
        t[2] = t[0] * A1[2] + t[1] * A2[2] + t[2] * A3[2];
      }
    }
  *out = d;
  return PSPW_OK;
}

int read_fhi_file(const std::string &path, SpeciesData *sp, std::string *err) {
  std::ifstream f(path.c_str());
  if (!f.is_open()) return bad(err, "cannot open pseudopotential " + path);
  std::string line;
  int nang = 0;
  std::getline(f, line);
  std::sscanf(line.c_str(), "%lf %d", &sp->zv, &nang);
  if (nang < sp->lmax)
    return bad(err, path + ": pseudopotential has fewer angular momenta than L_MAX");
  for (int i = 0; i < 10; i++) std::getline(f, line);  // Gaussian fit parameters, unused
  nang = std::min(nang, sp->lmax);
  if (nang > kMaxAM) return bad(err, path + ": more than 3 angular momenta", PSPW_ERR_NOT_IMPL);
  sp->r.assign(kMaxR, 0.0);
  for (int il = 0; il < kMaxAM; il++) {
    sp->psi[il].assign(kMaxR, 0.0);
    sp->vion[il].assign(kMaxR, 0.0);
  }
  for (int il = 0; il < nang; il++) {
    std::getline(f, line);
    double ratio = 0.0;
    if (std::sscanf(line.c_str(), "%d %lf", &sp->mmax, &ratio) != 2)
      return bad(err, path + ": missing mesh header");
    if (sp->mmax < 1 || sp->mmax > kMaxR)
      return bad(err, path + ": mesh size outside 1..570 (MAXR)");
    sp->clog = std::log(ratio);
    for (int ir = 0; ir < sp->mmax; ir++) {
      std::getline(f, line);
      int idx = 0;
      if (std::sscanf(line.c_str(), "%d %lf %lf %lf", &idx, &sp->r[ir], &sp->psi[il][ir],
                      &sp->vion[il][ir]) != 4)
        return bad(err, path + ": truncated radial table");
    }
  }
  return PSPW_OK;
}

int write_3d_array(const double *a, long long n, const std::string &path) {
  FILE *fp = std::fopen(path.c_str(), "w");
  if (!fp) return PSPW_ERR_ARG;
  for (long long i = 0; i < n; i++) std::fprintf(fp, "%18.10f\n", a[i]);
  return std::fclose(fp) == 0 ? PSPW_OK : PSPW_ERR_ARG;
}

}  // namespace pspw
