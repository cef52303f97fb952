// Internal interface of basis.cpp shared with the device set-up (geom.cu).
#pragma once

#include <vector>

namespace pspw {

// The one-dimensional phase tables EI1, EI2, EI3 of PhaseFactor.cpp:23-64:
// ei[d][2*((s*nax + a)*len[d] + zero[d]-1 + n) + {0,1}] = exp(-2 pi i n tau'_d)
// for the crystal coordinate tau'_d of atom a of species s and
// -(NR+1)/2 <= n <= (NR+1)/2; zero for atoms a >= na[s].
struct PhaseTables {
  int len[3] = {0, 0, 0}, zero[3] = {0, 0, 0};
  int nax = 0, nsp = 0;
  std::vector<double> ei[3];
};
// 3x3 inverse by cofactors in the operation order of matinv3x3.cpp,
// column-major HM(i,j) = hm[(j-1)*3 + i-1]
void matinv3(const double *hm, double *hi);
void phase_tables(const double *lattice9, const int nr[3], int nsp, const int *na,
                  const double *tau, PhaseTables *pt);

}  // namespace pspw
