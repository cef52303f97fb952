// Plane-wave basis for one Gamma-point cell, built the way the reference's
// set-up builds it, so that a cell made here indexes its G vectors exactly
// like the reference program does (same sphere, same heap-sort order, same
// FFT-grid map and phase factors, bit for bit):
//   grid rule           Setup.cpp:20-34
//   ALAT/OMEGA/recip    Setup.cpp:39-46, determinant3x3.cpp, CalcRecipLatt.cpp:5-23
//   sphere counts       GVectorsGen0.cpp:5-64, NGWX rule Setup.cpp:64-66
//   half-space list,
//   heap-sort order,
//   +/-G expansion      GVectorsGen.cpp:5-137, sort1.cpp:5-55
//   wavefunction sphere GkVectorsGen.cpp:5-38
//   phase factors EIGR  PhaseFactor.cpp:5-80, matinv3x3.cpp
// The engine itself never needs this file: a caller of the drop-in hands over
// its own arrays.  It exists so the engine's workloads can be generated
// without the reference.  Compiled with -ffp-contract=off so every product
// and sum rounds as the reference's scalar code does.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pspw_gpu.h"
#include "basis.h"

namespace {

struct Lattice {
  double a1[3], a2[3], a3[3];
  double b1[3], b2[3], b3[3];
  double alat, omega;
};

double det3(const double *x, const double *y, const double *z) {
  return x[0] * (y[1] * z[2] - y[2] * z[1]) - x[1] * (y[0] * z[2] - y[2] * z[0]) +
         x[2] * (y[0] * z[1] - y[1] * z[0]);
}

// Reciprocal vectors in units of 2 pi / ALAT.  The component formulas are the
// reference's (CalcRecipLatt.cpp:9-21); they treat A1, A2, A3 as the columns of
// the cell matrix, which only matters for non-orthogonal cells.
void recip(Lattice &L) {
  const double s = L.alat / L.omega;
  const double *A1 = L.a1, *A2 = L.a2, *A3 = L.a3;
  L.b1[0] = (A2[1] * A3[2] - A2[2] * A3[1]) * s;
  L.b1[1] = (A1[2] * A3[1] - A1[1] * A3[2]) * s;
  L.b1[2] = (A1[1] * A2[2] - A1[2] * A2[1]) * s;
  L.b2[0] = (A2[2] * A3[0] - A2[0] * A3[2]) * s;
  L.b2[1] = (A1[0] * A3[2] - A1[2] * A3[0]) * s;
  L.b2[2] = (A1[2] * A2[0] - A1[0] * A2[2]) * s;
  L.b3[0] = (A2[0] * A3[1] - A2[1] * A3[0]) * s;
  L.b3[1] = (A1[1] * A3[0] - A1[0] * A3[1]) * s;
  L.b3[2] = (A1[0] * A2[1] - A1[1] * A2[0]) * s;
}

Lattice make_lattice(const double *lat9) {
  Lattice L;
  for (int i = 0; i < 3; i++) {
    L.a1[i] = lat9[i];
    L.a2[i] = lat9[3 + i];
    L.a3[i] = lat9[6 + i];
  }
  L.alat = L.a1[0];
  L.omega = det3(L.a1, L.a2, L.a3);
  recip(L);
  return L;
}

int grid_rule(double ecut, const double *a) {
  int n = (int)(2.0 * std::sqrt(ecut * (a[0] * a[0] + a[1] * a[1] + a[2] * a[2])) / M_PI);
  n += 2;
  if (n % 2 == 1) n += 1;
  return n;
}

inline void gvec(const Lattice &L, int i, int j, int k, double g[3]) {
  for (int c = 0; c < 3; c++) g[c] = i * L.b1[c] + j * L.b2[c] + k * L.b3[c];
}

inline double norm2(const double g[3]) { return g[0] * g[0] + g[1] * g[1] + g[2] * g[2]; }

// The half-space enumeration shared by both sphere passes: k >= 0, and for
// k == 0 only j >= 0, and for j == k == 0 only i >= 1.
template <class F>
void half_space(int nr1, int nr2, int nr3, F &&visit) {
  for (int k = 0; k <= nr3 / 2; k++) {
    const int j0 = (k == 0) ? 0 : -nr2 / 2;
    for (int j = j0; j <= nr2 / 2; j++) {
      const int i0 = (j == 0 && k == 0) ? 1 : -nr1 / 2;
      for (int i = i0; i <= nr1 / 2; i++) visit(i, j, k);
    }
  }
}

// Index heap sort of arr[0..n) into 1-based idx[0..n): the exact sift-down
// sequence of the reference's sort1 (Numerical-Recipes indexx form), which is
// not stable, so the order of equal-|G| vectors depends on it.
void heap_index_sort(int n, const double *arr, int *idx) {
  for (int i = 0; i < n; i++) idx[i] = i + 1;
  if (n < 2) return;
  int l = n / 2 + 1;
  int ir = n;
  for (;;) {
    int it;
    double q;
    if (l > 1) {
      --l;
      it = idx[l - 1];
      q = arr[it - 1];
    } else {
      it = idx[ir - 1];
      q = arr[it - 1];
      idx[ir - 1] = idx[0];
      if (--ir == 1) {
        idx[0] = it;
        return;
      }
    }
    int i = l;
    int j = l + l;
    while (j <= ir) {
      if (j < ir && arr[idx[j - 1] - 1] < arr[idx[j] - 1]) j++;
      if (q < arr[idx[j - 1] - 1]) {
        idx[i - 1] = idx[j - 1];
        i = j;
        j += j;
      } else {
        j = ir + 1;
      }
    }
    idx[i - 1] = it;
  }
}

// 3x3 inverse by cofactors, with the reference's operation order
// (matinv3x3.cpp), column-major HM(i,j) = hm[(j-1)*3 + i-1].
void inv3(const double *hm, double *hi) {
#define M(i, j) hm[((j)-1) * 3 + (i)-1]
#define O(i, j) hi[((j)-1) * 3 + (i)-1]
  double d11 = M(2, 2) * M(3, 3) - M(2, 3) * M(3, 2);
  double d12 = M(2, 3) * M(3, 1) - M(2, 1) * M(3, 3);
  double d13 = M(2, 1) * M(3, 2) - M(3, 1) * M(2, 2);
  double d22 = M(1, 1) * M(3, 3) - M(1, 3) * M(3, 1);
  double d23 = M(1, 1) * M(3, 2) - M(3, 1) * M(1, 2);
  double d33 = M(1, 1) * M(2, 2) - M(1, 2) * M(2, 1);
  double d21 = M(3, 2) * M(1, 3) - M(1, 2) * M(3, 3);
  double d31 = M(1, 2) * M(2, 3) - M(2, 2) * M(1, 3);
  double d32 = M(1, 3) * M(2, 1) - M(1, 1) * M(2, 3);
  double dh = M(1, 1) * d11 + M(1, 2) * d12 + M(1, 3) * d13;
  d23 = -d23;
  O(1, 1) = d11 / dh;
  O(2, 2) = d22 / dh;
  O(3, 3) = d33 / dh;
  O(1, 2) = d21 / dh;
  O(1, 3) = d31 / dh;
  O(2, 3) = d32 / dh;
  O(2, 1) = d12 / dh;
  O(3, 1) = d13 / dh;
  O(3, 2) = d23 / dh;
#undef M
#undef O
}

void fill_info(const Lattice &L, double ecut, const int *nr_forced, pspw_basis_info *info) {
  int nr1, nr2, nr3;
  if (nr_forced && nr_forced[0] > 0) {
    nr1 = nr_forced[0];
    nr2 = nr_forced[1];
    nr3 = nr_forced[2];
  } else {
    nr1 = grid_rule(ecut, L.a1);
    nr2 = grid_rule(ecut, L.a2);
    nr3 = grid_rule(ecut, L.a3);
  }
  info->nr[0] = nr1;
  info->nr[1] = nr2;
  info->nr[2] = nr3;
  info->alat = L.alat;
  info->omega = L.omega;
  info->tpiba = 2. * M_PI / L.alat;
  info->tpiba2 = info->tpiba * info->tpiba;
  info->gcut = 4. * ecut / info->tpiba / info->tpiba;
  info->gcutw = info->gcut / 4.0;
  // sphere counts (Gamma: the +k and -k tests coincide, each G counts twice)
  int ngw = 1, jg = 2;
  half_space(nr1, nr2, nr3, [&](int i, int j, int k) {
    double g[3];
    gvec(L, i, j, k, g);
    const double t = norm2(g);
    if (t <= info->gcutw) ngw += 2;
    if (t < info->gcut) jg++;
  });
  int ngx = 2 * (jg - 1) + 1;
  if (ngx < 8 * ngw) ngx = 8 * ngw;
  int ngwx = ngx / 8 + 8;
  ngx = ngwx * 8 + 8;
  ngwx = ngwx + 1;
  info->ngx = ngx;
  info->ngwx = ngwx;
  info->ngw = -1;  // known after the sphere is built
  info->ng = -1;
}

}  // namespace

namespace pspw {

void phase_tables(const double *lattice9, const int nr[3], int nsp, const int *na,
                  const double *tau, PhaseTables *pt) {
  Lattice L = make_lattice(lattice9);
  int nax = 0;
  for (int s = 0; s < nsp; s++) nax = na[s] > nax ? na[s] : nax;
  pt->nax = nax;
  pt->nsp = nsp;
  double xmat[9], xmati[9];
  for (int i = 0; i < 3; i++) {
    xmat[0 * 3 + i] = L.a1[i];
    xmat[1 * 3 + i] = L.a2[i];
    xmat[2 * 3 + i] = L.a3[i];
  }
  inv3(xmat, xmati);
  for (int d = 0; d < 3; d++) {
    pt->zero[d] = (nr[d] + 1) / 2 + 1;
    // The reference sizes these tables NR+1 (AllocateArrays.cpp:29-34) but its
    // loops (PhaseFactor.cpp:44-61) reach index NR+2 when NR is odd, one
    // past the end; one spare slot keeps that write inside the table here.
    pt->len[d] = nr[d] + 2;
    // zero for atoms a >= na[s] (the reference's zero-filled arrays)
    pt->ei[d].assign((size_t)2 * pt->len[d] * nax * nsp, 0.0);
  }
  for (int s = 0; s < nsp; s++) {
    for (int a = 0; a < na[s]; a++) {
      const double *tp = tau + ((size_t)s * nax + a) * 3;
      const size_t sa = (size_t)s * nax + a;
      for (int d = 0; d < 3; d++) {
        double acc = xmati[0 * 3 + d] * tp[0];
        acc = acc + xmati[1 * 3 + d] * tp[1];
        acc = acc + xmati[2 * 3 + d] * tp[2];
        const double ar = -2.0 * M_PI * acc;
        std::vector<double> &e = pt->ei[d];
        const size_t b = sa * pt->len[d] + pt->zero[d] - 1;
        e[2 * b] = 1.0;
        e[2 * b + 1] = 0.0;
        for (int i = 1; i <= (nr[d] + 1) / 2; i++) {
          const double c = std::cos(i * ar), sn = std::sin(i * ar);
          e[2 * (b + i)] = c;
          e[2 * (b + i) + 1] = sn;
          e[2 * (b - i)] = c;
          e[2 * (b - i) + 1] = -sn;
        }
      }
    }
  }
}

void matinv3(const double *hm, double *hi) { inv3(hm, hi); }

}  // namespace pspw

extern "C" int pspw_basis_info_gamma(const double *lattice9, double ecut_ry, const int *nr_forced,
                                     pspw_basis_info *info) {
  if (!lattice9 || !info || !(ecut_ry > 0.0)) return PSPW_ERR_ARG;
  Lattice L = make_lattice(lattice9);
  if (!(L.omega > 0.0)) return PSPW_ERR_ARG;
  fill_info(L, ecut_ry, nr_forced, info);
  return PSPW_OK;
}

extern "C" int pspw_basis_build_gamma(const double *lattice9, double ecut_ry, const int *nr_forced,
                                      int nsp, const int *na, const double *tau,
                                      pspw_basis_info *info, unsigned int *n123, double *xkg,
                                      int *igk, int *n1, int *n2, int *n3, int *in1, int *in2,
                                      int *in3, double *g, double *gg, double *eigr) {
  int rc = pspw_basis_info_gamma(lattice9, ecut_ry, nr_forced, info);
  if (rc != PSPW_OK) return rc;
  if (nsp < 1 || !na) return PSPW_ERR_ARG;
  Lattice L = make_lattice(lattice9);
  const int nr1 = info->nr[0], nr2 = info->nr[1], nr3 = info->nr[2];
  const int ngx = info->ngx, ngwx = info->ngwx;
  const int ngx21 = ngx / 2 + 1;
  // half-space list with |G|^2 <= GCUT; entry 1 is the implicit G = 0
  std::vector<double> dum(ngx21, 0.0);
  std::vector<int> idum((size_t)ngx21 * 3, 0);
  int jg = 2;
  bool overflow = false;
  half_space(nr1, nr2, nr3, [&](int i, int j, int k) {
    double gv[3];
    gvec(L, i, j, k, gv);
    const double t = norm2(gv);
    if (t <= info->gcut) {
      if (jg > ngx21) {
        overflow = true;
        return;
      }
      dum[jg - 1] = t;
      idum[(size_t)0 * ngx21 + jg - 1] = i;
      idum[(size_t)1 * ngx21 + jg - 1] = j;
      idum[(size_t)2 * ngx21 + jg - 1] = k;
      jg++;
    }
  });
  if (overflow) return PSPW_ERR_SHAPE;
  const int ng_stop = jg - 1;
  std::vector<int> order(ng_stop);
  heap_index_sort(ng_stop, dum.data(), order.data());
  if (dum[order[0] - 1] != 0 || order[0] != 1) return PSPW_ERR_SHAPE;
  for (int i = 0; i < ngx; i++) {
    n1[i] = n2[i] = n3[i] = in1[i] = in2[i] = in3[i] = 0;
    g[i] = 0.0;
  }
  for (int i = 0; i < (ngx + 1) * 3; i++) gg[i] = 0.0;
  const int ldg = ngx + 1;
  n1[0] = n2[0] = n3[0] = 1;
  int ng = 2;
  for (int jj = 2; jj <= ng_stop; jj++) {
    if (ng + 1 > ngx) return PSPW_ERR_SHAPE;
    const int src = order[jj - 1];
    int i = idum[(size_t)0 * ngx21 + src - 1];
    int j = idum[(size_t)1 * ngx21 + src - 1];
    int k = idum[(size_t)2 * ngx21 + src - 1];
    const double t = dum[src - 1];
    in1[ng - 1] = i;
    in2[ng - 1] = j;
    in3[ng - 1] = k;
    in1[ng] = -i;
    in2[ng] = -j;
    in3[ng] = -k;
    double gv[3];
    gvec(L, i, j, k, gv);
    for (int c = 0; c < 3; c++) {
      gg[(size_t)c * ldg + ng - 1] = gv[c];
      gg[(size_t)c * ldg + ng] = -gv[c];
    }
    g[ng - 1] = t;
    g[ng] = t;
    n1[ng - 1] = i + 1 + (i < 0 ? nr1 : 0);
    n2[ng - 1] = j + 1 + (j < 0 ? nr2 : 0);
    n3[ng - 1] = k + 1 + (k < 0 ? nr3 : 0);
    n1[ng] = -i + 1 + (-i < 0 ? nr1 : 0);
    n2[ng] = -j + 1 + (-j < 0 ? nr2 : 0);
    n3[ng] = -k + 1 + (-k < 0 ? nr3 : 0);
    ng += 2;
  }
  ng -= 1;
  info->ng = ng;
  // wavefunction sphere (Gamma: k = 0)
  for (int i = 0; i < ngwx; i++) {
    n123[i] = 0;
    xkg[i] = 0.0;
    igk[i] = 0;
  }
  int ngw = 0;
  for (int ig = 1; ig <= ng; ig++) {
    const double gx = gg[(size_t)0 * ldg + ig - 1] + 0.0;
    const double gy = gg[(size_t)1 * ldg + ig - 1] + 0.0;
    const double gz = gg[(size_t)2 * ldg + ig - 1] + 0.0;
    const double t = gx * gx + gy * gy + gz * gz;
    if (t <= info->gcutw) {
      ngw++;
      if (ngw > ngwx) return PSPW_ERR_SHAPE;
      igk[ngw - 1] = ig;
      xkg[ngw - 1] = t;
      n123[ngw - 1] =
          (unsigned)(n1[ig - 1] + nr1 * ((n2[ig - 1] - 1) + nr2 * (n3[ig - 1] - 1)));
    }
  }
  info->ngw = ngw;
  // phase factors EIGR(NGWX, NAX, NSP), interleaved complex
  if (eigr && tau) {
    pspw::PhaseTables pt;
    const int nr[3] = {nr1, nr2, nr3};
    pspw::phase_tables(lattice9, nr, nsp, na, tau, &pt);
    const int nax = pt.nax;
    for (long i = 0; i < 2L * ngwx * nax * nsp; i++) eigr[i] = 0.0;
    for (int s = 0; s < nsp; s++) {
      for (int a = 0; a < nax; a++) {
        const size_t sa = (size_t)s * nax + a;
        for (int ig = 0; ig < ngw; ig++) {
          const int igp = igk[ig];
          const size_t p1 = sa * pt.len[0] + pt.zero[0] + in1[igp - 1] - 1,
                       p2 = sa * pt.len[1] + pt.zero[1] + in2[igp - 1] - 1,
                       p3 = sa * pt.len[2] + pt.zero[2] + in3[igp - 1] - 1;
          const double ar = pt.ei[0][2 * p1], ai = pt.ei[0][2 * p1 + 1];
          const double br = pt.ei[1][2 * p2], bi = pt.ei[1][2 * p2 + 1];
          const double cr = pt.ei[2][2 * p3], ci = pt.ei[2][2 * p3 + 1];
          const double tr = ar * br - ai * bi, ti = ar * bi + ai * br;
          const size_t o = (sa * ngwx + ig) * 2;
          eigr[o] = tr * cr - ti * ci;
          eigr[o + 1] = tr * ci + ti * cr;
        }
      }
    }
  }
  return PSPW_OK;
}
