// Drop-in replacement of the reference's hot-path translation units.
//
// Exports the reference's C++ functions with their exact signatures (and so
// the same g++ mangled names, common_pspw.h:176-222 and 252-259), reading
// the reference program's globals (common_pspw.h:43-148) as that code does,
// and forwards to the C ABI in include/pspw_gpu.h.  A program links this
// library in place of ApplyHam_block.o, ApplyHam.o, chebyfilt.o,
// davidson_cpu.o, lobpcg_cpu.o, ortho_qr.o, eig_zheevd.o, eig_zhegv.o,
// GenPrec.o, EvalRhoPsi.o, EvalENL.o, lanczos.o and Diagon_cpu.o.
//
// Device state: one pspw_cell per k-point, built from N123/XKG/EIGR/PKG_A/
// WNL on first use (or by SetupArrays_ApplyHam_cuda) and reused while those
// arrays keep their addresses and sizes.  A program that rewrites them in
// place (new atomic positions) calls SetupArrays_ApplyHam_cuda again.  V_eff
// (the `rho` argument) is uploaded on every call, as the reference passes it
// on every call.
//
// Arithmetic: FP64 throughout by default, matching the reference to
// rounding.  PSPW_DROPIN_FILTER_PREC=f32 runs chebyfilt in FP32 on the device
// (the mixed-precision filter; the host block stays FP64).
//
// Errors keep the reference's behaviour: the invariant checks of
// ApplyHam_block.cpp:18-21 (nnr != NNR) and :70-73 (lm_end > 4) print the
// same message and abort; an engine failure prints the engine's message and
// aborts (the reference has no error return on these paths).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "pspw_gpu.h"

typedef double _Complex zcomplex;

// ---- the reference program's globals (defined by its global_variables.cpp)
extern int NSP;
extern int *NA;
extern int NAX;
extern int NLMAX;
extern int *L_MAX;
extern int *L_LOC;
extern int NX;
extern int NR1, NR2, NR3, NNR;
extern int NKPT;
extern double TPIBA2;
extern int NGWX;
extern int *NGW;
extern double *XKG;
extern unsigned int *N123;
extern zcomplex *EIGR;
extern double *PKG_A;
extern double *WNL;
extern int NEMPTY;
extern bool USER_MAX_DIAG_ITER;
extern int MAX_DIAG_ITER;
extern bool DIAG_VERBOSE;
extern zcomplex *C0;
extern double *FOCC;
extern double *WKPT;
extern double OMEGA;
extern double EKIN;
extern double ENL;
extern zcomplex *FNL;

#define DROPIN_API __attribute__((visibility("default")))

namespace {

struct KCell {
  pspw_cell *cell = nullptr;
  const void *key[5] = {};
  int ngw = -1, ngwx = -1, nnr = -1;
};

std::vector<KCell> g_cells;  // index ik-1
int g_device = 0;
bool g_device_set = false;

[[noreturn]] void die(const char *where, int rc) {
  std::printf("ERROR in %s: pspw engine error %d (%s): %s\n", where, rc, pspw_error_string(rc),
              pspw_last_error());
  std::fflush(stdout);
  std::abort();
}

void check_nnr(int nnr) {
  if (nnr != NNR) {  // ApplyHam_block.cpp:18-21
    std::printf("nnr != NNR : %d %d\n", nnr, NNR);
    std::abort();
  }
}

std::vector<int> lm_ends() {
  std::vector<int> lm(NSP);
  for (int is = 0; is < NSP; is++) {
    lm[is] = L_MAX[is] * L_MAX[is] - 2 * L_LOC[is] + 1;  // ApplyHam_block.cpp:69
    if (lm[is] > 4) {                                    // :70-73
      std::printf("ERROR: lm_end > 4 is not implemented\n");
      std::abort();
    }
  }
  return lm;
}

int device() {
  if (!g_device_set) {
    const char *d = std::getenv("PSPW_DEVICE");
    g_device = d ? std::atoi(d) : 0;
    g_device_set = true;
  }
  return g_device;
}

void drop_cell(KCell &k) {
  if (k.cell) pspw_cell_destroy(k.cell);
  k = KCell();
}

pspw_cell *build_cell(int ik, const unsigned int *n123, const double *xkg, const zcomplex *eigr,
                      const double *pkg_a) {
  if ((int)g_cells.size() < ik) g_cells.resize(ik);
  KCell &k = g_cells[ik - 1];
  const void *key[5] = {n123, xkg, eigr, pkg_a, WNL};
  const int ngw = NGW[ik - 1];
  bool same = k.cell && k.ngw == ngw && k.ngwx == NGWX && k.nnr == NNR;
  for (int i = 0; same && i < 5; i++) same = (k.key[i] == key[i]);
  if (same) return k.cell;
  drop_cell(k);
  std::vector<int> lm = lm_ends();
  const size_t col = (size_t)ik - 1;
  pspw_cell *c = nullptr;
  int rc = pspw_cell_create(
      &c, device(), NR1, NR2, NR3, ngw, NGWX, n123 + col * NGWX, xkg + col * NGWX, TPIBA2, NSP, NA,
      NAX, lm.data(), NLMAX,
      reinterpret_cast<const double *>(eigr + col * (size_t)NGWX * NAX * NSP),
      pkg_a + col * (size_t)NLMAX * NGWX * NSP, WNL);
  if (rc) die("pspw_cell_create", rc);
  k.cell = c;
  for (int i = 0; i < 5; i++) k.key[i] = key[i];
  k.ngw = ngw;
  k.ngwx = NGWX;
  k.nnr = NNR;
  return c;
}

pspw_cell *cell_for(int ik) { return build_cell(ik, N123, XKG, EIGR, PKG_A); }

int filter_prec() {
  const char *p = std::getenv("PSPW_DROPIN_FILTER_PREC");
  return (p && (!std::strcmp(p, "f32") || !std::strcmp(p, "F32"))) ? PSPW_PREC_F32 : PSPW_PREC_F64;
}

}  // namespace

// ------------------------------------------------------------ host signatures

// ApplyHam_block.cpp:5 / common_pspw.h:177
DROPIN_API void ApplyHam_block(zcomplex *vin, zcomplex *vout, int NGW_ik, int ik, double *rho,
                               int nnr, int nstates) {
  check_nnr(nnr);
  pspw_cell *c = cell_for(ik);
  int rc = pspw_cell_set_veff(c, rho, nnr);
  if (rc) die("ApplyHam_block", rc);
  rc = pspw_apply_ham_block(c, reinterpret_cast<const double *>(vin),
                            reinterpret_cast<double *>(vout), NGW_ik, nstates);
  if (rc) die("ApplyHam_block", rc);
}

// ApplyHam.cpp:5 / common_pspw.h:176
DROPIN_API void ApplyHam(zcomplex *vin, zcomplex *vout, int NGW_ik, int ik, double *rho, int nnr) {
  ApplyHam_block(vin, vout, NGW_ik, ik, rho, nnr, 1);
}

// chebyfilt.cpp:6 / common_pspw.h:187.  The block width is the global NX+2
// (chebyfilt.cpp:20,26,44), as in the reference.
DROPIN_API void chebyfilt(int ik, zcomplex *X, int degree, double lb, double ub, double *rhoe,
                          int nnr) {
  check_nnr(nnr);
  pspw_cell *c = cell_for(ik);
  int rc = pspw_cell_set_veff(c, rhoe, nnr);
  if (rc) die("chebyfilt", rc);
  rc = pspw_chebyfilt(c, reinterpret_cast<double *>(X), NGW[ik - 1], NX + 2, degree, lb, ub,
                      filter_prec());
  if (rc) die("chebyfilt", rc);
}

// ------------------------------------------------------------ device API
// (the CUDA layer the reference declares, common_pspw.h:252-259)

DROPIN_API void SetupCUDA() { (void)device(); }

DROPIN_API void ShutdownCUDA() {
  for (auto &k : g_cells) drop_cell(k);
  g_cells.clear();
}

DROPIN_API int SetupArrays_ApplyHam_cuda(unsigned int *n123, double *xkg, zcomplex *eigr,
                                         double *pkg_a) {
  for (auto &k : g_cells) drop_cell(k);
  for (int ik = 1; ik <= NKPT; ik++) build_cell(ik, n123, xkg, eigr, pkg_a);
  return 0;
}

DROPIN_API int SetupRho_ApplyHam_cuda() { return 0; }

DROPIN_API int CopyRho_ApplyHam_cuda(double *rho) {
  for (int ik = 1; ik <= NKPT; ik++) {
    int rc = pspw_cell_set_veff(cell_for(ik), rho, NNR);
    if (rc) return rc;
  }
  return 0;
}

// d_vin, d_vout: device FP64 blocks, ld = NGW_ik
DROPIN_API int ApplyHam_block_cuda(zcomplex *d_vin, zcomplex *d_vout, int NGW_ik, int ik,
                                   int nstates) {
  pspw_cell *c = cell_for(ik);
  int rc = pspw_apply_ham_block_dev(c, PSPW_PREC_F64, d_vin, d_vout, NGW_ik, NGW_ik, nstates);
  if (rc) return rc;
  return pspw_cell_synchronize(c);
}

DROPIN_API void FreeArrays_ApplyHam_cuda() { ShutdownCUDA(); }

DROPIN_API void FreeRho_ApplyHam_cuda() {}

// ------------------------------------------------------------ solvers

namespace {

double *dp(zcomplex *z) { return reinterpret_cast<double *>(z); }

int solver_max_iter() { return USER_MAX_DIAG_ITER ? MAX_DIAG_ITER : 0; }

}  // namespace

// ortho_qr.cpp:3
DROPIN_API void ortho_qr(zcomplex *X, int nbasis, int nstates) {
  int rc = pspw_ortho_qr(cell_for(1), dp(X), nbasis, nstates);
  if (rc == PSPW_ERR_LAPACK) {  // ortho_qr.cpp:20-29 prints and returns
    std::printf("ERROR calling zgeqrf_ : %s\n", pspw_last_error());
    return;
  }
  if (rc) die("ortho_qr", rc);
}

// eig_zheevd.cpp:5
DROPIN_API void eig_zheevd(zcomplex *A, int ldA, double *lambda, int N) {
  int rc = pspw_eig_zheevd(cell_for(1), dp(A), ldA, lambda, N);
  if (rc == PSPW_ERR_LAPACK) {  // eig_zheevd.cpp:26-29 prints and returns
    std::printf("ERROR calling zheevd_ : %s\n", pspw_last_error());
    return;
  }
  if (rc) die("eig_zheevd", rc);
}

// eig_zhegv.cpp:5
DROPIN_API void eig_zhegv(zcomplex *A, int ldA, zcomplex *B, int ldB, zcomplex *evec, int ldE,
                          int N) {
  int rc = pspw_eig_zhegv(cell_for(1), dp(A), ldA, dp(B), ldB, dp(evec), ldE, N);
  if (rc == PSPW_ERR_LAPACK) {
    std::printf("ERROR calling zheevd in eig_zhegv : %s\n", pspw_last_error());
    return;
  }
  if (rc) die("eig_zhegv", rc);
}

// eig_zhegv.cpp:86
DROPIN_API void eig_zhegv_eval(zcomplex *A, int ldA, zcomplex *B, int ldB, double *eval,
                               zcomplex *evec, int ldE, int N) {
  int rc = pspw_eig_zhegv_eval(cell_for(1), dp(A), ldA, dp(B), ldB, eval, dp(evec), ldE, N);
  if (rc == PSPW_ERR_LAPACK) {
    std::printf("ERROR calling zheevd in eig_zhegv : %s\n", pspw_last_error());
    return;
  }
  if (rc) die("eig_zhegv_eval", rc);
}

// GenPrec.cpp:5
DROPIN_API void GenPrec(int ik, double *prec, int nbasis, double tau) {
  int rc = pspw_gen_prec(cell_for(ik), prec, nbasis, tau);
  if (rc) die("GenPrec", rc);
}

// lobpcg_cpu.cpp:15-27 (ChebySCFLoop.cpp uses it on host matrices)
DROPIN_API void symmetrize(zcomplex *v, int ldv, int nrow, int ncol) {
  (void)nrow;
  for (int j = 0; j < ncol; j++)
    for (int i = 0; i <= j; i++) {
      double *a = dp(v + (size_t)j * ldv + i), *b = dp(v + (size_t)i * ldv + j);
      const double tr = 0.5 * (a[0] + b[0]), ti = 0.5 * (a[1] - b[1]);
      a[0] = tr;
      a[1] = ti;
      b[0] = tr;
      b[1] = -ti;
    }
}

static void print_solver_table(const char *title, int nstates, const double *ev, const double *res) {
  std::printf("%s\n", title);
  for (int i = 0; i < nstates; i++) std::printf("%d %18.10f %18.10f\n", i + 1, ev[i], res[i]);
}

// davidson_cpu.cpp:9
DROPIN_API void davidson_cpu(int ik, double *evals, zcomplex *X, int nbasis, int nstates,
                             double *rhoe, int nnr, double *prec) {
  check_nnr(nnr);
  pspw_cell *c = cell_for(ik);
  int rc = pspw_cell_set_veff(c, rhoe, nnr);
  if (rc) die("davidson_cpu", rc);
  std::vector<double> res(nstates);
  int iters = 0;
  rc = pspw_davidson(c, evals, dp(X), nbasis, nstates, prec, NEMPTY, solver_max_iter(),
                     PSPW_PREC_F64, res.data(), &iters);
  if (rc) die("davidson_cpu", rc);
  print_solver_table("Final Davidson result (GPU engine):", nstates, evals, res.data());
}

// lobpcg_cpu.cpp:31
DROPIN_API void lobpcg_cpu(int ik, double *lambda, zcomplex *X, int nbasis, int nstates,
                           double *rhoe, int nnr, double *prec) {
  check_nnr(nnr);
  pspw_cell *c = cell_for(ik);
  int rc = pspw_cell_set_veff(c, rhoe, nnr);
  if (rc) die("lobpcg_cpu", rc);
  std::vector<double> res(nstates);
  int iters = 0;
  rc = pspw_lobpcg(c, lambda, dp(X), nbasis, nstates, prec, NEMPTY, solver_max_iter(),
                   PSPW_PREC_F64, res.data(), &iters);
  if (rc == PSPW_ERR_LAPACK) {  // lobpcg_cpu.cpp:163-166 aborts on a failed Cholesky
    std::printf("%s\n", pspw_last_error());
    std::abort();
  }
  if (rc) die("lobpcg_cpu", rc);
  print_solver_table("Final LOBPCG result (GPU engine)", nstates, lambda, res.data());
}

// Diagon_cpu.cpp:5-57: preconditioner, solver on NGW_ik x NX, then the
// NGWX-padded copy with zero tails
static void diagon(bool lobpcg, int ik, double *eigval, zcomplex *eigvec, int NGW_ik, double *rhoe,
                   int nnr, double tau) {
  std::vector<zcomplex> tmp((size_t)NGW_ik * NX);
  std::vector<double> prec(NGW_ik);
  GenPrec(ik, prec.data(), NGW_ik, tau);
  if (lobpcg)
    lobpcg_cpu(ik, eigval, tmp.data(), NGW_ik, NX, rhoe, nnr, prec.data());
  else
    davidson_cpu(ik, eigval, tmp.data(), NGW_ik, NX, rhoe, nnr, prec.data());
  for (int ist = 0; ist < NX; ist++) {
    zcomplex *dst = eigvec + (size_t)ist * NGWX;
    std::memcpy(dst, tmp.data() + (size_t)ist * NGW_ik, sizeof(zcomplex) * NGW_ik);
    std::memset(dst + NGW_ik, 0, sizeof(zcomplex) * (NGWX - NGW_ik));
  }
}

DROPIN_API void Diagon_lobpcg_cpu(int ik, double *eigval, zcomplex *eigvec, int NGW_ik,
                                  double *rhoe, int nnr, double tau) {
  diagon(true, ik, eigval, eigvec, NGW_ik, rhoe, nnr, tau);
}

DROPIN_API void Diagon_davidson_cpu(int ik, double *eigval, zcomplex *eigvec, int NGW_ik,
                                    double *rhoe, int nnr, double tau) {
  diagon(false, ik, eigval, eigvec, NGW_ik, rhoe, nnr, tau);
}

// lanczos.cpp:8
DROPIN_API void lanczos(int ik, zcomplex *v0, int k, double *T, int ldT, zcomplex *f, double *rhoe,
                        int nnr) {
  check_nnr(nnr);
  pspw_cell *c = cell_for(ik);
  int rc = pspw_cell_set_veff(c, rhoe, nnr);
  if (rc) die("lanczos", rc);
  rc = pspw_lanczos(c, dp(v0), NGW[ik - 1], k, T, ldT, dp(f));
  if (rc) die("lanczos", rc);
}

// EvalRhoPsi.cpp:83: C0(:,ist,ik) copies NGWX entries of column ist (with
// leading dimension ldEigvec, reading into the next column when it is
// shorter, as the reference does), then the density and EKIN on the device.
DROPIN_API void EvalRhoPsi(int ik, double *rhoe, zcomplex *eigvec, int ldEigvec, int NGW_ik) {
  for (int ist = 0; ist < NX; ist++)
    std::memcpy(C0 + ((size_t)(ik - 1) * NX + ist) * NGWX, eigvec + (size_t)ist * ldEigvec,
                sizeof(zcomplex) * NGWX);
  int rc = pspw_eval_rho_psi(cell_for(ik), rhoe, dp(eigvec), ldEigvec, NGW_ik, NX,
                             FOCC + (size_t)(ik - 1) * NX, WKPT[ik - 1], OMEGA, &EKIN);
  if (rc == PSPW_ERR_CHARGE) {  // EvalRhoPsi.cpp:129-133
    std::printf("%s\n", pspw_last_error());
    std::abort();
  }
  if (rc) die("EvalRhoPsi", rc);
}

// EvalENL.cpp:5-49: FNL of every k-point on the device (unconjugated C0
// against PKG_A conj(EIGR)), written into the global FNL, then ENL summed on
// the host in the reference's loop order (species, atom, k-point, lm).
DROPIN_API void EvalENL() {
  std::vector<std::vector<double>> fnl(NKPT);
  int nproj = 0;
  for (int is = 0; is < NSP; is++) nproj += NA[is] * (L_MAX[is] * L_MAX[is] - 2 * L_LOC[is] + 1);
  for (int ik = 1; ik <= NKPT; ik++) {
    fnl[ik - 1].assign(2 * (size_t)NX * nproj, 0.0);
    double e = 0.0;
    const int rc = pspw_eval_enl(cell_for(ik), dp(C0 + (size_t)(ik - 1) * NGWX * NX), NGWX,
                                 NGW[ik - 1], NX, FOCC + (size_t)(ik - 1) * NX, WKPT[ik - 1], &e,
                                 fnl[ik - 1].data());
    if (rc) die("EvalENL", rc);
  }
  ENL = 0.0;
  int p0 = 0;  // first projector of (is, ia)
  for (int is = 1; is <= NSP; is++) {
    const int lm_end = L_MAX[is - 1] * L_MAX[is - 1] - 2 * L_LOC[is - 1] + 1;
    for (int ia = 1; ia <= NA[is - 1]; ia++, p0 += lm_end) {
      for (int ik = 1; ik <= NKPT; ik++) {
        for (int lm = 1; lm <= lm_end; lm++) {
          const double *f = fnl[ik - 1].data() + 2 * (size_t)(p0 + lm - 1) * NX;
          double enl_m = 0.0;
          for (int ist = 1; ist <= NX; ist++) {
            const double re = f[2 * (ist - 1)], im = f[2 * (ist - 1) + 1];
            // FNL(ist, ik, is, ia, lm), dimensions NX x NKPT x NSP x NAX
            const size_t at =
                ((((size_t)(lm - 1) * NAX + (ia - 1)) * NSP + (is - 1)) * NKPT + (ik - 1)) * NX +
                (ist - 1);
            double *g = reinterpret_cast<double *>(FNL + at);
            g[0] = re;
            g[1] = im;
            const double a = std::hypot(re, im);
            enl_m = enl_m + FOCC[(size_t)(ik - 1) * NX + ist - 1] * (a * a);
          }
          ENL = ENL + WKPT[ik - 1] * enl_m * WNL[(size_t)(lm - 1) * NSP + (is - 1)];
        }
      }
    }
  }
}

// EvalRhoPsi.cpp:5 (eigvec with leading dimension NGWX)
DROPIN_API void EvalRhoPsi(int ik, double *rhoe, zcomplex *eigvec, int NGW_ik) {
  EvalRhoPsi(ik, rhoe, eigvec, NGWX, NGW_ik);
}
