/*
 * TEST INFRASTRUCTURE (oracle build only) -- never linked into the product.
 *
 * Harness around the reference implementation compiled from its own
 * sources.  It fills the common_pspw.h globals for a synthetic cell (the
 * steps of Setup.cpp:5-145 that do not read pseudopotential files, using the
 * reference's own CalcRecipLatt, GVectorsGen0, AllocateArrays, InitOcc,
 * GVectorsGen, GkVectorsGen and PhaseFactor), accepts synthetic KB form
 * factors, and exposes the reference hot-path functions through extern "C"
 * wrappers so a test can call them with ctypes.
 *
 * The same file is linked twice: against the reference's own hot-path
 * objects (libref.so, the oracle) and against the GPU drop-in library in
 * their place (libref_dropin.so), which is how the drop-in is shown to link
 * and run in the reference's host program unchanged.
 */
#include "common_pspw.h"

extern void random_col(double complex *A, int nelem, long a);

extern "C" {

/* Geometry and basis for one k-point (Gamma) cell.
 * a: 9 doubles, lattice vectors A1, A2, A3 (bohr).  ecut: wavefunction cutoff
 * in Rydberg as in the reference INPUT.  nr: forced FFT grid (all > 0) or
 * zeros for the reference rule.  tau: 3*nax*nsp positions (bohr), Fortran
 * order TAU(3,NAX,NSP).  zv, lmax, lloc: per species. */
int ref_setup_cell(const double *a, double ecut, const int *nr, int nsp, const int *na,
                   const double *tau, const double *zv, const int *lmax, const int *lloc,
                   int nempty) {
  int is, ia, i, lm;
  NSP = nsp;
  NA = (int *)malloc(NSP * sizeof(int));
  NAX = 0;
  for (is = 0; is < NSP; is++) {
    NA[is] = na[is];
    if (NA[is] > NAX) NAX = NA[is];
  }
  for (i = 0; i < 3; i++) {
    A1[i] = a[i];
    A2[i] = a[3 + i];
    A3[i] = a[6 + i];
  }
  TAU = (double *)malloc(3 * NAX * NSP * sizeof(double));
  for (i = 0; i < 3 * NAX * NSP; i++) TAU[i] = tau[i];
  ZV = (double *)malloc(NSP * sizeof(double));
  L_MAX = (int *)malloc(NSP * sizeof(int));
  L_LOC = (int *)malloc(NSP * sizeof(int));
  for (is = 0; is < NSP; is++) {
    ZV[is] = zv[is];
    L_MAX[is] = lmax[is];
    L_LOC[is] = lloc[is];
  }
  ECUT = ecut;
  NEMPTY = nempty;
  NKPT = 1;
  XK = (double *)malloc(3 * sizeof(double));
  XK[0] = XK[1] = XK[2] = 0.0;
  WKPT = (double *)malloc(sizeof(double));
  WKPT[0] = 1.0;
  TMETAL = false;
  USER_FFT_GRID = (nr[0] > 0);
  if (USER_FFT_GRID) {
    NR1 = nr[0];
    NR2 = nr[1];
    NR3 = nr[2];
    NNR = NR1 * NR2 * NR3;
  }
  /* Setup.cpp:11-17 */
  NLMAX = 0;
  for (is = 1; is <= NSP; is++) {
    lm = L_MAX[is - 1] * L_MAX[is - 1] - 2 * L_LOC[is - 1] + 1;
    if (lm > NLMAX) NLMAX = lm;
  }
  if (NLMAX < 4) NLMAX = 4;
  /* Setup.cpp:20-34 */
  if (!USER_FFT_GRID) {
    NR1 = 2.0 * sqrt(ECUT * (A1[0] * A1[0] + A1[1] * A1[1] + A1[2] * A1[2])) / M_PI;
    NR2 = 2.0 * sqrt(ECUT * (A2[0] * A2[0] + A2[1] * A2[1] + A2[2] * A2[2])) / M_PI;
    NR3 = 2.0 * sqrt(ECUT * (A3[0] * A3[0] + A3[1] * A3[1] + A3[2] * A3[2])) / M_PI;
    NR1 += 2;
    NR2 += 2;
    NR3 += 2;
    if (NR1 % 2 == 1) NR1++;
    if (NR2 % 2 == 1) NR2++;
    if (NR3 % 2 == 1) NR3++;
    NNR = NR1 * NR2 * NR3;
  }
  /* Setup.cpp:39-66 */
  ALAT = A1[0];
  OMEGA = determinant3x3(A1, A2, A3);
  CalcRecipLatt();
  NGW = (int *)malloc(NKPT * sizeof(int));
  TPIBA = 2. * M_PI / ALAT;
  TPIBA2 = TPIBA * TPIBA;
  GCUT = 4. * ECUT / TPIBA / TPIBA;
  GCUTW = GCUT / 4.0;
  GVectorsGen0();
  NGWX = NGX / 8 + 8;
  NGX = NGWX * 8 + 8;
  NGWX = NGWX + 1;
  /* Setup.cpp:75-87 */
  NEL = 0.0;
  for (is = 1; is <= NSP; is++) NEL = NEL + NA[is - 1] * ZV[is - 1];
  NX = NEMPTY + (int)((NEL + 1.0) / 2.0);
  NSTATX = NX * NKPT;
  AllocateArrays();
  InitOcc();
  GVectorsGen();
  GkVectorsGen();
  /* PrepareSCF.cpp:10: phase factors; the synthetic run skips the
   * pseudopotential-file form factors (set by ref_set_nl instead). */
  PhaseFactor();
  (void)ia;
  return 0;
}

void ref_get_dims(int *out) {
  out[0] = NR1;
  out[1] = NR2;
  out[2] = NR3;
  out[3] = NNR;
  out[4] = NGW[0];
  out[5] = NGWX;
  out[6] = NGX;
  out[7] = NG;
  out[8] = NX;
  out[9] = NLMAX;
  out[10] = NAX;
  out[11] = NSP;
}

void ref_get_scalars(double *out) {
  out[0] = TPIBA;
  out[1] = TPIBA2;
  out[2] = OMEGA;
  out[3] = ALAT;
  out[4] = GCUT;
  out[5] = GCUTW;
  out[6] = NEL;
  out[7] = EKIN;
}

/* Copies of the basis arrays for column ik=1 (NGWX entries each). */
void ref_get_basis(unsigned int *n123, double *xkg, int *igk) {
  for (int i = 0; i < NGWX; i++) {
    n123[i] = N123[i];
    xkg[i] = XKG[i];
    igk[i] = IGK[i];
  }
}

/* G-vector tables (NGX entries) */
void ref_get_gvec(int *n1, int *n2, int *n3, int *in1, int *in2, int *in3, double *g) {
  for (int i = 0; i < NGX; i++) {
    n1[i] = N1[i];
    n2[i] = N2[i];
    n3[i] = N3[i];
    in1[i] = IN1[i];
    in2[i] = IN2[i];
    in3[i] = IN3[i];
    g[i] = G[i];
  }
}

/* EIGR(NGWX,NAX,NSP) for ik=1 */
void ref_get_eigr(double complex *eigr) {
  for (long i = 0; i < (long)NGWX * NAX * NSP; i++) eigr[i] = EIGR[i];
}

/* Overwrite PKG_A(NLMAX,NGWX,NSP) and WNL(NSP,NLMAX) */
void ref_set_nl(const double *pkg_a, const double *wnl) {
  for (long i = 0; i < (long)NLMAX * NGWX * NSP; i++) PKG_A[i] = pkg_a[i];
  for (int i = 0; i < NSP * NLMAX; i++) WNL[i] = wnl[i];
}

void ref_set_nx(int nx, int nempty) {
  NX = nx;
  NEMPTY = nempty;
}

void ref_set_diag(int user_max, int max_iter, int verbose) {
  USER_MAX_DIAG_ITER = user_max != 0;
  MAX_DIAG_ITER = max_iter;
  DIAG_VERBOSE = verbose != 0;
}

void ref_set_focc(const double *focc, int nx) {
  free(FOCC);
  FOCC = (double *)malloc(nx * sizeof(double));
  for (int i = 0; i < nx; i++) FOCC[i] = focc[i];
}

/* C0 sized for the current NX, zeroed (EvalRhoPsi writes NGWX x NX). */
void ref_alloc_c0(void) {
  free(C0);
  C0 = (double complex *)malloc((size_t)NGWX * NX * sizeof(double complex));
  for (long i = 0; i < (long)NGWX * NX; i++) C0[i] = Z_ZERO;
  free(FNL);
  FNL = (double complex *)malloc((size_t)NX * NSP * NAX * NLMAX * sizeof(double complex));
}

void ref_get_c0(double complex *c0) {
  for (long i = 0; i < (long)NGWX * NX; i++) c0[i] = C0[i];
}

void ref_set_ekin(double v) { EKIN = v; }
double ref_get_ekin(void) { return EKIN; }
double ref_get_enl(void) { return ENL; }

/* ---- hot-path entry points (ik = 1) ---- */
void ref_ApplyHam_block(double complex *vin, double complex *vout, int ngw, double *rho,
                        int nstates) {
  ApplyHam_block(vin, vout, ngw, 1, rho, NNR, nstates);
}

void ref_ApplyHam(double complex *vin, double complex *vout, int ngw, double *rho) {
  ApplyHam(vin, vout, ngw, 1, rho, NNR);
}

void ref_chebyfilt(double complex *X, int degree, double lb, double ub, double *rho) {
  chebyfilt(1, X, degree, lb, ub, rho, NNR);
}

void ref_lanczos(double complex *v0, int k, double *T, int ldT, double complex *f, double *rho) {
  lanczos(1, v0, k, T, ldT, f, rho, NNR);
}

void ref_davidson(double *evals, double complex *X, int nbasis, int nstates, double *rho,
                  double *prec) {
  davidson_cpu(1, evals, X, nbasis, nstates, rho, NNR, prec);
}

void ref_lobpcg(double *evals, double complex *X, int nbasis, int nstates, double *rho,
                double *prec) {
  lobpcg_cpu(1, evals, X, nbasis, nstates, rho, NNR, prec);
}

void ref_Diagon_davidson(double *eigval, double complex *eigvec, int ngw, double *rho,
                         double tau) {
  Diagon_davidson_cpu(1, eigval, eigvec, ngw, rho, NNR, tau);
}

void ref_Diagon_lobpcg(double *eigval, double complex *eigvec, int ngw, double *rho, double tau) {
  Diagon_lobpcg_cpu(1, eigval, eigvec, ngw, rho, NNR, tau);
}

void ref_ortho_qr(double complex *X, int nbasis, int nstates) { ortho_qr(X, nbasis, nstates); }

void ref_eig_zheevd(double complex *A, int ldA, double *lambda, int N) {
  eig_zheevd(A, ldA, lambda, N);
}

void ref_eig_zhegv(double complex *A, int ldA, double complex *B, int ldB, double complex *evec,
                   int ldE, int N) {
  eig_zhegv(A, ldA, B, ldB, evec, ldE, N);
}

void ref_eig_zhegv_eval(double complex *A, int ldA, double complex *B, int ldB, double *eval,
                        double complex *evec, int ldE, int N) {
  eig_zhegv_eval(A, ldA, B, ldB, eval, evec, ldE, N);
}

void ref_GenPrec(double *prec, int nbasis, double tau) { GenPrec(1, prec, nbasis, tau); }

void ref_EvalRhoPsi(double *rhoe, double complex *eigvec, int ld, int ngw) {
  EvalRhoPsi(1, rhoe, eigvec, ld, ngw);
}

void ref_EvalENL(void) { EvalENL(); }

void ref_random_col(double complex *A, int nelem, long seed) { random_col(A, nelem, seed); }

void ref_fft(double complex *data, int inverse) { fft_fftw3(data, NR1, NR2, NR3, inverse != 0); }

/* ---- SCF pieces (EvalEnergy.cpp, xc_PZ.cpp, NormalizeRho.cpp, the mixers) ---- */

/* The local-potential data EvalEnergy reads: SFAC(is,ig) complex, VPS(is,ig),
 * RHOPS(is,ig) real (NSP x NG, species fastest), and the scalars. */
void ref_set_local(const double complex *sfac, const double *vps, const double *rhops, double esr,
                   double eself, double nel) {
  const long n = (long)NSP * NG;
  free(SFAC);
  free(VPS);
  free(RHOPS);
  SFAC = (double complex *)malloc(n * sizeof(double complex));
  VPS = (double *)malloc(n * sizeof(double));
  RHOPS = (double *)malloc(n * sizeof(double));
  for (long i = 0; i < n; i++) {
    SFAC[i] = sfac[i];
    VPS[i] = vps[i];
    RHOPS[i] = rhops[i];
  }
  ESR = esr;
  ESELF = eself;
  NEL = nel;
}

/* EvalEnergy(rhoe): rhoe in = density, out = V_eff; e = {ETOT, EKIN, EHT,
 * EPSEU, ENL, EXC} with EKIN and ENL taken from the arguments. */
void ref_EvalEnergy(double *rhoe, double ekin, double enl, double *e) {
  EKIN = ekin;
  ENL = enl;
  EvalEnergy(rhoe);
  e[0] = ETOT;
  e[1] = EKIN;
  e[2] = EHT;
  e[3] = EPSEU;
  e[4] = ENL;
  e[5] = EXC;
}

double ref_xc_PZ(double *rho, double *vxc, int nnr) {
  double exc = 0.0;
  xc_PZ(rho, vxc, exc, nnr);
  return exc;
}

void ref_NormalizeRho(double *rho, int nnr, double omega, double nel) {
  NormalizeRho(rho, nnr, omega, nel);
}

void ref_KerkerPrec(double *diff, int idx1, int nnr, double beta, double q0) {
  KerkerPrec(diff, idx1, nnr, beta, q0);
}

void ref_set_mixing(double kerker_q0) { KERKER_Q0 = kerker_q0; }

double ref_PulayRhoMix(int iter, double *rhoe, double *rho_old, double *f, int mixdim, int nnr) {
  double d = 0.0;
  PulayRhoMix(iter, rhoe, rho_old, f, mixdim, nnr, d);
  return d;
}

double ref_AndersonRhoMix(int iter, double beta, double *rhoe, double *rho_old, double *f,
                          double *g, int nnr) {
  double d = 0.0;
  AndersonRhoMix(iter, beta, rhoe, rho_old, f, g, nnr, d);
  return d;
}

double ref_BroydenRhoMix(int iter, double alpha, double w0, double *rho, double *rho_old,
                         double *f, double *df, double *u, double *a, int mixdim, int nnr) {
  double d = 0.0;
  BroydenRhoMix(iter, alpha, w0, rho, rho_old, f, df, u, a, mixdim, nnr, d);
  return d;
}

double ref_KerkerRhoMix(double beta, double q0, double *rhoe, double *rho_old, int nnr) {
  double d = 0.0;
  KerkerRhoMix(beta, q0, rhoe, rho_old, nnr, d);
  return d;
}

/* ---- the reference program's own set-up and SCF loop (main.cpp) ---- */

/* ReadInputFile + Setup + PrepareSCF on the INPUT in the current directory */
void ref_prog_setup(void) {
  ReadInputFile();
  Setup();
  PrepareSCF();
}

/* the starting density of ChebySCFLoop.cpp:157-168 and EwaldEnergy() */
void ref_prog_start_density(double *rho) {
  double complex *c = (double complex *)malloc(NNR * sizeof(double complex));
  for (int i = 0; i < NNR; i++) c[i] = Z_ZERO;
  FormFactorAtomic(c);
  fft_fftw3(c, NR1, NR2, NR3, true);
  for (int i = 0; i < NNR; i++) rho[i] = creal(c[i]);
  NormalizeRho(rho, NNR, OMEGA, NEL);
  free(c);
  EwaldEnergy();
}

/* SFAC (NSP x NG complex), VPS, RHOPS (NSP x NG of NSP x NGX), and
 * scal = {ESR, ESELF, NEL, OMEGA} */
void ref_get_local(double complex *sfac, double *vps, double *rhops, double *scal) {
  for (long i = 0; i < (long)NSP * NG; i++) {
    sfac[i] = SFAC[i];
    vps[i] = VPS[i];
    rhops[i] = RHOPS[i];
  }
  scal[0] = ESR;
  scal[1] = ESELF;
  scal[2] = NEL;
  scal[3] = OMEGA;
}

/* PKG_A (NLMAX x NGWX x NSP, k-point 1) and WNL (NSP x NLMAX) */
void ref_get_nl(double *pkg_a, double *wnl) {
  for (long i = 0; i < (long)NLMAX * NGWX * NSP; i++) pkg_a[i] = PKG_A[i];
  for (long i = 0; i < (long)NSP * NLMAX; i++) wnl[i] = WNL[i];
}

/* TAU(3, NAX, NSP) in bohr after ReadInputFile's conversions */
void ref_get_tau(double *tau) {
  for (int i = 0; i < 3 * NAX * NSP; i++) tau[i] = TAU[i];
}

/* NA, L_MAX, L_LOC per species (NSP entries each) */
void ref_get_species(int *na, int *lmax, int *lloc) {
  for (int is = 0; is < NSP; is++) {
    na[is] = NA[is];
    lmax[is] = L_MAX[is];
    lloc[is] = L_LOC[is];
  }
}

/* iv = {NX, NEMPTY, CHEBYPOL_DEGREE, MAX_SCF_ITER, IMIX, MIXDIM, IDIAG,
 *       USER_MAX_DIAG_ITER, MAX_DIAG_ITER},
 * dv = {SCF_CONV_CRIT, RHO_MIX_FAC, KERKER_Q0}, focc = FOCC (NX) */
void ref_get_ctrl(int *iv, double *dv, double *focc) {
  iv[0] = NX;
  iv[1] = NEMPTY;
  iv[2] = CHEBYPOL_DEGREE;
  iv[3] = MAX_SCF_ITER;
  iv[4] = IMIX;
  iv[5] = MIXDIM;
  iv[6] = IDIAG;
  iv[7] = USER_MAX_DIAG_ITER ? 1 : 0;
  iv[8] = MAX_DIAG_ITER;
  dv[0] = SCF_CONV_CRIT;
  dv[1] = RHO_MIX_FAC;
  dv[2] = KERKER_Q0;
  for (int i = 0; i < NX; i++) focc[i] = FOCC[i];
}

/* ChebySCFLoop() with rand() seeded by srand(1); eig = EIG (NX), e6 =
 * {ETOT, EKIN, EHT, EPSEU, ENL, EXC} at the end */
void ref_prog_cheby_scf(double *eig, double *e6) {
  srand(1);
  ChebySCFLoop();
  for (int i = 0; i < NX; i++) eig[i] = EIG[i];
  e6[0] = ETOT;
  e6[1] = EKIN;
  e6[2] = EHT;
  e6[3] = EPSEU;
  e6[4] = ENL;
  e6[5] = EXC;
}

double ref_SimpleRhoMix(double beta, double *rhoe, double *rho_old, int nnr) {
  double d = 0.0;
  SimpleRhoMix(beta, rhoe, rho_old, nnr, d);
  return d;
}

}  // extern "C"
