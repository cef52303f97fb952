/*
 * pspw_gpu.h -- C ABI of the B200 Hamiltonian-application and eigensolver
 * engine for the plane-wave Kohn-Sham method of f-fathurrahman/ffr-pspw-dft-c.
 *
 * Plain pointers and sizes only.  Complex arrays are interleaved (re, im)
 * doubles (layout-identical to C99 `double complex`) or floats, column-major
 * with an explicit leading dimension, exactly as the reference stores them.
 * Every entry point returns a status code (PSPW_OK = 0); pspw_last_error()
 * gives the message of the last failure on the calling thread.
 *
 * Handle model: one pspw_cell per geometry and k-point holds device copies of
 * the basis and projector arrays and of V_eff(r), plus a CUDA stream and
 * persistent workspaces.  Calls on one cell are serialised by the caller;
 * different cells are independent.
 *
 * Reference interfaces replaced (file:line in the reference repository):
 *   pspw_cell_create         SetupArrays_ApplyHam_cuda   common_pspw.h:255
 *   pspw_cell_set_veff       CopyRho_ApplyHam_cuda       common_pspw.h:257
 *   pspw_cell_destroy        FreeArrays_ApplyHam_cuda    common_pspw.h:258
 *   pspw_apply_ham_block     ApplyHam_block              common_pspw.h:177, ApplyHam_block.cpp:5
 *   pspw_apply_ham_block_dev ApplyHam_block_cuda         common_pspw.h:254
 *   pspw_chebyfilt           chebyfilt                   common_pspw.h:187, chebyfilt.cpp:6
 */
#ifndef PSPW_GPU_H
#define PSPW_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* status codes */
#define PSPW_OK 0
#define PSPW_ERR_ARG 1       /* invalid argument (null pointer, negative size)   */
#define PSPW_ERR_SHAPE 2     /* inconsistent sizes (nnr != NNR, ngw > cell ngw)  */
#define PSPW_ERR_CUDA 3      /* CUDA runtime / library failure                    */
#define PSPW_ERR_OOM 4       /* device allocation failed                          */
#define PSPW_ERR_NONFINITE 5 /* NaN/Inf detected in an input that is checked      */
#define PSPW_ERR_TIMEOUT 6   /* a bounded device-side wait ran out                */
#define PSPW_ERR_LAPACK 7    /* dense factorisation/eigensolver info != 0         */
#define PSPW_ERR_CHARGE 8    /* EvalRhoPsi: |sum |c|^2 - 1| > 6e-3                */
#define PSPW_ERR_NOT_IMPL 9  /* e.g. more than 4 KB projectors per atom           */

/* arithmetic of device-resident wavefunction blocks */
#define PSPW_PREC_F64 0 /* complex128 (interleaved double) */
#define PSPW_PREC_F32 1 /* complex64  (interleaved float)  */

typedef struct pspw_cell pspw_cell;

typedef struct {
  int nr[3];   /* FFT grid NR1, NR2, NR3                 */
  int ngw;     /* wavefunction sphere size NGW(1)        */
  int ngwx;    /* padded leading dimension NGWX          */
  int ngx;     /* NGX                                    */
  int ng;      /* density sphere size NG                 */
  double alat, omega, tpiba, tpiba2, gcut, gcutw;
} pspw_basis_info;

const char *pspw_error_string(int code);
const char *pspw_last_error(void);
int pspw_version(void);

/* ------------------------------------------------------------------ basis
 * Gamma-point basis generation with the reference's set-up rules
 * (Setup.cpp:20-66, GVectorsGen0.cpp, GVectorsGen.cpp, GkVectorsGen.cpp,
 * PhaseFactor.cpp).  lattice9 = A1, A2, A3 (bohr), ecut_ry = ECUT in Rydberg,
 * nr_forced = {NR1,NR2,NR3} or NULL/{0,..} for the reference grid rule.
 * _info fills sizes (ngw and ng stay -1 until _build); _build fills the
 * arrays: n123/xkg/igk [ngwx]; n1..in3, g [ngx]; gg [(ngx+1)*3];
 * eigr [2*ngwx*nax*nsp] (may be NULL), tau = TAU(3,NAX,NSP) in bohr. */
int pspw_basis_info_gamma(const double *lattice9, double ecut_ry, const int *nr_forced,
                          pspw_basis_info *info);
int pspw_basis_build_gamma(const double *lattice9, double ecut_ry, const int *nr_forced, int nsp,
                           const int *na, const double *tau, pspw_basis_info *info,
                           unsigned int *n123, double *xkg, int *igk, int *n1, int *n2, int *n3,
                           int *in1, int *in2, int *in3, double *g, double *gg, double *eigr);

/* ------------------------------------------------------------------ cell
 * Device copy of one k-point's Hamiltonian data (replaces
 * SetupArrays_ApplyHam_cuda, common_pspw.h:255).  Arguments are the
 * reference globals for column ik:
 *   n123[ngwx]   N123(:,ik), 1-based FFT-grid index        (GkVectorsGen.cpp:379)
 *   xkg[ngwx]    XKG(:,ik), |k+G|^2 in (2 pi/ALAT)^2
 *   eigr         EIGR(:,:,:,ik), 2*ngwx*nax*nsp doubles
 *   pkg_a        PKG_A(:,:,:,ik), nlmax*ngwx*nsp doubles
 *   wnl          WNL(nsp, nlmax)
 *   lm_end[nsp]  L_MAX^2 - 2 L_LOC + 1 per species (<= 4, ApplyHam_block.cpp:69-73)
 * ngw is the number of plane waves of this k-point (NGW(ik)). */
int pspw_cell_create(pspw_cell **cell, int device, int nr1, int nr2, int nr3, int ngw, int ngwx,
                     const unsigned int *n123, const double *xkg, double tpiba2, int nsp,
                     const int *na, int nax, const int *lm_end, int nlmax, const double *eigr,
                     const double *pkg_a, const double *wnl);
int pspw_cell_destroy(pspw_cell *cell);
/* V_eff(r) on the FFT grid, NR1 fastest (the `rho` argument of ApplyHam*;
 * replaces CopyRho_ApplyHam_cuda, common_pspw.h:257).  nnr must equal
 * NR1*NR2*NR3 (ApplyHam_block.cpp:18-21). */
int pspw_cell_set_veff(pspw_cell *cell, const double *veff, int nnr);
int pspw_cell_set_veff_device(pspw_cell *cell, const double *d_veff, int nnr);
/* the cell's CUDA stream (cudaStream_t), a wait for its queued work, and
 * basic sizes {n1,n2,n3,ngw,sticks,active x,atoms,projectors} */
int pspw_cell_get_stream(pspw_cell *cell, void **stream);
int pspw_cell_synchronize(pspw_cell *cell);
int pspw_cell_sizes(pspw_cell *cell, int *out8);
/* cap the number of bands transformed per batch of the FFT passes
 * (0 = automatic); results do not depend on it */
int pspw_cell_set_band_batch(pspw_cell *cell, int nbatch);

/* Kernels of the FP32 projector GEMMs (no reference counterpart: the
 * reference has one CPU path).  AUTO takes the tensor-core (tcgen05, 3xTF32)
 * kernels when every species with projectors has at most 256 atoms and at
 * most 4 projectors per atom (one projection and one back-projection per
 * such species), else the SIMT kernels; TENSOR_CORE on a cell outside that
 * range is PSPW_ERR_NOT_IMPL.  The FP64 path does not depend on it: it stores the
 * projectors once per cell and runs both products on the FP64 tensor-core
 * GEMM (the allocation-free entry point keeps SIMT kernels). */
#define PSPW_NL_AUTO 0
#define PSPW_NL_SIMT 1
#define PSPW_NL_TENSOR_CORE 2
int pspw_cell_set_nl_path(pspw_cell *cell, int path);

/* Whether the projection of H*psi runs on the cell's second stream,
 * concurrently with the FFT passes (AUTO, ON), or after them on the cell
 * stream (OFF); no reference counterpart.  Results do not depend on it (the
 * same kernels run in the same order of arithmetic).  The allocation-free
 * entry point always keeps one stream. */
#define PSPW_OVERLAP_AUTO 0
#define PSPW_OVERLAP_ON 1
#define PSPW_OVERLAP_OFF 2
int pspw_cell_set_nl_overlap(pspw_cell *cell, int mode);

/* Check of the device timeout path (no reference counterpart).  Every
 * barrier wait in the engine's tensor-core kernels gives up after about one
 * second and raises the cell's error word, which the next call that
 * synchronises reports as PSPW_ERR_TIMEOUT; the context and the cell stay
 * usable.  This runs one such wait on the cell stream: with complete == 0
 * nothing completes the barrier and the call returns PSPW_ERR_TIMEOUT after
 * about a second; with complete != 0 it returns PSPW_OK. */
int pspw_cell_check_device_wait(pspw_cell *cell, int complete);

/* ------------------------------------------------------------------ H*psi
 * vout = H vin for nstates bands (ApplyHam_block.cpp:5-172): kinetic
 * 0.5*XKG*TPIBA2, local V_eff through an FFT sandwich, KB nonlocal
 * sum_a,lm beta W beta^H.  Host FP64 buffers, ld = ngw. */
int pspw_apply_ham_block(pspw_cell *cell, const double *vin, double *vout, int ngw, int nstates);
/* Device buffers of precision `prec`, leading dimension ld >= ngw
 * (replaces ApplyHam_block_cuda, common_pspw.h:254).  Enqueued on the cell
 * stream; returns without synchronising. */
int pspw_apply_ham_block_dev(pspw_cell *cell, int prec, const void *d_vin, void *d_vout, int ld,
                             int ngw, int nstates);

/* The same H*psi as pspw_apply_ham_block_dev, with no device allocation on
 * the call path.  No counterpart in the reference.  For callers that cannot
 * let a library allocate when it is called: code being captured into a CUDA
 * graph, applications whose memory manager owns all device memory, services
 * that must not fail for lack of memory mid-request.  All scratch comes from
 * one static 16 MiB device array in the library (held by every GPU that
 * loads it until exit); cell/block sizes whose scratch does not fit are
 * rejected with PSPW_ERR_SHAPE.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and should come before any
 * stream capture.  The address is kept per device index for the life of the
 * process; cudaDeviceReset unloads the library's device image, so after a
 * reset this entry point must not be called again in that process.  All
 * calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller.  Set V_eff with
 * pspw_cell_set_veff_device, which does not allocate either. */
int pspw_apply_ham_block_dev_noalloc(pspw_cell *cell, int prec, const void *d_vin, void *d_vout,
                                     int ld, int ngw, int nstates);

/* ------------------------------------------------------------------ filter
 * Degree-`degree` scaled Chebyshev filter of chebyfilt.cpp:6-74 applied to
 * the ngw x nstates block X in place.  Host FP64 X; `prec` selects the
 * arithmetic on the device (F64 = the reference's, F32 = mixed precision). */
int pspw_chebyfilt(pspw_cell *cell, double *X, int ngw, int nstates, int degree, double lb,
                   double ub, int prec);
int pspw_chebyfilt_dev(pspw_cell *cell, int prec, void *d_X, int ld, int ngw, int nstates,
                       int degree, double lb, double ub);

/* ------------------------------------------------------------------ solvers
 * Host-buffer entry points with the reference routines' semantics; all
 * arithmetic on the device.  `prec`/`hprec` arrays are host.
 *
 * random_col      util_random_cpu.cpp:5   (host, bit-exact LCG start vectors)
 * gen_prec        GenPrec.cpp:5           prec[nbasis] from XKG, tau
 * ortho_qr        ortho_qr.cpp:3          X (nbasis x nstates) <- Q of its QR
 * eig_zheevd      eig_zheevd.cpp:5        A <- eigenvectors, lambda <- eigenvalues
 * eig_zhegv(_eval) eig_zhegv.cpp:5,86     generalised problem via B^-1/2
 * davidson        davidson_cpu.cpp:9      block Davidson, 2nb subspace
 * lobpcg          lobpcg_cpu.cpp:31       LOBPCG with Cholesky-orthonormalised W, P
 * lanczos         lanczos.cpp:8           k-step Lanczos: T (k x k), residual f
 * eval_rho_psi    EvalRhoPsi.cpp:83       rhoe += sum_i w f_i |psi_i(r)|^2 / Omega
 *
 * davidson/lobpcg overwrite X with their random start and return the
 * eigenvectors there; nempty = NEMPTY; max_iter <= 0 selects the reference
 * default max(30, nstates/2); hprec is the arithmetic of H*psi inside the
 * solver (the rest is FP64); resnrm[nstates] and iters may be NULL.
 * Davidson with hprec = PSPW_PREC_F32 is supported for small blocks only:
 * its 2 nstates subspace overlap becomes nearly singular on large blocks
 * (measured on a 512-state, 216-atom cell), and the reference's eig_zhegv
 * scales every overlap direction above 1.2e-15 by 1/sqrt(eigenvalue)
 * (eig_zhegv.cpp:39-47), which turns the FP32 rounding of H R into
 * spurious Ritz values.  Use FP64 H*psi with Davidson on large blocks, or
 * LOBPCG, which stays bounded with FP32 H*psi.
 * eval_rho_psi: eigvec columns with leading dimension ld, the last plane
 * wave of each band is left out as in the reference, *ekin += EKIN part;
 * returns PSPW_ERR_CHARGE when a band's norm is off by more than 6e-3. */
int pspw_random_col(double *A, int nelem, long seed);
int pspw_gen_prec(pspw_cell *cell, double *prec, int nbasis, double tau);
int pspw_ortho_qr(pspw_cell *cell, double *X, int nbasis, int nstates);
int pspw_eig_zheevd(pspw_cell *cell, double *A, int lda, double *lambda, int n);
int pspw_eig_zhegv(pspw_cell *cell, double *A, int lda, double *B, int ldb, double *evec, int lde,
                   int n);
int pspw_eig_zhegv_eval(pspw_cell *cell, double *A, int lda, double *B, int ldb, double *eval,
                        double *evec, int lde, int n);
int pspw_davidson(pspw_cell *cell, double *evals, double *X, int nbasis, int nstates,
                  const double *prec, int nempty, int max_iter, int hprec, double *resnrm,
                  int *iters);
int pspw_lobpcg(pspw_cell *cell, double *lambda, double *X, int nbasis, int nstates,
                const double *prec, int nempty, int max_iter, int hprec, double *resnrm,
                int *iters);
/* LOBPCG with an orthonormal search basis (no reference counterpart; an
 * opt-in alternative to pspw_lobpcg with the same arguments, start and
 * convergence test).  The reference's lobpcg_cpu orthonormalises W and P
 * each on its own and solves a generalised Rayleigh-Ritz problem whose
 * overlap becomes nearly singular near convergence; here W and P are made
 * orthogonal to X (W also to P) before their Cholesky QR, so [X W P] is
 * orthonormal and the Rayleigh-Ritz step is a standard Hermitian
 * eigenproblem; P is dropped for one iteration when it cannot be
 * orthonormalised. */
int pspw_lobpcg_ortho(pspw_cell *cell, double *lambda, double *X, int nbasis, int nstates,
                      const double *prec, int nempty, int max_iter, int hprec, double *resnrm,
                      int *iters);
/* The same solver started from the caller's block: X (host, nbasis x
 * nstates) is read as the start (orthonormalised first) and overwritten
 * with the result. */
int pspw_lobpcg_ortho_from(pspw_cell *cell, double *lambda, double *X, int nbasis, int nstates,
                           const double *prec, int nempty, int max_iter, int hprec,
                           double *resnrm, int *iters);
int pspw_lanczos(pspw_cell *cell, double *v0, int ngw, int k, double *T, int ldT, double *f);
int pspw_eval_rho_psi(pspw_cell *cell, double *rhoe, const double *eigvec, int ld, int ngw,
                      int nx, const double *focc, double wkpt, double omega, double *ekin);

/* Nonlocal energy of one k-point (EvalENL.cpp:5-49): with C0 (host,
 * ngw x nx complex, leading dimension ld, used unconjugated)
 *   FNL(ist, p) = sum_{G < ngw} C0(G, ist) PKG_A(lm_p, G) conj(EIGR(G, atom_p))
 *   *enl        = wkpt * sum_p WNL(p) sum_ist focc[ist] |FNL(ist, p)|^2
 * accumulated over projectors in the reference's (species, atom, lm) order.
 * fnl (may be null) receives FNL as nx x nproj complex, column-major.  FP64
 * on the device. */
int pspw_eval_enl(pspw_cell *cell, const double *c0, int ld, int ngw, int nx,
                  const double *focc, double wkpt, double *enl, double *fnl);
/* the same two on device pointers (rhoe, eigvec, c0: device FP64; focc, enl,
 * fnl, ekin: host) */
int pspw_eval_rho_psi_dev(pspw_cell *cell, double *d_rhoe, const double *d_eigvec, int ld,
                          int ngw, int nx, const double *focc, double wkpt, double omega,
                          double *ekin);
int pspw_eval_enl_dev(pspw_cell *cell, const double *d_c0, int ld, int ngw, int nx,
                      const double *focc, double wkpt, double *enl, double *fnl);

/* ------------------------------------------------------------------ dense steps, device pointers
 * The subspace products of the solvers and of the SCF loop (the zgemm_
 * calls of davidson_cpu.cpp:120-178, lobpcg_cpu.cpp:103-309,
 * eig_zhegv.cpp:50-60 and ChebySCFLoop.cpp:296-306) on device FP64 complex
 * column-major matrices, enqueued on the cell stream.
 *
 * zgemm_dev   C = alpha op(A) B + beta C; op(A) = A ('N') or A^H ('C'),
 *             any other opa is PSPW_ERR_ARG; alpha, beta: host {re, im}.
 *             More than 8 columns run on the FP64 tensor-core instruction
 *             (DMMA); long K with a small output is split over blocks and
 *             reduced in a fixed order (bitwise repeatable). */
int pspw_zgemm_dev(pspw_cell *cell, char opa, int m, int n, int k, const double *alpha,
                   const double *d_A, int lda, const double *d_B, int ldb, const double *beta,
                   double *d_C, int ldc);
/* eig_zheevd_dev  eig_zheevd.cpp:5-34 on device pointers: A (n x n, lda,
 *             upper triangle read) <- orthonormal eigenvectors, w[n] (device)
 *             <- eigenvalues ascending.  n <= 150 (the Rayleigh-Ritz matrix
 *             of the Chebyshev SCF loop is (NX+2) x (NX+2)) runs on the
 *             engine's own kernels: Householder tridiagonalisation in one
 *             block's shared memory, bisection, twisted factorisations
 *             (inverse iteration for clusters); larger n on cuSOLVER
 *             zheevd.  Bitwise repeatable. */
int pspw_eig_zheevd_dev(pspw_cell *cell, double *d_A, int lda, double *d_w, int n);
/* ortho_span_dev  an orthonormal basis of span(X) in place, the step that
 *             ortho_qr performs in the Chebyshev SCF loop
 *             (ChebySCFLoop.cpp:288-291): columns scaled to unit norm, then
 *             CholeskyQR2 (Gram matrices and products by U^-1 on the DMMA
 *             GEMM, Cholesky factor and inverse in one block) for n <= 150,
 *             the Householder QR when the first Cholesky factor shows
 *             cond(X) above 1e6 or n > 150.  X: device, ngw x n, ld ngw.
 *             The basis spans the same space as ortho_qr's and Rayleigh-Ritz
 *             gives the same Ritz pairs; the columns themselves differ. */
int pspw_ortho_span_dev(pspw_cell *cell, double *d_X, int ngw, int n);

/* ------------------------------------------------------------------ SCF pieces
 * The steps of the SCF iteration around the eigensolver, on the device in
 * FP64, with the local-potential data and the density-mixing history kept
 * in a pspw_scf handle bound to a cell (same grid, same stream).
 *
 * pspw_scf_create   the data EvalEnergy.cpp reads besides the density: the
 *                   NG density G vectors as 1-based grid indices N1, N2, N3
 *                   (G = 0 first) and |G|^2 in (2 pi/alat)^2 units (the
 *                   global G), SFAC (complex), VPS and RHOPS (real), each
 *                   NSP x NG with the species index fastest, OMEGA, NEL,
 *                   ESR, ESELF.
 * eval_energy       EvalEnergy.cpp:5-163: rhoe in = density, out = V_eff =
 *                   Re(V_H + V_loc) + V_xc; e6 = {ETOT, EKIN, EHT, EPSEU,
 *                   ENL, EXC} with EKIN and ENL supplied by the caller.
 *                   Grid points outside the density sphere keep the
 *                   transformed density before the inverse transform, as in
 *                   the reference.
 * xc_pz             xc_PZ.cpp:7-63 (Perdew-Zunger LDA): vxc and Exc (the
 *                   plain sum of rho (ex + ec), not yet x OMEGA/NNR).
 * normalize_rho     NormalizeRho.cpp:7-33 with the handle's OMEGA and NEL;
 *                   *warn = 1 where the reference prints its warning;
 *                   PSPW_ERR_CHARGE where it aborts (sum < 1e-15).
 * kerker_prec       KerkerRhoMix.cpp:53-81: x <- FFT^-1 [beta gg/(gg+q0)
 *                   FFT x] on the wavefunction sphere of the cell (other
 *                   components unchanged, as in the reference).
 * mix_init / mix    SimpleRhoMix.cpp, KerkerRhoMix.cpp:5-50,
 *                   AndersonRhoMix.cpp:8-91, PulayRhoMix.cpp:5-91,
 *                   BroydenRhoMix.cpp:10-104 (beta is a parameter; the
 *                   reference's Pulay uses 0.25 and its Broyden alpha = 0.25,
 *                   w0 = 0.01, ChebySCFLoop.cpp:240,336).  The history
 *                   starts at zero as in ChebySCFLoop.cpp:123-148; rho_old
 *                   (may be null) fills its first column.  iter counts from
 *                   1; *d = the mixer's residual measure. */
typedef struct pspw_scf pspw_scf;
#define PSPW_MIX_SIMPLE 0
#define PSPW_MIX_KERKER 1
#define PSPW_MIX_ANDERSON 2
#define PSPW_MIX_PULAY 3
#define PSPW_MIX_BROYDEN 4
int pspw_scf_create(pspw_cell *cell, int ng, const int *n1, const int *n2, const int *n3,
                    const double *g, int nsp, const double *sfac, const double *vps,
                    const double *rhops, double omega, double nel, double esr, double eself,
                    pspw_scf **out);
int pspw_scf_destroy(pspw_scf *scf);
int pspw_eval_energy(pspw_scf *scf, double *rhoe, double ekin, double enl, double *e6);
int pspw_eval_energy_dev(pspw_scf *scf, double *d_rhoe, double ekin, double enl, double *e6);
int pspw_xc_pz(pspw_scf *scf, const double *rho, double *vxc, double *exc);
int pspw_normalize_rho(pspw_scf *scf, double *rho, int *warn);
int pspw_kerker_prec(pspw_scf *scf, double *x, double beta, double q0);
/* the same three on device vectors (NNR doubles on the cell's device) */
int pspw_xc_pz_dev(pspw_scf *scf, const double *d_rho, double *d_vxc, double *exc);
int pspw_normalize_rho_dev(pspw_scf *scf, double *d_rho, int *warn);
int pspw_kerker_prec_dev(pspw_scf *scf, double *d_x, double beta, double q0);
int pspw_mix_init(pspw_scf *scf, int kind, int mixdim, double beta, double q0,
                  const double *rho_old);
int pspw_mix(pspw_scf *scf, int iter, double *rhoe, double *d);
int pspw_mix_dev(pspw_scf *scf, int iter, double *d_rhoe, double *d);

/* ------------------------------------------------------------------ SCF loop
 * pspw_cheby_scf: the Chebyshev-filtered SCF iteration of ChebySCFLoop.cpp:
 * 36-378 (one k-point) with V_eff, the densities, the mixing history and the
 * wavefunction block on the device.
 *   params     the reference's INPUT controls (below)
 *   focc       NX occupations (FOCC)
 *   rho_start  the normalised starting density (NNR; the reference builds it
 *              with FormFactorAtomic + NormalizeRho, ChebySCFLoop.cpp:160-168)
 *   v0         the Lanczos start vector (NGW complex; the reference draws it
 *              with rand(), ChebySCFLoop.cpp:100-106)
 *   X          NGW x (NX+2) complex: the start block when idiag < 0 (it is
 *              orthonormalised), the final block on return
 *   eig        NX eigenvalues (EIG); rho_out (may be null) the final mixed
 *              density; hist (may be null) 4 x max_scf_iter: per iteration
 *              ETOT, |dETOT|, the mixer's d, and the milliseconds from the
 *              start of the call to the end of the iteration (host clock,
 *              taken after the iteration's results reached the host); e6 the final {ETOT, EKIN, EHT,
 *              EPSEU, ENL, EXC}; *iterations the last iteration done;
 *              *converged = 1 if |dETOT| <= conv was reached.
 * The pspw_scf handle supplies the local potential data, OMEGA and NEL. */
typedef struct {
  int nx;             /* NX: occupied + empty states; the filter works on NX + 2 */
  int nempty;         /* NEMPTY (Davidson's convergence count) */
  int degree;         /* CHEBYPOL_DEGREE */
  int max_scf_iter;   /* MAX_SCF_ITER */
  double conv;        /* SCF_CONV_CRIT on |ETOT - ETOT_old| (Ha) */
  int imix;           /* IMIX: 1 Kerker, 2 Anderson, 3 Pulay, 4 Broyden,
                         other: simple */
  int mixdim;         /* MIXDIM (Pulay) */
  double mix_beta;    /* RHO_MIX_FAC (simple, Kerker, Anderson) */
  double pulay_beta;  /* the Pulay warm-up beta and Broyden alpha (0.25 in the
                         reference) */
  double kerker_q0;   /* KERKER_Q0 */
  int idiag;          /* IDIAG: >= 0 first iteration by Davidson, < 0 start from X */
  int max_diag_iter;  /* Davidson iteration cap; 0 = the reference's default */
  int filter_prec;    /* PSPW_PREC_F64, or PSPW_PREC_F32 for the filter and the H*v
                         products of the Lanczos filter bounds (the rest FP64) */
  int tmetal;         /* TMETAL: 0 fixed occupations (the reference's loop);
                         1 Fermi-Dirac occupations of the Ritz values after
                         every Rayleigh-Ritz step (FermiEnergy.cpp, which the
                         reference reads but never calls) */
  double ekt;         /* EKT: the electronic temperature of TMETAL, in eV */
} pspw_scf_params;
int pspw_cheby_scf(pspw_scf *scf, const pspw_scf_params *params, const double *focc,
                   const double *rho_start, const double *v0, double *X, double *eig,
                   double *rho_out, double *hist, int *iterations, int *converged, double *e6);

/* ------------------------------------------------------------------ system
 * One system set up from the reference's own input files, the way its main
 * program does before the SCF loop (main.cpp:20-30):
 *   pspw_system_load      ReadInputFile (INPUT in `dir`), ReadPseudopotentials
 *                         (FHI98 files named in INPUT, relative to `dir`),
 *                         Setup, PrepareSCF (PhaseFactor, StructureFactor,
 *                         FormFactor, NLFormFactor), the starting density of
 *                         ChebySCFLoop.cpp:157-168 and EwaldEnergy.  The
 *                         G-vector list and its heap-sort order are built on
 *                         the host; EIGR, SFAC, VPS/RHOPS, PKG_A, the
 *                         starting density and ESR on the device, which then
 *                         holds a ready pspw_cell and pspw_scf.
 *   pspw_system_cheby_scf ChebySCFLoop() on that system (rand() seeded 1 as in
 *                         a fresh reference process, drawn from a private
 *                         generator state); with outdir it writes
 *                         STARTING_RHO.dat and FINAL_RHO.dat (Print3DArray).
 * device < 0 stops after the host part (readers, basis, occupations, WNL,
 * ESELF): no GPU is touched, the device arrays, cell and SCF are absent.
 * One Gamma-point k-point only (ChebySCFLoop.cpp:74-77); L_MAX <= 3.
 * info: dims16 = {NR1, NR2, NR3, NNR, NGW, NGWX, NG, NGX, NX, NLMAX, NAX, NSP,
 * NEMPTY, ISCF, NKPT, IDIAG}; scal16 = {TPIBA, TPIBA2, OMEGA, ALAT, GCUT,
 * GCUTW, NEL, ESR, ESELF, ECUT, WKPT, 0...}.
 * array: a copy of one set-up array, nbytes must equal its size:
 *   EIGR 16*NGWX*NAX*NSP, SFAC 16*NSP*NG (NSP leading), VPS and RHOPS
 *   8*NSP*NG, PKG_A 8*NLMAX*NGWX*NSP, RHO_START 8*NNR, WNL 8*NSP*NLMAX,
 *   FOCC 8*NX, N123 4*NGWX, XKG 8*NGWX, TAU 8*3*NAX*NSP, G 8*NG.
 * timing: ms8 = {host input + basis, phase + structure factors, local form
 * factors, nonlocal form factors, cell + SCF handles, starting density,
 * Ewald sum, total}. */
typedef struct pspw_system pspw_system;
#define PSPW_SYS_EIGR 0
#define PSPW_SYS_SFAC 1
#define PSPW_SYS_VPS 2
#define PSPW_SYS_RHOPS 3
#define PSPW_SYS_PKG_A 4
#define PSPW_SYS_RHO_START 5
#define PSPW_SYS_WNL 6
#define PSPW_SYS_FOCC 7
#define PSPW_SYS_N123 8
#define PSPW_SYS_XKG 9
#define PSPW_SYS_TAU 10
#define PSPW_SYS_G 11
int pspw_system_load(const char *dir, int device, pspw_system **out);
int pspw_system_destroy(pspw_system *sys);
int pspw_system_info(pspw_system *sys, int *dims16, double *scal16);
int pspw_system_params(pspw_system *sys, pspw_scf_params *params);
int pspw_system_array(pspw_system *sys, int which, void *host, long long nbytes);
int pspw_system_cell(pspw_system *sys, pspw_cell **cell);
int pspw_system_scf(pspw_system *sys, pspw_scf **scf);
int pspw_system_timing(pspw_system *sys, double *ms8);
int pspw_system_cheby_scf(pspw_system *sys, int filter_prec, const char *outdir, double *eig,
                          double *e6, int *iterations, int *converged, double *hist);
/* The same loop with explicit controls (no reference counterpart: the
 * reference reads them from INPUT and hard-codes the Pulay warm-up beta
 * 0.25, PulayRhoMix.cpp:10).  Start from pspw_system_params and change what
 * differs, e.g. pulay_beta and mixdim; params->nx must be the system's NX. */
int pspw_system_cheby_scf_with(pspw_system *system, const pspw_scf_params *params,
                               const char *outdir, double *eig, double *e6, int *iterations,
                               int *converged, double *hist);
/* Print3DArray.cpp:5-22: n1*n2*n3 values, one `%18.10f` per line */
/* Atoms and KB projectors of a system (no reference counterpart; the
 * reference keeps them in the globals NA, L_MAX, L_LOC): natoms = sum NA,
 * nproj = sum over species of NA * lm_end.  Valid for host-only systems. */
int pspw_system_species(pspw_system *system, int *natoms, int *nproj);

/* ------------------------------------------------------------------ batches
 * Block H*psi on many independent cells in one launch (no reference
 * counterpart; the reference applies ApplyHam_block to one cell per
 * process).  create: ncells cells on one device, each with V_eff set, and
 * nbands[i] bands per cell, in precision prec; the batch allocates each
 * cell's input and output block (NGW x nbands, ld = the cell's NGW), which
 * blocks returns.  tune: for every cell, times the schedules that give the
 * same result (band batches of the FFT passes; tensor-core or SIMT
 * projector kernels for FP32 cells of one species), `reps` timed calls
 * each, keeps the fastest (cached per cell shape for the process) and
 * drops the captured graph.  apply: one CUDA graph launch on the batch
 * stream doing H*psi for every cell (captured on the first apply after
 * create or tune; the cells' kernels run on concurrent branches), returns
 * without synchronising.  A cell's result is the same alone and in the
 * batch.  The cells must stay alive and unchanged (V_eff, schedules) while
 * the batch exists. */
typedef struct pspw_batch pspw_batch;
int pspw_batch_create(int ncells, pspw_cell *const *cells, const int *nbands, int prec,
                      pspw_batch **out);
int pspw_batch_blocks(pspw_batch *batch, int i, void **d_in, void **d_out);
/* host copies of cell i's input (before apply) and output (after; waits for
 * the batch stream); complex values of the batch's precision, NGW x nbands */
int pspw_batch_upload(pspw_batch *batch, int i, const void *host_in);
int pspw_batch_download(pspw_batch *batch, int i, void *host_out);
int pspw_batch_tune(pspw_batch *batch, int reps);
int pspw_batch_schedule(pspw_batch *batch, int i, int *band_batch, int *nl_path, double *ms);
int pspw_batch_apply(pspw_batch *batch);
/* kernel launches one apply replays (0 before the first apply) */
int pspw_batch_kernels(pspw_batch *batch, long long *kernels);
int pspw_batch_stream(pspw_batch *batch, void **stream);
int pspw_batch_synchronize(pspw_batch *batch);
int pspw_batch_destroy(pspw_batch *batch);

/* ------------------------------------------------------------------ serving
 * Independent SCF jobs on one GPU with continuous batching (no reference
 * counterpart: the reference runs one job per process, main.cpp:20-50).  A
 * job is a directory holding an INPUT and the pseudopotential files it
 * names.  The server runs `slots` jobs at a time on `device`; a job is
 * admitted when a slot is free and the estimated device footprints of the
 * running jobs plus its own stay within hbm_budget_bytes (<= 0: 80 % of the
 * free memory at creation; a job larger than the budget runs alone); jobs
 * that arrive while others run are admitted as slots and memory free up.
 * Each job runs pspw_system_load + pspw_system_cheby_scf_with on its own
 * streams, with its blocks, densities and mixing history on the device from
 * admission to completion, so the kernels of concurrent jobs overlap.  SCF
 * controls: the job's INPUT, with filter_prec, and, where positive,
 * conv_per_atom (|dETOT| <= conv_per_atom * natoms), max_scf_iter,
 * pulay_beta and mixdim overriding it.  Times are seconds since the
 * server's creation.  submit returns at once; wait blocks until the job has
 * finished and copies its result (and up to neig eigenvalues; eig may be
 * NULL).  destroy waits for the submitted jobs to finish. */
typedef struct pspw_server pspw_server;
typedef struct {
  int slots;               /* jobs running at the same time */
  double hbm_budget_bytes; /* admission limit on the summed footprints */
  int filter_prec;         /* PSPW_PREC_F64 or PSPW_PREC_F32 (the mixed form) */
  double conv_per_atom;    /* Ha per atom; <= 0: the INPUT's SCF_CONV_CRIT */
  int max_scf_iter;        /* <= 0: the INPUT's */
  double pulay_beta;       /* <= 0: 0.25, the reference's */
  int mixdim;              /* <= 0: the INPUT's */
} pspw_server_config;
typedef struct {
  int id, status;          /* status: PSPW_OK or the job's error code */
  int natoms, nbands, ngw, nnr, iterations, converged;
  double etot;             /* final total energy (Ha) */
  double footprint_bytes;  /* the estimate the admission used */
  double t_submit, t_admit, t_scf, t_done;  /* submitted, admitted, SCF start, done */
  char error[160];         /* the job's error message when status != PSPW_OK */
} pspw_job_result;
int pspw_server_create(int device, const pspw_server_config *cfg, pspw_server **out);
int pspw_server_submit(pspw_server *server, const char *dir, int *job_id);
int pspw_server_wait(pspw_server *server, int job_id, pspw_job_result *result, double *eig,
                     int neig);
int pspw_server_now(pspw_server *server, double *seconds);
int pspw_server_destroy(pspw_server *server);

int pspw_print_3d_array(const double *a, int n1, int n2, int n3, const char *path);

/* ------------------------------------------------------------------ timing
 * Optional device timing on the cell stream: CUDA events around each launch
 * of the enabled families, summed until reset.  Families (bit i of the mask):
 * 0 whole H*psi / filter call, 1 FFT pass chain, 2 projector GEMMs,
 * 3 sticks_inv, 4 planes_inv, 5 xlines, 6 planes_fwd, 7 sticks_fwd,
 * 8 projection GEMM (+ reduction), 9 back-projection GEMM, 10 subspace GEMMs;
 * phases of a pspw_cheby_scf iteration: 11 filter, 12 QR, 13 Rayleigh-Ritz
 * products (H X, X^H H X, rotation), 14 symmetrize + eigendecomposition,
 * 15 EvalRhoPsi, 16 EvalENL, 17 mixing + EvalEnergy + V_eff, 18 Lanczos
 * bounds. */
int pspw_timing_enable(pspw_cell *cell, int family_mask);
int pspw_timing_read(pspw_cell *cell, int family, double *total_ms, long long *launches);
int pspw_timing_reset(pspw_cell *cell);
/* number of kernels the cell has enqueued since creation */
int pspw_kernel_launches(pspw_cell *cell, long long *count);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif
