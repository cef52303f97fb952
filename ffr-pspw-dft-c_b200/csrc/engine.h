// Internal state of one cell (one geometry and k-point) and the kernel
// launchers shared by the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "pspw_gpu.h"

namespace pspw {

constexpr int kMaxStages = 16;

// One 1D FFT length: radix schedule and the table of its n-th roots of unity
// exp(+2 pi i t / n) (both precisions).
struct FftDim {
  int n = 0;
  int nf = 0;
  int rad[kMaxStages] = {};
  double2 *d_w64 = nullptr;
  float2 *d_w32 = nullptr;
};

// Device copy of the basis in the layouts the kernels read.
//
// The wavefunction sphere is organised in "sticks": the distinct (i1,i2)
// grid columns that hold at least one G of the sphere, numbered in (i2,i1)
// order.  A G entry of stick c sits at z = i3.  The x values that carry a
// stick form the active-x set (nxa of the n1 planes' x positions).
struct Basis {
  int n1 = 0, n2 = 0, n3 = 0, nnr = 0;
  int ngw = 0;
  int ncol = 0;  // sticks
  int nxa = 0;   // active x positions
  int *d_col_start = nullptr;  // [ncol+1] CSR over G entries sorted by stick
  int *d_sg_ig = nullptr;      // [ngw] G index (0-based, caller order)
  int *d_sg_z = nullptr;       // [ngw] i3 of that G
  int *d_sg_col = nullptr;     // [ngw] stick of that G
  // [ngw] (stick mod stick_tile(n3)) * (n3 + 1) + i3: the G's offset in the
  // register-FFT stick kernels' tile
  unsigned short *d_sg_off = nullptr;
  int *d_col_of_xy = nullptr;  // [n1*n2] stick at (i1,i2) or -1
  int *d_xa_list = nullptr;    // [nxa] i1 of active x
  int *d_xa_of_x = nullptr;    // [n1] active index or -1
  double *d_kin64 = nullptr;   // [ngw] 0.5*XKG*TPIBA2
  float *d_kin32 = nullptr;
  double *d_xkg64 = nullptr;   // [ngw] XKG (the preconditioner and EKIN read it)
  int *d_wgrid = nullptr;      // [ngw] 0-based grid index of G (N123 - 1)
  FftDim dim[3];
  // register-FFT path (every length has a two-factor split): stick
  // coordinates, and per axis the natural index held at each position of
  // the digit-permuted order
  bool fast = false;
  int *d_col_x = nullptr;  // [ncol]
  int *d_col_y = nullptr;  // [ncol]
  int *d_pinv[3] = {nullptr, nullptr, nullptr};
};

// KB projectors beta_p(G) = EIGR(G, atom_p) * PKG_A(lm_p, G, species_p).
struct Projectors {
  int nat = 0, nsp = 0, nproj = 0;
  double2 *d_eigr64 = nullptr;  // [nat][ngw], atoms species-major
  float2 *d_eigr32 = nullptr;
  double *d_pkga64 = nullptr;  // [nsp][ngw][4]
  float *d_pkga32 = nullptr;
  // FP64 path: beta_p(G) = EIGR(G, atom_p) PKG_A(lm_p, G) as an NGW x nproj
  // column-major matrix, built on the first FP64 projector call (the DMMA
  // GEMMs of gemm.cu use it as an operand)
  double2 *d_beta64 = nullptr;
  int *d_patom = nullptr;    // [nproj] atom (species-major global index)
  int *d_psp = nullptr;      // [nproj] species
  int *d_plm = nullptr;      // [nproj] lm (0..3)
  double *d_pw64 = nullptr;  // [nproj] WNL(species, lm)
  float *d_pw32 = nullptr;
  // EIGR split into TF32 hi/lo operand tiles of the tensor-core projector
  // GEMMs (one species only; built at cell creation, nl_tc.cu)
  float *d_etp = nullptr;  // projection: per 8 G, [npad atoms x 16] hi then lo
  float *d_etb = nullptr;  // back-projection: per (128 G, 8 atoms), [128 x 16] hi then lo
  // (both hold one block of tiles per species with projectors, species in order)
  int tc_npad = 0;         // atoms padded to a multiple of 16 (largest species)
  std::vector<int> sp_na, sp_lm;  // per species: atoms, projectors per atom (host)
};

// Timing families (bit i of the mask enables family i).
enum Family {
  kFamAll = 0,       // a whole H*psi / filter call
  kFamLocal = 1,     // the five FFT passes of a band batch
  kFamNonlocal = 2,  // projector GEMMs
  kFamSticksInv = 3,
  kFamPlanesInv = 4,
  kFamXlines = 5,
  kFamPlanesFwd = 6,
  kFamSticksFwd = 7,
  kFamProj = 8,
  kFamBackproj = 9,
  kFamGemm = 10,     // subspace GEMMs of the solvers
  // phases of one ChebySCF iteration (pspw_cheby_scf)
  kFamScfFilter = 11,
  kFamScfQr = 12,
  kFamScfRayleigh = 13,  // H X, X^H H X, rotation
  kFamScfEig = 14,       // symmetrize + eigendecomposition of the NX+2 matrix
  kFamScfDensity = 15,   // EvalRhoPsi
  kFamScfEnl = 16,       // EvalENL
  kFamScfMixEnergy = 17, // mixing + EvalEnergy + V_eff upload
  kFamScfLanczos = 18,   // bounds for the next filter
  kNumFamilies = 19
};

// Workspace slots of a cell (grown on demand, kept until the cell is freed).
enum WsSlot {
  kWsSticks = 0,   // FFT stick buffer
  kWsPlanes = 1,   // FFT plane buffer (generic path)
  kWsProjPart = 2, // projector partial sums
  kWsProj = 3,     // projections W beta^H psi
  kWsHostIn = 4,   // host-facing calls: input block
  kWsHostOut = 5,  // host-facing calls: output block
  kWsFilt1 = 6,    // Chebyshev filter blocks
  kWsFilt2 = 7,
  kWsConv = 8,     // FP32 copy of a host block
  kWsGemmPart = 9, // split-K partial sums of the subspace GEMMs
  kWsRhoPart = 10, // density: per-group partial planes
  kWsVeffTmp = 11, // V_eff staging
  kWsSolver = 12,  // cuSOLVER work
  kWsInfo = 13,    // cuSOLVER info
  kWsTau = 14,     // Householder scalars
  kWsEval = 15,    // eigenvalues of the overlap in eig_zhegv
  kWsSolverBase = 16,  // eigensolver blocks 16..31
  kWsWTile = 32,       // projections as tensor-core operand tiles
  kWsEnl = 33,         // EvalENL projections
  kWsScfA = 34,        // SCF-piece host entry points: vectors on the device
  kWsScfB = 35,
  kWsStickX = 36,      // the filter's block in stick order
  kWsHeev = 37,        // the small Hermitian eigensolver's workspace
  kWsSpan = 38,        // pspw_ortho_span_dev: G, U, W, norms (38..41)
  kWsChol = 42,        // the Cholesky factor handed to the triangular inverse
  kWsCount = 43
};

struct Timing {
  int mask = 0;
  double ms[kNumFamilies] = {};
  long long launches[kNumFamilies] = {};
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
};

struct Workspace {
  void *ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace pspw

struct pspw_cell {
  int device = 0;
  cudaStream_t stream = nullptr;
  // second stream for the projection, which runs concurrently with the local
  // part of H*psi (fork and join events on the cell stream)
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // copy stream of the host-facing filter, which moves band chunks in and out
  // while the cell stream filters the other chunk (events per chunk)
  cudaStream_t stream_copy = nullptr;
  cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
  int ngwx = 0;
  double tpiba2 = 0.0;
  int band_batch = 0;
  int nl_path = 0;     // PSPW_NL_AUTO / _SIMT / _TENSOR_CORE
  int nl_overlap = 0;  // PSPW_OVERLAP_AUTO / _ON / _OFF
  pspw::Basis basis;
  pspw::Projectors proj;
  double *d_veff64 = nullptr;  // V_eff / NNR on the grid (forward-FFT scale folded in)
  float *d_veff32 = nullptr;
  double *d_vperm64 = nullptr;  // the same, indexed in the register path's permuted order
  float *d_vperm32 = nullptr;
  bool veff_set = false;
  // persistent scratch: 0 = FFT sticks, 1 = FFT planes, 2 = projector
  // partial sums, 3 = projections, 4.. = block buffers of the filter/solvers
  pspw::Workspace ws[pspw::kWsCount];
  void *cusolver = nullptr;  // cusolverDnHandle_t, created on first use
  void *cublas = nullptr;    // cublasHandle_t, created on first use
  pspw::Timing timing;
  long long kernel_launches = 0;  // kernels this cell has enqueued
  // Stick-order copies of the per-G arrays, for the Chebyshev filter: the
  // filter permutes its block into the order of the stick lists once, runs
  // all its H*psi with these arrays swapped in (the stick gathers and
  // scatters then read and write contiguous runs), and permutes back.
  // Built on the first filter call; swap_stick_order() exchanges them with
  // the cell's own (a second call swaps back).
  struct {
    bool built = false;
    bool active = false;   // the stick-order copies are the ones swapped in
    int *sg_ig = nullptr;  // identity: G k of the stick list is G k
    double *kin64 = nullptr;
    float *kin32 = nullptr;
    double2 *eigr64 = nullptr;
    float2 *eigr32 = nullptr;
    double *pkga64 = nullptr;
    float *pkga32 = nullptr;
    float *etp = nullptr, *etb = nullptr;
    double2 *beta64 = nullptr;
  } stick;
  // Error word the kernels raise when a bounded wait gives up (pinned,
  // mapped host memory: d_err is its device alias).  Read after every
  // stream synchronisation by device_status().
  int *h_err = nullptr;
  int *d_err = nullptr;
};

namespace pspw {

// error state
int fail(int code, const std::string &msg);
// pspw_cell_create, with the projector arrays taken from device copies of
// EIGR(NGWX, NAX, NSP) and PKG_A(NLMAX, NGWX, NSP) when d_eigr and d_pkg_a
// are given (eigr and pkg_a are then unused).
int cell_create(pspw_cell **out, int device, int nr1, int nr2, int nr3, int ngw, int ngwx,
                const unsigned int *n123, const double *xkg, double tpiba2, int nsp, const int *na,
                int nax, const int *lm_end, int nlmax, const double *eigr, const double *pkg_a,
                const double *wnl, const double2 *d_eigr, const double *d_pkg_a);
int cuda_fail(cudaError_t e, const char *what);
// build the stick-order copies (once) and exchange them with the cell's
// per-G arrays; calling it again restores the cell
int swap_stick_order(pspw_cell *c);
#define PSPW_CUDA(call)                                   \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return ::pspw::cuda_fail(_e, #call); \
  } while (0)

int ws_reserve(pspw_cell *c, int slot, size_t bytes, void **out);

// After a stream synchronisation: PSPW_ERR_TIMEOUT (and the flag cleared)
// when a kernel gave up on a bounded wait since the last check.
int device_status(pspw_cell *c);

// Raises a kernel's dynamic shared-memory limit on the current device to the
// most the device allows beside the kernel's static shared memory, once per
// (device, kernel).  Kernels whose dynamic size depends on the problem use
// this instead of setting the limit to each launch's size: the limit is a
// per-kernel setting shared by every host thread, so per-size values set by
// concurrent callers (several cells or jobs at once) could leave it below
// what another thread's launch requests.
int smem_allow_max(const void *kernel);
template <typename K>
int smem_allow_max(K *kernel) {
  return smem_allow_max(reinterpret_cast<const void *>(kernel));
}

// timing hooks (no-ops unless the family is enabled)
void timing_begin(pspw_cell *c, int family, cudaEvent_t *ev);
void timing_end(pspw_cell *c, int family, cudaEvent_t ev);

// Scratch supplied by the caller of hpsi_apply instead of the cell's
// workspaces: stick and plane buffers for `nbatch` bands, `max_split` slices
// of projector partial sums, the projections, and (FP32 on the tensor-core
// path) their operand tiles.
struct ScratchPlan {
  void *S, *P, *part, *wp;
  void *wt;  // projection operand tiles of the tensor-core back-projection
  int nbatch;
  int max_split;
};

// H*psi on device blocks of precision R.  out = a*(H in) + b*in + g*xm2
// (xm2 may be null when g == 0).  ld_in/ld_out >= ngw.  With `plan`, all
// scratch comes from it and no workspace is reserved.
template <typename R>
int hpsi_apply(pspw_cell *c, const void *in, int ld_in, void *out, int ld_out, int ngw,
               int nb, double a, double b, double g, const void *xm2, int ld_xm2,
               const ScratchPlan *plan = nullptr);

// Unweighted FP64 projections P[b*nproj + p] = sum_G conj(beta_p) psi_b
// (hpsi.cu), on the cell stream.
int project_fp64(pspw_cell *c, const double2 *psi, int ld, int ngw, int nb, double2 *P);

}  // namespace pspw
