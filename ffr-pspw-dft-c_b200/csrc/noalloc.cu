// Block H*psi without any device allocation on the call path.
//
// pspw_apply_ham_block_dev allocates its scratch (the FFT stick and plane
// buffers and the projector partial sums) on first use and whenever a
// larger problem arrives.  Some callers cannot let a library allocate at
// call time: code that is being recorded into a CUDA graph (an allocation
// there is not part of the graph and a free during capture is an error),
// applications whose memory manager owns every byte of the device and
// forbids libraries from calling cudaMalloc behind its back, and services
// that must never hit an out-of-memory failure in the middle of a request.
// For them pspw_apply_ham_block_dev_noalloc takes all of its scratch from
// the fixed array below, which is part of the library image: every GPU that
// loads the library holds these 16 MiB until the process exits.
//
// Host code may not use the array's name as a device address (on the host it
// names a stand-in object), so the address is looked up once per device with
// cudaGetSymbolAddress, with that device current, and cached.  The first call
// on each device performs that lookup, so it should be made before any
// stream capture begins.  The cache lives as long as the process: a
// cudaDeviceReset unloads the device image and leaves the cached address
// stale, so the entry point is not to be called after a reset.
//
// All calls on a device share the one array and it keeps whatever the last
// call left in it.  Nothing in it needs to start at zero: every element a
// call reads was written earlier in the same call.  Calls whose work can
// overlap on the GPU (different streams, different cells on one device)
// race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "common.cuh"
#include "engine.h"
#include "nl_tc.h"

#define PSPW_NOALLOC_SCRATCH_BYTES (16u << 20)

static __device__ __align__(256) unsigned char g_noalloc_scratch[PSPW_NOALLOC_SCRATCH_BYTES];

namespace pspw {
namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {};

// Device address of the scratch array on `dev` (which must be current).
int scratch_address(int dev, void **out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(PSPW_ERR_ARG, "noalloc: device index out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return PSPW_OK;
}

inline size_t up256(size_t n) { return (n + 255) / 256 * 256; }

}  // namespace
}  // namespace pspw

using namespace pspw;

extern "C" int pspw_apply_ham_block_dev_noalloc(pspw_cell *c, int prec, const void *d_vin,
                                                void *d_vout, int ld, int ngw, int nstates) {
  if (!c) return fail(PSPW_ERR_ARG, "noalloc: null cell");
  if (prec != PSPW_PREC_F64 && prec != PSPW_PREC_F32)
    return fail(PSPW_ERR_ARG, "noalloc: unknown precision");
  if (nstates <= 0) return PSPW_OK;
  PSPW_CUDA(cudaSetDevice(c->device));
  void *base = nullptr;
  int rc = scratch_address(c->device, &base);
  if (rc) return rc;
  const Basis &B = c->basis;
  const size_t sc = prec == PSPW_PREC_F64 ? sizeof(double2) : sizeof(float2);
  const size_t cap = PSPW_NOALLOC_SCRATCH_BYTES;
  const size_t per_band = ((size_t)B.n3 * B.ncol + (size_t)B.n3 * B.n2 * B.nxa) * sc;
  const size_t slice = (size_t)nstates * c->proj.nproj * sc;  // one projection block
  // FP32 on the tensor-core path: the projections as operand tiles
  const size_t wt_bytes =
      prec == PSPW_PREC_F32 && nl_tc_usable(c) ? up256(nl_tc_wtile_bytes(c, nstates)) : 0;
  const size_t wp_bytes = up256(slice) + wt_bytes;
  // partial-sum slices: up to a quarter of the array, at least one
  int nsplit = slice ? (int)std::max<size_t>(1, std::min<size_t>(64, cap / 4 / slice)) : 1;
  auto fit_bands = [&](int ns) -> long long {
    const size_t used = wp_bytes + up256((size_t)ns * slice);
    if (used >= cap) return 0;
    return (long long)((cap - used) / (per_band + 512));
  };
  long long nbatch = fit_bands(nsplit);
  if (nbatch < 1) {
    nsplit = 1;
    nbatch = fit_bands(1);
  }
  if (nbatch < 1) {
    const size_t need = wp_bytes + up256(slice) + up256(per_band) * 2;
    return fail(PSPW_ERR_SHAPE, "noalloc: this cell and block need at least " +
                                    std::to_string(need) + " bytes of scratch; the static array "
                                    "holds " + std::to_string(cap) + " (16 MiB); use "
                                    "pspw_apply_ham_block_dev or fewer bands per call");
  }
  nbatch = std::min<long long>(nbatch, nstates);
  unsigned char *p = static_cast<unsigned char *>(base);
  ScratchPlan plan;
  plan.wp = p;
  plan.wt = p + up256(slice);
  p += wp_bytes;
  plan.part = p;
  p += up256((size_t)nsplit * slice);
  plan.S = p;
  p += up256((size_t)nbatch * B.n3 * B.ncol * sc);
  plan.P = p;
  plan.nbatch = (int)nbatch;
  plan.max_split = nsplit;
  if (prec == PSPW_PREC_F64)
    return hpsi_apply<double>(c, d_vin, ld, d_vout, ld, ngw, nstates, 1.0, 0.0, 0.0, nullptr, ld,
                              &plan);
  return hpsi_apply<float>(c, d_vin, ld, d_vout, ld, ngw, nstates, 1.0, 0.0, 0.0, nullptr, ld,
                           &plan);
}
