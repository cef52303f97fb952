// Block H*psi on many independent cells in one launch (no reference
// counterpart: the reference applies ApplyHam_block.cpp:5-172 to one cell
// per process).  A batch holds cells of different grids, sphere sizes and
// band counts, with each cell's input and output blocks in device memory.
//
// Schedules: for every cell the batch times the H*psi variants that give
// the same result (band-batch sizes of the FFT passes; for FP32 cells of
// one species the tensor-core or SIMT projector kernels) and keeps the
// fastest.  Results are cached per cell shape (grid, sphere, bands, atoms,
// species, precision) for the life of the process, so cells of a shape
// seen before are not timed again.
//
// Launch: the whole batch is captured once into a CUDA graph, each cell's
// kernels on its own stream branch forked from and joined back into the
// batch stream, and every apply is one cudaGraphLaunch: the host pays one
// launch for all cells and the device runs the cells' kernels side by side.
// Each cell's kernels and arguments are the ones an eager call would
// launch, so a cell's result is the same alone and in the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "engine.h"
#include "nl_tc.h"

struct pspw_batch {
  int device = 0, prec = 0;
  std::vector<pspw_cell *> cells;
  std::vector<int> nb;
  std::vector<void *> in, out;
  std::vector<double> ms;  // tuned time per cell (ms), 0 before tuning
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long kernels = 0;  // kernel launches in one apply (counted at capture)
};

namespace pspw {
namespace {

using Key = std::tuple<int, int, int, int, int, int, int, int, int>;
struct Sched {
  int band_batch, nl_path;
  double ms;
};
std::mutex g_sched_mu;
std::map<Key, Sched> g_sched;

Key key_of(const pspw_cell *c, int nb, int prec) {
  return Key(c->basis.n1, c->basis.n2, c->basis.n3, c->basis.ngw, nb, c->proj.nat,
             c->proj.nsp, c->proj.nproj, prec);
}

int apply_cell(pspw_batch *b, int i) {
  pspw_cell *c = b->cells[i];
  const int ngw = c->basis.ngw;
  if (b->prec == PSPW_PREC_F64)
    return hpsi_apply<double>(c, b->in[i], ngw, b->out[i], ngw, ngw, b->nb[i], 1.0, 0.0, 0.0,
                              nullptr, ngw);
  return hpsi_apply<float>(c, b->in[i], ngw, b->out[i], ngw, ngw, b->nb[i], 1.0, 0.0, 0.0,
                           nullptr, ngw);
}

void drop_graph(pspw_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// mean time (ms) of `reps` eager applications of cell i, after one untimed
int time_cell(pspw_batch *b, int i, int reps, double *ms) {
  pspw_cell *c = b->cells[i];
  cudaEvent_t e0, e1;
  PSPW_CUDA(cudaEventCreate(&e0));
  PSPW_CUDA(cudaEventCreate(&e1));
  int rc = apply_cell(b, i);
  if (!rc) {
    cudaEventRecord(e0, c->stream);
    for (int r = 0; r < reps && !rc; r++) rc = apply_cell(b, i);
    cudaEventRecord(e1, c->stream);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / std::max(1, reps);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc) rc = device_status(c);
  return rc;
}

int capture(pspw_batch *b) {
  drop_graph(b);
  // first, one eager pass: every workspace the graph will use is allocated
  // now, outside the capture
  for (size_t i = 0; i < b->cells.size(); i++) {
    int rc = apply_cell(b, (int)i);
    if (rc) return rc;
  }
  for (pspw_cell *c : b->cells) PSPW_CUDA(cudaStreamSynchronize(c->stream));
  long long before = 0;
  for (pspw_cell *c : b->cells) before += c->kernel_launches;
  PSPW_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
  int rc = PSPW_OK;
  cudaEventRecord(b->fork, b->stream);
  for (size_t i = 0; i < b->cells.size() && !rc; i++) {
    pspw_cell *c = b->cells[i];
    cudaStreamWaitEvent(c->stream, b->fork, 0);
    rc = apply_cell(b, (int)i);
    cudaEventRecord(b->join[i], c->stream);
    cudaStreamWaitEvent(b->stream, b->join[i], 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(e, "batch: stream capture");
  b->graph = g;
  long long after = 0;
  for (pspw_cell *c : b->cells) after += c->kernel_launches;
  b->kernels = after - before;
  PSPW_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
  return PSPW_OK;
}

}  // namespace
}  // namespace pspw

using namespace pspw;

extern "C" {

int pspw_batch_create(int ncells, pspw_cell *const *cells, const int *nbands, int prec,
                      pspw_batch **out) {
  if (!out || ncells < 1 || !cells || !nbands) return fail(PSPW_ERR_ARG, "batch_create: bad arguments");
  if (prec != PSPW_PREC_F64 && prec != PSPW_PREC_F32)
    return fail(PSPW_ERR_ARG, "batch_create: unknown precision");
  const int dev = cells[0] ? cells[0]->device : 0;
  for (int i = 0; i < ncells; i++) {
    if (!cells[i] || cells[i]->device != dev || nbands[i] < 1)
      return fail(PSPW_ERR_ARG, "batch_create: null cell, mixed devices or no bands");
    if (!cells[i]->d_veff64) return fail(PSPW_ERR_ARG, "batch_create: a cell without V_eff");
  }
  PSPW_CUDA(cudaSetDevice(dev));
  auto *b = new pspw_batch;
  b->device = dev;
  b->prec = prec;
  const size_t sc = prec == PSPW_PREC_F64 ? sizeof(double2) : sizeof(float2);
  int rc = PSPW_OK;
  for (int i = 0; i < ncells && !rc; i++) {
    b->cells.push_back(cells[i]);
    b->nb.push_back(nbands[i]);
    void *p = nullptr, *q = nullptr;
    const size_t bytes = sc * (size_t)cells[i]->basis.ngw * nbands[i];
    if (cudaMalloc(&p, bytes) != cudaSuccess || cudaMalloc(&q, bytes) != cudaSuccess) {
      if (p) cudaFree(p);
      rc = fail(PSPW_ERR_OOM, "batch_create: device blocks");
      break;
    }
    cudaMemset(p, 0, bytes);
    cudaMemset(q, 0, bytes);
    b->in.push_back(p);
    b->out.push_back(q);
    b->ms.push_back(0.0);
  }
  if (!rc && (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess))
    rc = fail(PSPW_ERR_CUDA, "batch_create: stream");
  for (int i = 0; i < ncells && !rc; i++) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
      rc = fail(PSPW_ERR_CUDA, "batch_create: events");
    else
      b->join.push_back(e);
  }
  if (rc) {
    pspw_batch_destroy(b);
    return rc;
  }
  PSPW_CUDA(cudaDeviceSynchronize());  // the blocks' zero fill before any cell stream uses them
  *out = b;
  return PSPW_OK;
}

int pspw_batch_blocks(pspw_batch *b, int i, void **d_in, void **d_out) {
  if (!b || i < 0 || i >= (int)b->cells.size() || !d_in || !d_out)
    return fail(PSPW_ERR_ARG, "batch_blocks: bad arguments");
  *d_in = b->in[i];
  *d_out = b->out[i];
  return PSPW_OK;
}

int pspw_batch_upload(pspw_batch *b, int i, const void *host_in) {
  if (!b || i < 0 || i >= (int)b->cells.size() || !host_in)
    return fail(PSPW_ERR_ARG, "batch_upload: bad arguments");
  PSPW_CUDA(cudaSetDevice(b->device));
  PSPW_CUDA(cudaStreamSynchronize(b->stream));  // no apply still reading the block
  const size_t sc = b->prec == PSPW_PREC_F64 ? sizeof(double2) : sizeof(float2);
  PSPW_CUDA(cudaMemcpy(b->in[i], host_in, sc * (size_t)b->cells[i]->basis.ngw * b->nb[i],
                       cudaMemcpyHostToDevice));
  // the copy from pageable memory may return before its DMA lands; the
  // batch stream is non-blocking, so the legacy stream is synchronised here
  PSPW_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
  return PSPW_OK;
}

int pspw_batch_download(pspw_batch *b, int i, void *host_out) {
  if (!b || i < 0 || i >= (int)b->cells.size() || !host_out)
    return fail(PSPW_ERR_ARG, "batch_download: bad arguments");
  PSPW_CUDA(cudaSetDevice(b->device));
  PSPW_CUDA(cudaStreamSynchronize(b->stream));
  const size_t sc = b->prec == PSPW_PREC_F64 ? sizeof(double2) : sizeof(float2);
  PSPW_CUDA(cudaMemcpy(host_out, b->out[i], sc * (size_t)b->cells[i]->basis.ngw * b->nb[i],
                       cudaMemcpyDeviceToHost));
  return PSPW_OK;
}

int pspw_batch_tune(pspw_batch *b, int reps) {
  if (!b) return fail(PSPW_ERR_ARG, "batch_tune: null batch");
  PSPW_CUDA(cudaSetDevice(b->device));
  drop_graph(b);
  reps = std::max(1, reps);
  for (size_t i = 0; i < b->cells.size(); i++) {
    pspw_cell *c = b->cells[i];
    const int nb = b->nb[i];
    const Key k = key_of(c, nb, b->prec);
    {
      std::lock_guard<std::mutex> lk(g_sched_mu);
      auto it = g_sched.find(k);
      if (it != g_sched.end()) {
        c->band_batch = it->second.band_batch;
        c->nl_path = it->second.nl_path;
        b->ms[i] = it->second.ms;
        continue;
      }
    }
    std::vector<int> batches = {0, nb, (nb + 1) / 2, (nb + 3) / 4, std::min(nb, 16)};
    std::sort(batches.begin(), batches.end());
    batches.erase(std::unique(batches.begin(), batches.end()), batches.end());
    std::vector<int> paths = {PSPW_NL_AUTO};
    if (b->prec == PSPW_PREC_F32 && c->proj.nproj > 0) {
      c->nl_path = PSPW_NL_AUTO;
      if (nl_tc_usable(c)) paths = {PSPW_NL_TENSOR_CORE, PSPW_NL_SIMT};
    }
    Sched best{0, PSPW_NL_AUTO, 1e30};
    for (int path : paths)
      for (int bb : batches) {
        c->nl_path = path;
        c->band_batch = bb;
        double t = 0.0;
        const int rc = time_cell(b, (int)i, reps, &t);
        if (rc) return rc;
        if (t < best.ms) best = Sched{bb, path, t};
      }
    c->band_batch = best.band_batch;
    c->nl_path = best.nl_path;
    b->ms[i] = best.ms;
    std::lock_guard<std::mutex> lk(g_sched_mu);
    g_sched[k] = best;
  }
  return PSPW_OK;
}

int pspw_batch_schedule(pspw_batch *b, int i, int *band_batch, int *nl_path, double *ms) {
  if (!b || i < 0 || i >= (int)b->cells.size() || !band_batch || !nl_path || !ms)
    return fail(PSPW_ERR_ARG, "batch_schedule: bad arguments");
  *band_batch = b->cells[i]->band_batch;
  *nl_path = b->cells[i]->nl_path;
  *ms = b->ms[i];
  return PSPW_OK;
}

int pspw_batch_apply(pspw_batch *b) {
  if (!b) return fail(PSPW_ERR_ARG, "batch_apply: null batch");
  PSPW_CUDA(cudaSetDevice(b->device));
  if (!b->exec) {
    const int rc = capture(b);
    if (rc) return rc;
  }
  PSPW_CUDA(cudaGraphLaunch(b->exec, b->stream));
  return PSPW_OK;
}

int pspw_batch_kernels(pspw_batch *b, long long *kernels) {
  if (!b || !kernels) return fail(PSPW_ERR_ARG, "batch_kernels: bad arguments");
  *kernels = b->kernels;
  return PSPW_OK;
}

int pspw_batch_stream(pspw_batch *b, void **stream) {
  if (!b || !stream) return fail(PSPW_ERR_ARG, "batch_stream: bad arguments");
  *stream = b->stream;
  return PSPW_OK;
}

int pspw_batch_synchronize(pspw_batch *b) {
  if (!b) return fail(PSPW_ERR_ARG, "batch_synchronize: null batch");
  PSPW_CUDA(cudaSetDevice(b->device));
  PSPW_CUDA(cudaStreamSynchronize(b->stream));
  for (pspw_cell *c : b->cells) {
    const int rc = device_status(c);
    if (rc) return rc;
  }
  return PSPW_OK;
}

int pspw_batch_destroy(pspw_batch *b) {
  if (!b) return PSPW_OK;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (void *p : b->in) cudaFree(p);
  for (void *p : b->out) cudaFree(p);
  for (cudaEvent_t e : b->join) cudaEventDestroy(e);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return PSPW_OK;
}

}  // extern "C"
