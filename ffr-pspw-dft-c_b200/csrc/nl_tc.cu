// Kleinman-Bylander projector GEMMs of the FP32 H*psi on the tensor cores
// (tcgen05.mma kind::tf32, accumulators in tensor memory), with 3xTF32
// splitting (hi*hi + hi*lo + lo*hi) so the sums keep FP32 accuracy.
//
// With beta_{a,lm}(G) = EIGR(G,a) PKG_A(lm,G) (ApplyHam_block.cpp:88-117) and
// one species, both GEMMs are real GEMMs with the complex parts interleaved
// along K, and beta is never stored:
//
// projection   P[a][(b,lm)] = sum_G conj(E[a][G]) PKG[G][lm] psi[G][b]
//   D[(b,lm,p)][a] = sum_{(G,c)} A'[(b,lm,p)][(G,c)] B'[a][(G,c)]
//   B'[a][(G,0)] = Re E, B'[a][(G,1)] = Im E   (EIGR as stored)
//   A'[(b,lm,re)][(G,*)] = PKG (Re psi,  Im psi)
//   A'[(b,lm,im)][(G,*)] = PKG (Im psi, -Re psi)
//   M = (band, lm, re/im) in tiles of 128, N = atoms, K = 2*NGW split over
//   blocks; slices reduced in a fixed order with the weights WNL.
// back-projection NL[G][b] = sum_lm PKG[G][lm] sum_a E[a][G] W[(a,lm)][b]
//   D[G][(b,lm,p)] = sum_{(a,c)} A'[G][(a,c)] B'[(b,lm,p)][(a,c)]
//   A'[G][(a,0)] = Re E, A'[G][(a,1)] = Im E
//   B'[(b,lm,re)][(a,*)] = (Re W, -Im W), B'[(b,lm,im)][(a,*)] = (Im W, Re W)
//   M = G in tiles of 128, N = (band, lm, re/im) in tiles of up to 256,
//   K = 2*atoms; the epilogue contracts lm with PKG and applies the
//   Chebyshev update out = a (H psi) + b psi + g x.
//
// Operands go global -> registers -> (TF32 hi/lo split) -> shared memory in
// the K-major no-swizzle layout of tc.cuh, two stages deep: the global loads
// of step k+1 are in flight while the MMAs of step k run.  One thread issues
// the MMAs and commits them to the stage's mbarrier; every wait is bounded and
// raises the cell's error word instead of hanging.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "common.cuh"
#include "engine.h"
#include "nl_tc.h"
#include "tc.cuh"

namespace pspw {
namespace {

constexpr int kBK = 16;                                 // fp32 of K per stage (8 complex)
constexpr int kTileBytes128 = 128 * kBK * 4;            // 128 rows x BK fp32
constexpr uint32_t kLBO = 128, kSBO = (kBK / 4) * 128;  // core-matrix strides

__device__ __forceinline__ void st_split(unsigned char *hi, unsigned char *lo, uint32_t off,
                                         float x) {
  uint32_t h, l;
  tc::split_tf32(x, h, l);
  *reinterpret_cast<uint32_t *>(hi + off) = h;
  *reinterpret_cast<uint32_t *>(lo + off) = l;
}

// The 3xTF32 MMAs of one stage (K = 16 as two K = 8 steps), from one thread.
__device__ __forceinline__ void issue_stage(uint32_t tmem, uint32_t a_hi, uint32_t a_lo,
                                            uint32_t b_hi, uint32_t b_lo, uint32_t idesc,
                                            bool first) {
#pragma unroll
  for (int s = 0; s < kBK / 8; s++) {
    const uint32_t o = s * 256;
    const uint64_t ah = tc::sdesc(a_hi + o, kLBO, kSBO), al = tc::sdesc(a_lo + o, kLBO, kSBO);
    const uint64_t bh = tc::sdesc(b_hi + o, kLBO, kSBO), bl = tc::sdesc(b_lo + o, kLBO, kSBO);
    tc::mma_tf32(tmem, ah, bh, idesc, (first && s == 0) ? 0u : 1u);
    tc::mma_tf32(tmem, ah, bl, idesc, 1u);
    tc::mma_tf32(tmem, al, bh, idesc, 1u);
  }
}

__host__ __device__ constexpr uint32_t tmem_cols(int n) {
  return n <= 32 ? 32u : (n <= 64 ? 64u : (n <= 128 ? 128u : 256u));
}

// Shared state of one block: stage barriers and the TMEM base address.
struct Pipe {
  uint64_t bar[2];
  uint32_t tmem;
};

__device__ __forceinline__ void pipe_open(Pipe &p, uint32_t ncols) {
  if (threadIdx.x < 32) {
    tc::tmem_alloc(&p.tmem, ncols);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    tc::mbar_init(&p.bar[0], 1);
    tc::mbar_init(&p.bar[1], 1);
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

// Wait (bounded, block-uniform result) until the MMAs reading stage `st`
// have finished.
__device__ __forceinline__ bool stage_free(Pipe &p, int st, uint32_t *nphase) {
  const bool done = tc::mbar_wait(&p.bar[st], nphase[st] & 1);
  nphase[st]++;
  return __syncthreads_and(done) != 0;
}

// Staged tile written: make it visible to the tensor core and issue.
__device__ __forceinline__ void stage_issue(Pipe &p, int st, unsigned char *a_hi,
                                            unsigned char *b_hi, int bbytes, uint32_t idesc,
                                            bool first) {
  tc::fence_proxy_async();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc::fence_after_sync();
    issue_stage(p.tmem, tc::smem_addr(a_hi), tc::smem_addr(a_hi + kTileBytes128),
                tc::smem_addr(b_hi), tc::smem_addr(b_hi + bbytes), idesc, first);
    tc::mma_commit(&p.bar[st]);
  }
}

// After the main loop: wait for the last commit (it covers every earlier
// MMA of the thread that issued them).  Block-uniform result.
__device__ __forceinline__ bool pipe_drain(Pipe &p, int nissued, uint32_t *nphase) {
  bool done = true;
  if (nissued > 0) {
    const int st = (nissued - 1) & 1;
    done = tc::mbar_wait(&p.bar[st], nphase[st] & 1);
  }
  const bool ok = __syncthreads_and(done) != 0;
  tc::fence_after_sync();
  return ok;
}

__device__ __forceinline__ void pipe_close(Pipe &p, uint32_t ncols) {
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) tc::tmem_dealloc(p.tmem, ncols);
}

// ------------------------------------------------------------------ projection
// grid (M tiles of 128 rows, K splits of ksplit_g G each); block 128.
// part[split][m][a] with m = b*2L + 2*lm + p.
__global__ void __launch_bounds__(128) k_proj_tc(const float2 *__restrict__ psi, int ld, int ngw,
                                                 int nb, const float2 *__restrict__ eigr,
                                                 int ngw_cell, const float *__restrict__ pkga,
                                                 int L, int nat, int npad, int ksplit_g,
                                                 float *__restrict__ part, int *err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ Pipe pipe;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int Mtot = nb * 2 * L;
  const int m0 = blockIdx.x * 128;
  const int gb = blockIdx.y * ksplit_g, ge = min(ngw, gb + ksplit_g);
  const int bbytes = npad * kBK * 4;
  const int stage_bytes = 2 * kTileBytes128 + 2 * bbytes;
  const uint32_t ncols = tmem_cols(npad);
  pipe_open(pipe, ncols);
  const uint32_t idesc = tc::idesc_tf32(128, npad);
  // this thread's row of A'
  const int m = m0 + tid;
  const bool mvalid = m < Mtot;
  const int b = mvalid ? m / (2 * L) : 0;
  const int lm = mvalid ? (m % (2 * L)) >> 1 : 0;
  const int p = m & 1;
  const float2 *pcol = psi + (size_t)b * ld;
  uint32_t nphase[2] = {0, 0};
  bool ok = true;
  const int nsteps = ge > gb ? (ge - gb + 7) / 8 : 0;
  int issued = 0;
  for (int step = 0; step < nsteps; step++) {
    const int st = step & 1;
    const int g0 = gb + step * 8;
    // global loads of this step
    float2 v[8];
    float f[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int g = g0 + j;
      const bool in = mvalid && g < ge;
      v[j] = in ? pcol[g] : make_float2(0.f, 0.f);
      f[j] = in ? pkga[(size_t)g * 4 + lm] : 0.f;
    }
    float2 e[2][8];
#pragma unroll
    for (int rr = 0; rr < 2; rr++) {
      const int r = tid + 128 * rr;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int g = g0 + j;
        e[rr][j] = (r < nat && g < ge) ? eigr[(size_t)r * ngw_cell + g] : make_float2(0.f, 0.f);
      }
    }
    if (step >= 2 && !(ok = stage_free(pipe, st, nphase))) break;
    unsigned char *a_hi = sm + st * stage_bytes, *a_lo = a_hi + kTileBytes128;
    unsigned char *b_hi = a_lo + kTileBytes128, *b_lo = b_hi + bbytes;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const float x0 = p ? f[j] * v[j].y : f[j] * v[j].x;
      const float x1 = p ? -f[j] * v[j].x : f[j] * v[j].y;
      st_split(a_hi, a_lo, tc::core_off<kBK>(tid, 2 * j), x0);
      st_split(a_hi, a_lo, tc::core_off<kBK>(tid, 2 * j + 1), x1);
    }
#pragma unroll
    for (int rr = 0; rr < 2; rr++) {
      const int r = tid + 128 * rr;
      if (r < npad) {
#pragma unroll
        for (int j = 0; j < 8; j++) {
          st_split(b_hi, b_lo, tc::core_off<kBK>(r, 2 * j), e[rr][j].x);
          st_split(b_hi, b_lo, tc::core_off<kBK>(r, 2 * j + 1), e[rr][j].y);
        }
      }
    }
    stage_issue(pipe, st, a_hi, b_hi, bbytes, idesc, step == 0);
    issued++;
  }
  const bool drained = pipe_drain(pipe, issued, nphase);
  if (!(ok && drained)) {
    if (tid == 0) atomicOr(err, 1);
  } else {
    const int mg = m0 + 32 * warp + (tid & 31);
    float acc[16];
    for (int c0 = 0; c0 < npad; c0 += 16) {
      if (issued > 0) {
        tc::tmem_ld16(pipe.tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, acc);
      } else {
#pragma unroll
        for (int i = 0; i < 16; i++) acc[i] = 0.f;
      }
      if (mg < Mtot) {
        float *dst = part + ((size_t)blockIdx.y * Mtot + mg) * nat;
#pragma unroll
        for (int i = 0; i < 16; i++)
          if (c0 + i < nat) dst[c0 + i] = acc[i];
      }
    }
  }
  pipe_close(pipe, ncols);
}

// wp[b*nproj + a*L + lm] = W * sum_s (part[s][(b,lm,re)][a] + i part[s][(b,lm,im)][a]),
// the slices summed in a fixed order.
__global__ void k_proj_tc_reduce(const float *__restrict__ part, int nsplit, int nb, int L,
                                 int nat, const float *__restrict__ w, float2 *__restrict__ wp) {
  const int nproj = nat * L;
  const int Mtot = nb * 2 * L;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb * nproj) return;
  const int b = i / nproj, pj = i - b * nproj;
  const int a = pj / L, lm = pj - a * L;
  const int mre = b * 2 * L + 2 * lm;
  float re = 0.f, im = 0.f;
  for (int s = 0; s < nsplit; s++) {
    re += part[((size_t)s * Mtot + mre) * nat + a];
    im += part[((size_t)s * Mtot + mre + 1) * nat + a];
  }
  const float wl = w[pj];
  wp[i] = make_float2(wl * re, wl * im);
}

// ------------------------------------------------------------------ back-projection
// grid (G tiles of 128, N tiles of nbt bands); block 128.
__global__ void __launch_bounds__(128) k_backproj_tc(
    const float2 *__restrict__ wp, int nproj, int ngw, int nb, int nbt,
    const float2 *__restrict__ eigr, int ngw_cell, const float *__restrict__ pkga, int L, int nat,
    float2 *out, int ldo, const float2 *__restrict__ in, int ldi, const float2 *__restrict__ xm2,
    int ldx, float ca, float cb, float cg, int *err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ Pipe pipe;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int g0 = blockIdx.x * 128;
  const int b0 = blockIdx.y * nbt;
  const int nbb = min(nbt, nb - b0);
  const int per = 2 * L;             // columns per band
  const int ncolN = nbt * per;       // N of the MMA: a multiple of 16, <= 256
  const int bbytes = ncolN * kBK * 4;
  const int stage_bytes = 2 * kTileBytes128 + 2 * bbytes;
  const uint32_t ncols = tmem_cols(ncolN);
  pipe_open(pipe, ncols);
  const uint32_t idesc = tc::idesc_tf32(128, ncolN);
  const int ga = g0 + tid;  // this thread's G row of A'
  uint32_t nphase[2] = {0, 0};
  bool ok = true;
  const int nsteps = (nat + 7) / 8;  // 8 atoms = 16 fp32 of K per stage
  int issued = 0;
  for (int step = 0; step < nsteps; step++) {
    const int st = step & 1;
    const int a0 = step * 8;
    float2 e[8];
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int a = a0 + j;
      e[j] = (a < nat && ga < ngw) ? eigr[(size_t)a * ngw_cell + ga] : make_float2(0.f, 0.f);
    }
    float2 w[2][8];
#pragma unroll
    for (int rr = 0; rr < 2; rr++) {
      const int r = tid + 128 * rr;
      const int bl = r / per, lm = (r % per) >> 1;
      const bool rv = r < ncolN && bl < nbb;
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int a = a0 + j;
        w[rr][j] = (rv && a < nat) ? wp[(size_t)(b0 + bl) * nproj + a * L + lm]
                                   : make_float2(0.f, 0.f);
      }
    }
    if (step >= 2 && !(ok = stage_free(pipe, st, nphase))) break;
    unsigned char *a_hi = sm + st * stage_bytes, *a_lo = a_hi + kTileBytes128;
    unsigned char *b_hi = a_lo + kTileBytes128, *b_lo = b_hi + bbytes;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      st_split(a_hi, a_lo, tc::core_off<kBK>(tid, 2 * j), e[j].x);
      st_split(a_hi, a_lo, tc::core_off<kBK>(tid, 2 * j + 1), e[j].y);
    }
#pragma unroll
    for (int rr = 0; rr < 2; rr++) {
      const int r = tid + 128 * rr;
      if (r < ncolN) {
        const int pr = r & 1;
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const float x0 = pr ? w[rr][j].y : w[rr][j].x;
          const float x1 = pr ? w[rr][j].x : -w[rr][j].y;
          st_split(b_hi, b_lo, tc::core_off<kBK>(r, 2 * j), x0);
          st_split(b_hi, b_lo, tc::core_off<kBK>(r, 2 * j + 1), x1);
        }
      }
    }
    stage_issue(pipe, st, a_hi, b_hi, bbytes, idesc, step == 0);
    issued++;
  }
  const bool drained = pipe_drain(pipe, issued, nphase);
  if (!(ok && drained)) {
    if (tid == 0) atomicOr(err, 1);
  } else {
    // epilogue: this thread owns G row g of the warp's 32-lane slice
    const int g = g0 + 32 * warp + (tid & 31);
    float pk[4] = {0.f, 0.f, 0.f, 0.f};
    if (g < ngw)
      for (int l = 0; l < L; l++) pk[l] = pkga[(size_t)g * 4 + l];
    float acc[16];
    float accr = 0.f, acci = 0.f;
    int col = 0;
    for (int c0 = 0; c0 < ncolN; c0 += 16) {
      if (issued > 0) {
        tc::tmem_ld16(pipe.tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, acc);
      } else {
#pragma unroll
        for (int i = 0; i < 16; i++) acc[i] = 0.f;
      }
#pragma unroll
      for (int i = 0; i < 16; i++, col++) {
        const int cc = col % per;
        const float pv = pk[cc >> 1];
        if (cc & 1)
          acci += pv * acc[i];
        else
          accr += pv * acc[i];
        if (cc == per - 1) {
          const int bl = col / per;
          if (bl < nbb && g < ngw) {
            const size_t bb = (size_t)(b0 + bl);
            const float2 h = out[bb * ldo + g];
            float rr = ca * (h.x + accr), ii = ca * (h.y + acci);
            if (cb != 0.f) {
              const float2 u = in[bb * ldi + g];
              rr += cb * u.x;
              ii += cb * u.y;
            }
            if (cg != 0.f) {
              const float2 u = xm2[bb * ldx + g];
              rr += cg * u.x;
              ii += cg * u.y;
            }
            out[bb * ldo + g] = make_float2(rr, ii);
          }
          accr = acci = 0.f;
        }
      }
    }
  }
  pipe_close(pipe, ncols);
}

// Dynamic shared memory of a block whose B' tile has nrows_b rows: the two
// stages, raised where needed so that no more blocks fit on an SM than its
// 512 TMEM columns can serve at once (an allocation would otherwise wait for
// a resident block to finish).
int tile_smem(int nrows_b) {
  const int stages = 2 * (2 * kTileBytes128 + 2 * nrows_b * kBK * 4);
  const int per_sm = 512 / (int)tmem_cols(nrows_b);
  const int floor_bytes = 233472 / (per_sm + 1) + 1024;
  return std::max(stages, floor_bytes);
}

}  // namespace

bool nl_tc_usable(const pspw_cell *c) {
  static const bool off = std::getenv("PSPW_NL_SIMT") != nullptr;
  const Projectors &P = c->proj;
  if (c->nl_path == PSPW_NL_SIMT || (off && c->nl_path != PSPW_NL_TENSOR_CORE)) return false;
  return P.nsp == 1 && P.nat >= 1 && P.nat <= 256 && P.nproj > 0 &&
         P.nproj % P.nat == 0 && P.nproj / P.nat <= 4 && c->d_err != nullptr;
}

int nl_tc_project(pspw_cell *c, const float2 *in, int ld, int ngw, int nb, float2 *wp,
                  float *part, int max_split) {
  const Projectors &P = c->proj;
  const int nat = P.nat, L = P.nproj / P.nat;
  const int npad = (nat + 15) / 16 * 16;
  const int Mtot = nb * 2 * L;
  const int mt = (Mtot + 127) / 128;
  // split G so the grid covers the GPU about twice, at least 64 G per split
  int nsplit = std::max(1, std::min((ngw + 63) / 64, (2 * 148 + mt - 1) / mt));
  if (part) nsplit = std::max(1, std::min(nsplit, max_split));
  int kg = (ngw + nsplit - 1) / nsplit;
  kg = (kg + 7) / 8 * 8;
  nsplit = (ngw + kg - 1) / kg;
  if (!part) {
    int rc = ws_reserve(c, kWsProjPart, sizeof(float) * (size_t)nsplit * Mtot * nat, (void **)&part);
    if (rc) return rc;
  }
  const int smem = tile_smem(npad);
  PSPW_CUDA(cudaFuncSetAttribute(k_proj_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_proj_tc<<<dim3(mt, nsplit), 128, smem, c->stream>>>(in, ld, ngw, nb, P.d_eigr32, c->basis.ngw,
                                                        P.d_pkga32, L, nat, npad, kg, part,
                                                        c->d_err);
  k_proj_tc_reduce<<<(nb * P.nproj + 255) / 256, 256, 0, c->stream>>>(part, nsplit, nb, L, nat,
                                                                      P.d_pw32, wp);
  c->kernel_launches += 2;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int nl_tc_backproject(pspw_cell *c, const float2 *wp, int ngw, int nb, float2 *out, int ldo,
                      const float2 *in, int ldi, const float2 *xm2, int ldx, float a, float b,
                      float g) {
  const Projectors &P = c->proj;
  const int L = P.nproj / P.nat, per = 2 * L;
  // bands per N tile: nbt*2L a multiple of 16 and at most 256
  int nmax = 256 / per;
  while (nmax > 0 && (nmax * per) % 16) nmax--;
  int nbt = std::min(nmax, nb);
  while (nbt > 0 && (nbt * per) % 16) nbt++;
  if (nbt < 1 || nbt * per > 256) return fail(PSPW_ERR_NOT_IMPL, "tensor-core back-projection: tile");
  const int smem = tile_smem(nbt * per);
  PSPW_CUDA(cudaFuncSetAttribute(k_backproj_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  dim3 grid((ngw + 127) / 128, (nb + nbt - 1) / nbt);
  k_backproj_tc<<<grid, 128, smem, c->stream>>>(wp, P.nproj, ngw, nb, nbt, P.d_eigr32, c->basis.ngw,
                                                P.d_pkga32, L, P.nat, out, ldo, in, ldi, xm2, ldx,
                                                a, b, g, c->d_err);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

}  // namespace pspw
