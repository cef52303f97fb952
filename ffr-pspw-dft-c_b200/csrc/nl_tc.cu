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
//   blocks; the slices are reduced in a fixed order with the weights WNL.
// back-projection NL[G][b] = sum_lm PKG[G][lm] sum_a E[a][G] W[(a,lm)][b]
//   D[G][(b,lm,p)] = sum_{(a,c)} A'[G][(a,c)] B'[(b,lm,p)][(a,c)]
//   A'[G][(a,0)] = Re E, A'[G][(a,1)] = Im E
//   B'[(b,lm,re)][(a,*)] = (Re W, -Im W), B'[(b,lm,im)][(a,*)] = (Im W, Re W)
//   M = G in tiles of 128, N = (band, lm, re/im) in tiles of at most 128,
//   K = 2*atoms; the epilogue contracts lm with PKG and applies the
//   Chebyshev update out = a (H psi) + b psi + g x.
//
// Operands that do not depend on psi (both EIGR operands) are split into
// TF32 hi/lo tiles once per cell, in the K-major no-swizzle layout of tc.cuh,
// and reach shared memory as single bulk copies.  The psi operand of the
// projection is built on the fly by the row threads and stored straight into
// tensor memory (the MMA reads A from TMEM), so it never passes through
// shared memory.  The reduction of the projection writes W' as operand
// tiles, so the back-projection is a GEMM fed by bulk copies alone.
//
// Both GEMM kernels are warp-specialised (320 threads, 352 for the projection):
//   warps 0-7  row threads: warp w serves TMEM lanes 32 (w % 4) .. + 31
//              (rows of the 128-row M tile) and half w / 4 of the columns;
//              they build the A' operand (projection) and run the epilogue;
//   warp 8     producer: cp.async of psi / PKG_A into a raw ring
//              (projection) or the bulk copies of the fixed tiles
//              (back-projection);
//   warp 9     one thread issues the MMAs of a K step once its operand slot
//              is full and commits them to the slot's "empty" barrier;
//   warp 10    (projection) one thread bulk-copies the EIGR tiles, so the
//              raw producer never waits on the MMAs.
// Slots are handed over with mbarriers only; there is no block-wide barrier
// in the main loop.  Every wait is bounded and gives up as soon as any
// thread of the block has given up; the block then raises the cell's error
// word.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "nl_tc.h"
#include "tc.cuh"

namespace pspw {
namespace {

constexpr int kBK = 16;                                 // fp32 of K per step
constexpr int kTileBytes128 = 128 * kBK * 4;            // 128 rows x BK fp32
constexpr uint32_t kLBO = 128, kSBO = (kBK / 4) * 128;  // core-matrix strides
constexpr int kNTP = 4;                                 // operand slots, projection
constexpr int kNTB = 2;                                 // operand slots, back-projection
constexpr int kNR = 6;                                  // raw slots, projection
constexpr int kRowWarps = 8;                            // row / epilogue warps
constexpr int kRowThreads = 32 * kRowWarps;
constexpr int kThreads = kRowThreads + 64;              // + producer + MMA warps
constexpr int kThreadsP = kThreads + 32;                // projection: + tile producer
constexpr int kMaxBackN = 128;  // N tile of the back-projection

__host__ __device__ constexpr int round16(int x) { return (x + 15) & ~15; }

// TMEM columns to allocate for n: a power of two from 32 to 512
__host__ __device__ constexpr uint32_t tmem_cols(int n) {
  return n <= 32 ? 32u : (n <= 64 ? 64u : (n <= 128 ? 128u : (n <= 256 ? 256u : 512u)));
}

// The 3xTF32 MMAs of one K step (K = 16 as two K = 8 instructions).
__device__ __forceinline__ void issue_step(uint32_t tmem, uint32_t a_hi, uint32_t a_lo,
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

// Barriers and state shared by the roles of one block.
struct Sync {
  uint64_t full[kNTP];   // projection: A' written by the row warps and EIGR landed
  uint64_t bfull[kNTP];  // back-projection: bulk-copied operands landed
  uint64_t empty[kNTP];  // MMAs reading the slot finished
  uint64_t rfull[kNR];   // raw slot landed (projection)
  uint64_t rempty[kNR];  // raw slot consumed (projection)
  uint64_t done;         // every MMA of the block finished
  uint32_t tmem;
  int abort;
};

__device__ __forceinline__ void open_block(Sync &sy, uint32_t ncols, int nt, int nfull, int nraw) {
  if (threadIdx.x < 32) {
    tc::tmem_alloc(&sy.tmem, ncols);
    tc::tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    for (int i = 0; i < nt; i++) {
      tc::mbar_init(&sy.full[i], nfull);
      tc::mbar_init(&sy.bfull[i], 1);
      tc::mbar_init(&sy.empty[i], 1);
    }
    for (int i = 0; i < nraw; i++) {
      tc::mbar_init(&sy.rfull[i], 32);
      tc::mbar_init(&sy.rempty[i], kRowWarps);
    }
    tc::mbar_init(&sy.done, 1);
    sy.abort = 0;
    tc::fence_mbar_init();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

__device__ __forceinline__ void close_block(Sync &sy, uint32_t ncols, int *err) {
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x == 0 && sy.abort) atomicOr(err, 1);
  if (threadIdx.x < 32) tc::tmem_dealloc(sy.tmem, ncols);
}

// Producer tail: wait (bounded) until the bulk copies of the last `nt`
// issued steps have landed, so none is in flight when the block exits.
__device__ __forceinline__ void drain_bulk(Sync &sy, int issued, int nt) {
  for (int k = max(0, issued - nt); k < issued; k++) tc::mbar_wait(&sy.bfull[k % nt], (k / nt) & 1);
}

// ------------------------------------------------------------------ projection
// grid (M tiles of 128 rows, K splits of ksplit_g G each, ksplit_g % 16 == 0);
// kThreadsP threads.  One K step = 16 G = 32 fp32 of K = two EIGR tiles.
// etp: per 8 G, [npad x 16] hi then lo.  part[split][m][a], m = b*2L + 2lm + p.
//
// The A' operand lives in tensor memory: D occupies columns [0, dcols) and
// A' slot ts the 64 columns acol + 64 ts: hi of the step's 32 fp32 of K, then
// lo.  Row thread (warp w, lane l) owns TMEM lane 32 (w % 4) + l = row
// m - m0 and K half w / 4 (8 of the step's 16 G).  Slot ts is "ready" when
// the 8 row warps have arrived and the EIGR bulk copy has landed.
__host__ __device__ constexpr int proj_slots(int npad) { return tmem_cols(npad) <= 64 ? 3 : 2; }
constexpr int kStepG = 16;  // G per projection step

template <int L>
__global__ void __launch_bounds__(kThreadsP) k_proj_tc(const float2 *__restrict__ psi, int ld,
                                                      int ngw, int nb,
                                                      const float *__restrict__ etp,
                                                      const float *__restrict__ pkga, int nat,
                                                      int npad, int ksplit_g,
                                                      float *__restrict__ part, int *err) {
  constexpr int per = 2 * L;
  constexpr int nbr_max = 127 / per + 2;  // bands a 128-row tile touches
  constexpr int prow = kStepG + 1;        // raw psi row (float2), padded
  constexpr int raw_psi = round16(nbr_max * prow * 8);
  constexpr int raw_bytes = raw_psi + kStepG * 16;
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ Sync sy;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int Mtot = nb * per;
  const int m0 = blockIdx.x * 128;
  const int bfirst = m0 / per;
  const int nbr = min(Mtot - 1, m0 + 127) / per - bfirst + 1;
  const int gb = blockIdx.y * ksplit_g, ge = min(ngw, gb + ksplit_g);
  const int nsteps = ge > gb ? (ge - gb + kStepG - 1) / kStepG : 0;
  const int nts = proj_slots(npad);
  const uint32_t ebytes = (uint32_t)npad * 128;  // hi + lo EIGR tile of 8 G
  unsigned char *raw0 = sm + nts * 2 * ebytes;
  const uint32_t acol = tmem_cols(npad);
  const uint32_t ncols = tmem_cols(acol + 64 * nts);
  open_block(sy, ncols, nts, kRowWarps + 1, kNR);

  if (warp < kRowWarps) {
    // ---- A' rows
    const int row = 32 * (warp & 3) + lane, half = warp >> 2;
    const uint32_t lane_base = sy.tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const int m = m0 + row;
    const bool mv = m < Mtot;
    const int bl = mv ? m / per - bfirst : 0;
    const int lm = (m % per) >> 1, p = m & 1;
    for (int k = 0; k < nsteps; k++) {
      const int rs = k % kNR, ts = k % nts;
      if (!tc::mbar_wait_abort(&sy.rfull[rs], (k / kNR) & 1, &sy.abort)) break;
      if (k >= nts && !tc::mbar_wait_abort(&sy.empty[ts], ((k / nts) - 1) & 1, &sy.abort)) break;
      tc::fence_after_sync();
      const unsigned char *r = raw0 + rs * raw_bytes;
      const float2 *rp = reinterpret_cast<const float2 *>(r) + bl * prow + 8 * half;
      const float *rk = reinterpret_cast<const float *>(r + raw_psi) + 32 * half + lm;
      uint32_t hi[16], lo[16];
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const float2 v = rp[j];
        const float f = rk[4 * j];
        const float x0 = p ? f * v.y : f * v.x;
        const float x1 = p ? -f * v.x : f * v.y;
        tc::split_tf32(mv ? x0 : 0.f, hi[2 * j], lo[2 * j]);
        tc::split_tf32(mv ? x1 : 0.f, hi[2 * j + 1], lo[2 * j + 1]);
      }
      const uint32_t ca = lane_base + acol + 64 * ts + 16 * half;
      tc::tmem_st16(ca, hi);
      tc::tmem_st16(ca + 32, lo);
      tc::tmem_wait_st();
      tc::fence_before_sync();
      __syncwarp();  // one arrival per warp: the barriers count warps
      if (lane == 0) {
        tc::mbar_arrive(&sy.full[ts]);
        tc::mbar_arrive(&sy.rempty[rs]);
      }
    }
    // ---- epilogue: D row m, this warp's half of the atom columns -> part
    // (tcgen05.ld is warp-collective: decided per warp, rows past Mtot load
    // without storing)
    const bool ok = __all_sync(0xffffffffu, tc::mbar_wait_abort(&sy.done, 0, &sy.abort));
    tc::fence_after_sync();
    if (ok) {
      float *dst = part + ((size_t)blockIdx.y * Mtot + m) * nat;
      const int hw = npad / 2;
      for (int c0 = half * hw; c0 < (half + 1) * hw; c0 += 8) {
        uint32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        if (nsteps > 0) {
          tc::tmem_ld<8>(lane_base + (uint32_t)c0, acc);
          tc::tmem_wait_ld();
        }
        if (mv) {
#pragma unroll
          for (int i = 0; i < 8; i++)
            if (c0 + i < nat) dst[c0 + i] = __uint_as_float(acc[i]);
        }
      }
    }
  } else if (warp == kRowWarps) {
    // ---- raw producer: psi / PKG_A by all lanes
    for (int k = 0; k < nsteps; k++) {
      const int rs = k % kNR;
      if (k >= kNR && !tc::mbar_wait_abort(&sy.rempty[rs], ((k / kNR) - 1) & 1, &sy.abort))
        break;
      unsigned char *r = raw0 + rs * raw_bytes;
      float2 *rp = reinterpret_cast<float2 *>(r);
      float *rk = reinterpret_cast<float *>(r + raw_psi);
      const int g0 = gb + kStepG * k;
      for (int e = lane; e < nbr * kStepG; e += 32) {
        const int b = e / kStepG, j = e % kStepG, g = g0 + j;
        const bool v = g < ge;
        tc::cp_async8(rp + b * prow + j, psi + (size_t)(bfirst + b) * ld + (v ? g : 0), v);
      }
      if (lane < kStepG) {
        const int g = g0 + lane;
        const bool v = g < ge;
        tc::cp_async16(rk + 4 * lane, pkga + (size_t)(v ? g : 0) * 4, v);
      }
      tc::cp_async_mbar_arrive_noinc(&sy.rfull[rs]);
    }
    tc::cp_async_wait<0>();
  } else if (warp == kRowWarps + 2) {
    // ---- tile producer: two EIGR tiles (one bulk copy) per step
    if (lane == 0) {
      int issued = 0;
      for (int k = 0; k < nsteps; k++) {
        const int ts = k % nts;
        if (k >= nts && !tc::mbar_wait_abort(&sy.empty[ts], ((k / nts) - 1) & 1, &sy.abort))
          break;
        tc::mbar_arrive_expect_tx(&sy.full[ts], 2 * ebytes);
        tc::bulk_g2s(sm + ts * 2 * ebytes, etp + (size_t)(gb / 8 + 2 * k) * (ebytes / 4),
                     2 * ebytes, &sy.full[ts]);
        issued = k + 1;
      }
      // let the copies still in flight land before the block can exit
      for (int k = max(0, issued - nts); k < issued; k++)
        tc::mbar_wait(&sy.full[k % nts], (k / nts) & 1);
    }
  } else if (lane == 0) {
    // ---- MMA issuer
    const uint32_t idesc = tc::idesc_tf32(128, npad);
    for (int k = 0; k < nsteps; k++) {
      const int ts = k % nts;
      if (!tc::mbar_wait_abort(&sy.full[ts], (k / nts) & 1, &sy.abort)) break;
      tc::fence_after_sync();
      const uint32_t b = tc::smem_addr(sm + ts * 2 * ebytes);
      const uint32_t a = sy.tmem + acol + 64 * ts;
#pragma unroll
      for (int s = 0; s < 4; s++) {
        const uint32_t bt = b + (s >> 1) * ebytes + (s & 1) * 256;
        const uint64_t bh = tc::sdesc(bt, kLBO, kSBO);
        const uint64_t bl = tc::sdesc(bt + npad * 64, kLBO, kSBO);
        tc::mma_tf32_ts(sy.tmem, a + 8 * s, bh, idesc, (k == 0 && s == 0) ? 0u : 1u);
        tc::mma_tf32_ts(sy.tmem, a + 8 * s, bl, idesc, 1u);
        tc::mma_tf32_ts(sy.tmem, a + 32 + 8 * s, bh, idesc, 1u);
      }
      tc::mma_commit(&sy.empty[ts]);
    }
    tc::mma_commit(&sy.done);  // arrives once every MMA issued above has finished
  }
  close_block(sy, ncols, err);
}

// Reduction of the projection slices, written as the B' operand tiles of the
// back-projection: tile (band tile bt, atom step s) holds ncolN = nbt*2L rows
// x 16 fp32 (8 atoms x re/im), hi then lo.  Every element of every tile is
// written (zeros outside nb x nat).
// grid (ceil(4 nsa / 32), nbtiles * nbt * L); 128 threads.  Block y is one
// (band, lm); lane l of warp q serves atom pair 32 blockIdx.x + l (atoms
// 2 pair, 2 pair + 1) over slices q, q + 4, ..., so a warp reads whole rows
// of part; the four partial sums are added in the order q = 0..3, so the
// result does not depend on scheduling.
constexpr int kWtWarps = 4;
template <int L>
__global__ void __launch_bounds__(32 * kWtWarps) k_proj_tc_wtiles(
    const float *__restrict__ part, int nsplit, int nb, int nat, const float *__restrict__ w,
    int nbt, int nsa, float *__restrict__ wt) {
  constexpr int per = 2 * L;
  __shared__ float4 ps[kWtWarps][32];
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int pair = blockIdx.x * 32 + lane;
  const int lm = blockIdx.y % L, b = blockIdx.y / L;
  const int a0 = 2 * pair;
  const int Mtot = nb * per;
  // x = (Re, Im) of atom a0, (Re, Im) of atom a0 + 1
  float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
  if (b < nb && a0 < nat) {
    const bool two = a0 + 1 < nat;
    const size_t rs = (size_t)Mtot * nat;  // slice stride
    const float *p0 = part + (size_t)(b * per + 2 * lm) * nat + a0;
#pragma unroll 4
    for (int sl = q; sl < nsplit; sl += kWtWarps) {
      const float *r0 = p0 + sl * rs, *r1 = r0 + nat;
      x.x += r0[0];
      x.y += r1[0];
      if (two) {
        x.z += r0[1];
        x.w += r1[1];
      }
    }
  }
  ps[q][lane] = x;
  __syncthreads();
  if (q != 0 || pair >= 4 * nsa) return;
#pragma unroll
  for (int i = 1; i < kWtWarps; i++) {
    const float4 y = ps[i][lane];
    x.x += y.x;
    x.y += y.y;
    x.z += y.z;
    x.w += y.w;
  }
  const float w0 = a0 < nat ? w[a0 * L + lm] : 0.f;
  const float w1 = a0 + 1 < nat ? w[(a0 + 1) * L + lm] : 0.f;
  const float2 W0 = make_float2(w0 * x.x, w0 * x.y), W1 = make_float2(w1 * x.z, w1 * x.w);
  const int s = pair >> 2, c = pair & 3;
  const int bt = b / nbt, bl = b % nbt;
  const int ncolN = nbt * per;
  unsigned char *hi = reinterpret_cast<unsigned char *>(wt + ((size_t)bt * nsa + s) * ncolN * 32);
  unsigned char *lo = hi + ncolN * 64;
  const int r = bl * per + 2 * lm;
  tc::st_split4(hi, lo, tc::core_off<kBK>(r, 4 * c), make_float4(W0.x, -W0.y, W1.x, -W1.y));
  tc::st_split4(hi, lo, tc::core_off<kBK>(r + 1, 4 * c), make_float4(W0.y, W0.x, W1.y, W1.x));
}

// ------------------------------------------------------------------ back-projection
// The 2L TMEM columns of one band (warp-collective).
template <int per>
__device__ __forceinline__ void ld_band(uint32_t taddr, uint32_t *v) {
  if constexpr (per == 8) {
    tc::tmem_ld<8>(taddr, v);
  } else if constexpr (per == 4) {
    tc::tmem_ld<4>(taddr, v);
  } else if constexpr (per == 2) {
    tc::tmem_ld<2>(taddr, v);
  } else {
    tc::tmem_ld<2>(taddr, v);
    tc::tmem_ld<2>(taddr + 2, v + 2);
    tc::tmem_ld<2>(taddr + 4, v + 4);
  }
  tc::tmem_wait_ld();
}

// grid (G tiles of 128, band tiles of nbt); kThreads threads.
// etb: per (G tile, 8 atoms), [128 x 16] hi then lo.  wt: see k_proj_tc_wtiles.
// Epilogue thread (warp w, lane l): G row 32 (w % 4) + l, bands of half w / 4
// of the band tile.
// PRE: the recurrence's other terms are in out already (stick pass), so the
// epilogue only adds ca times the projector term.
template <int L, bool PRE>
__global__ void __launch_bounds__(kThreads) k_backproj_tc(
    const float *__restrict__ etb, const float *__restrict__ wt, int nsa, int ngw, int nb, int nbt,
    const float *__restrict__ pkga, float2 *out, int ldo, const float2 *__restrict__ in, int ldi,
    const float2 *__restrict__ xm2, int ldx, float ca, float cb, float cg, int *err) {
  constexpr int per = 2 * L;
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ Sync sy;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int gt = blockIdx.x, bt = blockIdx.y;
  const int g0 = gt * 128, b0 = bt * nbt;
  const int nbb = min(nbt, nb - b0);
  const int ncolN = nbt * per;  // a multiple of 16, <= 128; nbt is even
  const uint32_t abytes = 2 * kTileBytes128, bbytes = (uint32_t)ncolN * 128;
  const int slot_bytes = (int)(abytes + bbytes);
  const uint32_t ncols = tmem_cols(ncolN);
  open_block(sy, ncols, kNTB, 1, 0);

  if (warp == kRowWarps) {
    if (lane == 0) {
      int issued = 0;
      for (int k = 0; k < nsa; k++) {
        const int ts = k % kNTB;
        if (k >= kNTB && !tc::mbar_wait_abort(&sy.empty[ts], ((k / kNTB) - 1) & 1, &sy.abort))
          break;
        unsigned char *slot = sm + ts * slot_bytes;
        tc::mbar_arrive_expect_tx(&sy.bfull[ts], abytes + bbytes);
        tc::bulk_g2s(slot, etb + ((size_t)gt * nsa + k) * (abytes / 4), abytes, &sy.bfull[ts]);
        tc::bulk_g2s(slot + abytes, wt + ((size_t)bt * nsa + k) * (bbytes / 4), bbytes,
                     &sy.bfull[ts]);
        issued = k + 1;
      }
      drain_bulk(sy, issued, kNTB);
    }
  } else if (warp == kRowWarps + 1) {
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_tf32(128, ncolN);
      for (int k = 0; k < nsa; k++) {
        const int ts = k % kNTB;
        if (!tc::mbar_wait_abort(&sy.bfull[ts], (k / kNTB) & 1, &sy.abort)) break;
        tc::fence_after_sync();
        const uint32_t a = tc::smem_addr(sm + ts * slot_bytes);
        issue_step(sy.tmem, a, a + kTileBytes128, a + abytes, a + abytes + ncolN * 64, idesc,
                   k == 0);
        tc::mma_commit(&sy.empty[ts]);
      }
      tc::mma_commit(&sy.done);
    }
  } else {
    // ---- epilogue
    const int row = 32 * (warp & 3) + lane, half = warp >> 2;
    const uint32_t lane_base = sy.tmem + ((uint32_t)(32 * (warp & 3)) << 16);
    const int g = g0 + row;
    const bool gv = g < ngw;
    const int nbh = nbt / 2;
    const int bstart = half * nbh;
    float pk[4] = {0.f, 0.f, 0.f, 0.f};
    if (gv) {
      const float4 p4 = *reinterpret_cast<const float4 *>(pkga + (size_t)g * 4);
      pk[0] = p4.x;
      pk[1] = p4.y;
      pk[2] = p4.z;
      pk[3] = p4.w;
    }
    // the operands of CH bands are loaded at once (the first CH while the
    // MMAs run), so one memory latency covers CH bands
    constexpr int CH = PRE ? 8 : 4;
    float2 hv[CH], uv[CH], xv[CH];
    auto fetch = [&](int j0) {
#pragma unroll
      for (int i = 0; i < CH; i++) {
        const int bl = bstart + j0 + i;
        hv[i] = uv[i] = xv[i] = make_float2(0.f, 0.f);
        if (gv && j0 + i < nbh && bl < nbb) {
          const size_t bb = (size_t)(b0 + bl);
          hv[i] = out[bb * ldo + g];
          if (!PRE && cb != 0.f) uv[i] = in[bb * ldi + g];
          if (!PRE && cg != 0.f) xv[i] = xm2[bb * ldx + g];
        }
      }
    };
    fetch(0);
    const bool ok = __all_sync(0xffffffffu, tc::mbar_wait_abort(&sy.done, 0, &sy.abort));
    tc::fence_after_sync();
    if (ok) {
      for (int j0 = 0; j0 < nbh; j0 += CH) {
        if (j0 > 0) fetch(j0);
#pragma unroll
        for (int i = 0; i < CH; i++) {
          const int j = j0 + i;
          if (j >= nbh) break;  // block-uniform: the TMEM load below is warp-collective
          uint32_t v[per];
          ld_band<per>(lane_base + (uint32_t)((bstart + j) * per), v);
          float accr = 0.f, acci = 0.f;
#pragma unroll
          for (int l = 0; l < L; l++) {
            accr += pk[l] * __uint_as_float(v[2 * l]);
            acci += pk[l] * __uint_as_float(v[2 * l + 1]);
          }
          const int bl = bstart + j;
          if (!gv || bl >= nbb) continue;
          const float2 hc = hv[i];
          if (PRE) {
            out[(size_t)(b0 + bl) * ldo + g] = make_float2(hc.x + ca * accr, hc.y + ca * acci);
          } else {
            float rr = ca * (hc.x + accr), ii = ca * (hc.y + acci);
            if (cb != 0.f) {
              rr += cb * uv[i].x;
              ii += cb * uv[i].y;
            }
            if (cg != 0.f) {
              rr += cg * xv[i].x;
              ii += cg * xv[i].y;
            }
            out[(size_t)(b0 + bl) * ldo + g] = make_float2(rr, ii);
          }
        }
      }
    }
  }
  close_block(sy, ncols, err);
}

// ------------------------------------------------------------------ EIGR tiles
__global__ void k_build_etp(const float2 *__restrict__ eigr, int ngw, int nat, int npad, int nst,
                            float *__restrict__ etp) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)nst * npad * 4) return;
  const int c = (int)(idx & 3);
  const int r = (int)((idx >> 2) % npad);
  const int s = (int)(idx / (4 * npad));
  float v[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int k = 4 * c + q, g = 8 * s + (k >> 1);
    float x = 0.f;
    if (r < nat && g < ngw) {
      const float2 e = eigr[(size_t)r * ngw + g];
      x = (k & 1) ? e.y : e.x;
    }
    v[q] = x;
  }
  unsigned char *hi = reinterpret_cast<unsigned char *>(etp + (size_t)s * npad * 32);
  tc::st_split4(hi, hi + npad * 64, tc::core_off<kBK>(r, 4 * c), make_float4(v[0], v[1], v[2], v[3]));
}

__global__ void k_build_etb(const float2 *__restrict__ eigr, int ngw, int nat, int nsa, int ngt,
                            float *__restrict__ etb) {
  const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (idx >= (long long)ngt * nsa * 512) return;
  const int c = (int)(idx & 3);
  const int gg = (int)((idx >> 2) & 127);
  const int s = (int)((idx >> 9) % nsa);
  const int t = (int)(idx / (512LL * nsa));
  float v[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int k = 4 * c + q, a = 8 * s + (k >> 1), g = 128 * t + gg;
    float x = 0.f;
    if (a < nat && g < ngw) {
      const float2 e = eigr[(size_t)a * ngw + g];
      x = (k & 1) ? e.y : e.x;
    }
    v[q] = x;
  }
  unsigned char *hi = reinterpret_cast<unsigned char *>(etb + ((size_t)t * nsa + s) * 4096);
  tc::st_split4(hi, hi + 8192, tc::core_off<kBK>(gg, 4 * c), make_float4(v[0], v[1], v[2], v[3]));
}

// ------------------------------------------------------------------ host side
struct Shape {
  int L, per, nat, npad, nsa, nbt, ncolN, nbtiles;
};

// A species with projectors: its atoms (a range of the species-major atom
// order), its projectors per atom, its first projector, and the offsets
// (floats) of its blocks in the EIGR tile buffers, which hold one block per
// such species in species order.
struct Group {
  int sp, atom0, nat, L, p0;
  size_t etp_off, etb_off;
};

std::vector<Group> groups_of(const Projectors &P, int ngw_cell) {
  std::vector<Group> g;
  const size_t nst = (size_t)(ngw_cell + kStepG - 1) / kStepG * (kStepG / 8);
  const size_t ngt = (size_t)(ngw_cell + 127) / 128;
  int atom0 = 0, p0 = 0;
  size_t eo = 0, bo = 0;
  for (int s = 0; s < (int)P.sp_na.size(); s++) {
    const int na = P.sp_na[s], L = P.sp_lm[s];
    if (na > 0 && L > 0) {
      g.push_back({s, atom0, na, L, p0, eo, bo});
      eo += nst * (size_t)((na + 15) / 16 * 16) * 32;  // npad x 128 bytes per 8 G
      bo += ngt * (size_t)((na + 7) / 8) * 4096;       // 16 KB per (128 G, 8 atoms)
    }
    atom0 += na;
    p0 += na * std::max(0, L);
  }
  return g;
}

bool fits(const Projectors &P) {
  if (P.nproj <= 0 || (int)P.sp_na.size() != P.nsp || (int)P.sp_lm.size() != P.nsp) return false;
  bool any = false;
  for (int s = 0; s < P.nsp; s++) {
    if (P.sp_na[s] <= 0 || P.sp_lm[s] <= 0) continue;
    if (P.sp_na[s] > 256 || P.sp_lm[s] > 4) return false;
    any = true;
  }
  return any;
}

Shape shape_of(const Group &gp, int nb) {
  Shape s;
  s.nat = gp.nat;
  s.L = gp.L;
  s.per = 2 * s.L;
  s.npad = (gp.nat + 15) / 16 * 16;
  s.nsa = (gp.nat + 7) / 8;
  // bands per back-projection N tile: nbt*2L a multiple of 16, at most 128
  int nmax = kMaxBackN / s.per;
  while ((nmax * s.per) % 16) nmax--;
  int nbt = std::min(nmax, nb);
  while ((nbt * s.per) % 16) nbt++;
  s.nbt = nbt;
  s.ncolN = nbt * s.per;
  s.nbtiles = (nb + nbt - 1) / nbt;
  return s;
}

size_t up256(size_t n) { return (n + 255) / 256 * 256; }

size_t group_wtile_bytes(const Shape &s) { return up256((size_t)s.nbtiles * s.nsa * s.ncolN * 128); }

// Dynamic shared memory, raised where needed so that no more blocks fit on
// an SM than its 512 TMEM columns can serve at once (an allocation would
// otherwise wait for a resident block to finish).
int block_smem(int need, int ncols) {
  const int per_sm = 512 / ncols;
  const int floor_bytes = 233472 / (per_sm + 1) + 1024;
  return std::max(need, floor_bytes);
}

int proj_tmem_cols(const Shape &s) {
  return tmem_cols(tmem_cols(s.npad) + 64 * proj_slots(s.npad));
}

int proj_smem(const Shape &s) {
  const int nbr_max = 127 / s.per + 2;
  const int raw = round16(nbr_max * (kStepG + 1) * 8) + kStepG * 16;
  return block_smem(proj_slots(s.npad) * 2 * s.npad * 128 + kNR * raw, proj_tmem_cols(s));
}

int back_smem(const Shape &s) {
  return block_smem(kNTB * (2 * kTileBytes128 + s.ncolN * 128), tmem_cols(s.ncolN));
}

int sm_count() {
  static const int n = [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }();
  return n;
}

// splits of the projection's K range: enough blocks to fill the GPU once
int proj_splits(const Shape &s, int ngw, int nb, int *kg_out) {
  const int mt = (nb * s.per + 127) / 128;
  const int smem = proj_smem(s);
  const int per_sm = std::max(1, std::min(233472 / (smem + 1024), 512 / proj_tmem_cols(s)));
  int nsplit = std::max(1, std::min((ngw + 63) / 64, per_sm * sm_count() / mt));
  int kg = (ngw + nsplit - 1) / nsplit;
  kg = (kg + kStepG - 1) / kStepG * kStepG;
  *kg_out = kg;
  return (ngw + kg - 1) / kg;
}

template <int L>
int launch_project(pspw_cell *c, const Shape &s, const float2 *psi, int ld, int ngw, int nb,
                   float *part, int nsplit, int kg, float *wt, const float *etp,
                   const float *pkga, const float *pw) {
  const int mt = (nb * s.per + 127) / 128;
  const int smem = proj_smem(s);
  int rc = smem_allow_max(k_proj_tc<L>);
  if (rc) return rc;
  k_proj_tc<L><<<dim3(mt, nsplit), kThreadsP, smem, c->stream>>>(
      psi, ld, ngw, nb, etp, pkga, s.nat, s.npad, kg, part, c->d_err);
  const dim3 wgrid((4 * s.nsa + 31) / 32, s.nbtiles * s.nbt * L);
  k_proj_tc_wtiles<L><<<wgrid, 32 * kWtWarps, 0, c->stream>>>(part, nsplit, nb, s.nat, pw, s.nbt,
                                                               s.nsa, wt);
  c->kernel_launches += 2;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

template <int L>
int launch_back(pspw_cell *c, const Shape &s, const float *wt, const float *etb,
                const float *pkga, int ngw, int nb, float2 *out, int ldo, const float2 *in,
                int ldi, const float2 *xm2, int ldx, float a, float b, float g, bool pre) {
  const int smem = back_smem(s);
  auto kern = pre ? k_backproj_tc<L, true> : k_backproj_tc<L, false>;
  int rc = smem_allow_max(kern);
  if (rc) return rc;
  dim3 grid((ngw + 127) / 128, s.nbtiles);
  kern<<<grid, kThreads, smem, c->stream>>>(etb, wt, s.nsa, ngw, nb, s.nbt, pkga, out, ldo, in,
                                            ldi, xm2, ldx, a, b, g, c->d_err);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

}  // namespace

// One bounded barrier wait, the one every tensor-core kernel uses: with
// complete == 0 nothing arrives on the barrier, so the wait gives up after
// about a second and raises the cell's error word; otherwise the waiting
// thread arrives first and the wait succeeds at once.
__global__ void k_wait_check(int complete, int *err) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
    if (complete) tc::mbar_arrive(&bar);
    if (!tc::mbar_wait(&bar, 0)) atomicOr(err, 1);
  }
}

int nl_tc_wait_check(pspw_cell *c, int complete) {
  if (!c->d_err) return fail(PSPW_ERR_NOT_IMPL, "the cell has no device error word");
  k_wait_check<<<1, 32, 0, c->stream>>>(complete, c->d_err);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  return device_status(c);
}

bool nl_tc_usable(const pspw_cell *c) {
  static const bool off = std::getenv("PSPW_NL_SIMT") != nullptr;
  if (c->nl_path == PSPW_NL_SIMT || (off && c->nl_path != PSPW_NL_TENSOR_CORE)) return false;
  return fits(c->proj) && c->proj.d_etp && c->proj.d_etb && c->d_err;
}

int nl_tc_build_tiles(pspw_cell *c, const float2 *eigr32, float **etp, float **etb) {
  Projectors &P = c->proj;
  if (!fits(P)) return PSPW_OK;
  const int ngw = c->basis.ngw;
  const std::vector<Group> gs = groups_of(P, ngw);
  // projection tiles: every 8 G of the sphere, rounded up to whole steps of
  // kStepG G (the tail tiles hold zeros); one block per species
  const int nst = (ngw + kStepG - 1) / kStepG * (kStepG / 8), ngt = (ngw + 127) / 128;
  size_t fe = 0, fb = 0;
  int npad_max = 0;
  for (const Group &g : gs) {
    const int npad = (g.nat + 15) / 16 * 16, nsa = (g.nat + 7) / 8;
    fe = g.etp_off + (size_t)nst * npad * 32;
    fb = g.etb_off + (size_t)ngt * nsa * 4096;
    npad_max = std::max(npad_max, npad);
  }
  if (cudaMalloc(etp, fe * sizeof(float)) != cudaSuccess ||
      cudaMalloc(etb, fb * sizeof(float)) != cudaSuccess)
    return fail(PSPW_ERR_OOM, "EIGR operand tiles");
  P.tc_npad = npad_max;
  for (const Group &g : gs) {
    const int npad = (g.nat + 15) / 16 * 16, nsa = (g.nat + 7) / 8;
    const float2 *e = eigr32 + (size_t)g.atom0 * ngw;
    const long long n1 = (long long)nst * npad * 4, n2 = (long long)ngt * nsa * 512;
    k_build_etp<<<(unsigned)((n1 + 255) / 256), 256, 0, c->stream>>>(e, ngw, g.nat, npad, nst,
                                                                     *etp + g.etp_off);
    k_build_etb<<<(unsigned)((n2 + 255) / 256), 256, 0, c->stream>>>(e, ngw, g.nat, nsa, ngt,
                                                                     *etb + g.etb_off);
    c->kernel_launches += 2;
  }
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int nl_tc_prepare(pspw_cell *c) {
  Projectors &P = c->proj;
  if (!fits(P) || P.d_etp) return PSPW_OK;
  return nl_tc_build_tiles(c, P.d_eigr32, &P.d_etp, &P.d_etb);
}

size_t nl_tc_wtile_bytes(const pspw_cell *c, int nb) {
  if (!fits(c->proj)) return 0;
  size_t n = 0;
  for (const Group &g : groups_of(c->proj, c->basis.ngw)) n += group_wtile_bytes(shape_of(g, nb));
  return n;
}

int nl_tc_reserve(pspw_cell *c, int ngw, int nb, float **part, int *max_split, float **wt) {
  int ms = 1;
  for (const Group &g : groups_of(c->proj, c->basis.ngw)) {
    int kg = 0;
    ms = std::max(ms, proj_splits(shape_of(g, nb), ngw, nb, &kg));
  }
  // the partial sums of any one species fit max_split x 2 nb nproj floats
  int rc = ws_reserve(c, kWsProjPart, sizeof(float) * (size_t)ms * 2 * nb * c->proj.nproj,
                      (void **)part);
  if (rc) return rc;
  rc = ws_reserve(c, kWsWTile, nl_tc_wtile_bytes(c, nb), (void **)wt);
  if (rc) return rc;
  *max_split = ms;
  return PSPW_OK;
}

int nl_tc_project(pspw_cell *c, const float2 *psi, int ld, int ngw, int nb, float *part,
                  int max_split, float *wt) {
  const Projectors &P = c->proj;
  const size_t cap = (size_t)std::max(1, max_split) * 2 * nb * P.nproj;  // floats of part
  size_t woff = 0;
  for (const Group &g : groups_of(P, c->basis.ngw)) {
    const Shape s = shape_of(g, nb);
    int kg = 0;
    int nsplit = proj_splits(s, ngw, nb, &kg);
    const int lim = (int)std::max<size_t>(1, cap / ((size_t)nb * s.per * s.nat));
    if (nsplit > lim) {
      nsplit = lim;
      kg = ((ngw + nsplit - 1) / nsplit + kStepG - 1) / kStepG * kStepG;
      nsplit = (ngw + kg - 1) / kg;
    }
    float *w = wt + woff / sizeof(float);
    const float *etp = P.d_etp + g.etp_off, *pk = P.d_pkga32 + (size_t)g.sp * c->basis.ngw * 4,
                *pw = P.d_pw32 + g.p0;
    int rc;
    switch (s.L) {
      case 1: rc = launch_project<1>(c, s, psi, ld, ngw, nb, part, nsplit, kg, w, etp, pk, pw); break;
      case 2: rc = launch_project<2>(c, s, psi, ld, ngw, nb, part, nsplit, kg, w, etp, pk, pw); break;
      case 3: rc = launch_project<3>(c, s, psi, ld, ngw, nb, part, nsplit, kg, w, etp, pk, pw); break;
      default: rc = launch_project<4>(c, s, psi, ld, ngw, nb, part, nsplit, kg, w, etp, pk, pw);
    }
    if (rc) return rc;
    woff += group_wtile_bytes(s);
  }
  return PSPW_OK;
}

int nl_tc_backproject(pspw_cell *c, const float *wt, int ngw, int nb, float2 *out, int ldo,
                      const float2 *in, int ldi, const float2 *xm2, int ldx, float a, float b,
                      float g, bool pre) {
  const Projectors &P = c->proj;
  size_t woff = 0;
  bool first = true;
  for (const Group &gp : groups_of(P, c->basis.ngw)) {
    const Shape s = shape_of(gp, nb);
    const float *w = wt + woff / sizeof(float);
    const float *etb = P.d_etb + gp.etb_off, *pk = P.d_pkga32 + (size_t)gp.sp * c->basis.ngw * 4;
    // the first species applies the recurrence's update; the others add
    // their a * sum to it (the `pre` form)
    const bool pr = first ? pre : true;
    int rc;
    switch (s.L) {
      case 1: rc = launch_back<1>(c, s, w, etb, pk, ngw, nb, out, ldo, in, ldi, xm2, ldx, a, b, g, pr); break;
      case 2: rc = launch_back<2>(c, s, w, etb, pk, ngw, nb, out, ldo, in, ldi, xm2, ldx, a, b, g, pr); break;
      case 3: rc = launch_back<3>(c, s, w, etb, pk, ngw, nb, out, ldo, in, ldi, xm2, ldx, a, b, g, pr); break;
      default: rc = launch_back<4>(c, s, w, etb, pk, ngw, nb, out, ldo, in, ldi, xm2, ldx, a, b, g, pr);
    }
    if (rc) return rc;
    woff += group_wtile_bytes(s);
    first = false;
  }
  return PSPW_OK;
}

}  // namespace pspw
