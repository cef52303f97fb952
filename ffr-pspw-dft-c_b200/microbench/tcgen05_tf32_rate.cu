// Issue rate of tcgen05.mma kind::tf32 (M = 128, K = 8) with one block per
// SM: cycles per MMA for N = 64, 128, 256, A from shared or tensor memory.
// The operand contents are irrelevant (zeros / uninitialised TMEM); every
// wait is bounded.  Prints one line per shape.
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 \
//        -I ffr-pspw-dft-c_b200/csrc ffr-pspw-dft-c_b200/microbench/tcgen05_tf32_rate.cu \
//        -o /tmp/tcgen05_tf32_rate && /tmp/tcgen05_tf32_rate
#include <cuda_runtime.h>

#include <cstdio>

#include "tc.cuh"

using namespace pspw;

template <int N, bool TS>
__global__ void k_rate(unsigned long long *out, int reps, int *err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  constexpr uint32_t cols = (N + 32 > 256) ? 512 : 256;
  if (threadIdx.x < 32) {
    tc::tmem_alloc(&tbase, cols);
    tc::tmem_relinquish();
  }
  for (int i = threadIdx.x; i < (128 + N) * 8; i += blockDim.x) reinterpret_cast<float *>(sm)[i] = 0.f;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
  }
  tc::fence_proxy_async();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (threadIdx.x == 0) {
    const uint32_t a = tc::smem_addr(sm), b = a + 128 * 32;
    const uint64_t ad = tc::sdesc(a, 128, 256), bd = tc::sdesc(b, 128, 256);
    const uint32_t id = tc::idesc_tf32(128, N);
    const uint32_t atm = tbase + N;  // A in TMEM after the accumulator
    const long long t0 = clock64();
    for (int r = 0; r < reps; r++) {
      if (TS)
        tc::mma_tf32_ts(tbase, atm, bd, id, r ? 1u : 0u);
      else
        tc::mma_tf32(tbase, ad, bd, id, r ? 1u : 0u);
    }
    tc::mma_commit(&bar);
    if (!tc::mbar_wait(&bar, 0)) atomicOr(err, 1);
    const long long t1 = clock64();
    if (blockIdx.x == 0) out[0] = (unsigned long long)(t1 - t0);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (threadIdx.x < 32) tc::tmem_dealloc(tbase, cols);
}

template <int N, bool TS>
static void run(unsigned long long *d, int *e, int sms) {
  const int reps = 1024, smem = (128 + N) * 32;
  k_rate<N, TS><<<sms, 128, smem>>>(d, reps, e);
  const cudaError_t st = cudaDeviceSynchronize();
  unsigned long long cyc = 0;
  int he = 0;
  cudaMemcpy(&cyc, d, sizeof(cyc), cudaMemcpyDeviceToHost);
  cudaMemcpy(&he, e, sizeof(he), cudaMemcpyDeviceToHost);
  const double per = (double)cyc / reps;
  printf("M=128 N=%3d K=8 A=%s: %.1f cycles/MMA = %.0f flop/cycle/SM%s%s\n", N,
         TS ? "tmem" : "smem", per, 128.0 * N * 8 * 2 / per, he ? " [wait timed out]" : "",
         st == cudaSuccess ? "" : cudaGetErrorString(st));
}

int main() {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  unsigned long long *d;
  int *e;
  cudaMalloc(&d, sizeof(*d));
  cudaMalloc(&e, sizeof(*e));
  cudaMemset(e, 0, sizeof(*e));
  run<64, false>(d, e, sms);
  run<128, false>(d, e, sms);
  run<256, false>(d, e, sms);
  run<64, true>(d, e, sms);
  run<128, true>(d, e, sms);
  run<256, true>(d, e, sms);
  return 0;
}
