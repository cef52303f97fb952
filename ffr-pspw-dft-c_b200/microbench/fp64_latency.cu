// Latency of dependent chains on one SM, in SM cycles per operation: FP64
// fma, square root, division, 64-bit shuffle, block barrier, dependent
// shared-memory load, FP64 add and a five-level warp sum.  One block of 32,
// 640 and 1024 threads (every warp runs the same chain), so the figures also
// show how the latency grows with the warps sharing the SM.  The numbers set
// the per-step budgets of the one-block dense kernels (heev.cu).
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 fp64_latency.cu -o fp64_latency
#include <cstdio>
#include <cuda_runtime.h>

__global__ void k_latency(double *out, long long *cyc, double seed, int n) {
  __shared__ int chase[1024];
  const int tid = threadIdx.x;
  for (int i = tid; i < 1024; i += blockDim.x) chase[i] = (i * 37 + 11) & 1023;
  __syncthreads();
  double x = seed + tid * 1e-9, y = 1.0 + seed, z = 3.0 + seed;
  long long t0, t1;
  t0 = clock64();
  for (int i = 0; i < n; i++) x = fma(x, 0.999999, 1e-7);
  t1 = clock64();
  if (tid == 0) cyc[0] = t1 - t0;
  t0 = clock64();
  for (int i = 0; i < n; i++) y = sqrt(y) + 1.0;
  t1 = clock64();
  if (tid == 0) cyc[1] = t1 - t0;
  t0 = clock64();
  for (int i = 0; i < n; i++) z = 1.0 / z + 1.0;
  t1 = clock64();
  if (tid == 0) cyc[2] = t1 - t0;
  double s = x;
  t0 = clock64();
  for (int i = 0; i < n; i++) s = __shfl_xor_sync(0xffffffffu, s, 1) + 1e-9;
  t1 = clock64();
  if (tid == 0) cyc[3] = t1 - t0;
  t0 = clock64();
  for (int i = 0; i < n; i++) __syncthreads();
  t1 = clock64();
  if (tid == 0) cyc[4] = t1 - t0;
  int p = tid & 1023;  // chase[] holds indices in [0, 1024)
  t0 = clock64();
  for (int i = 0; i < n; i++) p = chase[p];
  t1 = clock64();
  if (tid == 0) cyc[5] = t1 - t0;
  double a = x;
  t0 = clock64();
  for (int i = 0; i < n; i++) a = a + 1e-9;
  t1 = clock64();
  if (tid == 0) cyc[6] = t1 - t0;
  double w = x;
  t0 = clock64();
  for (int i = 0; i < n; i++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    w *= 1e-3;
  }
  t1 = clock64();
  if (tid == 0) cyc[7] = t1 - t0;
  out[tid] = x + y + z + s + a + w + p;
}

int main() {
  double *out;
  long long *cyc;
  if (cudaMalloc(&out, 1024 * sizeof(double)) != cudaSuccess ||
      cudaMalloc(&cyc, 8 * sizeof(long long)) != cudaSuccess)
    return 1;
  const int n = 256;
  const char *name[8] = {"fp64 fma", "fp64 sqrt + add", "fp64 division + add",
                         "shuffle (f64) + add", "block barrier", "shared load (chase)",
                         "fp64 add", "5-level warp sum + mul"};
  const int sizes[3] = {32, 640, 1024};
  for (int b = 0; b < 3; b++) {
    k_latency<<<1, sizes[b]>>>(out, cyc, 0.5, n);
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      printf("error: %s\n", cudaGetErrorString(e));
      return 1;
    }
    long long h[8];
    cudaMemcpy(h, cyc, sizeof(h), cudaMemcpyDeviceToHost);
    printf("block of %d threads, cycles per dependent operation:\n", sizes[b]);
    for (int i = 0; i < 8; i++) printf("  %-24s %6.1f\n", name[i], (double)h[i] / n);
  }
  cudaFree(out);
  cudaFree(cyc);
  return 0;
}
