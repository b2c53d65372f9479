// FMA throughput of the current GPU: every thread runs 8 independent FMA
// chains, all SMs fully occupied; flops = 2 per FMA.
#include "common.cuh"
#include "peaks.cuh"

namespace b2 {

namespace {

template <typename T>
__global__ void k_fma(T* out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; k++) x[k] = (T)(threadIdx.x + k);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = x[k] * a + b;
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == (T)-12345.678) out[0] = s;  // keep the chains alive
}

template <typename T>
double run(int iters) {
  int dev = 0, nsm = 0;
  B2_CHECK(cudaGetDevice(&dev));
  B2_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  DBuf<T> out(0);
  out.alloc(1, 0);
  int blocks = nsm * 8, threads = 256;
  cudaEvent_t e0, e1;
  B2_CHECK(cudaEventCreate(&e0));
  B2_CHECK(cudaEventCreate(&e1));
  k_fma<T><<<blocks, threads>>>(out.p, iters / 8, (T)0.999999, (T)1e-7);  // warm-up
  B2_LAUNCH_CHECK();
  B2_CHECK(cudaEventRecord(e0));
  k_fma<T><<<blocks, threads>>>(out.p, iters, (T)0.999999, (T)1e-7);
  B2_LAUNCH_CHECK();
  B2_CHECK(cudaEventRecord(e1));
  B2_CHECK(cudaEventSynchronize(e1));
  float ms = 0;
  B2_CHECK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double flops = 2.0 * 8.0 * iters * (double)blocks * threads;
  return flops / (ms * 1e-3);
}

}  // namespace

double fma_peak_flops(bool fp64) { return fp64 ? run<double>(4096) : run<float>(16384); }

}  // namespace b2
