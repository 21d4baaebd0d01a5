// Benchmark infrastructure: the measured denominator of the pairwise kernels'
// roofline.
//
// The pairwise kernels are bound by the FP64 (plain form) or FP32 (mixed form)
// CUDA-core pipes, for which no measured figure exists on this machine. This
// kernel keeps every SM's FMA pipe busy with independent dependency chains and
// reports the sustained fused-multiply-add rate (2 flops per FMA); bench.py
// reports it beside the rate derived from the SM count and clock.
#include "device_math.cuh"
#include "kernels.cuh"

namespace btk {

namespace {

constexpr int kChains = 8;

template <class T>
__global__ void __launch_bounds__(256) k_fma_peak(T* out, int iters, T b, T c) {
  T a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = (T)(threadIdx.x + k) * (T)1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == (T)12345.678) out[0] = s;  // keeps the chains live; never true in practice
}

}  // namespace

}  // namespace btk

using namespace btk;

extern "C" btk_status btk_measure_pipe_peak(int which, double* tflops, btk_stream_t stream) {
  BTK_CHECK(tflops && (which == 0 || which == 1), BTK_ERR_INVALID_ARGUMENT, "btk_measure_pipe_peak: bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  BTK_CUDA(cudaGetDevice(&dev));
  BTK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  double* sink = nullptr;
  BTK_CUDA(cudaMallocAsync(&sink, 16, st));
  const int threads = 256, blocks = sms * 8, iters = which == 0 ? 8192 : 32768;
  cudaEvent_t e0, e1;
  BTK_CUDA(cudaEventCreate(&e0));
  BTK_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    BTK_CUDA(cudaEventRecord(e0, st));
    if (which == 0)
      k_fma_peak<double><<<blocks, threads, 0, st>>>(sink, iters, 0.999999, 1e-7);
    else
      k_fma_peak<float><<<blocks, threads, 0, st>>>((float*)sink, iters, 0.999999f, 1e-7f);
    count_launch();
    BTK_CUDA(cudaGetLastError());
    BTK_CUDA(cudaEventRecord(e1, st));
    BTK_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    BTK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0 && ms < best) best = ms;  // first launch warms up
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(sink, st);
  const double flops = 2.0 * kChains * (double)iters * threads * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return BTK_OK;
}
