// Pipe-peak probes: the denominators for the pairwise kernels' roofline.
//
// The pairwise kernels are bound by the FP64 (plain form) or FP32 (mixed form)
// CUDA-core pipes, which no vendor figure on this machine states as measured.
// These kernels keep every SM's FMA pipe busy with independent dependency
// chains and report the sustained fused-multiply-add rate (2 flops per FMA).
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

// Packed FP32: one sm_100 FFMA2 per step (two FMAs, 4 flops).
__global__ void __launch_bounds__(256) k_ffma2_peak(float* out, int iters, float b, float c) {
  float2 a[kChains];
  const float2 b2 = make_float2(b, b), c2 = make_float2(c, c);
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = make_float2((threadIdx.x + k) * 1e-3f, (threadIdx.x + 2 * k) * 1e-3f);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = __ffma2_rn(a[k], b2, c2);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k].x + a[k].y;
  if (s == 12345.678f) out[0] = s;
}

// MUFU reciprocal square root (rsqrt.approx.ftz.f32) per step.
__global__ void __launch_bounds__(256) k_rsqrt_peak(float* out, int iters) {
  float a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = 1.0f + (threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = rsqrt_fp32(a[k]);
  }
  float s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == 12345.678f) out[0] = s;
}

}  // namespace

}  // namespace btk

using namespace btk;

extern "C" btk_status btk_measure_pipe_peak(int which, double* tflops, btk_stream_t stream) {
  BTK_CHECK(tflops && which >= 0 && which <= 3, BTK_ERR_INVALID_ARGUMENT, "btk_measure_pipe_peak: bad argument");
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
    else if (which == 1)
      k_fma_peak<float><<<blocks, threads, 0, st>>>((float*)sink, iters, 0.999999f, 1e-7f);
    else if (which == 2)
      k_ffma2_peak<<<blocks, threads, 0, st>>>((float*)sink, iters, 0.999999f, 1e-7f);
    else
      k_rsqrt_peak<<<blocks, threads, 0, st>>>((float*)sink, iters / 8);
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
  const double per_step = which == 2 ? 4.0 : (which == 3 ? 1.0 / 8.0 : 2.0);
  const double flops = per_step * kChains * (double)iters * threads * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return BTK_OK;
}
