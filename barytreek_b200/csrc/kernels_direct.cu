// FP64 direct sum over every (target, source) pair, target == source included
// (src/direct_sum_impl.hpp:9-94). Used for accuracy measurement against the
// treecode (the reference's examples do the same, e.g.
// examples/example_poisson_3d.cpp:163-183) and by the degree selector's audit.
// It uses IEEE sqrt and division, independent of the treecode's fast
// reciprocal square root.
#include "kernels.cuh"

namespace btk {

namespace {

constexpr int kDirectThreads = 256;
constexpr int kDirectChunk = 512;

template <int DIM, int KIND>
__global__ void __launch_bounds__(kDirectThreads) k_direct(double eps2, int nt, const double* xt, const double* yt,
                                                           const double* zt, int ns, const double4* src, double* out) {
  constexpr int NC = KIND == BTK_KIND_POT ? 1 : (KIND == BTK_KIND_VEL ? 3 : 1 + DIM);
  __shared__ double4 sb[kDirectChunk];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int ii = i < nt ? i : nt - 1;
  const double tx = xt[ii], ty = yt[ii], tz = DIM == 3 ? zt[ii] : 0.0;
  double acc[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
  for (int s0 = 0; s0 < ns; s0 += kDirectChunk) {
    const int cnt = min(kDirectChunk, ns - s0);
    __syncthreads();
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) sb[j] = src[s0 + j];
    __syncthreads();
    for (int j = 0; j < cnt; ++j) {
      const double4 s = sb[j];
      const double dx = tx - s.x, dy = ty - s.y, dz = DIM == 3 ? tz - s.z : 0.0;
      const double r2 = dx * dx + dy * dy + dz * dz + eps2;
      if (DIM == 2) {
        acc[0] += log(r2) * s.w;
        if (KIND == BTK_KIND_FIELD) {
          const double g = s.w / r2;
          acc[1] += dx * g;
          acc[2] += dy * g;
        }
      } else if (KIND == BTK_KIND_VEL) {
        const double g = s.w / r2;
        acc[0] += dx * g;
        acc[1] += dy * g;
        acc[2] += dz * g;
      } else {
        const double ri = 1.0 / sqrt(r2);
        acc[0] += ri * s.w;
        if (KIND == BTK_KIND_FIELD) {
          const double g = s.w * ri * ri * ri;
          acc[1] += dx * g;
          acc[2] += dy * g;
          acc[3] += dz * g;
        }
      }
    }
  }
  if (i >= nt) return;
  const double pi = 3.141592653589793238462643383279502884;
  const double q4 = 1.0 / (4.0 * pi);
  if (DIM == 2) {
    out[i] = q4 * acc[0];
    if (KIND == BTK_KIND_FIELD) {
      out[(size_t)nt + i] = -acc[1] / (2.0 * pi);
      out[2 * (size_t)nt + i] = -acc[2] / (2.0 * pi);
    }
  } else {
#pragma unroll
    for (int c = 0; c < NC; ++c) out[(size_t)c * nt + i] = -q4 * acc[c];
  }
}

}  // namespace

cudaError_t launch_direct(int dim, int kind, double eps, int nt, const double* xt, const double* yt, const double* zt,
                          int ns, const double4* src, double* out, cudaStream_t s) {
  if (nt <= 0) return cudaSuccess;
  const int grid = (nt + kDirectThreads - 1) / kDirectThreads;
  const double e2 = eps * eps;
  if (dim == 2) {
    if (kind == BTK_KIND_POT) k_direct<2, BTK_KIND_POT><<<grid, kDirectThreads, 0, s>>>(e2, nt, xt, yt, zt, ns, src, out);
    else k_direct<2, BTK_KIND_FIELD><<<grid, kDirectThreads, 0, s>>>(e2, nt, xt, yt, zt, ns, src, out);
  } else {
    if (kind == BTK_KIND_POT) k_direct<3, BTK_KIND_POT><<<grid, kDirectThreads, 0, s>>>(e2, nt, xt, yt, zt, ns, src, out);
    else if (kind == BTK_KIND_VEL) k_direct<3, BTK_KIND_VEL><<<grid, kDirectThreads, 0, s>>>(e2, nt, xt, yt, zt, ns, src, out);
    else k_direct<3, BTK_KIND_FIELD><<<grid, kDirectThreads, 0, s>>>(e2, nt, xt, yt, zt, ns, src, out);
  }
  count_launch();
  return cudaGetLastError();
}

}  // namespace btk
