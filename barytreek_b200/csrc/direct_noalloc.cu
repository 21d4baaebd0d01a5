// btk_direct_sum_noalloc: the FP64 direct sum of btk_direct_sum, with that
// entry point's one piece of per-call scratch (the packed double4 source
// array) held in a file-scope device array instead of memory allocated on
// every call. Same kernel, same packing, so the results are bit-identical.
//
// Who needs it: callers that cannot allocate device memory inside the call.
//  * A host code whose own caching allocator has reserved the device's memory
//    (a PyTorch process, a simulation code with a pooled allocator): a
//    cudaMallocAsync inside the call can fail there, or fragment the pool.
//  * A time-stepping loop that evaluates the field every step and cannot take
//    an allocation's latency and stream-ordered free on each step.
//
// Limit: kNoAllocMaxSources = 262,144 sources, i.e. 8 MiB of device memory
// held by the module for the life of the process. Larger calls are rejected
// with BTK_ERR_INVALID_ARGUMENT before any device work; btk_direct_sum (which
// allocates) has no such limit. Targets are not limited (the output is the
// caller's).
//
// One scratch array per device. Calls on one device that overlap in time (two
// host threads, or two streams not ordered against each other) race on it;
// calls ordered on one stream do not. The first call on each device looks up
// the scratch address with cudaGetSymbolAddress, with that device current, and
// caches it; make that first call before any stream capture begins on that
// device. The cached address belongs to the device's current primary context:
// after cudaDeviceReset (or any teardown of that context) the module is
// loaded anew and its scratch may move, so a process must not call this entry
// point on a device again once it has reset that device. Nothing in the
// scratch must start at zero: the packing kernel of the
// same call writes every slot the summation kernel reads.
#include <cstdint>
#include <mutex>
#include <string>

#include "kernels.cuh"

namespace btk {
namespace {

constexpr int kNoAllocMaxSources = 1 << 18;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double4 g_direct_scratch[kNoAllocMaxSources];

std::mutex g_scratch_mu;
double4* g_scratch_addr[kMaxDevices];  // per device, filled on first use

btk_status scratch_for_current_device(double4** out) {
  int dev = -1;
  BTK_CUDA(cudaGetDevice(&dev));
  BTK_CHECK(dev >= 0 && dev < kMaxDevices, BTK_ERR_UNSUPPORTED, "direct_sum_noalloc: device index above 63");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    BTK_CUDA(cudaGetSymbolAddress(&p, g_direct_scratch));
    BTK_CHECK(p && reinterpret_cast<uintptr_t>(p) % 256 == 0, BTK_ERR_CUDA,
              "direct_sum_noalloc: scratch symbol address missing or misaligned");
    g_scratch_addr[dev] = static_cast<double4*>(p);
  }
  *out = g_scratch_addr[dev];
  return BTK_OK;
}

// Packs (x, y, z, q) into double4 in the original source order; the same
// values k_gather produces through an identity permutation.
__global__ void k_pack_sources(int n, const double* x, const double* y, const double* z, const double* q,
                               double4* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = make_double4(x[i], y[i], z ? z[i] : 0.0, q[i]);
}

}  // namespace
}  // namespace btk

using namespace btk;

extern "C" btk_status btk_direct_sum_noalloc(int dim, int kind, double eps, int nt, const double* xt,
                                             const double* yt, const double* zt, int ns, const double* xs,
                                             const double* ys, const double* zs, const double* charges, double* out,
                                             btk_stream_t stream) {
  BTK_CHECK(dim == 2 || dim == 3, BTK_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
  BTK_CHECK(!(kind == BTK_KIND_VEL && dim != 3) && kind >= 0 && kind <= 2, BTK_ERR_INVALID_ARGUMENT, "bad kind");
  BTK_CHECK(nt >= 0 && ns >= 0, BTK_ERR_INVALID_ARGUMENT, "direct_sum_noalloc: negative count");
  BTK_CHECK(ns <= kNoAllocMaxSources, BTK_ERR_INVALID_ARGUMENT,
            "direct_sum_noalloc: " + std::to_string(ns) + " sources exceed the static scratch of " +
                std::to_string(kNoAllocMaxSources) + "; use btk_direct_sum");
  BTK_CHECK(xt && yt && xs && ys && charges && out && (dim == 2 || (zt && zs)), BTK_ERR_INVALID_ARGUMENT,
            "direct_sum_noalloc: null argument");
  double4* src = nullptr;
  BTK_TRY(scratch_for_current_device(&src));
  cudaStream_t st = (cudaStream_t)stream;
  if (ns > 0) {
    k_pack_sources<<<(ns + 255) / 256, 256, 0, st>>>(ns, xs, ys, dim == 3 ? zs : nullptr, charges, src);
    count_launch();
    BTK_CUDA(cudaGetLastError());
  }
  BTK_CUDA(launch_direct(dim, kind, eps, nt, xt, yt, dim == 3 ? zt : nullptr, ns, src, out, st));
  return BTK_OK;
}
