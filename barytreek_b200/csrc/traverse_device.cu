// Dual-tree traversal on the device, producing exactly the interaction list
// of btk_dual_tree_traversal_2d/3d (src/interaction_list.cpp:5-117,
// :119-250), pairs in the same order.
//
// The reference walks a FIFO of (target, source) panel pairs from the roots:
// a pair that meets the MAC (r_T + r_S) / dist < theta becomes an interaction
// (type by point_count > thresh on each side); otherwise two leaves become PP,
// and anything else pushes the 2^dim children of one side (the non-leaf side,
// or the side with more points when both can be refined). A FIFO visits the
// pairs generation by generation, each generation in the order its parents
// pushed them, so processing a whole generation at once, placing the
// interactions and the children with exclusive scans over the generation,
// reproduces the list pair for pair. The MAC uses the reference's expression
// order with correctly rounded operations (no fused multiply-add).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "btk_internal.h"

namespace btk {
namespace {

constexpr int kScanBlock = 1024;

struct TravPanel {
  double c[3];  // box centre 0.5 * (min + max)
  double radius;
  int count;
  int leaf;
  int child[8];
};

// Exclusive scan within blocks of kScanBlock elements; block totals to sums.
__global__ void __launch_bounds__(kScanBlock) k_scan_block(const int* in, int* out, int n, int* sums) {
  __shared__ int warp_tot[kScanBlock / 32];
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int v = i < n ? in[i] : 0;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int t = warp_tot[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    warp_tot[lane] = t;  // inclusive over warps
  }
  __syncthreads();
  const int incl = x + (warp > 0 ? warp_tot[warp - 1] : 0);
  if (i < n) out[i] = incl - v;
  if (threadIdx.x == kScanBlock - 1 && sums) sums[blockIdx.x] = incl;
}

__global__ void k_scan_add(int* out, int n, const int* offs) {
  const int i = blockIdx.x * kScanBlock + threadIdx.x;
  if (i < n) out[i] += offs[blockIdx.x];
}

// Device buffers of one traversal, freed on every exit path.
struct Arena2 {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit Arena2(cudaStream_t s) : st(s) {}
  ~Arena2() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
  template <class U>
  cudaError_t alloc(U** p, size_t n) {
    cudaError_t e = cudaMallocAsync((void**)p, sizeof(U) * std::max<size_t>(n, 1), st);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

// out = exclusive scan of in (n elements).
btk_status exclusive_scan(const int* in, int* out, int n, Arena2& A, cudaStream_t st) {
  if (n <= 0) return BTK_OK;
  const int blocks = (n + kScanBlock - 1) / kScanBlock;
  int* sums = nullptr;
  if (blocks > 1) BTK_CUDA(A.alloc(&sums, (size_t)blocks));
  k_scan_block<<<blocks, kScanBlock, 0, st>>>(in, out, n, sums);
  count_launch();
  BTK_CUDA(cudaGetLastError());
  if (blocks > 1) {
    int* offs = nullptr;
    BTK_CUDA(A.alloc(&offs, (size_t)blocks));
    BTK_TRY(exclusive_scan(sums, offs, blocks, A, st));
    k_scan_add<<<blocks, kScanBlock, 0, st>>>(out, n, offs);
    count_launch();
    BTK_CUDA(cudaGetLastError());
  }
  return BTK_OK;
}

// One generation: what each pair does. act: 0..3 interaction of that type,
// 4 refine target, 5 refine source.
template <int D>
__global__ void k_trav_eval(int F, const int* ft, const int* fs, const TravPanel* T, const TravPanel* S, double theta,
                            int thresh, int* act, int* n_int, int* n_child) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= F) return;
  const TravPanel& t = T[ft[k]];
  const TravPanel& s = S[fs[k]];
  const double x_ex = __dadd_rn(s.c[0], -t.c[0]), y_ex = __dadd_rn(s.c[1], -t.c[1]);
  double d2 = __dadd_rn(__dmul_rn(x_ex, x_ex), __dmul_rn(y_ex, y_ex));
  if (D == 3) {
    const double z_ex = __dadd_rn(s.c[2], -t.c[2]);
    d2 = __dadd_rn(d2, __dmul_rn(z_ex, z_ex));
  }
  const double dist = __dsqrt_rn(d2);
  double separation = 100;
  if (dist > 0) separation = __ddiv_rn(__dadd_rn(t.radius, s.radius), dist);
  int a;
  if (separation < theta) {
    a = (t.count > thresh ? 2 : 0) + (s.count > thresh ? 1 : 0);
  } else if (t.leaf && s.leaf) {
    a = 0;
  } else if (t.leaf) {
    a = 5;
  } else if (s.leaf) {
    a = 4;
  } else {
    a = t.count > s.count ? 4 : 5;
  }
  act[k] = a;
  n_int[k] = a < 4 ? 1 : 0;
  n_child[k] = a >= 4 ? (1 << D) : 0;
}

template <int D>
__global__ void k_trav_emit(int F, const int* ft, const int* fs, const TravPanel* T, const TravPanel* S, const int* act,
                            const int* pos_int, const int* pos_child, btk_interact_pair* list, int* nt, int* ns) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= F) return;
  const int a = act[k], it = ft[k], is = fs[k];
  if (a < 4) {
    list[pos_int[k]] = btk_interact_pair{it, is, a};
  } else {
    const int p = pos_child[k];
#pragma unroll
    for (int c = 0; c < (1 << D); ++c) {
      nt[p + c] = a == 4 ? T[it].child[c] : it;
      ns[p + c] = a == 4 ? is : S[is].child[c];
    }
  }
}

// Host copy of the fields the traversal reads; refuses child links outside
// the array (the device follows them without further checks).
template <class P>
btk_status pack_panels(const P* p, int n, std::vector<TravPanel>& out) {
  const int nc = sizeof(P) == sizeof(btk_panel_2d) ? 4 : 8;
  out.resize(std::max(n, 1));
  for (int i = 0; i < n; ++i) {
    if (!p[i].is_leaf)
      for (int c = 0; c < nc; ++c)
        BTK_CHECK((&p[i].child1)[c] >= 0 && (&p[i].child1)[c] < n, BTK_ERR_INVALID_ARGUMENT,
                  "dual_tree_traversal_device: a non-leaf panel's child index is outside the panel array");
    TravPanel& q = out[i];
    std::memset(&q, 0, sizeof(q));
    q.c[0] = 0.5 * (p[i].min_x + p[i].max_x);
    q.c[1] = 0.5 * (p[i].min_y + p[i].max_y);
    if constexpr (sizeof(P) == sizeof(btk_panel_3d)) q.c[2] = 0.5 * (p[i].min_z + p[i].max_z);
    q.radius = p[i].radius;
    q.count = p[i].point_count;
    q.leaf = p[i].is_leaf ? 1 : 0;
    for (int c = 0; c < nc; ++c) q.child[c] = (&p[i].child1)[c];
  }
  return BTK_OK;
}

template <int D, class P>
btk_status traverse_device(btk_run_config* cfg, const P* Tp, int t_count, const P* Sp, int s_count,
                           btk_interact_pair** list_out, cudaStream_t st) {
  BTK_CHECK(cfg && Tp && Sp && list_out, BTK_ERR_INVALID_ARGUMENT, "dual_tree_traversal_device: null argument");
  BTK_CHECK(t_count > 0 && s_count > 0, BTK_ERR_INVALID_ARGUMENT, "dual_tree_traversal_device: empty panel array");
  const bool same = (const void*)Tp == (const void*)Sp && t_count == s_count;
  std::vector<TravPanel> ht, hs;
  BTK_TRY(pack_panels(Tp, t_count, ht));
  if (!same) BTK_TRY(pack_panels(Sp, s_count, hs));
  Arena2 A(st);
  TravPanel *dT = nullptr, *dS = nullptr;
  BTK_CUDA(A.alloc(&dT, ht.size()));
  BTK_CUDA(cudaMemcpyAsync(dT, ht.data(), sizeof(TravPanel) * ht.size(), cudaMemcpyHostToDevice, st));
  if (same) {
    dS = dT;
  } else {
    BTK_CUDA(A.alloc(&dS, hs.size()));
    BTK_CUDA(cudaMemcpyAsync(dS, hs.data(), sizeof(TravPanel) * hs.size(), cudaMemcpyHostToDevice, st));
  }
  // Generation 0: the root pair.
  int F = 1;
  int *ft = nullptr, *fs = nullptr;
  BTK_CUDA(A.alloc(&ft, 1));
  BTK_CUDA(A.alloc(&fs, 1));
  BTK_CUDA(cudaMemsetAsync(ft, 0, sizeof(int), st));
  BTK_CUDA(cudaMemsetAsync(fs, 0, sizeof(int), st));
  std::vector<btk_interact_pair> host_list;
  const double theta = cfg->fmm_theta;
  const int thresh = cfg->fmm_cluster_thresh;
  int generation = 0;
  while (F > 0) {
    BTK_CHECK(++generation < 4096, BTK_ERR_INTERNAL, "dual_tree_traversal_device: traversal does not terminate");
    int *act = nullptr, *ni = nullptr, *nc = nullptr, *pi = nullptr, *pc = nullptr;
    BTK_CUDA(A.alloc(&act, (size_t)F));
    BTK_CUDA(A.alloc(&ni, (size_t)F));
    BTK_CUDA(A.alloc(&nc, (size_t)F));
    BTK_CUDA(A.alloc(&pi, (size_t)F));
    BTK_CUDA(A.alloc(&pc, (size_t)F));
    const int blocks = (F + 255) / 256;
    k_trav_eval<D><<<blocks, 256, 0, st>>>(F, ft, fs, dT, dS, theta, thresh, act, ni, nc);
    count_launch();
    BTK_CUDA(cudaGetLastError());
    BTK_TRY(exclusive_scan(ni, pi, F, A, st));
    BTK_TRY(exclusive_scan(nc, pc, F, A, st));
    int last[4];  // exclusive prefix and own count of the last pair, for both scans
    BTK_CUDA(cudaMemcpyAsync(&last[0], pi + F - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    BTK_CUDA(cudaMemcpyAsync(&last[1], ni + F - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    BTK_CUDA(cudaMemcpyAsync(&last[2], pc + F - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    BTK_CUDA(cudaMemcpyAsync(&last[3], nc + F - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    BTK_CUDA(cudaStreamSynchronize(st));
    const int n_new_int = last[0] + last[1], n_next = last[2] + last[3];
    btk_interact_pair* dl = nullptr;
    int *nt = nullptr, *ns = nullptr;
    BTK_CUDA(A.alloc(&dl, (size_t)n_new_int));
    BTK_CUDA(A.alloc(&nt, (size_t)n_next));
    BTK_CUDA(A.alloc(&ns, (size_t)n_next));
    k_trav_emit<D><<<blocks, 256, 0, st>>>(F, ft, fs, dT, dS, act, pi, pc, dl, nt, ns);
    count_launch();
    BTK_CUDA(cudaGetLastError());
    if (n_new_int > 0) {
      const size_t old = host_list.size();
      host_list.resize(old + n_new_int);
      BTK_CUDA(cudaMemcpyAsync(host_list.data() + old, dl, sizeof(btk_interact_pair) * n_new_int,
                               cudaMemcpyDeviceToHost, st));
    }
    ft = nt;
    fs = ns;
    F = n_next;
  }
  BTK_CUDA(cudaStreamSynchronize(st));
  int counts[4] = {0, 0, 0, 0};
  for (const btk_interact_pair& p : host_list) counts[p.interact_type]++;
  cfg->fmm_interaction_count = (int)host_list.size();
  cfg->fmm_pp_count = counts[0];
  cfg->fmm_pc_count = counts[1];
  cfg->fmm_cp_count = counts[2];
  cfg->fmm_cc_count = counts[3];
  btk_interact_pair* out =
      (btk_interact_pair*)std::malloc(sizeof(btk_interact_pair) * (host_list.size() ? host_list.size() : 1));
  BTK_CHECK(out, BTK_ERR_OUT_OF_MEMORY, "dual_tree_traversal_device: host allocation failed");
  if (!host_list.empty()) std::memcpy(out, host_list.data(), sizeof(btk_interact_pair) * host_list.size());
  *list_out = out;
  return BTK_OK;
}

}  // namespace
}  // namespace btk

using namespace btk;

extern "C" {

btk_status btk_dual_tree_traversal_2d_device(btk_run_config* cfg, const btk_panel_2d* panels_target,
                                             int target_panel_count, const btk_panel_2d* panels_source,
                                             int source_panel_count, btk_interact_pair** interaction_list,
                                             btk_stream_t stream) {
  return traverse_device<2>(cfg, panels_target, target_panel_count, panels_source, source_panel_count,
                            interaction_list, (cudaStream_t)stream);
}

btk_status btk_dual_tree_traversal_3d_device(btk_run_config* cfg, const btk_panel_3d* panels_target,
                                             int target_panel_count, const btk_panel_3d* panels_source,
                                             int source_panel_count, btk_interact_pair** interaction_list,
                                             btk_stream_t stream) {
  return traverse_device<3>(cfg, panels_target, target_panel_count, panels_source, source_panel_count,
                            interaction_list, (cudaStream_t)stream);
}

}  // extern "C"
