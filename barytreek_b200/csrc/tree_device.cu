// Tree construction with the point work on the device, producing exactly the
// tree of btk_tree_construction_2d/3d (src/tree_construction.cpp:5-306).
//
// The reference refines panels breadth-first: a panel with more than
// fmm_cluster_thresh points gets 2^dim children (bisection of its box at the
// midpoint, in the reference's child order), its points are distributed by
// comparison with the midpoint, keeping their order, and children are
// numbered in the order their parents are refined. Done level by level, that
// is: at level l, every panel over the threshold, in index order, gets the
// next 2^dim ids. Here the O(panels) bookkeeping (boxes, midpoints, ids,
// radius) runs on the host with the same expressions as the host functions,
// and the O(points) work runs on the device:
//  * the root box: a min/max reduction that keeps, among equal extreme values,
//    the first in index order, and skips NaN, which is what the reference's
//    sequential std::min/std::max from max()/min() starting values yields
//    (signed zeros included);
//  * each level's point partition: a stable 2^dim-way split of every refined
//    panel's index range (per-chunk child counts, a scan per panel, then a
//    scatter that ranks points within a chunk with warp ballots).
// Points stay in original-index order inside every leaf, as in the
// reference's panel_points_inside rows.
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

#include "btk_internal.h"

namespace btk {
namespace {

constexpr int kTreeChunk = 4096;   // points per partition work unit
constexpr int kTreeThreads = 256;
constexpr int kTreeWarps = kTreeThreads / 32;

struct TreeChunk {
  int split;  // index of the refined panel among this level's refined panels
  int start;  // first position of the chunk in the permutation
  int len;
};

// Child of a point relative to the midpoint (tree_construction.cpp:81-93 for
// 2-D, :240-268 for 3-D): ties go to the lower half.
template <int D>
__device__ __forceinline__ int which_child_dev(double x, double y, double z, const double* mid) {
  int q = (x > mid[0]) ? ((y > mid[1]) ? 0 : 3) : ((y > mid[1]) ? 1 : 2);
  if (D == 3 && !(z > mid[2])) q += 4;
  return q;
}

// Extremes with their index: (value, index), first index among equal values.
struct Ext {
  double v;
  long long i;  // -1: none
};
__device__ __forceinline__ Ext better_min(Ext a, Ext b) {
  if (b.i < 0) return a;
  if (a.i < 0) return b;
  if (b.v < a.v || (b.v == a.v && b.i < a.i)) return b;
  return a;
}
__device__ __forceinline__ Ext better_max(Ext a, Ext b) {
  if (b.i < 0) return a;
  if (a.i < 0) return b;
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;
  return a;
}

// Per-block extremes of one coordinate array; out[2 * block] = min, [+1] = max.
__global__ void k_extremes(const double* __restrict__ v, int n, Ext* out) {
  Ext mn{0.0, -1}, mx{0.0, -1};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double x = v[i];
    if (x != x) continue;  // NaN never wins a comparison
    mn = better_min(mn, Ext{x, i});
    mx = better_max(mx, Ext{x, i});
  }
  __shared__ Ext smn[kTreeThreads], smx[kTreeThreads];
  smn[threadIdx.x] = mn;
  smx[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      smn[threadIdx.x] = better_min(smn[threadIdx.x], smn[threadIdx.x + s]);
      smx[threadIdx.x] = better_max(smx[threadIdx.x], smx[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = smn[0];
    out[2 * blockIdx.x + 1] = smx[0];
  }
}

// Second pass over the per-block results (one block).
__global__ void k_extremes_final(const Ext* in, int blocks, Ext* out) {
  __shared__ Ext smn[kTreeThreads], smx[kTreeThreads];
  Ext mn{0.0, -1}, mx{0.0, -1};
  for (int b = threadIdx.x; b < blocks; b += blockDim.x) {
    mn = better_min(mn, in[2 * b]);
    mx = better_max(mx, in[2 * b + 1]);
  }
  smn[threadIdx.x] = mn;
  smx[threadIdx.x] = mx;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      smn[threadIdx.x] = better_min(smn[threadIdx.x], smn[threadIdx.x + s]);
      smx[threadIdx.x] = better_max(smx[threadIdx.x], smx[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = smn[0];
    out[1] = smx[0];
  }
}

__global__ void k_iota(int* a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

// Child counts per chunk.
template <int D>
__global__ void __launch_bounds__(kTreeThreads) k_part_count(const TreeChunk* chunks, const double* mids,
                                                             const int* perm, const double* x, const double* y,
                                                             const double* z, int* chunk_counts) {
  __shared__ int cnt[8];
  if (threadIdx.x < 8) cnt[threadIdx.x] = 0;
  __syncthreads();
  const TreeChunk ch = chunks[blockIdx.x];
  const double* mid = mids + 3 * ch.split;
  for (int k = threadIdx.x; k < ch.len; k += blockDim.x) {
    const int i = perm[ch.start + k];
    atomicAdd(&cnt[which_child_dev<D>(x[i], y[i], D == 3 ? z[i] : 0.0, mid)], 1);
  }
  __syncthreads();
  if (threadIdx.x < 8) chunk_counts[8 * blockIdx.x + threadIdx.x] = cnt[threadIdx.x];
}

// Per refined panel: child totals, each child's first position, and every
// chunk's first position per child (children laid out in child order).
__global__ void k_part_scan(int n_split, const int* split_begin, const int* chunk_first, const int* chunk_counts,
                            int* chunk_off, int* split_counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_split) return;
  int tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int k = chunk_first[s]; k < chunk_first[s + 1]; ++k)
    for (int c = 0; c < 8; ++c) tot[c] += chunk_counts[8 * k + c];
  int run[8];
  int base = split_begin[s];
  for (int c = 0; c < 8; ++c) {
    run[c] = base;
    base += tot[c];
    split_counts[8 * s + c] = tot[c];
  }
  for (int k = chunk_first[s]; k < chunk_first[s + 1]; ++k)
    for (int c = 0; c < 8; ++c) {
      chunk_off[8 * k + c] = run[c];
      run[c] += chunk_counts[8 * k + c];
    }
}

// Stable scatter of each chunk's points to their children's ranges.
template <int D>
__global__ void __launch_bounds__(kTreeThreads) k_part_scatter(const TreeChunk* chunks, const double* mids,
                                                               const int* chunk_off, const int* perm, const double* x,
                                                               const double* y, const double* z, int* out) {
  __shared__ int wcnt[kTreeWarps][8];
  __shared__ int run[8];
  const TreeChunk ch = chunks[blockIdx.x];
  const double* mid = mids + 3 * ch.split;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x < 8) run[threadIdx.x] = chunk_off[8 * blockIdx.x + threadIdx.x];
  __syncthreads();
  for (int b0 = 0; b0 < ch.len; b0 += blockDim.x) {
    const int k = b0 + threadIdx.x;
    const bool valid = k < ch.len;
    int i = 0, c = -1;
    if (valid) {
      i = perm[ch.start + k];
      c = which_child_dev<D>(x[i], y[i], D == 3 ? z[i] : 0.0, mid);
    }
    const unsigned lt = (1u << lane) - 1u;
    int rank = 0;
#pragma unroll
    for (int cc = 0; cc < 8; ++cc) {
      const unsigned m = __ballot_sync(0xffffffffu, c == cc);
      if (c == cc) rank = __popc(m & lt);
      if (lane == 0) wcnt[warp][cc] = __popc(m);
    }
    __syncthreads();
    if (valid) {
      int off = 0;
      for (int w = 0; w < warp; ++w) off += wcnt[w][c];
      out[run[c] + off + rank] = i;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
      int t = 0;
      for (int w = 0; w < kTreeWarps; ++w) t += wcnt[w][threadIdx.x];
      run[threadIdx.x] += t;
    }
    __syncthreads();
  }
}

__global__ void k_part_copy(const TreeChunk* chunks, const int* src, int* dst) {
  const TreeChunk ch = chunks[blockIdx.x];
  for (int k = threadIdx.x; k < ch.len; k += blockDim.x) dst[ch.start + k] = src[ch.start + k];
}

// Leaves in panel order: their points (ascending original index) into
// leaf_order, and each point's leaf into leaf_of.
__global__ void k_leaf_rows(const int* leaf_id, const int* leaf_perm_begin, const int* leaf_out_begin,
                            const int* leaf_count, const int* perm, int* leaf_order, int* leaf_of) {
  const int L = blockIdx.x;
  const int pb = leaf_perm_begin[L], ob = leaf_out_begin[L], cnt = leaf_count[L], id = leaf_id[L];
  for (int k = threadIdx.x; k < cnt; k += blockDim.x) {
    const int i = perm[pb + k];
    if (leaf_order) leaf_order[ob + k] = i;
    leaf_of[i] = id;
  }
}

// ---- host side ----------------------------------------------------------
template <int D> struct DevPanelT;
template <> struct DevPanelT<2> { using type = btk_panel_2d; };
template <> struct DevPanelT<3> { using type = btk_panel_3d; };

inline int* child_slot_d(btk_panel_2d& p, int c) { return &p.child1 + c; }
inline int* child_slot_d(btk_panel_3d& p, int c) { return &p.child1 + c; }
inline void set_box_d(btk_panel_2d& p, const double* lo, const double* hi) {
  p.min_x = lo[0]; p.max_x = hi[0]; p.min_y = lo[1]; p.max_y = hi[1];
}
inline void set_box_d(btk_panel_3d& p, const double* lo, const double* hi) {
  p.min_x = lo[0]; p.max_x = hi[0]; p.min_y = lo[1]; p.max_y = hi[1]; p.min_z = lo[2]; p.max_z = hi[2];
}
inline void get_box_d(const btk_panel_2d& p, double* lo, double* hi) {
  lo[0] = p.min_x; hi[0] = p.max_x; lo[1] = p.min_y; hi[1] = p.max_y;
}
inline void get_box_d(const btk_panel_3d& p, double* lo, double* hi) {
  lo[0] = p.min_x; hi[0] = p.max_x; lo[1] = p.min_y; hi[1] = p.max_y; lo[2] = p.min_z; hi[2] = p.max_z;
}
template <class P>
P fresh_panel_d() {
  P p;
  std::memset(&p, 0, sizeof(P));
  p.parent_id = -1;
  const int nc = sizeof(P) == sizeof(btk_panel_2d) ? 4 : 8;
  for (int c = 0; c < nc; ++c) *child_slot_d(p, c) = -1;
  p.is_leaf = true;
  return p;
}
// Child boxes in the reference's child order: upper/lower z halves, each
// (hi x, hi y), (lo x, hi y), (lo x, lo y), (hi x, lo y).
template <int D>
void child_box_d(int c, const double* lo, const double* mid, const double* hi, double* clo, double* chi) {
  static const int hx[4] = {1, 0, 0, 1}, hy[4] = {1, 1, 0, 0};
  const int q = c & 3;
  clo[0] = hx[q] ? mid[0] : lo[0]; chi[0] = hx[q] ? hi[0] : mid[0];
  clo[1] = hy[q] ? mid[1] : lo[1]; chi[1] = hy[q] ? hi[1] : mid[1];
  if (D == 3) {
    const bool upper = c < 4;
    clo[2] = upper ? mid[2] : lo[2];
    chi[2] = upper ? hi[2] : mid[2];
  }
}

// Device buffers of one construction, freed on every exit path.
struct TreeScratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit TreeScratch(cudaStream_t s) : st(s) {}
  ~TreeScratch() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
  template <class T>
  cudaError_t alloc(T** p, size_t n) {
    cudaError_t e = cudaMallocAsync((void**)p, sizeof(T) * std::max<size_t>(n, 1), st);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

template <int D>
btk_status build_tree_device(const btk_run_config* cfg, btk_tree_info* info, const double* const* xyz, int n,
                             typename DevPanelT<D>::type** panels_out, int* leaf_of, int* leaf_order,
                             cudaStream_t st) {
  using P = typename DevPanelT<D>::type;
  constexpr int NC = 1 << D;
  BTK_CHECK(cfg && info && panels_out && (n == 0 || leaf_of), BTK_ERR_INVALID_ARGUMENT,
            "tree_construction_device: null argument");
  BTK_CHECK(n >= 0, BTK_ERR_INVALID_ARGUMENT, "tree_construction_device: negative point count");
  for (int d = 0; d < D; ++d)
    BTK_CHECK(n == 0 || xyz[d], BTK_ERR_INVALID_ARGUMENT, "tree_construction_device: null coordinates");
  const int thresh = cfg->fmm_cluster_thresh;
  BTK_CHECK(thresh > 0, BTK_ERR_INVALID_ARGUMENT, "tree_construction_device: fmm_cluster_thresh must be positive");
  const double* X = xyz[0];
  const double* Y = xyz[1];
  const double* Z = D == 3 ? xyz[2] : nullptr;
  TreeScratch S(st);

  // Root box (tree_construction.cpp:145-167): starting values max() and
  // min() (the smallest positive double), as the reference has them.
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int d = 0; d < D; ++d) {
    lo[d] = std::numeric_limits<double>::max();
    hi[d] = std::numeric_limits<double>::min();
  }
  if (n > 0) {
    const int blocks = std::min(1024, (n + kTreeThreads - 1) / kTreeThreads);
    Ext *part = nullptr, *res = nullptr;
    BTK_CUDA(S.alloc(&part, 2 * (size_t)blocks));
    BTK_CUDA(S.alloc(&res, 2 * (size_t)D));
    for (int d = 0; d < D; ++d) {
      k_extremes<<<blocks, kTreeThreads, 0, st>>>(xyz[d], n, part);
      k_extremes_final<<<1, kTreeThreads, 0, st>>>(part, blocks, res + 2 * d);
      count_launch(2);
    }
    BTK_CUDA(cudaGetLastError());
    Ext h[6];
    BTK_CUDA(cudaMemcpyAsync(h, res, sizeof(Ext) * 2 * D, cudaMemcpyDeviceToHost, st));
    BTK_CUDA(cudaStreamSynchronize(st));
    for (int d = 0; d < D; ++d) {
      if (h[2 * d].i >= 0 && h[2 * d].v < lo[d]) lo[d] = h[2 * d].v;
      if (h[2 * d + 1].i >= 0 && hi[d] < h[2 * d + 1].v) hi[d] = h[2 * d + 1].v;
    }
  }
  std::vector<P> panels(1, fresh_panel_d<P>());
  std::vector<int> begin(1, 0), count(1, n);
  panels[0].id = 0;
  panels[0].level = 0;
  panels[0].point_count = n;
  set_box_d(panels[0], lo, hi);

  int *perm = nullptr, *tmp = nullptr;
  BTK_CUDA(S.alloc(&perm, (size_t)n));
  BTK_CUDA(S.alloc(&tmp, (size_t)n));
  if (n > 0) {
    k_iota<<<(n + 255) / 256, 256, 0, st>>>(perm, n);
    count_launch();
    BTK_CUDA(cudaGetLastError());
  }

  size_t lev_begin = 0, lev_end = 1;
  while (lev_begin < lev_end) {
    std::vector<int> split;  // refined panels of this level, in index order
    for (size_t i = lev_begin; i < lev_end; ++i)
      if (panels[i].point_count > thresh && panels[i].is_leaf) split.push_back((int)i);
    if (split.empty()) break;
    const int ns = (int)split.size();
    std::vector<double> mids(3 * (size_t)ns, 0.0);
    std::vector<int> split_begin(ns), chunk_first(ns + 1, 0);
    std::vector<TreeChunk> chunks;
    for (int s = 0; s < ns; ++s) {
      const int i = split[s];
      BTK_CHECK(panels[i].level < 60, BTK_ERR_INVALID_ARGUMENT,
                "tree_construction: more than fmm_cluster_thresh coincident points (refinement does not terminate)");
      double plo[3], phi[3];
      get_box_d(panels[i], plo, phi);
      for (int d = 0; d < D; ++d) mids[3 * s + d] = 0.5 * (plo[d] + phi[d]);
      split_begin[s] = begin[i];
      chunk_first[s] = (int)chunks.size();
      for (int a = 0; a < count[i]; a += kTreeChunk)
        chunks.push_back(TreeChunk{s, begin[i] + a, std::min(kTreeChunk, count[i] - a)});
    }
    chunk_first[ns] = (int)chunks.size();
    const int nch = (int)chunks.size();
    TreeChunk* d_chunks = nullptr;
    double* d_mids = nullptr;
    int *d_split_begin = nullptr, *d_chunk_first = nullptr, *d_cc = nullptr, *d_off = nullptr, *d_sc = nullptr;
    BTK_CUDA(S.alloc(&d_chunks, (size_t)nch));
    BTK_CUDA(S.alloc(&d_mids, mids.size()));
    BTK_CUDA(S.alloc(&d_split_begin, (size_t)ns));
    BTK_CUDA(S.alloc(&d_chunk_first, (size_t)ns + 1));
    BTK_CUDA(S.alloc(&d_cc, 8 * (size_t)nch));
    BTK_CUDA(S.alloc(&d_off, 8 * (size_t)nch));
    BTK_CUDA(S.alloc(&d_sc, 8 * (size_t)ns));
    BTK_CUDA(cudaMemcpyAsync(d_chunks, chunks.data(), sizeof(TreeChunk) * nch, cudaMemcpyHostToDevice, st));
    BTK_CUDA(cudaMemcpyAsync(d_mids, mids.data(), sizeof(double) * mids.size(), cudaMemcpyHostToDevice, st));
    BTK_CUDA(cudaMemcpyAsync(d_split_begin, split_begin.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, st));
    BTK_CUDA(cudaMemcpyAsync(d_chunk_first, chunk_first.data(), sizeof(int) * (ns + 1), cudaMemcpyHostToDevice, st));
    k_part_count<D><<<nch, kTreeThreads, 0, st>>>(d_chunks, d_mids, perm, X, Y, Z, d_cc);
    k_part_scan<<<(ns + 127) / 128, 128, 0, st>>>(ns, d_split_begin, d_chunk_first, d_cc, d_off, d_sc);
    k_part_scatter<D><<<nch, kTreeThreads, 0, st>>>(d_chunks, d_mids, d_off, perm, X, Y, Z, tmp);
    k_part_copy<<<nch, kTreeThreads, 0, st>>>(d_chunks, tmp, perm);
    count_launch(4);
    BTK_CUDA(cudaGetLastError());
    std::vector<int> sc(8 * (size_t)ns);
    BTK_CUDA(cudaMemcpyAsync(sc.data(), d_sc, sizeof(int) * sc.size(), cudaMemcpyDeviceToHost, st));
    BTK_CUDA(cudaStreamSynchronize(st));
    // Children, numbered in the order their parents are refined.
    for (int s = 0; s < ns; ++s) {
      const int i = split[s];
      panels[i].is_leaf = false;
      const int base = (int)panels.size();
      const int lev = panels[i].level;
      double plo[3], phi[3];
      get_box_d(panels[i], plo, phi);
      int acc = begin[i];
      for (int c = 0; c < NC; ++c) {
        P ch = fresh_panel_d<P>();
        double clo[3], chi[3];
        child_box_d<D>(c, plo, &mids[3 * s], phi, clo, chi);
        set_box_d(ch, clo, chi);
        ch.parent_id = i;
        ch.level = lev + 1;
        ch.id = base + c;
        ch.point_count = sc[8 * s + c];
        *child_slot_d(panels[i], c) = ch.id;
        panels.push_back(ch);
        begin.push_back(acc);
        count.push_back(sc[8 * s + c]);
        acc += sc[8 * s + c];
      }
    }
    lev_begin = lev_end;
    lev_end = panels.size();
  }

  // Leaves in panel order: point rows and point -> leaf.
  const int P_count = (int)panels.size();
  std::vector<int> lid, lpb, lob, lcnt;
  int acc = 0;
  for (int i = 0; i < P_count; ++i)
    if (panels[i].is_leaf && panels[i].point_count > 0) {
      lid.push_back(i);
      lpb.push_back(begin[i]);
      lob.push_back(acc);
      lcnt.push_back(panels[i].point_count);
      acc += panels[i].point_count;
    }
  if (!lid.empty()) {
    const int nl = (int)lid.size();
    int *d_lid = nullptr, *d_lpb = nullptr, *d_lob = nullptr, *d_lcnt = nullptr;
    BTK_CUDA(S.alloc(&d_lid, (size_t)nl));
    BTK_CUDA(S.alloc(&d_lpb, (size_t)nl));
    BTK_CUDA(S.alloc(&d_lob, (size_t)nl));
    BTK_CUDA(S.alloc(&d_lcnt, (size_t)nl));
    BTK_CUDA(cudaMemcpyAsync(d_lid, lid.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, st));
    BTK_CUDA(cudaMemcpyAsync(d_lpb, lpb.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, st));
    BTK_CUDA(cudaMemcpyAsync(d_lob, lob.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, st));
    BTK_CUDA(cudaMemcpyAsync(d_lcnt, lcnt.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, st));
    k_leaf_rows<<<nl, kTreeThreads, 0, st>>>(d_lid, d_lpb, d_lob, d_lcnt, perm, leaf_order, leaf_of);
    count_launch();
    BTK_CUDA(cudaGetLastError());
  }
  // Finalise like tree_construction.cpp:278-305: radius, level_start.
  const int levels = panels.back().level + 1;
  int* ls = (int*)std::malloc(sizeof(int) * (levels + 1));
  P* out = (P*)std::malloc(sizeof(P) * P_count);
  if (!ls || !out) {
    std::free(ls);
    std::free(out);
    return set_error(BTK_ERR_OUT_OF_MEMORY, "tree_construction_device: host allocation failed");
  }
  ls[0] = 0;
  int target_level = 1;
  for (int i = 0; i < P_count; ++i) {
    P& p = panels[i];
    double plo[3], phi[3];
    get_box_d(p, plo, phi);
    const double x_ex = phi[0] - plo[0], y_ex = phi[1] - plo[1];
    if (D == 2) {
      p.radius = 0.5 * std::sqrt(x_ex * x_ex + y_ex * y_ex);
    } else {
      const double z_ex = phi[2] - plo[2];
      p.radius = 0.5 * std::sqrt(x_ex * x_ex + y_ex * y_ex + z_ex * z_ex);
    }
    if (p.level == target_level) {
      ls[target_level] = i;
      target_level += 1;
    }
    out[i] = p;
  }
  ls[levels] = P_count;
  BTK_CUDA(cudaStreamSynchronize(st));  // the leaf rows are written before returning
  info->panel_count = P_count;
  info->levels = levels;
  info->level_start = ls;
  *panels_out = out;
  return BTK_OK;
}

}  // namespace
}  // namespace btk

using namespace btk;

extern "C" {

btk_status btk_tree_construction_2d_device(const btk_run_config* cfg, btk_tree_info* info, const double* xcos,
                                           const double* ycos, int point_count, btk_panel_2d** panels,
                                           int* point_leaf_panel, int* leaf_order, btk_stream_t stream) {
  const double* xyz[3] = {xcos, ycos, nullptr};
  return build_tree_device<2>(cfg, info, xyz, point_count, panels, point_leaf_panel, leaf_order,
                              (cudaStream_t)stream);
}

btk_status btk_tree_construction_3d_device(const btk_run_config* cfg, btk_tree_info* info, const double* xcos,
                                           const double* ycos, const double* zcos, int point_count,
                                           btk_panel_3d** panels, int* point_leaf_panel, int* leaf_order,
                                           btk_stream_t stream) {
  const double* xyz[3] = {xcos, ycos, zcos};
  return build_tree_device<3>(cfg, info, xyz, point_count, panels, point_leaf_panel, leaf_order,
                              (cudaStream_t)stream);
}

}  // extern "C"
