// CC interactions as shared kernel matrices (an optional plan mode).
//
// The reference evaluates every cluster-cluster pair on its own
// (src/fmm_interactions/poisson_fmm_impl.hpp:376-442, poisson_vel_fmm_impl.hpp):
// Phi_T(j) += sum_k G(t_j, s_k) Q_S(k) over the ipc x ipc proxy points. The
// tree splits boxes at their midpoints (src/tree_construction.cpp:131-305), so
// all boxes of one level are translates of each other, and two pairs whose
// target and source levels and centre offset agree have the same proxy-point
// differences t_j - s_k: the same matrix G. Grouping the CC list by
// (target level, source level, lattice offset) turns each group into one
// matrix product, Phi[:, p] += G Q[:, p] over the group's pairs p, where G is
// evaluated once per block and reused by up to 32 pairs (2 FP64 flops per pair
// and kernel entry instead of a full kernel evaluation).
//
// G is built from the group's first pair's proxy coordinates (the same FP64
// differences the pairwise kernel forms for that pair); for the other pairs of
// the group the coordinates differ only in the last bits of the box bounds'
// midpoint rounding. Sums run in FP64 in both precisions.
//
// Block: kCcJ target proxies (one per thread) x PT pairs of one task. A thread
// evaluates G[j][k] for its target j and every source proxy k itself, in
// registers, and applies it to its PT pairs (NC x PT FP64 accumulators), so G
// never passes through shared memory; only the pairs' modified charges Q do,
// one x-node slab of source proxies (m^(dim-1) of them) at a time, read by
// every thread as broadcasts. Each G entry is evaluated once per block and
// reused PT times (PT = 16 for vector kinds, 32 for the potential). Tasks with
// fewer pairs run at PT/2 or PT/4. Results are added to the proxy target
// weights with FP64 atomics (pairs of one target panel sit in many groups).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <tuple>
#include <vector>

#include "device_math.cuh"
#include "kernels.cuh"

namespace btk {

namespace {

constexpr int kCcJ = 128;  // target proxies (threads) per block

template <int DIM, int KIND>
struct CcTraits {
  static constexpr int NC = KIND == BTK_KIND_POT ? 1 : (KIND == BTK_KIND_VEL ? 3 : 1 + DIM);
  static constexpr int PT = NC == 1 ? 32 : 16;  // pairs per task
};

// Dynamic shared memory: the per-axis node differences (padded to an even
// count, so what follows is 16-byte aligned), one slab of Q (FP64, or FP32 in
// the FP32 variant) and, in the FP32 variant, the FP64 accumulators
// [NC * PT][kCcJ] the per-slab FP32 partial sums are folded into.
__host__ __device__ constexpr size_t cc_diff_doubles(int dim, int m) { return ((size_t)dim * m * m + 1) & ~(size_t)1; }
__host__ __device__ constexpr size_t cc_slab(int dim, int m) { return dim == 3 ? (size_t)m * m : (size_t)m; }
__host__ __device__ constexpr size_t cc_q_bytes(int dim, int m, int pt, bool f32) {
  return ((cc_slab(dim, m) * pt * (f32 ? sizeof(float) : sizeof(double))) + 15) & ~(size_t)15;
}
constexpr size_t cc_smem_bytes(int dim, int nc, int m, int pt, bool f32) {
  return sizeof(double) * cc_diff_doubles(dim, m) + cc_q_bytes(dim, m, pt, f32) +
         (f32 ? sizeof(double) * nc * pt * kCcJ : 0);
}

// Kernel entries without the constant factor, as the pairwise FP64 kernel sums
// them (weight 1): POT 3-D 1/R, 2-D log R^2; VEL (t-s)/R^2; FIELD 3-D 1/R and
// (t-s)/R^3, 2-D log R^2 and (t-s)/R^2; R^2 = |t-s|^2 + eps^2.
template <int DIM, int KIND, bool GUARD>
__device__ __forceinline__ void cc_entry(double dx, double dy, double dz, double eps2, double* g) {
  if (DIM == 2) {
    const double r2 = fma(dx, dx, fma(dy, dy, eps2));
    g[0] = log(r2);
    if (KIND == BTK_KIND_FIELD) {
      const double rc = GUARD ? rcp_fp64_pos_guarded(r2) : rcp_fp64_pos(r2);
      g[1] = dx * rc;
      g[2] = dy * rc;
    }
  } else {
    const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
    if (KIND == BTK_KIND_VEL) {
      const double rc = GUARD ? rcp_fp64_pos_guarded(r2) : rcp_fp64_pos(r2);
      g[0] = dx * rc;
      g[1] = dy * rc;
      g[2] = dz * rc;
    } else {
      const double ri = GUARD ? rsqrt_fp64_guarded(r2) : rsqrt_fp64(r2);
      g[0] = ri;
      if (KIND == BTK_KIND_FIELD) {
        const double r3 = ri * (ri * ri);
        g[1] = dx * r3;
        g[2] = dy * r3;
        g[3] = dz * r3;
      }
    }
  }
}

// The same entries in FP32 with the hardware approximations the
// mixed-precision pairwise kernel uses (differences formed in FP64, rounded).
template <int DIM, int KIND>
__device__ __forceinline__ void cc_entry_f32(float dx, float dy, float dz, float eps2, float* g) {
  if (DIM == 2) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, eps2));
    g[0] = __logf(r2);
    if (KIND == BTK_KIND_FIELD) {
      const float rc = rcp_fp32(r2);
      g[1] = dx * rc;
      g[2] = dy * rc;
    }
  } else {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
    if (KIND == BTK_KIND_VEL) {
      const float rc = rcp_fp32(r2);
      g[0] = dx * rc;
      g[1] = dy * rc;
      g[2] = dz * rc;
    } else {
      const float ri = rsqrt_fp32(r2);
      g[0] = ri;
      if (KIND == BTK_KIND_FIELD) {
        const float r3 = ri * (ri * ri);
        g[1] = dx * r3;
        g[2] = dy * r3;
        g[3] = dz * r3;
      }
    }
  }
}

// One slab (source x node a2) of a thread's products: FP64 accumulators, or
// (F32) FP32 partial sums returned for folding.
template <int DIM, int KIND, int PT, bool GUARD, bool F32, class Acc>
__device__ __forceinline__ void cc_slab_products(const double* sD, const void* sQv, int m, int aj, int bj, int cj,
                                                 int a2, double eps2, Acc (*acc)[PT]) {
  constexpr int NC = CcTraits<DIM, KIND>::NC;
  const int mm = m * m;
  const double dx = sD[aj * m + a2];
  const int nb = DIM == 3 ? m : 1;
  for (int b2 = 0; b2 < nb; ++b2) {
    const double dy3 = DIM == 3 ? sD[mm + bj * m + b2] : 0.0;
#pragma unroll 2
    for (int c2 = 0; c2 < m; ++c2) {
      // 3-D: source node (a2, b2, c2); 2-D: (a2, c2)
      const double dy = DIM == 3 ? dy3 : sD[mm + bj * m + c2];
      const double dz = DIM == 3 ? sD[2 * mm + cj * m + c2] : 0.0;
      const int kk = b2 * m + c2;
      if constexpr (F32) {
        float g[NC];
        cc_entry_f32<DIM, KIND>((float)dx, (float)dy, (float)dz, (float)eps2, g);
        const float* q = static_cast<const float*>(sQv) + kk * PT;
#pragma unroll
        for (int pp = 0; pp < PT; pp += 4) {
          const float4 qv = *reinterpret_cast<const float4*>(q + pp);
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            acc[c][pp] = fmaf(g[c], qv.x, acc[c][pp]);
            acc[c][pp + 1] = fmaf(g[c], qv.y, acc[c][pp + 1]);
            acc[c][pp + 2] = fmaf(g[c], qv.z, acc[c][pp + 2]);
            acc[c][pp + 3] = fmaf(g[c], qv.w, acc[c][pp + 3]);
          }
        }
      } else {
        double g[NC];
        cc_entry<DIM, KIND, GUARD>(dx, dy, dz, eps2, g);
        const double* q = static_cast<const double*>(sQv) + kk * PT;
#pragma unroll
        for (int pp = 0; pp < PT; pp += 2) {
          const double2 qv = *reinterpret_cast<const double2*>(q + pp);
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            acc[c][pp] = fma(g[c], qv.x, acc[c][pp]);
            acc[c][pp + 1] = fma(g[c], qv.y, acc[c][pp + 1]);
          }
        }
      }
    }
  }
}

template <int DIM, int KIND, int PT, bool GUARD, bool F32>
__global__ void __launch_bounds__(kCcJ) k_cc_groups(CcParams p, int task0) {
  constexpr int NC = CcTraits<DIM, KIND>::NC;
  extern __shared__ __align__(16) double smem[];
  const int m = p.m, mm = m * m, ipc = p.ipc;
  const int slab = (int)cc_slab(DIM, m);  // source proxies per x node
  double* sD = smem;                       // [DIM][m][m]: target node a minus source node b, per axis
  void* sQ = smem + cc_diff_doubles(DIM, m);  // [slab][PT]: Q of the task's pairs for one x node
  double* sAcc = reinterpret_cast<double*>(reinterpret_cast<char*>(sQ) + cc_q_bytes(DIM, m, PT, F32));  // F32: [NC*PT][kCcJ]
  __shared__ int s_trow[PT], s_srow[PT];

  const CcTask task = p.tasks[task0 + blockIdx.x];
  const int tid = threadIdx.x;
  for (int e = tid; e < DIM * mm; e += kCcJ) {
    const int d = e / mm, a = (e / m) % m, b = e % m;
    sD[e] = p.nodes_t[(size_t)task.tp * kPanelNodes + d * kNodeStride + a] -
            p.nodes_s[(size_t)task.sp * kPanelNodes + d * kNodeStride + b];
  }
  if (tid < PT) {
    const bool ok = tid < task.p_count;
    const CcPair pr = p.pairs[task.p_begin + (ok ? tid : 0)];
    s_trow[tid] = pr.t_row;
    s_srow[tid] = ok ? pr.s_row : -1;
  }
  const int j = blockIdx.y * kCcJ + tid;
  const bool live = j < ipc;
  const bool warp_live = blockIdx.y * kCcJ + (tid & ~31) < ipc;  // warp-uniform
  const int jc = live ? j : ipc - 1;
  int aj, bj, cj = 0;
  if (DIM == 2) {
    aj = jc / m;
    bj = jc % m;
  } else {
    aj = jc / mm;
    bj = (jc / m) % m;
    cj = jc % m;
  }
  double acc[NC][F32 ? 1 : PT];
  if constexpr (F32) {
#pragma unroll
    for (int e = 0; e < NC * PT; ++e) sAcc[e * kCcJ + tid] = 0.0;
  } else {
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int q = 0; q < (F32 ? 1 : PT); ++q) acc[c][q] = 0.0;
  }

  for (int a2 = 0; a2 < m; ++a2) {
    __syncthreads();  // node differences and rows ready; previous slab consumed
    for (int e = tid; e < slab * PT; e += kCcJ) {
      const int kk = e % slab, pp = e / slab, row = s_srow[pp];
      const double v = row >= 0 ? p.psw[(size_t)row * ipc + (size_t)a2 * slab + kk] : 0.0;
      if constexpr (F32)
        static_cast<float*>(sQ)[kk * PT + pp] = (float)v;
      else
        static_cast<double*>(sQ)[kk * PT + pp] = v;
    }
    __syncthreads();
    if (!warp_live) continue;
    if constexpr (F32) {
      float part[NC][PT];
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int q = 0; q < PT; ++q) part[c][q] = 0.f;
      cc_slab_products<DIM, KIND, PT, GUARD, true>(sD, sQ, m, aj, bj, cj, a2, p.eps2, part);
#pragma unroll
      for (int c = 0; c < NC; ++c)
#pragma unroll
        for (int q = 0; q < PT; ++q) sAcc[(c * PT + q) * kCcJ + tid] += (double)part[c][q];
    } else {
      cc_slab_products<DIM, KIND, (F32 ? 1 : PT), GUARD, false>(sD, sQ, m, aj, bj, cj, a2, p.eps2, acc);
    }
  }
  if (!live) return;
#pragma unroll
  for (int pp = 0; pp < PT; ++pp) {
    if (pp >= task.p_count) break;
    const size_t row = (size_t)s_trow[pp] * ipc + j;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      const double v = F32 ? sAcc[(c * PT + pp) * kCcJ + tid] : acc[c][F32 ? 0 : pp];
      atomicAdd(p.ptw.p[c] + row, v * p.scale[c]);
    }
  }
}

template <int DIM, int KIND, int PT, bool GUARD, bool F32>
cudaError_t launch_cc_one(const CcParams& p, int t0, int t1, cudaStream_t s) {
  constexpr int NC = CcTraits<DIM, KIND>::NC;
  const size_t smem = cc_smem_bytes(DIM, NC, p.m, PT, F32);
  const dim3 grid(t1 - t0, (p.ipc + kCcJ - 1) / kCcJ);
  // The shared-memory opt-in is set once per kernel and device (for the
  // largest degree), at the first launch there.
  static std::atomic<uint64_t> opted{0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const uint64_t bit = 1ull << (dev & 63);
  if (!(opted.load(std::memory_order_acquire) & bit)) {
    e = cudaFuncSetAttribute(k_cc_groups<DIM, KIND, PT, GUARD, F32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)cc_smem_bytes(DIM, NC, kMaxNodes, PT, F32));
    if (e != cudaSuccess) return e;
    opted.fetch_or(bit, std::memory_order_release);
  }
  k_cc_groups<DIM, KIND, PT, GUARD, F32><<<grid, kCcJ, smem, s>>>(p, t0);
  count_launch();
  return cudaGetLastError();
}

template <int DIM, int KIND, int PT>
cudaError_t launch_cc_pt(bool guard, bool f32, const CcParams& p, int t0, int t1, cudaStream_t s) {
  if (t1 <= t0) return cudaSuccess;
  if (f32) return launch_cc_one<DIM, KIND, PT, false, true>(p, t0, t1, s);
  return guard ? launch_cc_one<DIM, KIND, PT, true, false>(p, t0, t1, s)
               : launch_cc_one<DIM, KIND, PT, false, false>(p, t0, t1, s);
}

// Tasks are sorted by pair count, largest first; bucket_end[0..2] end the
// runs with more than PT/2 pairs, more than PT/4, and the rest.
template <int DIM, int KIND>
cudaError_t launch_cc_kind(bool guard, bool f32, const CcParams& p, const int* bucket_end, cudaStream_t s) {
  constexpr int PT = CcTraits<DIM, KIND>::PT;
  cudaError_t e = launch_cc_pt<DIM, KIND, PT>(guard, f32, p, 0, bucket_end[0], s);
  if (e == cudaSuccess) e = launch_cc_pt<DIM, KIND, PT / 2>(guard, f32, p, bucket_end[0], bucket_end[1], s);
  if (e == cudaSuccess) e = launch_cc_pt<DIM, KIND, PT / 4>(guard, f32, p, bucket_end[1], bucket_end[2], s);
  return e;
}

// Lattice coordinates of a side's panel centres in units of the finest level's
// half width, or false when the tree is not a midpoint subdivision of one root
// box (a panel off the lattice or with the wrong width for its level).
bool lattice_coords(const HostTree& h, const PanelGeom& root, int finest, std::vector<long long>& out) {
  out.assign((size_t)h.panel_count * 3, 0);
  for (int i = 0; i < h.panel_count; ++i) {
    const int l = h.level[i];
    if (l < 0 || l > finest) return false;
    for (int d = 0; d < h.dim; ++d) {
      const double w = root.hi[d] - root.lo[d];
      if (w == 0.0) continue;  // flat axis: every box shares it
      const double unit = std::ldexp(w, -(finest + 1));
      const double c = 0.5 * (h.geom[i].lo[d] + h.geom[i].hi[d]);
      const double q = (c - root.lo[d]) / unit;
      const double qi = std::nearbyint(q);
      if (!(std::fabs(q - qi) <= 1e-6)) return false;
      const double wl = std::ldexp(w, -l), wi = h.geom[i].hi[d] - h.geom[i].lo[d];
      if (!(std::fabs(wi - wl) <= 1e-9 * w)) return false;
      out[(size_t)i * 3 + d] = (long long)qi;
    }
  }
  return true;
}

}  // namespace

int cc_pairs_per_task(int dim, int kind) {
  if (dim == 2) return kind == BTK_KIND_FIELD ? CcTraits<2, BTK_KIND_FIELD>::PT : CcTraits<2, BTK_KIND_POT>::PT;
  if (kind == BTK_KIND_FIELD) return CcTraits<3, BTK_KIND_FIELD>::PT;
  return kind == BTK_KIND_VEL ? CcTraits<3, BTK_KIND_VEL>::PT : CcTraits<3, BTK_KIND_POT>::PT;
}

cudaError_t launch_cc_groups(int dim, int kind, bool guard, bool f32, const CcParams& p, const int* bucket_end,
                             cudaStream_t s) {
  if (bucket_end[2] <= 0) return cudaSuccess;
  if (dim == 2)
    return kind == BTK_KIND_FIELD ? launch_cc_kind<2, BTK_KIND_FIELD>(guard, f32, p, bucket_end, s)
                                  : launch_cc_kind<2, BTK_KIND_POT>(guard, f32, p, bucket_end, s);
  if (kind == BTK_KIND_FIELD) return launch_cc_kind<3, BTK_KIND_FIELD>(guard, f32, p, bucket_end, s);
  if (kind == BTK_KIND_VEL) return launch_cc_kind<3, BTK_KIND_VEL>(guard, f32, p, bucket_end, s);
  return launch_cc_kind<3, BTK_KIND_POT>(guard, f32, p, bucket_end, s);
}

// Groups the CC list by (target level, source level, lattice offset of the box
// centres). Both trees must be midpoint subdivisions of the same single root
// box (one tree, or two trees over bitwise-equal root boxes); otherwise
// returns false and leaves the outputs empty. group_of[i] is pair i's group;
// groups are numbered in key order.
bool cc_group_pairs(const HostTree& T, const HostTree& S, const btk_interact_pair* cc, int n_cc,
                    std::vector<int>& group_of, int& n_groups) {
  group_of.clear();
  n_groups = 0;
  auto one_root = [](const HostTree& h) {
    return h.panel_count > 0 && h.levels >= 1 && h.level_start.size() >= 2 && h.level_start[0] == 0 &&
           h.level_start[1] == 1 && h.level[0] == 0;
  };
  if (n_cc <= 0 || !one_root(T) || !one_root(S) || T.dim != S.dim) return false;
  for (int d = 0; d < T.dim; ++d)
    if (T.geom[0].lo[d] != S.geom[0].lo[d] || T.geom[0].hi[d] != S.geom[0].hi[d]) return false;
  const int finest = std::max(T.levels, S.levels) - 1;
  if (finest > 60) return false;
  std::vector<long long> lt, ls;
  if (!lattice_coords(T, T.geom[0], finest, lt)) return false;
  if (&T == &S) {
    ls = lt;
  } else if (!lattice_coords(S, S.geom[0], finest, ls)) {
    return false;
  }
  using Key = std::tuple<int, int, long long, long long, long long>;
  std::vector<Key> key(n_cc);
  for (int i = 0; i < n_cc; ++i) {
    const int t = cc[i].target_panel, s = cc[i].source_panel;
    if (t < 0 || t >= T.panel_count || s < 0 || s >= S.panel_count) return false;
    key[i] = Key(T.level[t], S.level[s], lt[(size_t)t * 3] - ls[(size_t)s * 3], lt[(size_t)t * 3 + 1] - ls[(size_t)s * 3 + 1],
                 lt[(size_t)t * 3 + 2] - ls[(size_t)s * 3 + 2]);
  }
  std::vector<int> order(n_cc);
  for (int i = 0; i < n_cc; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return key[a] < key[b]; });
  group_of.assign(n_cc, -1);
  for (int r = 0; r < n_cc; ++r) {
    if (r == 0 || key[order[r]] != key[order[r - 1]]) ++n_groups;
    group_of[order[r]] = n_groups - 1;
  }
  return true;
}

// Tasks of at most pt pairs per group (groups in key order, pairs in list
// order), the group's first pair as the geometry of G; tasks sorted by pair
// count, largest first, with bucket_end[] closing the runs of more than pt/2
// pairs, more than pt/4, and the rest. pairs[] rows are panel indices (rows of
// the proxy weight arrays).
void cc_build_tasks(const btk_interact_pair* cc, int n_cc, const std::vector<int>& group_of, int n_groups, int pt,
                    std::vector<CcTask>& tasks, std::vector<CcPair>& pairs, int bucket_end[3]) {
  std::vector<int> head(n_groups + 1, 0);
  for (int i = 0; i < n_cc; ++i) head[group_of[i] + 1]++;
  for (int g = 0; g < n_groups; ++g) head[g + 1] += head[g];
  std::vector<int> pos(head.begin(), head.end() - 1), member(n_cc);
  for (int i = 0; i < n_cc; ++i) member[pos[group_of[i]]++] = i;
  pairs.resize(n_cc);
  tasks.clear();
  for (int g = 0; g < n_groups; ++g) {
    const int rep = member[head[g]];
    for (int b = head[g]; b < head[g + 1]; b += pt) {
      CcTask t;
      t.tp = cc[rep].target_panel;
      t.sp = cc[rep].source_panel;
      t.p_begin = b;
      t.p_count = std::min(pt, head[g + 1] - b);
      tasks.push_back(t);
    }
  }
  for (int r = 0; r < n_cc; ++r) pairs[r] = CcPair{cc[member[r]].target_panel, cc[member[r]].source_panel};
  std::stable_sort(tasks.begin(), tasks.end(), [](const CcTask& a, const CcTask& b) { return a.p_count > b.p_count; });
  const int n = (int)tasks.size();
  int k = 0;
  while (k < n && tasks[k].p_count > pt / 2) ++k;
  bucket_end[0] = k;
  while (k < n && tasks[k].p_count > pt / 4) ++k;
  bucket_end[1] = k;
  bucket_end[2] = n;
}

}  // namespace btk

extern "C" btk_status btk_cc_operator_groups(int dim, const void* panels_target, int n_target,
                                             const void* panels_source, int n_source,
                                             const btk_interact_pair* cc_list, int n_cc, int* group_of_pair,
                                             int* n_groups) {
  using namespace btk;
  BTK_CHECK(dim == 2 || dim == 3, BTK_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
  BTK_CHECK(panels_target && n_target > 0 && n_groups && (n_cc == 0 || (cc_list && group_of_pair)),
            BTK_ERR_INVALID_ARGUMENT, "btk_cc_operator_groups: null argument");
  HostTree T, S;
  BTK_CHECK(host_tree_from_panels_nolevels(dim, panels_target, n_target, T), BTK_ERR_INVALID_ARGUMENT,
            "target panels: levels are not in breadth-first order");
  const bool same = panels_source == nullptr || panels_source == panels_target;
  if (!same)
    BTK_CHECK(n_source > 0 && host_tree_from_panels_nolevels(dim, panels_source, n_source, S),
              BTK_ERR_INVALID_ARGUMENT, "source panels: levels are not in breadth-first order");
  std::vector<int> g;
  int ng = 0;
  cc_group_pairs(T, same ? T : S, cc_list, n_cc, g, ng);
  for (int i = 0; i < n_cc; ++i) group_of_pair[i] = ng > 0 ? g[i] : -1;
  *n_groups = ng;
  return BTK_OK;
}
