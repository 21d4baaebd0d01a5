// Per-pair interpolation degree (the learned-degree extension; no reference
// counterpart).
//
// The upward and downward passes run at the plan degree n. Every source
// cluster also gets its modified charges at each lower degree d by exact
// anterpolation, Q^d = (A_d x A_d x A_d) Q^n with A_d[a][i] = L^d_a(x^n_i)
// (the degree-d Lagrange basis at the degree-n nodes: exact because
// interpolation at n+1 points reproduces degree-d polynomials; the matrix is
// the same for every box since both node sets scale with the box). Target
// clusters collect CP/CC results at degree d in their own slots Phi^d, which
// are promoted exactly to degree n, Phi^n += (A_d^T x A_d^T x A_d^T) Phi^d,
// before the downward pass. Each (cluster, degree) pair owns a contiguous slot
// of (d+1)^dim proxies in the S4 / T4 arrays (slot tables built on the host).
//
// Work items: point-target items (PP + PC) keep their plan-time shape; only
// their PC entries are re-pointed at the chosen degree's slot. Every CP/CC pair
// owns a fixed block of item records (as many tiles as degree n needs); the
// tiles its chosen degree does not use are marked empty.
#include "kernels.cuh"

namespace btk {

namespace {

// out = M applied along axis `ax` of `in` (row-major dims n[0..dim-1]).
// M is rows x n[ax] with row stride `ms`; when `tr` is set M^T is applied
// (M given as n[ax] x rows). Output dims: n with n[ax] = rows.
__device__ void apply_rect(const double* in, double* out, int dim, const int* n, int ax, const double* M, int rows,
                           int ms, bool tr) {
  int no[3] = {n[0], n[1], dim == 3 ? n[2] : 1};
  int ni[3] = {n[0], n[1], dim == 3 ? n[2] : 1};
  no[ax] = rows;
  const int total = no[0] * no[1] * no[2];
  const int k_n = ni[ax];
  const int istr[3] = {ni[1] * ni[2], ni[2], 1};
  for (int o = threadIdx.x; o < total; o += blockDim.x) {
    int i0 = o / (no[1] * no[2]), i1 = (o / no[2]) % no[1], i2 = o % no[2];
    int idx[3] = {i0, i1, i2};
    const int r = idx[ax];
    idx[ax] = 0;
    const double* base = in + idx[0] * istr[0] + idx[1] * istr[1] + idx[2] * istr[2];
    double s = 0.0;
    for (int k = 0; k < k_n; ++k) {
      const double a = tr ? M[k * ms + r] : M[r * ms + k];
      s = fma(a, base[k * istr[ax]], s);
    }
    out[o] = s;
  }
}

constexpr int kMaxIpc = kMaxNodes * kMaxNodes * kMaxNodes;

// One block per (source cluster, degree slot): Q^d from Q^n, then the slot's
// proxy sources {x^d_a, y^d_b, z^d_c, Q^d[a,b,c]}.
__global__ void __launch_bounds__(256) k_src_slots(int dim, int n, const int* slot_cluster_panel,
                                                   const int* slot_degree, const long long* slot_offset,
                                                   const DevPanel* panels, const double* psw, const double* amat,
                                                   const int* amat_off, const double* ucos_all, const int* ucos_off,
                                                   const int* used, double4* S4) {
  __shared__ double bufA[kMaxIpc], bufB[kMaxIpc];
  const int slot = blockIdx.x;
  if (used && !used[slot]) return;  // no pair reads this slot this solve
  const int P = slot_cluster_panel[slot], d = slot_degree[slot];
  const int mn = n + 1, md = d + 1;
  const int ipc_n = dim == 3 ? mn * mn * mn : mn * mn;
  const int ipc_d = dim == 3 ? md * md * md : md * md;
  const double* A = amat + amat_off[d];  // md x mn
  for (int o = threadIdx.x; o < ipc_n; o += blockDim.x) bufA[o] = psw[(size_t)P * ipc_n + o];
  __syncthreads();
  const double* Q = bufA;
  if (d != n) {
    int dims[3] = {mn, mn, mn};
    apply_rect(bufA, bufB, dim, dims, 0, A, md, mn, false);
    __syncthreads();
    dims[0] = md;
    apply_rect(bufB, bufA, dim, dims, 1, A, md, mn, false);
    __syncthreads();
    if (dim == 3) {
      dims[1] = md;
      apply_rect(bufA, bufB, dim, dims, 2, A, md, mn, false);
      __syncthreads();
      Q = bufB;
    }
  }
  const DevPanel pn = panels[P];
  const double* uc = ucos_all + ucos_off[d];
  double4* out = S4 + slot_offset[slot];
  for (int k = threadIdx.x; k < ipc_d; k += blockDim.x) {
    int a, b, c = 0;
    if (dim == 2) {
      a = k / md;
      b = k % md;
    } else {
      a = k / (md * md);
      b = (k / md) % md;
      c = k % md;
    }
    double x[3];
    const int ab[3] = {a, b, c};
    for (int ax = 0; ax < dim; ++ax) {
      const double range = __dmul_rn(0.5, __dsub_rn(pn.hi[ax], pn.lo[ax]));
      const double mid = __dmul_rn(0.5, __dadd_rn(pn.hi[ax], pn.lo[ax]));
      x[ax] = __dadd_rn(__dmul_rn(uc[ab[ax]], range), mid);
    }
    out[k] = make_double4(x[0], x[1], dim == 3 ? x[2] : 0.0, Q[k]);
  }
}

// Target slots: proxy coordinates at degree d and their output offsets.
__global__ void k_tgt_slots(int dim, const int* slot_cluster_panel, const int* slot_degree,
                            const long long* slot_offset, const DevPanel* panels, const double* ucos_all,
                            const int* ucos_off, double4* T4, int* T_out, long long t4_base) {
  const int slot = blockIdx.x;
  const int P = slot_cluster_panel[slot], d = slot_degree[slot];
  const int md = d + 1;
  const int ipc_d = dim == 3 ? md * md * md : md * md;
  const DevPanel pn = panels[P];
  const double* uc = ucos_all + ucos_off[d];
  for (int k = threadIdx.x; k < ipc_d; k += blockDim.x) {
    int ab[3];
    if (dim == 2) {
      ab[0] = k / md;
      ab[1] = k % md;
      ab[2] = 0;
    } else {
      ab[0] = k / (md * md);
      ab[1] = (k / md) % md;
      ab[2] = k % md;
    }
    double x[3] = {0, 0, 0};
    for (int ax = 0; ax < dim; ++ax) {
      const double range = __dmul_rn(0.5, __dsub_rn(pn.hi[ax], pn.lo[ax]));
      const double mid = __dmul_rn(0.5, __dadd_rn(pn.hi[ax], pn.lo[ax]));
      x[ax] = __dadd_rn(__dmul_rn(uc[ab[ax]], range), mid);
    }
    const long long off = slot_offset[slot] + k;
    T4[t4_base + off] = make_double4(x[0], x[1], x[2], 0.0);
    T_out[t4_base + off] = (int)off;
  }
}

// One block per target cluster: Phi^n[cluster] += sum over its degree slots of
// the promoted Phi^d, for every component.
__global__ void __launch_bounds__(256) k_promote(int dim, int n, int ncomp, const int* cluster_panel,
                                                 const int* cluster_slot_begin, const int* slot_degree,
                                                 const long long* slot_offset, const double* amat,
                                                 const int* amat_off, Ptr4 ptwm, Ptr4 ptw) {
  // Each thread owns outputs o = tid + k*256 (apply_rect writes with the same
  // mapping), so the running sums stay in registers.
  constexpr int PER = (kMaxIpc + 255) / 256;
  __shared__ double bufA[kMaxIpc], bufB[kMaxIpc];
  const int c = blockIdx.x;
  const int P = cluster_panel[c];
  const int mn = n + 1;
  const int ipc_n = dim == 3 ? mn * mn * mn : mn * mn;
  const int s0 = cluster_slot_begin[c], s1 = cluster_slot_begin[c + 1];
  for (int comp = 0; comp < ncomp; ++comp) {
    double acc[PER];
#pragma unroll
    for (int k = 0; k < PER; ++k) acc[k] = 0.0;
    for (int s = s0; s < s1; ++s) {
      const int d = slot_degree[s], md = d + 1;
      const int ipc_d = dim == 3 ? md * md * md : md * md;
      const double* src = ptwm.p[comp] + slot_offset[s];
      __syncthreads();
      for (int o = threadIdx.x; o < ipc_d; o += blockDim.x) bufA[o] = src[o];
      __syncthreads();
      const double* R = bufA;
      if (d != n) {
        const double* A = amat + amat_off[d];  // md x mn; promotion applies A^T (mn x md)
        int dims[3] = {md, md, md};
        apply_rect(bufA, bufB, dim, dims, 0, A, mn, mn, true);
        __syncthreads();
        dims[0] = mn;
        apply_rect(bufB, bufA, dim, dims, 1, A, mn, mn, true);
        __syncthreads();
        R = bufA;
        if (dim == 3) {
          dims[1] = mn;
          apply_rect(bufA, bufB, dim, dims, 2, A, mn, mn, true);
          __syncthreads();
          R = bufB;
        }
      }
#pragma unroll
      for (int k = 0; k < PER; ++k) {
        const int o = threadIdx.x + k * 256;
        if (o < ipc_n) acc[k] += R[o];
      }
    }
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      const int o = threadIdx.x + k * 256;
      if (o < ipc_n) ptw.p[comp][(size_t)P * ipc_n + o] += acc[k];
    }
    __syncthreads();
  }
}

__device__ __forceinline__ int ipow_d(int b, int dim) { return dim == 3 ? b * b * b : b * b; }

// Re-points the PC entries of point-target items at the chosen degree's slot.
// Degree 0 (leaf pairs that may be approximated, kept direct): the source
// leaf's points, pc_direct[2 i] (first) and [2 i + 1] (count); degree -1 (the
// leaf pair's CC form taken instead): an empty entry.
__global__ void k_resolve_pc(int dim, int n_pc, const int* pc_entry, const int* pc_src_cluster, const int* degree,
                             const int* pc_direct, const long long* src_slot_offset, const int* cluster_slot_begin_s,
                             int slot_d_lo, long long s4_base, Entry* entries, int* slot_used) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pc) return;
  const int d = degree[i];
  Entry e;
  if (d < 0) {
    e.s_begin = 0;
    e.s_count = 0;
  } else if (d == 0) {
    e.s_begin = pc_direct[2 * i];
    e.s_count = pc_direct[2 * i + 1];
  } else {
    const int slot = cluster_slot_begin_s[pc_src_cluster[i]] + (d - slot_d_lo);
    e.s_begin = (int)(s4_base + src_slot_offset[slot]);
    e.s_count = ipow_d(d + 1, dim);
    if (slot_used) slot_used[slot] = 1;
  }
  const int k = pc_entry[i];
  if (k >= 0) entries[k] = e;
}

// Recomputes s_total of the point-target items (their entry counts changed).
__global__ void k_item_totals(int n_items, WorkItem* items, const Entry* entries) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_items) return;
  WorkItem w = items[i];
  int s = 0;
  for (int k = w.e_begin; k < w.e_end; ++k) s += entries[k].s_count;
  items[i].s_total = s;
}

// Builds the item records of the CP/CC pairs for the chosen degrees.
// Pair i owns items [far_item0 + i*tiles_max, ...) and entry far_entry0 + i.
__global__ void k_far_items(int dim, int n_far, int tiles_max, const int* far_type, const int* far_tgt_cluster,
                            const int* far_src, const int* degree, const long long* tgt_slot_offset,
                            const int* cluster_slot_begin_t, const long long* src_slot_offset,
                            const int* cluster_slot_begin_s, int slot_d_lo, long long t4_base, long long s4_base,
                            const double* tgt_centre, WorkItem* items, Entry* entries, int far_item0,
                            int far_entry0, int* slot_used, int tile) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_far) return;
  const int d = degree[i];
  if (d <= 0) {  // a leaf pair's CC form, not taken this solve: empty entry and tiles
    entries[far_entry0 + i] = Entry{0, 0};
    for (int k = 0; k < tiles_max; ++k) {
      WorkItem w{};
      w.e_begin = w.e_end = far_entry0 + i;
      items[far_item0 + (size_t)i * tiles_max + k] = w;
    }
    return;
  }
  const int ipc_d = ipow_d(d + 1, dim);
  Entry e;
  if (far_type[i] == 2) {  // CP: the source leaf's points (far_src packs begin, count)
    e.s_begin = far_src[2 * i];
    e.s_count = far_src[2 * i + 1];
  } else {  // CC: the source cluster's degree-d slot
    const int slot = cluster_slot_begin_s[far_src[2 * i]] + (d - slot_d_lo);
    e.s_begin = (int)(s4_base + src_slot_offset[slot]);
    e.s_count = ipc_d;
    if (slot_used) slot_used[slot] = 1;
  }
  entries[far_entry0 + i] = e;
  const int tc = far_tgt_cluster[i];
  const int tslot = cluster_slot_begin_t[tc] + (d - slot_d_lo);
  const long long t0 = t4_base + tgt_slot_offset[tslot];
  for (int k = 0; k < tiles_max; ++k) {
    WorkItem w{};
    const int a = k * tile;
    w.t_begin = (int)(t0 + a);
    w.t_count = a < ipc_d ? min(tile, ipc_d - a) : 0;
    w.e_begin = far_entry0 + i;
    w.e_end = far_entry0 + i + 1;
    w.s_total = e.s_count;
    w.flags = kItemProxyTargets | kItemAtomic;
    w.near_total = 0;
    w.cx = tgt_centre[3 * tc];
    w.cy = tgt_centre[3 * tc + 1];
    w.cz = tgt_centre[3 * tc + 2];
    items[far_item0 + (size_t)i * tiles_max + k] = w;
  }
}

}  // namespace

cudaError_t launch_src_slots(int dim, int n, int n_slots, const int* slot_cluster_panel, const int* slot_degree,
                             const long long* slot_offset, const DevPanel* panels, const double* psw,
                             const double* amat, const int* amat_off, const double* ucos_all, const int* ucos_off,
                             const int* used, double4* S4, cudaStream_t s) {
  if (n_slots <= 0) return cudaSuccess;
  k_src_slots<<<n_slots, 256, 0, s>>>(dim, n, slot_cluster_panel, slot_degree, slot_offset, panels, psw, amat,
                                     amat_off, ucos_all, ucos_off, used, S4);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_tgt_slots(int dim, int n_slots, const int* slot_cluster_panel, const int* slot_degree,
                             const long long* slot_offset, const DevPanel* panels, const double* ucos_all,
                             const int* ucos_off, double4* T4, int* T_out, long long t4_base, cudaStream_t s) {
  if (n_slots <= 0) return cudaSuccess;
  k_tgt_slots<<<n_slots, 128, 0, s>>>(dim, slot_cluster_panel, slot_degree, slot_offset, panels, ucos_all, ucos_off,
                                     T4, T_out, t4_base);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_promote(int dim, int n, int ncomp, int n_clusters, const int* cluster_panel,
                           const int* cluster_slot_begin, const int* slot_degree, const long long* slot_offset,
                           const double* amat, const int* amat_off, Ptr4 ptwm, Ptr4 ptw, cudaStream_t s) {
  if (n_clusters <= 0) return cudaSuccess;
  k_promote<<<n_clusters, 256, 0, s>>>(dim, n, ncomp, cluster_panel, cluster_slot_begin, slot_degree, slot_offset,
                                      amat, amat_off, ptwm, ptw);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_resolve(int dim, int n_pc, const int* pc_entry, const int* pc_src_cluster, const int* deg_pc,
                           const int* pc_direct, int n_far, int tiles_max, const int* far_type, const int* far_tgt_cluster,
                           const int* far_src, const int* deg_far, const long long* src_slot_offset,
                           const int* cluster_slot_begin_s, const long long* tgt_slot_offset,
                           const int* cluster_slot_begin_t, int slot_d_lo, long long t4_base, long long s4_base,
                           const double* tgt_centre, int n_point_items, WorkItem* items, Entry* entries,
                           int far_item0, int far_entry0, int* slot_used, int tile, cudaStream_t s) {
  if (n_pc > 0) {
    k_resolve_pc<<<(n_pc + 255) / 256, 256, 0, s>>>(dim, n_pc, pc_entry, pc_src_cluster, deg_pc, pc_direct,
                                                    src_slot_offset, cluster_slot_begin_s, slot_d_lo, s4_base,
                                                    entries, slot_used);
    count_launch();
  }
  if (n_point_items > 0) {
    k_item_totals<<<(n_point_items + 255) / 256, 256, 0, s>>>(n_point_items, items, entries);
    count_launch();
  }
  if (n_far > 0) {
    k_far_items<<<(n_far + 127) / 128, 128, 0, s>>>(dim, n_far, tiles_max, far_type, far_tgt_cluster, far_src, deg_far,
                                                    tgt_slot_offset, cluster_slot_begin_t, src_slot_offset,
                                                    cluster_slot_begin_s, slot_d_lo, t4_base, s4_base, tgt_centre,
                                                    items, entries, far_item0, far_entry0, slot_used, tile);
    count_launch();
  }
  return cudaGetLastError();
}

}  // namespace btk
