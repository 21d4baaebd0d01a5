// Host orchestration: tree sides on the device, interaction work lists, the
// plan API and the reference-named drop-in entry points.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "kernels.cuh"

namespace btk {

namespace {

// ---- device memory -----------------------------------------------------------
// Allocations of one plan or one drop-in call; freed together (stream-ordered).
struct Arena {
  cudaStream_t stream = nullptr;
  std::vector<void*> ptrs;
  size_t bytes = 0;
  explicit Arena(cudaStream_t s) : stream(s) {}
  ~Arena() {
    for (void* p : ptrs) cudaFreeAsync(p, stream);
  }
  template <class T>
  btk_status alloc(T** out, size_t n) {
    *out = nullptr;
    if (n == 0) return BTK_OK;
    void* p = nullptr;
    BTK_CUDA(cudaMallocAsync(&p, n * sizeof(T), stream));
    ptrs.push_back(p);
    bytes += n * sizeof(T);
    *out = static_cast<T*>(p);
    return BTK_OK;
  }
  template <class T>
  btk_status upload(T** out, const std::vector<T>& v) {
    BTK_TRY(alloc(out, v.size()));
    if (!v.empty()) BTK_CUDA(cudaMemcpyAsync(*out, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return BTK_OK;
  }
};

int ipow(int b, int e) {
  int r = 1;
  while (e-- > 0) r *= b;
  return r;
}

int ncomp_of(int dim, int kind) { return kind == BTK_KIND_POT ? 1 : (kind == BTK_KIND_VEL ? 3 : 1 + dim); }

int num_sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 1;
  }
  return n;
}

// ---- one side of the tree on the device ---------------------------------------
struct Side {
  HostTree h;
  int n_points = 0;
  int degree = 0, m = 0, ipc = 0;
  std::vector<int> leaf_begin;    // per panel (-1 for non-leaf)
  std::vector<int> leaves;        // non-empty leaves, panel order
  std::vector<int> clusters;      // non-leaf panels, panel order (proxy slots)
  std::vector<int> cluster_slot;  // per panel (-1 for leaves)
  std::vector<std::vector<int>> nonleaf_by_level, panels_by_level;
  std::vector<int> h_perm;  // leaf-order position -> original index (when built on the host)
  // device
  DevPanel* d_panels = nullptr;
  int *d_leaf_begin = nullptr, *d_point_count = nullptr, *d_leaves = nullptr, *d_clusters = nullptr;
  int *d_child = nullptr, *d_parent = nullptr, *d_perm = nullptr;
  double *d_nodes_shift = nullptr, *d_nodes_interp = nullptr, *d_xfer = nullptr;
  std::vector<int*> d_nonleaf_by_level, d_panels_by_level;
};

// Unit Chebyshev points in the reference's two evaluation orders, on the host
// with std::cos as the reference does: cos(pi/n*i) for bli_points_shift
// (src/bli_impl.hpp:74) and cos(pi*i/n) for interp_vals_bli (:25).
void unit_cosines(int n, std::vector<double>& shift, std::vector<double>& interp) {
  const double pi = 3.141592653589793238462643383279502884;
  shift.resize(n + 1);
  interp.resize(n + 1);
  for (int i = 0; i <= n; ++i) {
    shift[i] = std::cos(pi / n * i);
    interp[i] = std::cos(pi * i / n);
  }
}

btk_status side_layout(Side& S, int n_points, int degree) {
  const HostTree& h = S.h;
  S.n_points = n_points;
  S.degree = degree;
  S.m = degree + 1;
  S.ipc = ipow(S.m, h.dim);
  S.leaf_begin.assign(h.panel_count, -1);
  S.cluster_slot.assign(h.panel_count, -1);
  S.leaves.clear();
  S.clusters.clear();
  long long acc = 0;
  for (int i = 0; i < h.panel_count; ++i) {
    if (h.is_leaf[i]) {
      S.leaf_begin[i] = (int)acc;
      acc += h.point_count[i];
      if (h.point_count[i] > 0) S.leaves.push_back(i);
    } else {
      S.cluster_slot[i] = (int)S.clusters.size();
      S.clusters.push_back(i);
    }
  }
  BTK_CHECK(acc == n_points, BTK_ERR_INVALID_ARGUMENT,
            "tree: leaf point counts do not add up to the number of points");
  S.nonleaf_by_level.assign(h.levels, {});
  S.panels_by_level.assign(h.levels, {});
  for (int l = 0; l < h.levels; ++l)
    for (int i = h.level_start[l]; i < h.level_start[l + 1]; ++i) {
      BTK_CHECK(i >= 0 && i < h.panel_count, BTK_ERR_INVALID_ARGUMENT, "tree: level_start out of range");
      S.panels_by_level[l].push_back(i);
      if (!h.is_leaf[i]) S.nonleaf_by_level[l].push_back(i);
    }
  // Structural checks the kernels rely on.
  const int nc = 1 << h.dim;
  for (int i = 0; i < h.panel_count; ++i) {
    if (!h.is_leaf[i]) {
      for (int c = 0; c < nc; ++c) {
        int ch = h.child[(size_t)i * nc + c];
        BTK_CHECK(ch > i && ch < h.panel_count && h.parent[ch] == i, BTK_ERR_INVALID_ARGUMENT,
                  "tree: inconsistent child/parent links");
      }
    }
    // Level-0 panels are roots (one per tree: a forest of independent trees,
    // as a batch builds, has several); every other panel's parent precedes it.
    if (h.level[i] > 0)
      BTK_CHECK(h.parent[i] >= 0 && h.parent[i] < i, BTK_ERR_INVALID_ARGUMENT, "tree: bad parent link");
    else
      BTK_CHECK(h.parent[i] == -1, BTK_ERR_INVALID_ARGUMENT, "tree: a level-0 panel with a parent");
  }
  return BTK_OK;
}

btk_status side_upload(Side& S, Arena& A, const int* host_inside, const int* dev_inside, int thresh) {
  const HostTree& h = S.h;
  cudaStream_t st = A.stream;
  std::vector<DevPanel> dp(h.panel_count);
  for (int i = 0; i < h.panel_count; ++i) {
    for (int d = 0; d < 3; ++d) {
      dp[i].lo[d] = h.geom[i].lo[d];
      dp[i].hi[d] = h.geom[i].hi[d];
    }
    dp[i].parent = h.parent[i];
    dp[i].is_leaf = h.is_leaf[i];
    dp[i].point_count = h.point_count[i];
    dp[i].level = h.level[i];
  }
  BTK_TRY(A.upload(&S.d_panels, dp));
  BTK_TRY(A.upload(&S.d_leaf_begin, S.leaf_begin));
  BTK_TRY(A.upload(&S.d_point_count, h.point_count));
  BTK_TRY(A.upload(&S.d_leaves, S.leaves));
  BTK_TRY(A.upload(&S.d_clusters, S.clusters));
  BTK_TRY(A.upload(&S.d_child, h.child));
  BTK_TRY(A.upload(&S.d_parent, h.parent));
  S.d_nonleaf_by_level.assign(h.levels, nullptr);
  S.d_panels_by_level.assign(h.levels, nullptr);
  for (int l = 0; l < h.levels; ++l) {
    BTK_TRY(A.upload(&S.d_nonleaf_by_level[l], S.nonleaf_by_level[l]));
    BTK_TRY(A.upload(&S.d_panels_by_level[l], S.panels_by_level[l]));
  }
  // Geometry: nodes and transfer factors.
  std::vector<double> us, ui;
  unit_cosines(S.degree, us, ui);
  double *d_us = nullptr, *d_ui = nullptr;
  BTK_TRY(A.upload(&d_us, us));
  BTK_TRY(A.upload(&d_ui, ui));
  BTK_TRY(A.alloc(&S.d_nodes_shift, (size_t)h.panel_count * kPanelNodes));
  BTK_TRY(A.alloc(&S.d_nodes_interp, (size_t)h.panel_count * kPanelNodes));
  BTK_TRY(A.alloc(&S.d_xfer, (size_t)h.panel_count * kPanelXfer));
  BTK_CUDA(launch_panel_geometry(h.dim, S.degree, h.panel_count, S.d_panels, d_us, d_ui, S.d_nodes_shift,
                                 S.d_nodes_interp, S.d_xfer, st));
  // Leaf order permutation.
  BTK_TRY(A.alloc(&S.d_perm, (size_t)std::max(S.n_points, 1)));
  if (host_inside) {
    std::vector<int>& perm = S.h_perm;
    perm.assign(S.n_points, 0);
    for (int L : S.leaves)
      for (int j = 0; j < h.point_count[L]; ++j) {
        int v = host_inside[(size_t)L * thresh + j];
        BTK_CHECK(v >= 0 && v < S.n_points, BTK_ERR_INVALID_ARGUMENT, "panel_points_inside: index out of range");
        perm[S.leaf_begin[L] + j] = v;
      }
    if (S.n_points) BTK_CUDA(cudaMemcpyAsync(S.d_perm, perm.data(), sizeof(int) * S.n_points, cudaMemcpyHostToDevice, st));
  } else if (dev_inside) {
    BTK_CUDA(launch_perm_from_inside((int)S.leaves.size(), S.d_leaves, S.d_leaf_begin, S.d_point_count, dev_inside,
                                     thresh, S.d_perm, st));
  }
  return BTK_OK;
}

// Builds the leaf permutation from point_leaf_panel (stable counting sort:
// ascending original index inside each leaf, the order of panel_points_inside).
btk_status side_perm_from_leaf_of(Side& S, Arena& A, const std::vector<int>& leaf_of) {
  std::vector<int> cursor(S.leaf_begin);
  std::vector<int>& perm = S.h_perm;
  perm.assign(S.n_points, 0);
  for (int i = 0; i < S.n_points; ++i) {
    int L = leaf_of[i];
    BTK_CHECK(L >= 0 && L < S.h.panel_count && S.h.is_leaf[L], BTK_ERR_INVALID_ARGUMENT,
              "point_leaf_panel: not a leaf panel");
    int pos = cursor[L]++;
    BTK_CHECK(pos < S.leaf_begin[L] + S.h.point_count[L], BTK_ERR_INVALID_ARGUMENT,
              "point_leaf_panel: more points than the leaf's point_count");
    perm[pos] = i;
  }
  if (S.n_points)
    BTK_CUDA(cudaMemcpyAsync(S.d_perm, perm.data(), sizeof(int) * S.n_points, cudaMemcpyHostToDevice, A.stream));
  return BTK_OK;
}

// ---- interaction work lists -------------------------------------------------
struct WorkLists {
  std::vector<WorkItem> items;
  std::vector<Entry> entries;
  int64_t evals[4] = {0, 0, 0, 0};
};

// pc_begin (optional): S4 start of each PC pair's source proxies (default: the
// cluster's single-degree slot). pc_entry (optional, out): final entry index of
// each PC pair, for re-pointing when per-pair degrees change.
// split: work items per persistent-grid slot the cost cap aims at (longer
// source lists are cut into atomic pieces).
// Runs fn(begin, end) over [0, n) on up to `threads` host threads (serially
// when the range is small).
template <class F>
void parallel_ranges(int64_t n, int threads, int64_t min_per_thread, F fn) {
  const int t = (int)std::max<int64_t>(1, std::min<int64_t>(threads, n / std::max<int64_t>(1, min_per_thread)));
  if (t <= 1) {
    fn((int64_t)0, n, 0);
    return;
  }
  std::vector<std::thread> pool;
  for (int k = 1; k < t; ++k) pool.emplace_back(fn, n * k / t, n * (k + 1) / t, k);
  fn((int64_t)0, n / t, 0);
  for (auto& th : pool) th.join();
}

int host_threads() {
  static const int n = std::max(1, std::min(32, (int)std::thread::hardware_concurrency()));
  return n;
}

btk_status build_work(const Side& T, const Side& S, const btk_interact_pair* const lists[4], const int counts[4],
                      int grid_slots, WorkLists& W, const std::vector<long long>* pc_begin = nullptr,
                      std::vector<int>* pc_entry = nullptr, int split = 8, std::vector<int>* pp_entry = nullptr,
                      int tile = kTile) {
  const int ipc = S.ipc;
  const int nt = T.n_points, ns = S.n_points;
  const int Pt = T.h.panel_count, Ps = S.h.panel_count;
  // The four lists as one sequence (PP, PC, CP, CC, each in list order),
  // cut into chunks that host threads take in order.
  const int64_t off1 = counts[0], off2 = off1 + counts[1], off3 = off2 + counts[2], npairs = off3 + counts[3];
  auto pair_at = [&](int64_t g, int& t, int& i) {
    t = g < off1 ? 0 : (g < off2 ? 1 : (g < off3 ? 2 : 3));
    i = (int)(g - (t == 0 ? 0 : t == 1 ? off1 : t == 2 ? off2 : off3));
  };
  const int nthreads = host_threads();
  const int nchunk = (int)std::max<int64_t>(1, std::min<int64_t>(nthreads, npairs / 65536));
  auto chunk_lo = [&](int c) { return npairs * c / nchunk; };
  // Pass 1: validation and, per chunk, pairs per target panel.
  std::vector<std::vector<int>> hist(nchunk, std::vector<int>(Pt, 0));
  std::vector<int> bad(nchunk, 0);
  parallel_ranges(nchunk, nthreads, 1, [&](int64_t cb, int64_t ce, int) {
    for (int64_t c = cb; c < ce; ++c)
      for (int64_t g = chunk_lo((int)c); g < chunk_lo((int)c + 1); ++g) {
        int t, i;
        pair_at(g, t, i);
        const btk_interact_pair& pr = lists[t][i];
        if (!(pr.target_panel >= 0 && pr.target_panel < Pt && pr.source_panel >= 0 && pr.source_panel < Ps)) {
          bad[c] = 1;
          break;
        }
        const bool tgt_cluster = t >= 2, src_cluster = (t & 1) != 0;
        if (!(tgt_cluster == !T.h.is_leaf[pr.target_panel] && src_cluster == !S.h.is_leaf[pr.source_panel])) {
          bad[c] = 2;
          break;
        }
        hist[c][pr.target_panel]++;
      }
  });
  for (int c = 0; c < nchunk; ++c) {
    BTK_CHECK(bad[c] != 1, BTK_ERR_INVALID_ARGUMENT, "interaction list: panel index out of range");
    BTK_CHECK(bad[c] != 2, BTK_ERR_INVALID_ARGUMENT,
              "interaction list: pair type does not match the panels (PP/PC targets and PP/CP sources must be "
              "leaves, the others non-leaf)");
  }
  // Stable grouping by target panel: point targets take PP then PC pairs,
  // proxy targets CP then CC, each in list order. Chunk c writes target tp's
  // pairs from head[tp] + (pairs of tp in chunks before c).
  std::vector<int> head(Pt + 1, 0);
  for (int tp = 0; tp < Pt; ++tp) {
    int acc = 0;
    for (int c = 0; c < nchunk; ++c) {
      const int h = hist[c][tp];
      hist[c][tp] = acc;  // now the chunk's offset within tp's group
      acc += h;
    }
    head[tp + 1] = head[tp] + acc;
  }
  std::vector<Entry> grouped(head[Pt]);
  std::vector<char> touching(head[Pt], 0);
  std::vector<int> final_index(head[Pt], -1);
  std::vector<int> grouped_of_pc;
  if (pc_entry) grouped_of_pc.assign(counts[1], -1);
  std::vector<int> pp_at;  // PP pair at each grouped position (pp_entry only)
  if (pp_entry) pp_at.assign(head[Pt], -1);
  // A PP source leaf "touches" the target leaf when the gap between the boxes
  // is under half the target's smallest side. Only such pairs can be far
  // closer than their distance to the item's centre, so only their sources
  // take the mixed kernel's hi/lo coordinate path.
  auto touches = [&](int tp, int sp) {
    const PanelGeom &a = T.h.geom[tp], &b = S.h.geom[sp];
    double gap = 0.0, side = 1e300;
    for (int d = 0; d < T.h.dim; ++d) {
      gap = std::max(gap, std::max(b.lo[d] - a.hi[d], a.lo[d] - b.hi[d]));
      side = std::min(side, a.hi[d] - a.lo[d]);
    }
    return gap <= 0.5 * side;
  };
  std::vector<std::array<int64_t, 4>> evals_part(nchunk, std::array<int64_t, 4>{0, 0, 0, 0});
  parallel_ranges(nchunk, nthreads, 1, [&](int64_t cb, int64_t ce, int) {
    for (int64_t c = cb; c < ce; ++c) {
      std::vector<int>& cur = hist[c];
      for (int64_t g = chunk_lo((int)c); g < chunk_lo((int)c + 1); ++g) {
        int t, i;
        pair_at(g, t, i);
        const btk_interact_pair& pr = lists[t][i];
        const int sp = pr.source_panel, tp = pr.target_panel;
        const int pos = head[tp] + cur[tp]++;
        if (t == 0) touching[pos] = touches(tp, sp);
        Entry e;
        if (t & 1) {  // cluster source: its proxies
          e.s_begin = (t == 1 && pc_begin) ? (int)(*pc_begin)[i] : ns + S.cluster_slot[sp] * ipc;
          e.s_count = ipc;
        } else {
          e.s_begin = S.leaf_begin[sp];
          e.s_count = S.h.point_count[sp];
        }
        const int64_t nt_pts = (t >= 2) ? ipc : T.h.point_count[tp];
        evals_part[c][t] += nt_pts * (int64_t)e.s_count;
        if (t == 1 && pc_entry) grouped_of_pc[i] = pos;
        if (t == 0 && pp_entry) pp_at[pos] = i;
        grouped[pos] = e;
      }
    }
  });
  for (int c = 0; c < nchunk; ++c)
    for (int t = 0; t < 4; ++t) W.evals[t] += evals_part[c][t];
  // PP pairs lead every point target's group; count them per target.
  std::vector<int> n_near(Pt, 0);
  for (int i = 0; i < counts[0]; ++i) n_near[lists[0][i].target_panel]++;
  // Tiles and items. A warp evaluates its targets against every source of
  // its item, whatever the tile's fill, so an item runs for a time set by its
  // source count: long source lists are cut into pieces of at most
  // max_cost / tile sources whatever the tile's fill. Items are ordered by
  // their evaluations, largest first (the persistent grid's
  // longest-processing-time schedule; measured faster for the mixed kernel
  // than ordering by source count).
  auto tile_duration = [tile](int64_t st) { return (int64_t)tile * st; };
  auto order_key = [](int tc, int64_t st) { return (int64_t)tc * st; };
  int64_t total_cost = W.evals[0] + W.evals[1] + W.evals[2] + W.evals[3];
  const int64_t max_cost =
      std::max<int64_t>((int64_t)tile * 8192, total_cost / std::max<int64_t>(1, (int64_t)grid_slots * split));
  // Pass A per target: touching PP sources first (stable), then the other PP
  // sources, then the rest; count its non-empty entries and its items.
  std::vector<int> n_ent(Pt + 1, 0), n_itm(Pt + 1, 0), n_touch(Pt, 0), s_tot(Pt, 0);
  parallel_ranges(Pt, nthreads, 256, [&](int64_t pb, int64_t pe, int) {
    std::vector<Entry> seg;
    std::vector<int> segp;
    for (int64_t tp = pb; tp < pe; ++tp) {
      const int eb = head[tp], ee = head[tp + 1];
      if (eb == ee) continue;
      seg.clear();
      segp.clear();
      for (int k = eb; k < eb + n_near[tp]; ++k)
        if (touching[k]) {
          seg.push_back(grouped[k]);
          if (pp_entry) segp.push_back(pp_at[k]);
        }
      n_touch[tp] = (int)seg.size();
      for (int k = eb; k < eb + n_near[tp]; ++k)
        if (!touching[k]) {
          seg.push_back(grouped[k]);
          if (pp_entry) segp.push_back(pp_at[k]);
        }
      std::copy(seg.begin(), seg.end(), grouped.begin() + eb);
      if (pp_entry) std::copy(segp.begin(), segp.end(), pp_at.begin() + eb);
      int ne = 0, st = 0;
      for (int k = eb; k < ee; ++k)
        if (grouped[k].s_count > 0) {
          ++ne;
          st += grouped[k].s_count;
        }
      n_ent[tp] = ne;
      s_tot[tp] = st;
      if (st == 0) continue;
      const bool proxy = !T.h.is_leaf[tp];
      const int tn = proxy ? ipc : T.h.point_count[tp];
      int ni = 0;
      for (int a = 0; a < tn; a += tile) {
        const int64_t cost = tile_duration(st);
        const int nsplit = (int)std::min<int64_t>((cost + max_cost - 1) / max_cost, ne);
        if (nsplit <= 1) {
          ++ni;
          continue;
        }
        const int64_t per = (st + nsplit - 1) / nsplit;
        int k = eb, acc = 0;  // walk the non-empty entries like pass B
        bool open = false;
        int64_t piece = 0;
        for (; k < ee; ++k) {
          const int sc = grouped[k].s_count;
          if (sc <= 0) continue;
          if (open && piece + sc > per) {
            ++acc;
            piece = 0;
          }
          piece += sc;
          open = true;
        }
        if (open) ++acc;
        ni += acc;
      }
      n_itm[tp] = ni;
    }
  });
  // Offsets.
  std::vector<int64_t> ent_off(Pt + 1, 0), itm_off(Pt + 1, 0);
  for (int tp = 0; tp < Pt; ++tp) {
    ent_off[tp + 1] = ent_off[tp] + n_ent[tp];
    itm_off[tp + 1] = itm_off[tp] + n_itm[tp];
  }
  BTK_CHECK(ent_off[Pt] < (1ll << 31), BTK_ERR_UNSUPPORTED, "work lists: more than 2^31 entries");
  W.entries.resize(ent_off[Pt]);
  std::vector<std::pair<int64_t, WorkItem>> items(itm_off[Pt]);
  // Pass B per target: entries and items at the offsets.
  parallel_ranges(Pt, nthreads, 256, [&](int64_t pb, int64_t pe, int) {
    for (int64_t tp = pb; tp < pe; ++tp) {
      const int eb = head[tp], ee = head[tp + 1];
      if (eb == ee) continue;
      const int e0 = (int)ent_off[tp];
      int e = e0, e_near = e0;
      for (int k = eb; k < ee; ++k) {
        if (grouped[k].s_count > 0) {
          final_index[k] = e;
          W.entries[e++] = grouped[k];
        }
        if (k - eb < n_touch[tp]) e_near = e;
      }
      const int e1 = e;
      const int s_total = s_tot[tp];
      if (s_total == 0) continue;
      // Sources of entries [kb, ke) that are near-field (PP) points.
      auto near_of = [&](int kb, int ke) {
        int n = 0;
        for (int k = kb; k < std::min(ke, e_near); ++k) n += W.entries[k].s_count;
        return n;
      };
      const bool proxy = !T.h.is_leaf[tp];
      const int t0 = proxy ? nt + T.cluster_slot[tp] * ipc : T.leaf_begin[tp];
      const int tn = proxy ? ipc : T.h.point_count[tp];
      // Origin for relative coordinates (mixed precision): the target panel's
      // centre; its half widths bound the near-source test.
      const PanelGeom& g = T.h.geom[tp];
      const double c[3] = {0.5 * (g.lo[0] + g.hi[0]), 0.5 * (g.lo[1] + g.hi[1]), 0.5 * (g.lo[2] + g.hi[2])};
      const float bh[3] = {(float)(0.5 * (g.hi[0] - g.lo[0])), (float)(0.5 * (g.hi[1] - g.lo[1])),
                           T.h.dim == 3 ? (float)(0.5 * (g.hi[2] - g.lo[2])) : 0.f};
      auto item = [&](int tb, int tc, int kb, int ke, int st, int flags) {
        WorkItem w{};
        w.t_begin = tb;
        w.t_count = tc;
        w.e_begin = kb;
        w.e_end = ke;
        w.s_total = st;
        w.flags = flags;
        w.near_total = near_of(kb, ke);
        w.cx = c[0];
        w.cy = c[1];
        w.cz = c[2];
        w.hx = bh[0];
        w.hy = bh[1];
        w.hz = bh[2];
        return w;
      };
      int64_t out = itm_off[tp];
      for (int a = 0; a < tn; a += tile) {
        const int tc = std::min(tile, tn - a);
        const int64_t cost = tile_duration(s_total);
        const int nsplit = (int)std::min<int64_t>((cost + max_cost - 1) / max_cost, e1 - e0);
        if (nsplit <= 1) {
          items[out++] = {order_key(tc, s_total), item(t0 + a, tc, e0, e1, s_total, proxy ? kItemProxyTargets : 0)};
          continue;
        }
        // Split the entry range into nsplit pieces of similar source counts.
        const int64_t per = (s_total + nsplit - 1) / nsplit;
        int k = e0;
        while (k < e1) {
          int kb = k, st = 0;
          while (k < e1 && (st == 0 || st + W.entries[k].s_count <= per)) st += W.entries[k++].s_count;
          items[out++] = {order_key(tc, st), item(t0 + a, tc, kb, k, st, (proxy ? kItemProxyTargets : 0) | kItemAtomic)};
        }
      }
    }
  });
  if (pc_entry) {
    pc_entry->assign(counts[1], -1);
    for (int i = 0; i < counts[1]; ++i) {
      const int k = grouped_of_pc[i];
      (*pc_entry)[i] = k >= 0 ? final_index[k] : -1;
    }
  }
  if (pp_entry) {  // final entry of each PP pair (-1: empty source leaf, no entry)
    pp_entry->assign(counts[0], -1);
    for (size_t k = 0; k < pp_at.size(); ++k)
      if (pp_at[k] >= 0) (*pp_entry)[pp_at[k]] = final_index[k];
  }
  std::stable_sort(items.begin(), items.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  W.items.resize(items.size());
  for (size_t i = 0; i < items.size(); ++i) W.items[i] = items[i].second;
  return BTK_OK;
}

void kind_scales(int dim, int kind, double* sc) {
  const double pi = 3.141592653589793238462643383279502884;
  const double q4 = 1.0 / (4.0 * pi);
  for (int c = 0; c < 4; ++c) sc[c] = 0.0;
  if (dim == 2) {
    sc[0] = q4;                                    // +(1/4pi) log(r^2+eps^2)
    if (kind == BTK_KIND_FIELD) sc[1] = sc[2] = -1.0 / (2.0 * pi);
  } else if (kind == BTK_KIND_VEL) {
    sc[0] = sc[1] = sc[2] = -q4;                   // -(1/4pi) q (t-s)/(r^2+eps^2)
  } else {
    sc[0] = -q4;                                   // -(1/4pi)/sqrt(r^2+eps^2)
    if (kind == BTK_KIND_FIELD) sc[1] = sc[2] = sc[3] = -q4;
  }
}

// ---- the interaction phase on prepared device data ----------------------------
struct InteractCtx {
  int dim, kind, precision;
  double eps;
  WorkItem* d_items = nullptr;
  Entry* d_entries = nullptr;
  int n_items = 0;
  int* d_ticket_status = nullptr;  // [0] ticket, [1] status
  const double4* d_T4a = nullptr;  // audit targets and outputs (kItemAudit items)
  Ptr4 aout{};
  int n_audit_items = 0;  // audit items follow the n_items in d_items
  int audit_blocks = 0;   // blocks that start on the audit items
  uint32_t wait_limit = kWaitLimitDefault;
  int tile = kTile;  // targets per work item: 256 (128-thread blocks) or 128 (64-thread blocks)
};

btk_status run_interactions(const InteractCtx& C, const double4* S4, const double4* T4, const int* T_out,
                            Ptr4 out, Ptr4 ptw, cudaStream_t st, cudaEvent_t e0 = nullptr, cudaEvent_t e1 = nullptr) {
  if (C.n_items + C.n_audit_items == 0) return BTK_OK;
  InteractParams p{};
  p.items = C.d_items;
  p.n_items = C.n_items;
  p.entries = C.d_entries;
  p.S4 = S4;
  p.T4 = T4;
  p.T_out = T_out;
  for (int c = 0; c < 4; ++c) {
    p.out[c] = out.p[c];
    p.ptw[c] = ptw.p[c];
    p.aout[c] = C.aout.p[c];
  }
  p.T4a = C.d_T4a;
  p.eps2 = C.eps * C.eps;
  kind_scales(C.dim, C.kind, p.scale);
  p.ticket = C.d_ticket_status;
  p.status = C.d_ticket_status + 1;
  p.wait_limit = C.wait_limit;
  p.n_audit_items = C.n_audit_items;
  p.audit_ticket = C.d_ticket_status + 2;
  const bool guard = p.eps2 < 1.1754943508222875e-38;
  int per_sm = interact_blocks_per_sm(C.dim, C.kind, C.precision, guard, C.tile);
  if (per_sm <= 0) per_sm = 1;
  const int grid = std::min(C.n_items + C.n_audit_items, num_sms() * per_sm);
  p.audit_blocks = std::min(C.audit_blocks, grid);
  BTK_CUDA(cudaMemsetAsync(C.d_ticket_status, 0, sizeof(int), st));
  if (C.n_audit_items > 0) BTK_CUDA(cudaMemsetAsync(C.d_ticket_status + 2, 0, sizeof(int), st));
  if (e0) BTK_CUDA(cudaEventRecord(e0, st));
  BTK_CUDA(launch_interact(C.dim, C.kind, C.precision, guard, p, grid, st, C.tile));
  if (e1) BTK_CUDA(cudaEventRecord(e1, st));
  return BTK_OK;
}

btk_status validate_cfg(const btk_run_config* cfg, int dim) {
  BTK_CHECK(cfg, BTK_ERR_INVALID_ARGUMENT, "null run config");
  BTK_CHECK(cfg->dim == dim, BTK_ERR_INVALID_ARGUMENT, "run config dim does not match the entry point");
  BTK_CHECK(cfg->interp_degree >= 1 && cfg->interp_degree <= kMaxDegree, BTK_ERR_UNSUPPORTED,
            "interp_degree outside 1..12");
  BTK_CHECK(cfg->interp_point_count == ipow(cfg->interp_degree + 1, dim), BTK_ERR_INVALID_ARGUMENT,
            "interp_point_count != (interp_degree+1)^dim");
  BTK_CHECK(cfg->fmm_cluster_thresh > 0, BTK_ERR_INVALID_ARGUMENT, "fmm_cluster_thresh must be positive");
  BTK_CHECK(std::isfinite(cfg->ker_eps), BTK_ERR_INVALID_ARGUMENT, "ker_eps must be finite");
  return BTK_OK;
}

template <class P>
btk_status fetch_panels(const P* d_panels, int count, std::vector<P>& host, cudaStream_t st) {
  BTK_CHECK(d_panels || count == 0, BTK_ERR_INVALID_ARGUMENT, "null panel array");
  BTK_CHECK(count > 0, BTK_ERR_INVALID_ARGUMENT, "panel count must be positive");
  host.resize(count);
  BTK_CUDA(cudaMemcpyAsync(host.data(), d_panels, sizeof(P) * count, cudaMemcpyDeviceToHost, st));
  return BTK_OK;
}

template <class T>
btk_status fetch(const T* d, int count, std::vector<T>& host, cudaStream_t st) {
  host.resize(count);
  if (count == 0) return BTK_OK;
  BTK_CHECK(d, BTK_ERR_INVALID_ARGUMENT, "null device array");
  BTK_CUDA(cudaMemcpyAsync(host.data(), d, sizeof(T) * count, cudaMemcpyDeviceToHost, st));
  return BTK_OK;
}

btk_status check_status_word(const int* d_status, cudaStream_t st) {
  int h = 0;
  BTK_CUDA(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  BTK_CUDA(cudaStreamSynchronize(st));
  if (h != 0) return set_error((btk_status)h, "device-side wait timed out in the interaction kernel");
  return BTK_OK;
}

}  // namespace
}  // namespace btk

// =============================================================================
// Plan API
// =============================================================================
struct btk_plan {
  int dim = 3, degree = 8, m = 9, ipc = 729, kind = 0, precision = 0, ncomp = 1, thresh = 0;
  double eps = 0;
  bool same_tree = true;
  cudaStream_t stream = nullptr;
  std::unique_ptr<btk::Arena> arena;
  btk::Side tgt, src_own;
  btk::Side* src = nullptr;
  btk::InteractCtx ictx;
  int64_t evals[4] = {0, 0, 0, 0};
  // device work arrays
  double4 *d_S4 = nullptr, *d_T4 = nullptr;
  int* d_T_out = nullptr;
  double* d_psw = nullptr;
  double* d_ptw = nullptr;  // ncomp x Pt x ipc
  int* d_ticket_status = nullptr;  // [0] ticket, [1] device status, [2] audit ticket
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  bool timed = false;

  // ---- per-pair degrees (degree_mode == BTK_DEGREE_PER_PAIR) ----
  int degree_mode = BTK_DEGREE_FIXED, degree_min = 0;
  int n_pc = 0, n_cp = 0, n_far = 0, tiles_max = 0, n_static_items = 0, n_static_entries = 0;
  // Leaf pairs the degree choice may approximate (leaf_far_pairs): PC-block
  // pairs [n_pc_list, n_pc), degree 0 = direct.
  int leaf_far = 0, n_pc_list = 0, n_far_list = 0, n_tgt_slot_panels = 0;
  int n_conv_cc = 0;  // leaf pairs with a CC form: the first of them, CC entries closing the far block
  int n_pccc = 0;     // PC pairs with a CC form (large target leaf); their CC entries precede the leaf pairs'
  int n_cpcc = 0;     // CP pairs with a CC form (large source leaf); their CC entries follow the PC pairs'
  int *d_pccc_idx = nullptr, *d_pccc_coef = nullptr;  // their PC entries, target leaf points
  int *d_cpcc_idx = nullptr, *d_cpcc_coef = nullptr;  // their CP entries (pair array), source leaf points
  double leaf_theta = 0.8;  // separation bound of the leaf pairs
  int64_t conv_direct_total = 0;  // their direct evaluations (all included in evals[0])
  int64_t evals_pp_static = 0;     // PP evaluations with every leaf pair direct
  std::vector<int> h_conv;         // the leaf pairs' PP list indices, in plan order
  std::vector<int> h_pc_direct;    // per PC-block pair: source leaf first point, count (leaf pairs)
  int* d_pc_direct = nullptr;
  int n_src_slots = 0, n_tgt_slots = 0;
  long long total_src_slots = 0, total_tgt_slots = 0;
  int *d_s_slot_panel = nullptr, *d_s_slot_deg = nullptr, *d_s_cluster_slot_begin = nullptr;
  int* d_s_slot_used = nullptr;  // per source slot: read by this solve's work items
  int *d_t_slot_deg = nullptr, *d_t_cluster_slot_begin = nullptr, *d_t_cluster_panel = nullptr;
  long long *d_s_slot_off = nullptr, *d_t_slot_off = nullptr;
  double* d_amat = nullptr;
  int* d_amat_off = nullptr;
  double* d_ucos = nullptr;
  int* d_ucos_off = nullptr;
  int *d_pc_entry = nullptr, *d_pc_src_cluster = nullptr;
  int *d_far_type = nullptr, *d_far_tgt = nullptr, *d_far_src = nullptr;
  double* d_tgt_centre = nullptr;
  int *d_deg_pc = nullptr, *d_deg_far = nullptr;  // the degrees in force
  bool deg_learned = false;  // d_deg_* hold a learned solve's choice, not h_deg_*
  double* d_ptwm = nullptr;                       // ncomp x total_tgt_slots
  // host copies for work accounting
  std::vector<int> h_pc_tcount, h_cp_scount, h_deg_pc, h_deg_far;

  // ---- learned selector (per-pair plans) ----
  int n_pairs = 0;  // PC (the list, then the leaf pairs), then CP, then CC
  int *d_pair_type = nullptr, *d_pair_tgt = nullptr, *d_pair_src = nullptr;
  int *d_pc_tcount = nullptr, *d_cp_scount = nullptr;
  float *d_desc = nullptr, *d_feat = nullptr, *d_pred = nullptr;
  unsigned long long* d_evals = nullptr;
  double* d_gsum = nullptr;  // sum |q|, sum q
  double root_radius = 1.0, root_centre[3] = {0, 0, 0};
  // audit: a fixed 1% sample of the targets, direct sum over all sources; its
  // work items follow the solve's in ictx.d_items, [n_items_main, + n_audit_items)
  int n_audit = 0, n_items_main = 0, n_audit_items = 0;
  int work_split = 8;  // work items per persistent-grid slot
  // CC pairs as shared kernel matrices (fixed-degree plans, cc_operators = 1)
  int n_cc_groups = 0, n_cc_tasks = 0, cc_bucket_end[3] = {0, 0, 0};
  btk::CcTask* d_cc_tasks = nullptr;
  btk::CcPair* d_cc_pairs = nullptr;
  double adaptive_pair_tol = 0;  // learned solves with pair_tol <= 0 (0: not yet set)
  float build_ms_total = 0, build_ms_work = 0;  // host time of plan creation, of which work lists
  int degree_rule = BTK_DEGREE_RULE_COST;
  int* d_pair_weight = nullptr;       // points under each pair's target panel
  float inv_cbar = 1.f, inv_wbar = 1.f;  // 1 / mean pair cost at the plan degree, 1 / mean weight
  int* d_audit_orig = nullptr;
  double4* d_audit_T4 = nullptr;
  double *d_audit_out = nullptr, *d_audit_sums = nullptr;
  int* d_report = nullptr;  // degree histogram (kMaxNodes ints), copied with the audit sums
  int *d_cluster_slot_s = nullptr, *d_cluster_slot_t = nullptr;  // panel -> cluster index (or -1)
};

// Adaptive learned solves start at this fraction of the tolerance per pair.
constexpr double kAdaptiveStart = 0.05;

struct btk_selector {
  void* d_w = nullptr;  // BF16 parameters
  float norm[34] = {};  // feature mean[16], std[16], target mean, std
};

using namespace btk;

namespace {

// Barycentric basis of degree d on [-1, 1] (nodes cos(pi*a/d)) at x, with the
// reference's near-node rule (src/bli_impl.hpp:9-63).
void bary_row_unit(double x, int d, double* out) {
  const double pi = 3.141592653589793238462643383279502884;
  std::vector<double> node(d + 1), w(d + 1);
  for (int a = 0; a <= d; ++a) {
    node[a] = std::cos(pi * a / d);
    w[a] = (a % 2 ? -1.0 : 1.0) * ((a == 0 || a == d) ? 0.5 : 1.0);
  }
  for (int a = 0; a <= d; ++a)
    if (std::fabs(x - node[a]) < 2.220446049250313e-16) {
      for (int b = 0; b <= d; ++b) out[b] = b == a ? 1.0 : 0.0;
      return;
    }
  double den = 0.0;
  for (int a = 0; a <= d; ++a) {
    out[a] = w[a] / (x - node[a]);
    den += out[a];
  }
  for (int a = 0; a <= d; ++a) out[a] /= den;
}

// Far-field evaluation counts at the per-pair degrees in force.
void recount_far_evals(btk_plan* P) {
  auto sz = [&](int d) { return (int64_t)ipow(d + 1, P->dim); };
  P->evals[1] = P->evals[2] = P->evals[3] = 0;
  for (int i = 0; i < P->n_pc; ++i)
    if (P->h_deg_pc[i] > 0) P->evals[1] += P->h_pc_tcount[i] * sz(P->h_deg_pc[i]);
  // leaf pairs not direct leave the PP evaluations (the form taken is counted
  // above as PC, or below as CC)
  P->evals[0] = P->evals_pp_static;
  const int n_conv = P->n_pc - P->n_pc_list;
  for (int k = 0; k < n_conv; ++k) {
    const int i = P->n_pc_list + k;
    const int j = P->n_far_list + P->n_pccc + P->n_cpcc + k;  // CC entry (first n_conv_cc pairs)
    const bool direct = P->h_deg_pc[i] == 0 && (k >= P->n_conv_cc || P->h_deg_far[j] == 0);
    if (!direct) P->evals[0] -= (int64_t)P->h_pc_tcount[i] * P->h_pc_direct[2 * i + 1];
  }
  for (int i = 0; i < P->n_cp; ++i) P->evals[2] += sz(P->h_deg_far[i]) * P->h_cp_scount[i];
  for (int i = P->n_cp; i < P->n_far; ++i)
    if (P->h_deg_far[i] > 0) P->evals[3] += sz(P->h_deg_far[i]) * sz(P->h_deg_far[i]);
}

// The audit's targets and work items (built on the host; see build_audit_work).
struct AuditWork {
  std::vector<int> orig;  // audited targets (original indices), tile order
  std::vector<WorkItem> items;
  std::vector<Entry> entries;
};
void build_audit_work(const btk_plan* P, int entry_base, AuditWork& W);
btk_status setup_audit(btk_plan* P, Arena& A, const AuditWork& W, int item_base, int entry_base, cudaStream_t st);

btk_status plan_build_per_pair(btk_plan* P, const btk_interact_pair* const lists[4], const int counts[4], int slots,
                               cudaStream_t st) {
  Arena& A = *P->arena;
  Side& T = P->tgt;
  Side& S = *P->src;
  const int dim = P->dim, n = P->degree, dlo = P->degree_min;
  BTK_CHECK(dlo >= 1 && dlo <= n, BTK_ERR_INVALID_ARGUMENT, "degree_min must be in [1, interp_degree]");
  const int nd = n - dlo + 1;
  const int ncs = (int)S.clusters.size(), nct = (int)T.clusters.size();
  auto sz = [&](int d) { return (long long)ipow(d + 1, dim); };
  // Slot tables: cluster-major, degrees dlo..n.
  auto make_slots = [&](const std::vector<int>& slot_panels, std::vector<int>& panel, std::vector<int>& deg,
                        std::vector<long long>& off, std::vector<int>& begin) {
    const int nc = (int)slot_panels.size();
    long long o = 0;
    begin.resize(nc + 1);
    for (int c = 0; c < nc; ++c) {
      begin[c] = c * nd;
      for (int d = dlo; d <= n; ++d) {
        panel.push_back(slot_panels[c]);
        deg.push_back(d);
        off.push_back(o);
        o += sz(d);
      }
    }
    begin[nc] = nc * nd;
    return o;
  };
  // Leaf pairs the degree choice may approximate: PP pairs that satisfy the
  // traversal's MAC form, (r_t + r_s) / |c_t - c_s| < leaf_theta with r the
  // panels' half diagonals (src/interaction_list.cpp:142-156), whose source
  // leaf has more points than the proxies of degree_min. Their source leaves
  // get degree slots after the clusters'.
  std::vector<int> conv;                         // PP pair indices
  std::vector<int> slot_panels_s(S.clusters);    // source panels with degree slots
  std::vector<int> slot_of_s(S.cluster_slot);    // per source panel: its index there (-1: none)
  std::vector<int> slot_panels_t(T.clusters);    // target panels with degree slots
  std::vector<int> slot_of_t(T.cluster_slot);
  int n_conv_cc = 0;
  std::vector<int> pccc, cpcc;  // PC / CP list pairs with a CC form
  if (P->leaf_far) {
    for (int i = 0; i < counts[0]; ++i) {
      const btk_interact_pair& pr = lists[0][i];
      const int tp = pr.target_panel, sp = pr.source_panel;
      BTK_CHECK(tp >= 0 && tp < T.h.panel_count && sp >= 0 && sp < S.h.panel_count, BTK_ERR_INVALID_ARGUMENT,
                "interaction list: panel index out of range");
      if (T.h.point_count[tp] <= 0 || S.h.point_count[sp] <= sz(dlo)) continue;
      const PanelGeom &a = T.h.geom[tp], &b = S.h.geom[sp];
      double d2 = 0, ra = 0, rb = 0;
      for (int d = 0; d < dim; ++d) {
        const double dc = 0.5 * (b.lo[d] + b.hi[d]) - 0.5 * (a.lo[d] + a.hi[d]);
        d2 += dc * dc;
        ra += (a.hi[d] - a.lo[d]) * (a.hi[d] - a.lo[d]);
        rb += (b.hi[d] - b.lo[d]) * (b.hi[d] - b.lo[d]);
      }
      // (leaves within half the target's smallest side of each other stay
      // direct: their entries lead the items, on the near-field path)
      double gap = 0.0, side = 1e300;
      for (int d = 0; d < dim; ++d) {
        gap = std::max(gap, std::max(b.lo[d] - a.hi[d], a.lo[d] - b.hi[d]));
        side = std::min(side, a.hi[d] - a.lo[d]);
      }
      const double dist = std::sqrt(d2);
      if (dist > 0 && gap > 0.5 * side && (0.5 * std::sqrt(ra) + 0.5 * std::sqrt(rb)) / dist < P->leaf_theta)
        conv.push_back(i);
    }
    // Pairs whose target leaf holds more points than the plan degree's
    // proxies also get a CC form (target-leaf proxies x source-leaf proxies,
    // cheaper than the PC form at every degree): they go first, and their
    // target leaves get degree slots after the clusters'.
    std::stable_partition(conv.begin(), conv.end(),
                          [&](int i) { return T.h.point_count[lists[0][i].target_panel] > sz(n); });
    for (int i : conv) {
      const int sp = lists[0][i].source_panel, tp = lists[0][i].target_panel;
      if (slot_of_s[sp] < 0) {
        slot_of_s[sp] = (int)slot_panels_s.size();
        slot_panels_s.push_back(sp);
      }
      if (T.h.point_count[tp] > sz(n)) {
        ++n_conv_cc;
        if (slot_of_t[tp] < 0) {
          slot_of_t[tp] = (int)slot_panels_t.size();
          slot_panels_t.push_back(tp);
        }
      }
    }
    // The same holds for PC pairs (target leaf points x source-cluster
    // proxies): a large target leaf gets the CC form as the other choice.
    for (int i = 0; i < counts[1]; ++i) {
      const int tp = lists[1][i].target_panel;
      BTK_CHECK(tp >= 0 && tp < T.h.panel_count, BTK_ERR_INVALID_ARGUMENT, "interaction list: panel index out of range");
      if (T.h.point_count[tp] <= sz(n)) continue;
      pccc.push_back(i);
      if (slot_of_t[tp] < 0) {
        slot_of_t[tp] = (int)slot_panels_t.size();
        slot_panels_t.push_back(tp);
      }
    }
    // And for CP pairs (target proxies x source leaf points) with a large
    // source leaf, whose leaf then gets degree slots.
    for (int i = 0; i < counts[2]; ++i) {
      const int sp = lists[2][i].source_panel;
      BTK_CHECK(sp >= 0 && sp < S.h.panel_count, BTK_ERR_INVALID_ARGUMENT, "interaction list: panel index out of range");
      if (S.h.point_count[sp] <= sz(n)) continue;
      cpcc.push_back(i);
      if (slot_of_s[sp] < 0) {
        slot_of_s[sp] = (int)slot_panels_s.size();
        slot_panels_s.push_back(sp);
      }
    }
  }
  std::vector<int> s_panel, s_deg, s_begin, t_panel, t_deg, t_begin;
  std::vector<long long> s_off, t_off;
  P->total_src_slots = make_slots(slot_panels_s, s_panel, s_deg, s_off, s_begin);
  P->total_tgt_slots = make_slots(slot_panels_t, t_panel, t_deg, t_off, t_begin);
  P->n_tgt_slot_panels = (int)slot_panels_t.size();
  P->n_conv_cc = n_conv_cc;
  P->n_pccc = (int)pccc.size();
  P->n_cpcc = (int)cpcc.size();
  P->n_src_slots = (int)s_panel.size();
  P->n_tgt_slots = (int)t_panel.size();
  BTK_CHECK(S.n_points + P->total_src_slots < (1LL << 31) && T.n_points + P->total_tgt_slots < (1LL << 31),
            BTK_ERR_UNSUPPORTED, "per-pair degree slots exceed 2^31 entries");
  // Degree transfer matrices A_d[a][i] = L^d_a(x^n_i) (d < n) and unit nodes.
  std::vector<double> amat, ucos;
  std::vector<int> amat_off(kMaxNodes, 0), ucos_off(kMaxNodes, 0);
  const double pi = 3.141592653589793238462643383279502884;
  for (int d = dlo; d <= n; ++d) {
    amat_off[d] = (int)amat.size();
    if (d == n) continue;
    std::vector<double> row(d + 1);
    amat.resize(amat.size() + (size_t)(d + 1) * (n + 1));  // [a][i]: row a, n+1 columns
    for (int i = 0; i <= n; ++i) {
      bary_row_unit(std::cos(pi * i / n), d, row.data());
      for (int a = 0; a <= d; ++a) amat[amat_off[d] + a * (n + 1) + i] = row[a];
    }
  }
  if (amat.empty()) amat.push_back(0.0);
  for (int d = 1; d < kMaxNodes; ++d) {
    ucos_off[d] = (int)ucos.size();
    for (int i = 0; i <= d; ++i) ucos.push_back(std::cos(pi / d * i));
  }
  BTK_TRY(A.upload(&P->d_amat, amat));
  BTK_TRY(A.upload(&P->d_amat_off, amat_off));
  BTK_TRY(A.upload(&P->d_ucos, ucos));
  BTK_TRY(A.upload(&P->d_ucos_off, ucos_off));
  BTK_TRY(A.upload(&P->d_s_slot_panel, s_panel));
  BTK_TRY(A.alloc(&P->d_s_slot_used, (size_t)std::max(P->n_src_slots, 1)));
  BTK_TRY(A.upload(&P->d_s_slot_deg, s_deg));
  BTK_TRY(A.upload(&P->d_s_slot_off, s_off));
  BTK_TRY(A.upload(&P->d_s_cluster_slot_begin, s_begin));
  BTK_TRY(A.upload(&P->d_t_slot_deg, t_deg));
  BTK_TRY(A.upload(&P->d_t_slot_off, t_off));
  BTK_TRY(A.upload(&P->d_t_cluster_slot_begin, t_begin));
  BTK_TRY(A.upload(&P->d_t_cluster_panel, slot_panels_t));

  // Static items: PP and PC (PC entries start at the degree-n slot). The PC
  // block of the per-pair arrays is the PC list, then the leaf pairs (their
  // entries are the PP entries, direct until a degree is chosen).
  P->n_pc_list = counts[1];
  P->n_pc = counts[1] + (int)conv.size();
  P->n_cp = counts[2];
  P->n_far_list = counts[2] + counts[3];
  // CC forms of PC pairs, of CP pairs, then of leaf pairs close the far block
  P->n_far = P->n_far_list + P->n_pccc + P->n_cpcc + n_conv_cc;
  std::vector<long long> pc_begin(P->n_pc_list);
  std::vector<int> pc_src_cluster(P->n_pc), pc_direct(2 * (size_t)std::max(P->n_pc, 1), -1);
  P->h_pc_tcount.resize(P->n_pc);
  for (int i = 0; i < P->n_pc_list; ++i) {
    const int c = S.cluster_slot[lists[1][i].source_panel];
    BTK_CHECK(c >= 0, BTK_ERR_INVALID_ARGUMENT, "PC pair with a leaf source");
    pc_src_cluster[i] = c;
    pc_begin[i] = S.n_points + s_off[s_begin[c] + (n - dlo)];
    P->h_pc_tcount[i] = T.h.point_count[lists[1][i].target_panel];
  }
  P->conv_direct_total = 0;
  for (size_t k = 0; k < conv.size(); ++k) {
    const btk_interact_pair& pr = lists[0][conv[k]];
    const int i = P->n_pc_list + (int)k;
    pc_src_cluster[i] = slot_of_s[pr.source_panel];
    P->h_pc_tcount[i] = T.h.point_count[pr.target_panel];
    pc_direct[2 * i] = S.leaf_begin[pr.source_panel];
    pc_direct[2 * i + 1] = S.h.point_count[pr.source_panel];
    P->conv_direct_total += (int64_t)P->h_pc_tcount[i] * pc_direct[2 * i + 1];
  }
  const int counts_static[4] = {counts[0], counts[1], 0, 0};
  WorkLists W;
  std::vector<int> pc_entry, pp_entry;
  {
    const auto t0 = std::chrono::steady_clock::now();
    BTK_TRY(build_work(T, S, lists, counts_static, slots, W, &pc_begin, &pc_entry, P->work_split,
                       conv.empty() ? nullptr : &pp_entry, P->ictx.tile));
    P->build_ms_work += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
  for (int i : conv) {
    BTK_CHECK(pp_entry[i] >= 0, BTK_ERR_INTERNAL, "leaf pair without a work-list entry");
    pc_entry.push_back(pp_entry[i]);
  }
  BTK_TRY(A.upload(&P->d_pc_direct, pc_direct));
  P->h_pc_direct = pc_direct;
  P->h_conv = conv;
  P->evals[0] = W.evals[0];
  P->evals_pp_static = W.evals[0];
  P->n_static_items = (int)W.items.size();
  P->n_static_entries = (int)W.entries.size();
  // Far pairs: CP then CC.
  std::vector<int> far_type(P->n_far), far_tgt(P->n_far), far_src(2 * (size_t)P->n_far);
  P->h_cp_scount.resize(P->n_cp);
  for (int i = 0; i < P->n_far_list; ++i) {
    const bool cp = i < P->n_cp;
    const btk_interact_pair& pr = cp ? lists[2][i] : lists[3][i - P->n_cp];
    BTK_CHECK(pr.target_panel >= 0 && pr.target_panel < T.h.panel_count && pr.source_panel >= 0 &&
                  pr.source_panel < S.h.panel_count,
              BTK_ERR_INVALID_ARGUMENT, "interaction list: panel index out of range");
    far_type[i] = cp ? 2 : 3;
    far_tgt[i] = T.cluster_slot[pr.target_panel];
    BTK_CHECK(far_tgt[i] >= 0, BTK_ERR_INVALID_ARGUMENT, "CP/CC pair with a leaf target");
    if (cp) {
      BTK_CHECK(S.h.is_leaf[pr.source_panel], BTK_ERR_INVALID_ARGUMENT, "CP pair with a non-leaf source");
      far_src[2 * i] = S.leaf_begin[pr.source_panel];
      far_src[2 * i + 1] = S.h.point_count[pr.source_panel];
      P->h_cp_scount[i] = S.h.point_count[pr.source_panel];
    } else {
      far_src[2 * i] = S.cluster_slot[pr.source_panel];
      BTK_CHECK(far_src[2 * i] >= 0, BTK_ERR_INVALID_ARGUMENT, "CC pair with a leaf source");
      far_src[2 * i + 1] = 0;
    }
  }
  for (int k = 0; k < P->n_pccc; ++k) {
    const btk_interact_pair& pr = lists[1][pccc[k]];
    const int i = P->n_far_list + k;
    far_type[i] = 3;
    far_tgt[i] = slot_of_t[pr.target_panel];
    far_src[2 * i] = S.cluster_slot[pr.source_panel];
    BTK_CHECK(far_src[2 * i] >= 0, BTK_ERR_INVALID_ARGUMENT, "PC pair with a leaf source");
    far_src[2 * i + 1] = 0;
  }
  for (int k = 0; k < P->n_cpcc; ++k) {
    const btk_interact_pair& pr = lists[2][cpcc[k]];
    const int i = P->n_far_list + P->n_pccc + k;
    far_type[i] = 3;
    far_tgt[i] = T.cluster_slot[pr.target_panel];
    BTK_CHECK(far_tgt[i] >= 0, BTK_ERR_INVALID_ARGUMENT, "CP pair with a leaf target");
    far_src[2 * i] = slot_of_s[pr.source_panel];
    far_src[2 * i + 1] = 0;
  }
  {
    std::vector<int> ix(std::max<size_t>(pccc.size(), 1), 0), cf(ix.size(), 0);
    for (size_t k = 0; k < pccc.size(); ++k) {
      ix[k] = pccc[k];
      cf[k] = T.h.point_count[lists[1][pccc[k]].target_panel];
    }
    BTK_TRY(A.upload(&P->d_pccc_idx, ix));
    BTK_TRY(A.upload(&P->d_pccc_coef, cf));
    std::vector<int> jx(std::max<size_t>(cpcc.size(), 1), 0), cg(jx.size(), 0);
    for (size_t k = 0; k < cpcc.size(); ++k) {
      jx[k] = P->n_pc + cpcc[k];  // CP entry in the pair array: after the PC block
      cg[k] = S.h.point_count[lists[2][cpcc[k]].source_panel];
    }
    BTK_TRY(A.upload(&P->d_cpcc_idx, jx));
    BTK_TRY(A.upload(&P->d_cpcc_coef, cg));
  }
  for (int k = 0; k < n_conv_cc; ++k) {
    const btk_interact_pair& pr = lists[0][conv[k]];
    const int i = P->n_far_list + P->n_pccc + P->n_cpcc + k;
    far_type[i] = 3;
    far_tgt[i] = slot_of_t[pr.target_panel];
    far_src[2 * i] = slot_of_s[pr.source_panel];
    far_src[2 * i + 1] = 0;
  }
  const int n_tsp = P->n_tgt_slot_panels;
  std::vector<double> centre(3 * (size_t)std::max(n_tsp, 1), 0.0);
  for (int c = 0; c < n_tsp; ++c)
    for (int d = 0; d < 3; ++d) {
      const PanelGeom& g = T.h.geom[slot_panels_t[c]];
      centre[3 * c + d] = 0.5 * (g.lo[d] + g.hi[d]);
    }
  P->tiles_max = (int)((sz(n) + P->ictx.tile - 1) / P->ictx.tile);
  BTK_TRY(A.upload(&P->d_pc_entry, pc_entry));
  BTK_TRY(A.upload(&P->d_pc_src_cluster, pc_src_cluster));
  BTK_TRY(A.upload(&P->d_far_type, far_type));
  BTK_TRY(A.upload(&P->d_far_tgt, far_tgt));
  BTK_TRY(A.upload(&P->d_far_src, far_src));
  BTK_TRY(A.upload(&P->d_tgt_centre, centre));
  const size_t n_items = (size_t)P->n_static_items + (size_t)P->n_far * P->tiles_max;
  AuditWork audit;
  build_audit_work(P, P->n_static_entries + P->n_far, audit);
  const size_t n_audit_items = audit.items.size(), n_audit_entries = audit.entries.size();
  BTK_CHECK(n_items + n_audit_items < (1u << 31), BTK_ERR_UNSUPPORTED, "too many work items");
  // items: [static PP/PC | far CP/CC tiles | audit]; entries: [static | far | audit]
  BTK_TRY(A.alloc(&P->ictx.d_items, std::max<size_t>(n_items + n_audit_items, 1)));
  BTK_TRY(A.alloc(&P->ictx.d_entries,
                  std::max<size_t>((size_t)P->n_static_entries + P->n_far + n_audit_entries, 1)));
  if (!W.items.empty())
    BTK_CUDA(cudaMemcpyAsync(P->ictx.d_items, W.items.data(), sizeof(WorkItem) * W.items.size(),
                             cudaMemcpyHostToDevice, st));
  if (!W.entries.empty())
    BTK_CUDA(cudaMemcpyAsync(P->ictx.d_entries, W.entries.data(), sizeof(Entry) * W.entries.size(),
                             cudaMemcpyHostToDevice, st));
  P->ictx.n_items = (int)n_items;
  P->n_items_main = (int)n_items;
  // Degrees in force: all at n until set.
  P->h_deg_pc.assign(P->n_pc, n);
  std::fill(P->h_deg_pc.begin() + P->n_pc_list, P->h_deg_pc.end(), 0);  // leaf pairs: direct
  P->h_deg_far.assign(P->n_far, n);
  std::fill(P->h_deg_far.begin() + P->n_far_list, P->h_deg_far.end(), 0);  // leaf pairs' CC forms: not taken
  P->n_pairs = P->n_pc + P->n_far;
  {
    std::vector<int> all(std::max(P->n_pairs, 1), n);
    std::fill(all.begin() + P->n_pc_list, all.begin() + P->n_pc, 0);
    std::fill(all.begin() + P->n_pc + P->n_far_list, all.begin() + P->n_pairs, 0);
    BTK_TRY(A.upload(&P->d_deg_pc, all));  // one array: PC (list, leaf pairs) degrees, then CP, then CC
    P->d_deg_far = P->d_deg_pc + P->n_pc;
  }
  recount_far_evals(P);
  // Selector inputs: pair classes and panels (PC, CP, CC), per-pair point counts.
  {
    std::vector<int> ty(std::max(P->n_pairs, 1)), tg(std::max(P->n_pairs, 1)), sr(std::max(P->n_pairs, 1));
    for (int i = 0; i < P->n_pc; ++i) {
      const btk_interact_pair& pr = i < P->n_pc_list ? lists[1][i] : lists[0][conv[i - P->n_pc_list]];
      ty[i] = 1;
      tg[i] = pr.target_panel;
      sr[i] = pr.source_panel;
    }
    for (int i = 0; i < P->n_far; ++i) {
      const bool cp = i < P->n_cp;
      const btk_interact_pair& pr =
          cp ? lists[2][i]
             : (i < P->n_far_list
                    ? lists[3][i - P->n_cp]
                    : (i < P->n_far_list + P->n_pccc
                           ? lists[1][pccc[i - P->n_far_list]]
                           : (i < P->n_far_list + P->n_pccc + P->n_cpcc
                                  ? lists[2][cpcc[i - P->n_far_list - P->n_pccc]]
                                  : lists[0][conv[i - P->n_far_list - P->n_pccc - P->n_cpcc]])));
      ty[P->n_pc + i] = cp ? 2 : 3;
      tg[P->n_pc + i] = pr.target_panel;
      sr[P->n_pc + i] = pr.source_panel;
    }
    BTK_TRY(A.upload(&P->d_pair_type, ty));
    BTK_TRY(A.upload(&P->d_pair_tgt, tg));
    BTK_TRY(A.upload(&P->d_pair_src, sr));
    // Cost-aware degree rule: each pair's weight (targets carrying its error)
    // and the mean cost and weight that normalise its objective.
    std::vector<int> wt(std::max(P->n_pairs, 1), 1);
    double csum = 0, wsum = 0;
    const double m = (double)P->degree + 1, md = dim == 3 ? m * m * m : m * m;
    for (int i = 0; i < P->n_pairs; ++i) {
      wt[i] = std::max(1, T.h.point_count[tg[i]]);
      wsum += wt[i];
      csum += i < P->n_pc ? md * P->h_pc_tcount[i]
                          : (i < P->n_pc + P->n_cp ? md * P->h_cp_scount[i - P->n_pc] : md * md);
    }
    if (P->n_pairs > 0) {
      P->inv_cbar = (float)(P->n_pairs / std::max(csum, 1.0));
      P->inv_wbar = (float)(P->n_pairs / std::max(wsum, 1.0));
    }
    BTK_TRY(A.upload(&P->d_pair_weight, wt));
    std::vector<int> tc(P->h_pc_tcount), sc(P->h_cp_scount);
    tc.push_back(0);
    sc.push_back(0);
    BTK_TRY(A.upload(&P->d_pc_tcount, tc));
    BTK_TRY(A.upload(&P->d_cp_scount, sc));
    BTK_TRY(A.alloc(&P->d_desc, (size_t)S.h.panel_count * 6));
    BTK_TRY(A.alloc(&P->d_feat, (size_t)std::max(P->n_pairs, 1) * 16));
    BTK_TRY(A.alloc(&P->d_pred, (size_t)std::max(P->n_pairs, 1) * 9));
    BTK_TRY(A.alloc(&P->d_evals, 2));
    BTK_TRY(A.alloc(&P->d_gsum, 2));
    BTK_TRY(A.upload(&P->d_cluster_slot_s, slot_of_s));
    BTK_TRY(A.upload(&P->d_cluster_slot_t, slot_of_t));
    const PanelGeom& g = S.h.geom[0];
    double r2 = 0;
    for (int d = 0; d < dim; ++d) {
      r2 += (g.hi[d] - g.lo[d]) * (g.hi[d] - g.lo[d]);
      P->root_centre[d] = 0.5 * (g.lo[d] + g.hi[d]);
    }
    P->root_radius = std::max(0.5 * std::sqrt(r2), 1e-300);
  }
  BTK_TRY(setup_audit(P, A, audit, P->n_items_main, P->n_static_entries + P->n_far, st));
  BTK_CUDA(cudaStreamSynchronize(st));  // the copies read the audit's host vectors
  // Work arrays.
  BTK_TRY(A.alloc(&P->d_S4, (size_t)S.n_points + P->total_src_slots + 1));
  BTK_TRY(A.alloc(&P->d_T4, (size_t)T.n_points + P->total_tgt_slots + 1));
  BTK_TRY(A.alloc(&P->d_T_out, (size_t)T.n_points + P->total_tgt_slots + 1));
  BTK_TRY(A.alloc(&P->d_ptwm, (size_t)P->ncomp * P->total_tgt_slots + 1));
  if (T.n_points)
    BTK_CUDA(cudaMemcpyAsync(P->d_T_out, T.d_perm, sizeof(int) * T.n_points, cudaMemcpyDeviceToDevice, st));
  std::vector<int> t_slot_panel_dev(t_panel);
  int* d_t_slot_panel = nullptr;
  BTK_TRY(A.upload(&d_t_slot_panel, t_slot_panel_dev));
  BTK_CUDA(launch_tgt_slots(dim, P->n_tgt_slots, d_t_slot_panel, P->d_t_slot_deg, P->d_t_slot_off, T.d_panels,
                            P->d_ucos, P->d_ucos_off, P->d_T4, P->d_T_out, T.n_points, st));
  return BTK_OK;
}

btk_status plan_build(btk_plan* P, const btk_plan_desc* D, cudaStream_t st) {
  const btk_run_config& cfg = D->cfg;
  BTK_CHECK(cfg.dim == 2 || cfg.dim == 3, BTK_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
  BTK_TRY(validate_cfg(&cfg, cfg.dim));
  BTK_CHECK(D->kind >= 0 && D->kind <= 2, BTK_ERR_INVALID_ARGUMENT, "bad kind");
  BTK_CHECK(!(D->kind == BTK_KIND_VEL && cfg.dim != 3), BTK_ERR_UNSUPPORTED, "VEL kernel is 3-D only");
  BTK_CHECK(D->precision == BTK_PREC_FP64 || D->precision == BTK_PREC_MIXED, BTK_ERR_UNSUPPORTED,
            "precision must be BTK_PREC_FP64 or BTK_PREC_MIXED");
  BTK_CHECK(D->tree_target && D->panels_target && D->point_leaf_panel_source, BTK_ERR_INVALID_ARGUMENT,
            "plan: missing tree arrays");
  BTK_CHECK(D->panel_points_inside_target || D->panels_source == nullptr, BTK_ERR_INVALID_ARGUMENT,
            "plan: panel_points_inside_target may be NULL only with one tree (leaf order from point_leaf_panel)");
  P->dim = cfg.dim;
  P->degree = cfg.interp_degree;
  P->m = P->degree + 1;
  P->ipc = cfg.interp_point_count;
  P->kind = D->kind;
  P->precision = D->precision;
  P->ncomp = ncomp_of(cfg.dim, D->kind);
  P->thresh = cfg.fmm_cluster_thresh;
  P->eps = cfg.ker_eps;
  P->stream = st;
  P->same_tree = D->panels_source == nullptr;
  P->arena.reset(new Arena(st));
  Arena& A = *P->arena;

  host_tree_from_panels(cfg.dim, D->panels_target, D->tree_target->panel_count, D->tree_target->level_start,
                        D->tree_target->levels, P->tgt.h);
  BTK_TRY(side_layout(P->tgt, D->point_count_target, P->degree));
  BTK_TRY(side_upload(P->tgt, A, D->panel_points_inside_target, nullptr, P->thresh));
  if (!D->panel_points_inside_target)
    BTK_TRY(side_perm_from_leaf_of(P->tgt, A, std::vector<int>(D->point_leaf_panel_source,
                                                               D->point_leaf_panel_source + D->point_count_target)));
  if (P->same_tree) {
    P->src = &P->tgt;
    BTK_CHECK(D->point_count_source == D->point_count_target, BTK_ERR_INVALID_ARGUMENT,
              "one tree but different point counts");
  } else {
    BTK_CHECK(D->tree_source && D->panel_points_inside_source, BTK_ERR_INVALID_ARGUMENT, "plan: missing source tree");
    host_tree_from_panels(cfg.dim, D->panels_source, D->tree_source->panel_count, D->tree_source->level_start,
                          D->tree_source->levels, P->src_own.h);
    BTK_TRY(side_layout(P->src_own, D->point_count_source, P->degree));
    BTK_TRY(side_upload(P->src_own, A, D->panel_points_inside_source, nullptr, P->thresh));
    P->src = &P->src_own;
  }
  Side& T = P->tgt;
  Side& S = *P->src;
  const int nct = (int)T.clusters.size(), ncs = (int)S.clusters.size();
  const int Pt = T.h.panel_count, Ps = S.h.panel_count;

  // Work lists.
  const btk_interact_pair* lists[4] = {D->pp_list, D->pc_list, D->cp_list, D->cc_list};
  const int counts[4] = {cfg.fmm_pp_count, cfg.fmm_pc_count, cfg.fmm_cp_count, cfg.fmm_cc_count};
  for (int t = 0; t < 4; ++t) BTK_CHECK(counts[t] >= 0 && (counts[t] == 0 || lists[t]), BTK_ERR_INVALID_ARGUMENT,
                                        "plan: missing interaction list");
  const bool guard = P->eps * P->eps < 1.1754943508222875e-38;
  BTK_CHECK(D->tile_targets == 0 || D->tile_targets == 128 || D->tile_targets == 256, BTK_ERR_INVALID_ARGUMENT,
            "tile_targets must be 0, 128 or 256");
  P->ictx.tile = D->tile_targets ? D->tile_targets : kTile;
  const int slots =
      num_sms() * std::max(1, interact_blocks_per_sm(P->dim, P->kind, P->precision, guard, P->ictx.tile));
  P->ictx.dim = P->dim;
  P->ictx.kind = P->kind;
  P->ictx.precision = P->precision;
  P->ictx.eps = P->eps;
  BTK_TRY(A.alloc(&P->d_ticket_status, 3));  // ticket, status, audit ticket
  BTK_CUDA(cudaMemsetAsync(P->d_ticket_status, 0, 3 * sizeof(int), st));
  P->ictx.d_ticket_status = P->d_ticket_status;
  BTK_TRY(A.alloc(&P->d_psw, (size_t)Ps * P->ipc));
  BTK_TRY(A.alloc(&P->d_ptw, (size_t)P->ncomp * Pt * P->ipc));
  P->degree_mode = D->degree_mode;
  P->leaf_far = D->degree_mode == BTK_DEGREE_PER_PAIR && D->leaf_far_pairs ? 1 : 0;
  BTK_CHECK(std::isfinite(D->leaf_far_theta), BTK_ERR_INVALID_ARGUMENT, "leaf_far_theta must be finite");
  P->leaf_theta = D->leaf_far_theta > 0 ? D->leaf_far_theta : std::max(cfg.fmm_theta, 0.8);
  P->degree_min = D->degree_min;
  BTK_CHECK(D->work_split >= 0 && D->work_split <= 1024, BTK_ERR_INVALID_ARGUMENT, "work_split outside 0..1024");
  P->work_split = D->work_split > 0 ? D->work_split : 8;
  BTK_CHECK(D->degree_mode == BTK_DEGREE_FIXED || D->degree_mode == BTK_DEGREE_PER_PAIR, BTK_ERR_INVALID_ARGUMENT,
            "bad degree_mode");

  if (D->degree_mode == BTK_DEGREE_FIXED) {
    WorkLists W;
    const auto t0 = std::chrono::steady_clock::now();
    // CC pairs grouped by geometry leave the pairwise work lists.
    int counts_w[4] = {counts[0], counts[1], counts[2], counts[3]};
    if (D->cc_operators && counts[3] > 0) {
      std::vector<int> group_of;
      int ng = 0;
      if (cc_group_pairs(T.h, S.h, lists[3], counts[3], group_of, ng)) {
        for (int i = 0; i < counts[3]; ++i) {
          const btk_interact_pair& pr = lists[3][i];
          BTK_CHECK(!T.h.is_leaf[pr.target_panel] && !S.h.is_leaf[pr.source_panel], BTK_ERR_INVALID_ARGUMENT,
                    "interaction list: CC pair with a leaf panel");
        }
        std::vector<CcTask> tasks;
        std::vector<CcPair> pairs;
        cc_build_tasks(lists[3], counts[3], group_of, ng, cc_pairs_per_task(P->dim, P->kind), tasks, pairs,
                       P->cc_bucket_end);
        BTK_TRY(A.upload(&P->d_cc_tasks, tasks));
        BTK_TRY(A.upload(&P->d_cc_pairs, pairs));
        P->n_cc_groups = ng;
        P->n_cc_tasks = (int)tasks.size();
        counts_w[3] = 0;
      }
    }
    BTK_TRY(build_work(T, S, lists, counts_w, slots, W, nullptr, nullptr, P->work_split, nullptr, P->ictx.tile));
    P->build_ms_work += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    for (int t = 0; t < 4; ++t) P->evals[t] = W.evals[t];
    if (P->n_cc_tasks > 0) P->evals[3] = (int64_t)counts[3] * P->ipc * P->ipc;
    P->ictx.n_items = (int)W.items.size();
    BTK_TRY(A.upload(&P->ictx.d_items, W.items));
    BTK_TRY(A.upload(&P->ictx.d_entries, W.entries));
    BTK_TRY(A.alloc(&P->d_S4, (size_t)S.n_points + (size_t)ncs * P->ipc));
    BTK_TRY(A.alloc(&P->d_T4, (size_t)T.n_points + (size_t)nct * P->ipc));
    BTK_TRY(A.alloc(&P->d_T_out, (size_t)T.n_points + (size_t)nct * P->ipc));
    if (T.n_points)
      BTK_CUDA(cudaMemcpyAsync(P->d_T_out, T.d_perm, sizeof(int) * T.n_points, cudaMemcpyDeviceToDevice, st));
    BTK_CUDA(launch_tgt_proxies(P->dim, P->degree, nct, T.d_clusters, T.d_nodes_shift, P->d_T4 + T.n_points,
                                P->d_T_out + T.n_points, st));
  } else {
    BTK_TRY(plan_build_per_pair(P, lists, counts, slots, st));
  }
  for (int i = 0; i < 6; ++i) BTK_CUDA(cudaEventCreate(&P->ev[i]));
  BTK_CUDA(cudaStreamSynchronize(st));
  return BTK_OK;
}

// Upward pass on a side whose sorted points (S4 prefix) are in place.
btk_status run_upward(const Side& S, const double4* pts, double* psw, cudaStream_t st) {
  BTK_CUDA(launch_leaf_moments(S.h.dim, S.degree, (int)S.leaves.size(), S.d_leaves, S.d_leaf_begin, S.d_point_count,
                               pts, S.d_nodes_interp, psw, st));
  for (int l = S.h.levels - 2; l >= 0; --l)
    BTK_CUDA(launch_c2p(S.h.dim, S.degree, (int)S.nonleaf_by_level[l].size(), S.d_nonleaf_by_level[l], S.d_child,
                        S.d_xfer, psw, st));
  return BTK_OK;
}

btk_status run_downward(const Side& T, int ncomp, const double4* pts, Ptr4 ptw, Ptr4 out, cudaStream_t st) {
  for (int l = 1; l < T.h.levels; ++l)
    BTK_CUDA(launch_p2c(T.h.dim, T.degree, ncomp, (int)T.panels_by_level[l].size(), T.d_panels_by_level[l],
                        T.d_parent, T.d_xfer, ptw, T.ipc, st));
  BTK_CUDA(launch_l2p(T.h.dim, T.degree, ncomp, (int)T.leaves.size(), T.d_leaves, T.d_leaf_begin, T.d_point_count,
                      pts, T.d_perm, T.d_nodes_interp, ptw, out, st));
  return BTK_OK;
}

}  // namespace

extern "C" {

btk_status btk_plan_create(btk_plan** plan, const btk_plan_desc* desc, btk_stream_t stream) {
  BTK_CHECK(plan && desc, BTK_ERR_INVALID_ARGUMENT, "btk_plan_create: null argument");
  *plan = nullptr;
  btk_plan* P = new btk_plan();
  const auto t0 = std::chrono::steady_clock::now();
  btk_status s = plan_build(P, desc, (cudaStream_t)stream);
  if (s != BTK_OK) {
    btk_plan_destroy(P);
    return s;
  }
  P->build_ms_total = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *plan = P;
  return BTK_OK;
}

btk_status btk_plan_destroy(btk_plan* plan) {
  if (!plan) return BTK_OK;
  cudaDeviceSynchronize();
  for (auto& e : plan->ev)
    if (e) cudaEventDestroy(e);
  plan->arena.reset();
  cudaStreamSynchronize(plan->stream);
  delete plan;
  return BTK_OK;
}

btk_status btk_plan_stats_get(const btk_plan* plan, btk_plan_stats* st) {
  BTK_CHECK(plan && st, BTK_ERR_INVALID_ARGUMENT, "null argument");
  st->evals_pp = plan->evals[0];
  st->evals_pc = plan->evals[1];
  st->evals_cp = plan->evals[2];
  st->evals_cc = plan->evals[3];
  st->work_items = plan->ictx.n_items;
  st->device_bytes = (int64_t)plan->arena->bytes;
  st->levels_target = plan->tgt.h.levels;
  st->levels_source = plan->src->h.levels;
  st->build_ms_total = plan->build_ms_total;
  st->build_ms_work = plan->build_ms_work;
  st->cc_groups = plan->n_cc_groups;
  st->cc_tasks = plan->n_cc_tasks;
  st->leaf_far_pairs = plan->n_pc - plan->n_pc_list;
  return BTK_OK;
}

btk_status btk_plan_execute(btk_plan* P, const double* xt, const double* yt, const double* zt, const double* xs,
                            const double* ys, const double* zs, const double* charges, double* out,
                            btk_stream_t stream) {
  BTK_CHECK(P && xt && yt && xs && ys && charges && out, BTK_ERR_INVALID_ARGUMENT, "btk_plan_execute: null argument");
  BTK_CHECK(P->dim == 2 || (zt && zs), BTK_ERR_INVALID_ARGUMENT, "btk_plan_execute: null z coordinates");
  cudaStream_t st = (cudaStream_t)stream;
  Side& T = P->tgt;
  Side& S = *P->src;
  const int Pt = T.h.panel_count;
  if (P->deg_learned) {
    // A learned solve left its own degrees and forms on the device: this
    // solve uses the ones set by btk_plan_set_degrees / btk_plan_set_leaf_forms.
    BTK_CUDA(cudaMemcpyAsync(P->d_deg_pc, P->h_deg_pc.data(), sizeof(int) * P->n_pc, cudaMemcpyHostToDevice, st));
    BTK_CUDA(cudaMemcpyAsync(P->d_deg_far, P->h_deg_far.data(), sizeof(int) * P->n_far, cudaMemcpyHostToDevice, st));
    P->deg_learned = false;
  }
  BTK_CUDA(cudaMemsetAsync(P->d_ticket_status + 1, 0, sizeof(int), st));  // this solve's device status
  BTK_CUDA(cudaEventRecord(P->ev[0], st));
  // Upward.
  BTK_CUDA(launch_gather(S.n_points, S.d_perm, xs, ys, P->dim == 3 ? zs : nullptr, charges, P->d_S4, st));
  BTK_CUDA(cudaMemsetAsync(P->d_psw, 0, sizeof(double) * (size_t)S.h.panel_count * P->ipc, st));
  BTK_TRY(run_upward(S, P->d_S4, P->d_psw, st));
  const bool per_pair = P->degree_mode == BTK_DEGREE_PER_PAIR;
  if (!per_pair) {
    BTK_CUDA(launch_src_proxies(P->dim, P->degree, (int)S.clusters.size(), S.d_clusters, S.d_nodes_shift, P->d_psw,
                                P->d_S4 + S.n_points, st));
  } else {
    // Work items for the degrees in force (marking the source slots they
    // read), then those slots.
    BTK_CUDA(cudaMemsetAsync(P->d_s_slot_used, 0, sizeof(int) * (size_t)std::max(P->n_src_slots, 1), st));
    BTK_CUDA(launch_resolve(P->dim, P->n_pc, P->d_pc_entry, P->d_pc_src_cluster, P->d_deg_pc, P->d_pc_direct,
                            P->n_far, P->tiles_max,
                            P->d_far_type, P->d_far_tgt, P->d_far_src, P->d_deg_far, P->d_s_slot_off,
                            P->d_s_cluster_slot_begin, P->d_t_slot_off, P->d_t_cluster_slot_begin, P->degree_min,
                            T.n_points, S.n_points, P->d_tgt_centre, P->n_static_items, P->ictx.d_items,
                            P->ictx.d_entries, P->n_static_items, P->n_static_entries, P->d_s_slot_used,
                            P->ictx.tile, st));
    BTK_CUDA(launch_src_slots(P->dim, P->degree, P->n_src_slots, P->d_s_slot_panel, P->d_s_slot_deg, P->d_s_slot_off,
                              S.d_panels, P->d_psw, P->d_amat, P->d_amat_off, P->d_ucos, P->d_ucos_off,
                              P->d_s_slot_used, P->d_S4 + S.n_points, st));
  }
  BTK_CUDA(cudaEventRecord(P->ev[1], st));
  // Interactions.
  BTK_CUDA(launch_gather(T.n_points, T.d_perm, xt, yt, P->dim == 3 ? zt : nullptr, nullptr, P->d_T4, st));
  BTK_CUDA(cudaMemsetAsync(P->d_ptw, 0, sizeof(double) * (size_t)P->ncomp * Pt * P->ipc, st));
  BTK_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)P->ncomp * T.n_points, st));
  Ptr4 o{}, w{}, wm{};
  for (int c = 0; c < P->ncomp; ++c) {
    o.p[c] = out + (size_t)c * T.n_points;
    w.p[c] = P->d_ptw + (size_t)c * Pt * P->ipc;
    if (per_pair) wm.p[c] = P->d_ptwm + (size_t)c * P->total_tgt_slots;
  }
  if (per_pair) BTK_CUDA(cudaMemsetAsync(P->d_ptwm, 0, sizeof(double) * (size_t)P->ncomp * P->total_tgt_slots, st));
  // The kernel-tight pair is recorded only when there is a launch to bracket.
  BTK_CUDA(cudaEventRecord(P->ev[4], st));
  BTK_CUDA(cudaEventRecord(P->ev[5], st));
  BTK_TRY(run_interactions(P->ictx, P->d_S4, P->d_T4, P->d_T_out, o, per_pair ? wm : w, st, P->ev[4], P->ev[5]));
  if (P->n_cc_tasks > 0) {
    CcParams cp{};
    cp.tasks = P->d_cc_tasks;
    cp.pairs = P->d_cc_pairs;
    cp.nodes_t = T.d_nodes_shift;
    cp.nodes_s = S.d_nodes_shift;
    cp.psw = P->d_psw;
    cp.ptw = w;
    cp.eps2 = P->eps * P->eps;
    kind_scales(P->dim, P->kind, cp.scale);
    cp.m = P->m;
    cp.ipc = P->ipc;
    BTK_CUDA(launch_cc_groups(P->dim, P->kind, cp.eps2 < 1.1754943508222875e-38, P->precision == BTK_PREC_MIXED, cp,
                              P->cc_bucket_end, st));
  }
  if (per_pair)
    BTK_CUDA(launch_promote(P->dim, P->degree, P->ncomp, P->n_tgt_slot_panels, P->d_t_cluster_panel,
                            P->d_t_cluster_slot_begin, P->d_t_slot_deg, P->d_t_slot_off, P->d_amat, P->d_amat_off,
                            wm, w, st));
  BTK_CUDA(cudaEventRecord(P->ev[2], st));
  // Downward.
  BTK_TRY(run_downward(T, P->ncomp, P->d_T4, w, o, st));
  BTK_CUDA(cudaEventRecord(P->ev[3], st));
  P->timed = true;
  return BTK_OK;
}

}  // extern "C"

namespace {

// The audit: a fixed, seeded 1% sample of the targets (at least one when
// there are targets), spread evenly over the index range, and work items for
// its FP64 direct sum over every source, built on the host at plan creation:
// tiles of the plan's tile size of sampled targets x pieces of kAuditPiece consecutive sources
// of the leaf-ordered source array (kItemAudit | kItemAtomic; the interaction
// kernels evaluate them in FP64 whatever the plan's precision).
constexpr int kAuditPiece = 4096;

void build_audit_work(const btk_plan* P, int entry_base, AuditWork& W) {
  const int nt = P->tgt.n_points, ns = P->src->n_points;
  const int na = nt > 0 ? std::max(1, nt / 100) : 0;
  W.orig.assign(na, 0);
  // Evenly spread, seeded offsets (SplitMix64-style hash) over the index range.
  for (int k = 0; k < na; ++k) {
    uint64_t z = 0x9E3779B97F4A7C15ULL * (uint64_t)(k + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    const int64_t lo = (int64_t)k * nt / na, hi = (int64_t)(k + 1) * nt / na;
    W.orig[k] = (int)(lo + (int64_t)(z % (uint64_t)std::max<int64_t>(1, hi - lo)));
  }
  for (int s0 = 0; s0 < ns; s0 += kAuditPiece) W.entries.push_back(Entry{s0, std::min(kAuditPiece, ns - s0)});
  const int tile = P->ictx.tile;
  for (int t0 = 0; t0 < na; t0 += tile)
    for (int e = 0; e < (int)W.entries.size(); ++e) {
      WorkItem w{};
      w.t_begin = t0;
      w.t_count = std::min(tile, na - t0);
      w.e_begin = entry_base + e;
      w.e_end = entry_base + e + 1;
      w.s_total = W.entries[e].s_count;
      w.flags = kItemAtomic | kItemAudit;
      W.items.push_back(w);
    }
}

// Uploads the audit sample and its work items into ictx's arrays at
// item_base / entry_base (capacity reserved by the caller). The caller
// synchronises the stream before W goes out of scope.
btk_status setup_audit(btk_plan* P, Arena& A, const AuditWork& W, int item_base, int entry_base, cudaStream_t st) {
  const int na = (int)W.orig.size();
  BTK_TRY(A.upload(&P->d_audit_orig, W.orig.empty() ? std::vector<int>{0} : W.orig));
  BTK_TRY(A.alloc(&P->d_audit_T4, (size_t)std::max(na, 1)));
  BTK_TRY(A.alloc(&P->d_audit_out, (size_t)P->ncomp * std::max(na, 1)));
  BTK_TRY(A.alloc(&P->d_audit_sums, 2));
  BTK_TRY(A.alloc(&P->d_report, kMaxNodes));
  if (!W.items.empty()) {
    BTK_CUDA(cudaMemcpyAsync(P->ictx.d_items + item_base, W.items.data(), sizeof(WorkItem) * W.items.size(),
                             cudaMemcpyHostToDevice, st));
    BTK_CUDA(cudaMemcpyAsync(P->ictx.d_entries + entry_base, W.entries.data(), sizeof(Entry) * W.entries.size(),
                             cudaMemcpyHostToDevice, st));
  }
  P->n_audit = na;
  P->n_audit_items = (int)W.items.size();
  return BTK_OK;
}

}  // namespace

extern "C" {

btk_status btk_selector_create(btk_selector** out, const float* params, const float* norm) {
  BTK_CHECK(out && params && norm, BTK_ERR_INVALID_ARGUMENT, "btk_selector_create: null argument");
  const int np = selector_param_count();
  std::vector<uint16_t> bf(np);
  for (int i = 0; i < np; ++i) {  // round to nearest even BF16
    uint32_t u;
    std::memcpy(&u, &params[i], 4);
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7FFFu + lsb;
    bf[i] = (uint16_t)(u >> 16);
  }
  btk_selector* s = new btk_selector();
  std::memcpy(s->norm, norm, sizeof(s->norm));
  cudaError_t e = cudaMalloc(&s->d_w, sizeof(uint16_t) * np);
  if (e == cudaSuccess) e = cudaMemcpy(s->d_w, bf.data(), sizeof(uint16_t) * np, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(s->d_w);
    delete s;
    return cuda_error(e, "btk_selector_create");
  }
  *out = s;
  return BTK_OK;
}

btk_status btk_selector_destroy(btk_selector* s) {
  if (!s) return BTK_OK;
  cudaFree(s->d_w);
  delete s;
  return BTK_OK;
}

const void* btk_selector_weights(const btk_selector* s) { return s ? s->d_w : nullptr; }

btk_status btk_selector_predict(const btk_selector* s, int n, const float* features, float* out,
                                btk_stream_t stream) {
  BTK_CHECK(s && n >= 0 && (n == 0 || (features && out)), BTK_ERR_INVALID_ARGUMENT,
            "btk_selector_predict: bad argument");
  BTK_CUDA(launch_mlp_infer(n, s->d_w, s->norm, features, out, nullptr, (cudaStream_t)stream));
  return BTK_OK;
}

btk_status btk_plan_pair_count(const btk_plan* P, int* n_pairs) {
  BTK_CHECK(P && n_pairs, BTK_ERR_INVALID_ARGUMENT, "null argument");
  BTK_CHECK(P->degree_mode == BTK_DEGREE_PER_PAIR, BTK_ERR_INVALID_ARGUMENT, "plan is not BTK_DEGREE_PER_PAIR");
  *n_pairs = P->n_pairs;
  return BTK_OK;
}

// Upward pass, panel descriptors and far-pair features for the given charges.
btk_status btk_plan_pair_features(btk_plan* P, const double* xs, const double* ys, const double* zs,
                                  const double* charges, float* features, btk_stream_t stream) {
  BTK_CHECK(P && xs && ys && charges && features && (P->dim == 2 || zs), BTK_ERR_INVALID_ARGUMENT,
            "btk_plan_pair_features: null argument");
  BTK_CHECK(P->degree_mode == BTK_DEGREE_PER_PAIR, BTK_ERR_INVALID_ARGUMENT, "plan is not BTK_DEGREE_PER_PAIR");
  cudaStream_t st = (cudaStream_t)stream;
  Side& S = *P->src;
  BTK_CUDA(launch_gather(S.n_points, S.d_perm, xs, ys, P->dim == 3 ? zs : nullptr, charges, P->d_S4, st));
  BTK_CUDA(cudaMemsetAsync(P->d_psw, 0, sizeof(double) * (size_t)S.h.panel_count * P->ipc, st));
  BTK_TRY(run_upward(S, P->d_S4, P->d_psw, st));
  BTK_CUDA(launch_panel_desc(P->dim, P->degree, S.h.panel_count, P->d_psw, P->d_desc, st));
  BTK_CUDA(launch_pair_features(P->n_pairs, P->d_pair_type, P->d_pair_tgt, P->d_pair_src, P->tgt.d_panels,
                                S.d_panels, P->root_radius, P->eps, P->d_desc, S.n_points, P->d_S4, P->d_gsum,
                                features, st));
  return BTK_OK;
}

btk_status btk_plan_execute_learned(btk_plan* P, const btk_selector* sel, double tol, double pair_tol, int degree_lo,
                                    const double* xt, const double* yt, const double* zt, const double* xs,
                                    const double* ys, const double* zs, const double* charges, double* out,
                                    btk_learned_report* report, btk_stream_t stream) {
  BTK_CHECK(P && sel && xt && yt && xs && ys && charges && out && (P->dim == 2 || (zt && zs)),
            BTK_ERR_INVALID_ARGUMENT, "btk_plan_execute_learned: null argument");
  BTK_CHECK(P->degree_mode == BTK_DEGREE_PER_PAIR, BTK_ERR_INVALID_ARGUMENT, "plan is not BTK_DEGREE_PER_PAIR");
  BTK_CHECK(tol > 0, BTK_ERR_INVALID_ARGUMENT, "tol must be positive");
  const bool adaptive = !(pair_tol > 0);
  if (adaptive) pair_tol = P->adaptive_pair_tol > 0 ? P->adaptive_pair_tol : kAdaptiveStart * tol;
  cudaStream_t st = (cudaStream_t)stream;
  Side& T = P->tgt;
  Side& S = *P->src;
  const int Pt = T.h.panel_count;
  cudaEvent_t e[4];
  for (auto& x : e) BTK_CUDA(cudaEventCreate(&x));
  BTK_CUDA(cudaMemsetAsync(P->d_ticket_status + 1, 0, sizeof(int), st));  // this solve's device status
  BTK_CUDA(cudaEventRecord(e[0], st));
  P->deg_learned = true;
  // Upward pass and features, then the selector's degrees.
  BTK_TRY(btk_plan_pair_features(P, xs, ys, zs, charges, P->d_feat, stream));
  BTK_CUDA(launch_mlp_infer(P->n_pairs, sel->d_w, sel->norm, P->d_feat, P->d_pred, P->d_ticket_status + 1, st));
  const int lo = std::max(std::max(degree_lo, P->degree_min), 1);
  if (P->degree_rule == BTK_DEGREE_RULE_COST)
    BTK_CUDA(launch_choose_degrees_cost(P->n_pairs, P->dim, P->n_pc, P->n_cp, P->n_pc_list, P->d_pred,
                                        (float)std::log10(pair_tol), lo, P->degree, P->d_pc_tcount, P->d_cp_scount,
                                        P->d_pc_direct, P->d_pair_weight, P->inv_cbar, P->inv_wbar, P->d_deg_pc, st));
  else
    BTK_CUDA(launch_choose_degrees(P->n_pairs, P->d_pred, (float)std::log10(pair_tol), lo, P->degree, P->dim,
                                   P->n_pc_list, P->n_pc, P->d_pc_direct, P->d_deg_pc, st));
  BTK_CUDA(cudaMemsetAsync(P->d_evals, 0, 2 * sizeof(unsigned long long), st));
  BTK_CUDA(cudaMemsetAsync(P->d_report, 0, sizeof(int) * kMaxNodes, st));
  const int cost_rule = P->degree_rule == BTK_DEGREE_RULE_COST ? 1 : 0;
  BTK_CUDA(launch_choose_two_forms(P->n_pccc, P->dim, P->d_pccc_idx, P->d_pccc_coef, -1, P->n_pc + P->n_far_list,
                                   P->d_pred, (float)std::log10(pair_tol), lo, P->degree, cost_rule,
                                   P->d_pair_weight, P->inv_cbar, P->inv_wbar, P->d_deg_pc, st));
  BTK_CUDA(launch_choose_two_forms(P->n_cpcc, P->dim, P->d_cpcc_idx, P->d_cpcc_coef, 0,
                                   P->n_pc + P->n_far_list + P->n_pccc, P->d_pred, (float)std::log10(pair_tol), lo,
                                   P->degree, cost_rule, P->d_pair_weight, P->inv_cbar, P->inv_wbar, P->d_deg_pc,
                                   st));
  BTK_CUDA(launch_choose_leaf_pairs(P->n_pc - P->n_pc_list, P->n_conv_cc, P->dim, P->n_pc_list,
                                    P->n_pc + P->n_far_list + P->n_pccc + P->n_cpcc, P->d_pred,
                                    (float)std::log10(pair_tol), lo,
                                    P->degree,
                                    P->degree_rule == BTK_DEGREE_RULE_COST ? 1 : 0, P->d_pc_tcount, P->d_pc_direct,
                                    P->d_pair_weight, P->inv_cbar, P->inv_wbar, P->d_deg_pc, st));
  BTK_CUDA(launch_far_evals(P->dim, P->n_pc, P->n_cp, P->n_far - P->n_cp, P->n_pc_list, P->n_pc - P->n_pc_list,
                            P->n_conv_cc, P->d_deg_pc, P->d_pc_tcount, P->d_cp_scount, P->d_pc_direct, P->d_evals,
                            P->d_report, st));
  BTK_CUDA(cudaEventRecord(e[1], st));
  // Solve at the chosen degrees.
  Ptr4 o{}, w{}, wm{};
  for (int c = 0; c < P->ncomp; ++c) {
    o.p[c] = out + (size_t)c * T.n_points;
    w.p[c] = P->d_ptw + (size_t)c * Pt * P->ipc;
    wm.p[c] = P->d_ptwm + (size_t)c * P->total_tgt_slots;
  }
  cudaEvent_t ek[2];
  for (auto& x : ek) BTK_CUDA(cudaEventCreate(&x));
  BTK_CUDA(cudaEventRecord(ek[0], st));
  BTK_CUDA(cudaEventRecord(ek[1], st));
  bool first = true;
  auto solve = [&](const InteractCtx& ctx) -> btk_status {
    // Work items for the degrees in force (marking the source slots they
    // read), then those slots.
    BTK_CUDA(cudaMemsetAsync(P->d_s_slot_used, 0, sizeof(int) * (size_t)std::max(P->n_src_slots, 1), st));
    BTK_CUDA(launch_resolve(P->dim, P->n_pc, P->d_pc_entry, P->d_pc_src_cluster, P->d_deg_pc, P->d_pc_direct,
                            P->n_far, P->tiles_max,
                            P->d_far_type, P->d_far_tgt, P->d_far_src, P->d_deg_far, P->d_s_slot_off,
                            P->d_s_cluster_slot_begin, P->d_t_slot_off, P->d_t_cluster_slot_begin, P->degree_min,
                            T.n_points, S.n_points, P->d_tgt_centre, P->n_static_items, P->ictx.d_items,
                            P->ictx.d_entries, P->n_static_items, P->n_static_entries, P->d_s_slot_used,
                            P->ictx.tile, st));
    BTK_CUDA(launch_src_slots(P->dim, P->degree, P->n_src_slots, P->d_s_slot_panel, P->d_s_slot_deg, P->d_s_slot_off,
                              S.d_panels, P->d_psw, P->d_amat, P->d_amat_off, P->d_ucos, P->d_ucos_off,
                              P->d_s_slot_used, P->d_S4 + S.n_points, st));
    BTK_CUDA(launch_gather(T.n_points, T.d_perm, xt, yt, P->dim == 3 ? zt : nullptr, nullptr, P->d_T4, st));
    BTK_CUDA(cudaMemsetAsync(P->d_ptw, 0, sizeof(double) * (size_t)P->ncomp * Pt * P->ipc, st));
    BTK_CUDA(cudaMemsetAsync(P->d_ptwm, 0, sizeof(double) * (size_t)P->ncomp * P->total_tgt_slots, st));
    BTK_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * (size_t)P->ncomp * T.n_points, st));
    BTK_TRY(run_interactions(ctx, P->d_S4, P->d_T4, P->d_T_out, o, wm, st, first ? ek[0] : nullptr,
                             first ? ek[1] : nullptr));
    first = false;
    BTK_CUDA(launch_promote(P->dim, P->degree, P->ncomp, P->n_tgt_slot_panels, P->d_t_cluster_panel,
                            P->d_t_cluster_slot_begin, P->d_t_slot_deg, P->d_t_slot_off, P->d_amat, P->d_amat_off,
                            wm, w, st));
    BTK_TRY(run_downward(T, P->ncomp, P->d_T4, w, o, st));
    return BTK_OK;
  };
  // The audit (FP64 direct sum at the sampled targets) runs in the solve's
  // own interaction launch: its items have their own queue, which two blocks
  // per SM start on while the others start on the solve's items (measured
  // about 1 ms faster than queueing the audit after them).
  BTK_CUDA(launch_gather(P->n_audit, P->d_audit_orig, xt, yt, P->dim == 3 ? zt : nullptr, nullptr, P->d_audit_T4, st));
  BTK_CUDA(cudaMemsetAsync(P->d_audit_out, 0, sizeof(double) * (size_t)P->ncomp * std::max(P->n_audit, 1), st));
  BTK_CUDA(cudaMemsetAsync(P->d_audit_sums, 0, 2 * sizeof(double), st));
  InteractCtx with_audit = P->ictx;
  with_audit.n_audit_items = P->n_audit_items;
  with_audit.audit_blocks = P->precision == BTK_PREC_MIXED ? 2 * num_sms() : 0;
  with_audit.d_T4a = P->d_audit_T4;
  for (int c = 0; c < P->ncomp; ++c) with_audit.aout.p[c] = P->d_audit_out + (size_t)c * P->n_audit;
  BTK_TRY(solve(with_audit));
  BTK_CUDA(cudaEventRecord(e[2], st));
  BTK_CUDA(launch_audit_compare(P->n_audit, P->ncomp, T.n_points, P->d_audit_orig, nullptr, out, P->d_audit_out,
                                P->d_audit_sums, st));
  double sums[2] = {0, 0};
  unsigned long long ev[2] = {0, 0};  // far evaluations; direct ones of the leaf pairs kept direct
  int hist[kMaxNodes] = {0};  // degrees the selector chose (before any fallback)
  BTK_CUDA(cudaMemcpyAsync(sums, P->d_audit_sums, sizeof(sums), cudaMemcpyDeviceToHost, st));
  BTK_CUDA(cudaMemcpyAsync(ev, P->d_evals, sizeof(ev), cudaMemcpyDeviceToHost, st));
  BTK_CUDA(cudaMemcpyAsync(hist, P->d_report, sizeof(hist), cudaMemcpyDeviceToHost, st));
  BTK_CUDA(cudaStreamSynchronize(st));
  const double rel = std::sqrt(sums[0] / std::max(sums[1], 1e-300));
  if (adaptive) {
    // Close the loop on the audit: the global error grows about like
    // pair_tol^0.7, so this settles near an audit of tol / 2 without overshoot.
    const double r = rel > 0 ? 0.5 * tol / rel : 2.0;
    P->adaptive_pair_tol = std::min(tol, std::max(1e-4 * tol, pair_tol * std::min(2.0, std::max(0.5, r))));
  }
  int fell_back = 0;
  if (!(rel <= tol)) {
    // Fallback: the fixed-degree plain method (degree n everywhere, leaf pairs
    // direct, FP64).
    fell_back = 1;
    BTK_CUDA(launch_fill_int(P->n_pairs, P->degree, P->d_deg_pc, st));
    BTK_CUDA(launch_fill_int(P->n_pc - P->n_pc_list, 0, P->d_deg_pc + P->n_pc_list, st));
    BTK_CUDA(launch_fill_int(P->n_far - P->n_far_list, 0, P->d_deg_pc + P->n_pc + P->n_far_list, st));
    InteractCtx plain = P->ictx;
    plain.precision = BTK_PREC_FP64;
    BTK_TRY(solve(plain));
  }
  BTK_CUDA(cudaEventRecord(e[3], st));
  BTK_CUDA(cudaEventSynchronize(e[3]));
  if (report) {
    std::memset(report, 0, sizeof(*report));
    report->audit_rel_l2 = rel;
    report->audit_targets = P->n_audit;
    report->fell_back = fell_back;
    report->evals_far = (int64_t)ev[0];
    report->evals_near = P->evals[0] - P->conv_direct_total + (int64_t)ev[1];
    cudaEventElapsedTime(&report->ms_select, e[0], e[1]);
    cudaEventElapsedTime(&report->ms_solve, e[1], e[2]);
    cudaEventElapsedTime(&report->ms_total, e[0], e[3]);
    std::memcpy(report->degree_hist, hist, sizeof(hist));
    cudaEventElapsedTime(&report->ms_kernel, ek[0], ek[1]);
    report->pair_tol = pair_tol;
  }
  for (auto& x : e) cudaEventDestroy(x);
  for (auto& x : ek) cudaEventDestroy(x);
  return check_status_word(P->ictx.d_ticket_status + 1, st);
}

btk_status btk_plan_error_samples(btk_plan* P, const double* xt, const double* yt, const double* zt,
                                  const double* xs, const double* ys, const double* zs, const double* charges, int n,
                                  const int* pair_index, int K, const int* target_orig, const int* src_leaf_csr,
                                  const int* src_leaves, const double* ref, float* log10_err,
                                  btk_stream_t stream) {
  BTK_CHECK(P && xt && yt && xs && ys && charges && (P->dim == 2 || (zt && zs)), BTK_ERR_INVALID_ARGUMENT,
            "btk_plan_error_samples: null argument");
  BTK_CHECK(P->degree_mode == BTK_DEGREE_PER_PAIR, BTK_ERR_INVALID_ARGUMENT, "plan is not BTK_DEGREE_PER_PAIR");
  BTK_CHECK(n >= 0 && K >= 1 && K <= 128 && (n == 0 || (pair_index && target_orig && src_leaf_csr && src_leaves &&
                                                        log10_err)),
            BTK_ERR_INVALID_ARGUMENT, "btk_plan_error_samples: bad sample arrays (1 <= K <= 128)");
  if (n == 0) return BTK_OK;
  cudaStream_t st = (cudaStream_t)stream;
  Side& T = P->tgt;
  Side& S = *P->src;
  for (int i = 0; i < n; ++i) {
    BTK_CHECK(pair_index[i] >= 0 && pair_index[i] < P->n_pairs, BTK_ERR_INVALID_ARGUMENT, "sample pair out of range");
    BTK_CHECK(src_leaf_csr[i + 1] >= src_leaf_csr[i], BTK_ERR_INVALID_ARGUMENT, "bad source leaf CSR");
  }
  for (int i = 0; i < n * K; ++i)
    BTK_CHECK(target_orig[i] >= 0 && target_orig[i] < T.n_points, BTK_ERR_INVALID_ARGUMENT, "sample target out of range");
  for (int i = 0; i < src_leaf_csr[n]; ++i)
    BTK_CHECK(src_leaves[i] >= 0 && src_leaves[i] < S.h.panel_count && S.h.is_leaf[src_leaves[i]],
              BTK_ERR_INVALID_ARGUMENT, "sample source leaf is not a leaf panel");
  // Sources and all degree slots for these charges.
  BTK_CUDA(launch_gather(S.n_points, S.d_perm, xs, ys, P->dim == 3 ? zs : nullptr, charges, P->d_S4, st));
  BTK_CUDA(cudaMemsetAsync(P->d_psw, 0, sizeof(double) * (size_t)S.h.panel_count * P->ipc, st));
  BTK_TRY(run_upward(S, P->d_S4, P->d_psw, st));
  BTK_CUDA(launch_src_slots(P->dim, P->degree, P->n_src_slots, P->d_s_slot_panel, P->d_s_slot_deg, P->d_s_slot_off,
                            S.d_panels, P->d_psw, P->d_amat, P->d_amat_off, P->d_ucos, P->d_ucos_off, nullptr,
                            P->d_S4 + S.n_points, st));
  Arena A(st);
  int *d_pi = nullptr, *d_to = nullptr, *d_csr = nullptr, *d_sl = nullptr;
  double *d_exact = nullptr, *d_approx = nullptr;
  float* d_err = nullptr;
  const int n_deg = P->degree - P->degree_min + 1;
  BTK_TRY(A.upload(&d_pi, std::vector<int>(pair_index, pair_index + n)));
  BTK_TRY(A.upload(&d_to, std::vector<int>(target_orig, target_orig + (size_t)n * K)));
  BTK_TRY(A.upload(&d_csr, std::vector<int>(src_leaf_csr, src_leaf_csr + n + 1)));
  BTK_TRY(A.upload(&d_sl, std::vector<int>(src_leaves, src_leaves + std::max(1, src_leaf_csr[n]))));
  BTK_TRY(A.alloc(&d_exact, (size_t)n * K * P->ncomp));
  BTK_TRY(A.alloc(&d_approx, (size_t)n * n_deg * K * P->ncomp));
  BTK_TRY(A.alloc(&d_err, (size_t)n * n_deg));
  SampleArgs a{};
  a.dim = P->dim;
  a.kind = P->kind;
  a.ncomp = P->ncomp;
  a.K = K;
  a.n_deg = n_deg;
  a.deg_lo = P->degree_min;
  a.n = n;
  a.eps2 = P->eps * P->eps;
  a.pair_index = d_pi;
  a.ptype = P->d_pair_type;
  a.ptgt = P->d_pair_tgt;
  a.psrc = P->d_pair_src;
  a.xt = xt;
  a.yt = yt;
  a.zt = P->dim == 3 ? zt : nullptr;
  a.tgt_orig = d_to;
  a.src_leaf_csr = d_csr;
  a.src_leaves = d_sl;
  a.leaf_begin_s = S.d_leaf_begin;
  a.count_s = S.d_point_count;
  a.S4 = P->d_S4;
  a.s_slot_off = P->d_s_slot_off;
  a.s_slot_begin = P->d_s_cluster_slot_begin;
  a.cluster_slot_s = P->d_cluster_slot_s;
  a.T4 = P->d_T4;
  a.t_slot_off = P->d_t_slot_off;
  a.t_slot_begin = P->d_t_cluster_slot_begin;
  a.cluster_slot_t = P->d_cluster_slot_t;
  a.ns = S.n_points;
  a.nt = T.n_points;
  a.pt = T.d_panels;
  a.slot_d_lo = P->degree_min;
  a.exact = d_exact;
  a.approx = d_approx;
  a.ref = ref;
  BTK_CUDA(launch_error_samples(a, d_err, st));
  BTK_CUDA(cudaMemcpyAsync(log10_err, d_err, sizeof(float) * (size_t)n * n_deg, cudaMemcpyDeviceToHost, st));
  BTK_CUDA(cudaStreamSynchronize(st));
  return BTK_OK;
}

btk_status btk_plan_set_degree_rule(btk_plan* P, int rule) {
  BTK_CHECK(P, BTK_ERR_INVALID_ARGUMENT, "btk_plan_set_degree_rule: null plan");
  BTK_CHECK(rule == BTK_DEGREE_RULE_THRESHOLD || rule == BTK_DEGREE_RULE_COST, BTK_ERR_INVALID_ARGUMENT,
            "btk_plan_set_degree_rule: unknown rule");
  P->degree_rule = rule;
  return BTK_OK;
}

btk_status btk_plan_set_degrees(btk_plan* P, const int* deg_pc, const int* deg_cp, const int* deg_cc) {
  BTK_CHECK(P, BTK_ERR_INVALID_ARGUMENT, "null plan");
  BTK_CHECK(P->degree_mode == BTK_DEGREE_PER_PAIR, BTK_ERR_INVALID_ARGUMENT, "plan is not BTK_DEGREE_PER_PAIR");
  const int lo = P->degree_min, hi = P->degree;
  auto check = [&](const int* v, int n) {
    for (int i = 0; i < n; ++i)
      if (v[i] < lo || v[i] > hi) return false;
    return true;
  };
  const int n_cc = P->n_far_list - P->n_cp;  // the CC list (leaf pairs stay direct)
  BTK_CHECK(!deg_pc || check(deg_pc, P->n_pc_list), BTK_ERR_INVALID_ARGUMENT,
            "PC degree outside [degree_min, degree]");
  BTK_CHECK(!deg_cp || check(deg_cp, P->n_cp), BTK_ERR_INVALID_ARGUMENT, "CP degree outside [degree_min, degree]");
  BTK_CHECK(!deg_cc || check(deg_cc, n_cc), BTK_ERR_INVALID_ARGUMENT, "CC degree outside [degree_min, degree]");
  if (deg_pc) std::copy(deg_pc, deg_pc + P->n_pc_list, P->h_deg_pc.begin());  // leaf pairs stay direct
  if (deg_cp) std::copy(deg_cp, deg_cp + P->n_cp, P->h_deg_far.begin());
  if (deg_cc) std::copy(deg_cc, deg_cc + n_cc, P->h_deg_far.begin() + P->n_cp);
  BTK_CUDA(cudaMemcpyAsync(P->d_deg_pc, P->h_deg_pc.data(), sizeof(int) * P->n_pc, cudaMemcpyHostToDevice, P->stream));
  BTK_CUDA(cudaMemcpyAsync(P->d_deg_far, P->h_deg_far.data(), sizeof(int) * P->n_far, cudaMemcpyHostToDevice,
                           P->stream));
  BTK_CUDA(cudaStreamSynchronize(P->stream));
  P->deg_learned = false;
  recount_far_evals(P);
  return BTK_OK;
}

btk_status btk_plan_leaf_pairs(const btk_plan* P, int* n_pairs, int* n_with_cc, int* pp_index) {
  BTK_CHECK(P && n_pairs && n_with_cc, BTK_ERR_INVALID_ARGUMENT, "btk_plan_leaf_pairs: null argument");
  *n_pairs = (int)P->h_conv.size();
  *n_with_cc = P->n_conv_cc;
  if (pp_index) std::copy(P->h_conv.begin(), P->h_conv.end(), pp_index);
  return BTK_OK;
}

btk_status btk_plan_set_leaf_forms(btk_plan* P, const int* form, const int* degree) {
  BTK_CHECK(P && form && degree, BTK_ERR_INVALID_ARGUMENT, "btk_plan_set_leaf_forms: null argument");
  BTK_CHECK(P->degree_mode == BTK_DEGREE_PER_PAIR, BTK_ERR_INVALID_ARGUMENT, "plan is not BTK_DEGREE_PER_PAIR");
  const int n_conv = (int)P->h_conv.size();
  for (int k = 0; k < n_conv; ++k) {
    BTK_CHECK(form[k] >= 0 && form[k] <= 2 && (form[k] != 2 || k < P->n_conv_cc), BTK_ERR_INVALID_ARGUMENT,
              "leaf pair form must be 0 (direct), 1 (points x proxies) or 2 (proxies x proxies, first n_with_cc)");
    BTK_CHECK(form[k] == 0 || (degree[k] >= P->degree_min && degree[k] <= P->degree), BTK_ERR_INVALID_ARGUMENT,
              "leaf pair degree outside [degree_min, degree]");
  }
  for (int k = 0; k < n_conv; ++k) {
    P->h_deg_pc[P->n_pc_list + k] = form[k] == 1 ? degree[k] : (form[k] == 2 ? -1 : 0);
    if (k < P->n_conv_cc) P->h_deg_far[P->n_far_list + P->n_pccc + P->n_cpcc + k] = form[k] == 2 ? degree[k] : 0;
  }
  BTK_CUDA(cudaMemcpyAsync(P->d_deg_pc, P->h_deg_pc.data(), sizeof(int) * P->n_pc, cudaMemcpyHostToDevice, P->stream));
  BTK_CUDA(cudaMemcpyAsync(P->d_deg_far, P->h_deg_far.data(), sizeof(int) * P->n_far, cudaMemcpyHostToDevice,
                           P->stream));
  BTK_CUDA(cudaStreamSynchronize(P->stream));
  P->deg_learned = false;
  recount_far_evals(P);
  return BTK_OK;
}

btk_status btk_plan_set_wait_limit(btk_plan* P, long long polls) {
  BTK_CHECK(P, BTK_ERR_INVALID_ARGUMENT, "null plan");
  P->ictx.wait_limit = polls < 0 ? kWaitLimitDefault : (uint32_t)std::min<long long>(polls, 0xffffffffLL);
  return BTK_OK;
}

btk_status btk_plan_audit_targets(const btk_plan* P, int* n, int* orig) {
  BTK_CHECK(P && n, BTK_ERR_INVALID_ARGUMENT, "btk_plan_audit_targets: null argument");
  *n = P->n_audit;
  if (orig && P->n_audit > 0)
    BTK_CUDA(cudaMemcpy(orig, P->d_audit_orig, sizeof(int) * P->n_audit, cudaMemcpyDeviceToHost));
  return BTK_OK;
}

btk_status btk_plan_last_timing(btk_plan* P, float* ms) {
  BTK_CHECK(P && ms, BTK_ERR_INVALID_ARGUMENT, "null argument");
  BTK_CHECK(P->timed, BTK_ERR_INVALID_ARGUMENT, "plan has not executed");
  BTK_CUDA(cudaEventSynchronize(P->ev[3]));
  BTK_CUDA(cudaEventElapsedTime(&ms[0], P->ev[0], P->ev[1]));
  BTK_CUDA(cudaEventElapsedTime(&ms[1], P->ev[1], P->ev[2]));
  BTK_CUDA(cudaEventElapsedTime(&ms[2], P->ev[2], P->ev[3]));
  BTK_CUDA(cudaEventElapsedTime(&ms[3], P->ev[0], P->ev[3]));
  BTK_CUDA(cudaEventElapsedTime(&ms[4], P->ev[4], P->ev[5]));
  return check_status_word(P->d_ticket_status + 1, P->stream);
}

btk_status btk_solve_host(int dim, int kind, int precision, int degree, int cluster_size, double theta, double eps,
                          int n, const double* x, const double* y, const double* z, const double* charges,
                          double* out, btk_stream_t stream) {
  BTK_CHECK(dim == 2 || dim == 3, BTK_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
  BTK_CHECK(n > 0 && x && y && charges && out && (dim == 2 || z), BTK_ERR_INVALID_ARGUMENT,
            "btk_solve_host: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  btk_run_config cfg{};
  cfg.dim = dim;
  cfg.interp_degree = degree;
  cfg.interp_point_count = ipow(degree + 1, dim);
  cfg.fmm_cluster_thresh = cluster_size > 0 ? cluster_size : (1 << dim) * cfg.interp_point_count;
  cfg.fmm_theta = theta;
  cfg.ker_eps = eps;
  cfg.mpi_p = 1;
  btk_tree_info info{};
  void* panels = nullptr;
  int* inside = nullptr;
  std::vector<int> leaf_of(n);
  btk_status s = dim == 2 ? btk_tree_construction_2d(&cfg, &info, x, y, n, (btk_panel_2d**)&panels, leaf_of.data(), &inside)
                          : btk_tree_construction_3d(&cfg, &info, x, y, z, n, (btk_panel_3d**)&panels, leaf_of.data(), &inside);
  if (s != BTK_OK) return s;
  std::unique_ptr<void, void (*)(void*)> g1(panels, std::free), g2(inside, std::free), g3(info.level_start, std::free);
  btk_interact_pair* all = nullptr;
  s = dim == 2 ? btk_dual_tree_traversal_2d(&cfg, (btk_panel_2d*)panels, (btk_panel_2d*)panels, &all)
               : btk_dual_tree_traversal_3d(&cfg, (btk_panel_3d*)panels, (btk_panel_3d*)panels, &all);
  if (s != BTK_OK) return s;
  std::unique_ptr<void, void (*)(void*)> g4(all, std::free);
  std::vector<btk_interact_pair> L[4];
  L[0].resize(cfg.fmm_pp_count);
  L[1].resize(cfg.fmm_pc_count);
  L[2].resize(cfg.fmm_cp_count);
  L[3].resize(cfg.fmm_cc_count);
  BTK_TRY(btk_split_interactions(all, cfg.fmm_interaction_count, L[0].data(), L[1].data(), L[2].data(), L[3].data()));
  btk_plan_desc D{};
  D.cfg = cfg;
  D.point_count_target = D.point_count_source = n;
  D.tree_target = &info;
  D.panels_target = panels;
  D.panel_points_inside_target = inside;
  D.point_leaf_panel_source = leaf_of.data();
  D.pp_list = L[0].data();
  D.pc_list = L[1].data();
  D.cp_list = L[2].data();
  D.cc_list = L[3].data();
  D.kind = kind;
  D.precision = precision;
  btk_plan* P = nullptr;
  BTK_TRY(btk_plan_create(&P, &D, stream));
  std::unique_ptr<btk_plan, btk_status (*)(btk_plan*)> gp(P, btk_plan_destroy);
  const int nc = ncomp_of(dim, kind);
  Arena A(st);
  double *d_xyz = nullptr, *d_q = nullptr, *d_out = nullptr;
  BTK_TRY(A.alloc(&d_xyz, (size_t)3 * n));
  BTK_TRY(A.alloc(&d_q, (size_t)n));
  BTK_TRY(A.alloc(&d_out, (size_t)nc * n));
  BTK_CUDA(cudaMemcpyAsync(d_xyz, x, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  BTK_CUDA(cudaMemcpyAsync(d_xyz + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  if (dim == 3) BTK_CUDA(cudaMemcpyAsync(d_xyz + 2 * (size_t)n, z, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  BTK_CUDA(cudaMemcpyAsync(d_q, charges, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  const double* dz = dim == 3 ? d_xyz + 2 * (size_t)n : nullptr;
  BTK_TRY(btk_plan_execute(P, d_xyz, d_xyz + n, dz, d_xyz, d_xyz + n, dz, d_q, d_out, stream));
  BTK_CUDA(cudaMemcpyAsync(out, d_out, sizeof(double) * nc * (size_t)n, cudaMemcpyDeviceToHost, st));
  BTK_CUDA(cudaStreamSynchronize(st));
  return check_status_word(P->d_ticket_status + 1, st);
}

}  // extern "C"

// =============================================================================
// Drop-in entry points (reference names and argument order; device pointers)
// =============================================================================

// ---- drop-in entry points ---------------------------------------------------
// The reference-named calls take the tree, leaf rows and interaction lists as
// the caller's device arrays on every call. What is derived from them (the
// host tree, the device sides, the work lists and the solve's buffers) is kept
// between calls in a small cache keyed by the buffers' addresses, counts and
// run configuration, and validated on every call by a fingerprint of the
// buffers' contents computed on the device (an order-independent sum of a
// 64-bit mix of every 32-bit word and its position), so a tree rebuilt in the
// same buffers is detected and rebuilt. Calls hold one process-wide lock
// (they synchronise their stream before returning anyway).
namespace btk {
namespace {

__global__ void k_fingerprint(const uint32_t* w, long long n, unsigned long long* out) {
  unsigned long long acc = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    unsigned long long z = (unsigned long long)w[i] * 0x9E3779B97F4A7C15ULL ^ (unsigned long long)i * 0xD6E8FEB86659FD93ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    acc += z ^ (z >> 31);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

struct DevBuf {
  const void* p;
  size_t bytes;
};

// Fingerprints of the buffers (each a multiple of 4 bytes), one per buffer.
btk_status fingerprints(const std::vector<DevBuf>& bufs, std::vector<unsigned long long>& fp, cudaStream_t st) {
  static unsigned long long* d_fp[64] = {};
  static size_t cap[64] = {};
  int dev = 0;
  BTK_CUDA(cudaGetDevice(&dev));
  BTK_CHECK(dev >= 0 && dev < 64, BTK_ERR_UNSUPPORTED, "drop-in cache: device index above 63");
  if (cap[dev] < bufs.size()) {
    if (d_fp[dev]) cudaFree(d_fp[dev]);
    BTK_CUDA(cudaMalloc(&d_fp[dev], sizeof(unsigned long long) * 16));
    cap[dev] = 16;
  }
  BTK_CHECK(bufs.size() <= cap[dev], BTK_ERR_INTERNAL, "drop-in cache: too many buffers");
  BTK_CUDA(cudaMemsetAsync(d_fp[dev], 0, sizeof(unsigned long long) * bufs.size(), st));
  for (size_t k = 0; k < bufs.size(); ++k) {
    const long long n = (long long)(bufs[k].bytes / 4);
    if (!bufs[k].p || n == 0) continue;
    count_launch();
    k_fingerprint<<<num_sms() * 4, 256, 0, st>>>((const uint32_t*)bufs[k].p, n, d_fp[dev] + k);
    BTK_CUDA(cudaGetLastError());
  }
  fp.assign(bufs.size(), 0);
  BTK_CUDA(cudaMemcpyAsync(fp.data(), d_fp[dev], sizeof(unsigned long long) * bufs.size(), cudaMemcpyDeviceToHost,
                           st));
  BTK_CUDA(cudaStreamSynchronize(st));
  return BTK_OK;
}

// Key of a cache entry: addresses, counts and configuration values as words.
using DropinKey = std::vector<long long>;

struct DropinEntry {
  DropinKey key;
  std::vector<unsigned long long> fp;
  std::unique_ptr<Arena> arena;  // on the legacy stream: valid whatever the callers' streams
  Side T, S;                     // upward/downward use T only; interactions both
  double4 *S4 = nullptr, *T4 = nullptr, *pts = nullptr;
  int* T_out = nullptr;
  InteractCtx ctx;
  uint64_t last_use = 0;
};

std::mutex g_dropin_mu;
// At most kDropinEntries. Held on the heap and never destroyed, so no CUDA
// call runs from a static destructor at process exit (the runtime may be shut
// down by then); btk_dropin_cache_clear frees the entries.
std::vector<std::unique_ptr<DropinEntry>>& g_dropin = *new std::vector<std::unique_ptr<DropinEntry>>();
uint64_t g_dropin_clock = 0;
constexpr size_t kDropinEntries = 6;

// The entry for key/fp (valid), or a fresh one to build (its key/fp set); the
// least recently used entry makes room.
DropinEntry* dropin_lookup(const DropinKey& key, const std::vector<unsigned long long>& fp, bool& fresh) {
  for (auto& e : g_dropin)
    if (e->key == key) {
      e->last_use = ++g_dropin_clock;
      fresh = e->fp != fp;
      if (fresh) {  // same buffers, new contents: rebuild in place
        cudaDeviceSynchronize();
        e.reset(new DropinEntry());
        e->key = key;
        e->fp = fp;
        e->last_use = g_dropin_clock;
      }
      return e.get();
    }
  if (g_dropin.size() >= kDropinEntries) {
    auto lru = std::min_element(g_dropin.begin(), g_dropin.end(),
                                [](const auto& x, const auto& y) { return x->last_use < y->last_use; });
    cudaDeviceSynchronize();  // its buffers may still be read by earlier work
    g_dropin.erase(lru);
  }
  g_dropin.emplace_back(new DropinEntry());
  DropinEntry* e = g_dropin.back().get();
  e->key = key;
  e->fp = fp;
  e->last_use = ++g_dropin_clock;
  fresh = true;
  return e;
}

DropinKey key_of(int what, int dim, const btk_run_config* cfg, std::initializer_list<long long> more) {
  int dev = 0;
  cudaGetDevice(&dev);
  DropinKey k = {what, dev, dim, cfg->interp_degree, cfg->fmm_cluster_thresh};
  k.insert(k.end(), more.begin(), more.end());
  return k;
}

btk_status upward_dropin(int dim, const btk_run_config* cfg, const btk_tree_info* info, const double* x,
                         const double* y, const double* z, const double* q, const void* d_panels, double* psw,
                         const int* d_leaf_of, int n, cudaStream_t st) {
  BTK_TRY(validate_cfg(cfg, dim));
  BTK_CHECK(info && info->level_start && info->panel_count > 0 && info->levels > 0, BTK_ERR_INVALID_ARGUMENT,
            "upward_pass: bad tree_info");
  BTK_CHECK(n >= 0 && x && y && q && psw && d_leaf_of && (dim == 2 || z), BTK_ERR_INVALID_ARGUMENT,
            "upward_pass: null argument");
  const size_t panel_bytes = dim == 2 ? sizeof(btk_panel_2d) : sizeof(btk_panel_3d);
  std::lock_guard<std::mutex> lock(g_dropin_mu);
  DropinKey key = key_of(0, dim, cfg, {(long long)(uintptr_t)d_panels, info->panel_count, info->levels,
                                       (long long)(uintptr_t)d_leaf_of, n});
  key.insert(key.end(), info->level_start, info->level_start + info->levels + 1);
  std::vector<unsigned long long> fp;
  BTK_TRY(fingerprints({{d_panels, panel_bytes * info->panel_count}, {d_leaf_of, sizeof(int) * (size_t)n}}, fp, st));
  bool fresh = false;
  DropinEntry* E = dropin_lookup(key, fp, fresh);
  if (fresh) {
    Side& S = E->T;
    std::vector<int> leaf_of;
    if (dim == 2) {
      std::vector<btk_panel_2d> hp;
      BTK_TRY(fetch_panels((const btk_panel_2d*)d_panels, info->panel_count, hp, st));
      BTK_TRY(fetch(d_leaf_of, n, leaf_of, st));
      BTK_CUDA(cudaStreamSynchronize(st));
      host_tree_from_panels(2, hp.data(), info->panel_count, info->level_start, info->levels, S.h);
    } else {
      std::vector<btk_panel_3d> hp;
      BTK_TRY(fetch_panels((const btk_panel_3d*)d_panels, info->panel_count, hp, st));
      BTK_TRY(fetch(d_leaf_of, n, leaf_of, st));
      BTK_CUDA(cudaStreamSynchronize(st));
      host_tree_from_panels(3, hp.data(), info->panel_count, info->level_start, info->levels, S.h);
    }
    E->arena.reset(new Arena(nullptr));
    Arena& A = *E->arena;
    btk_status rc = side_layout(S, n, cfg->interp_degree);
    if (rc == BTK_OK) rc = side_upload(S, A, nullptr, nullptr, cfg->fmm_cluster_thresh);
    if (rc == BTK_OK) rc = side_perm_from_leaf_of(S, A, leaf_of);
    if (rc == BTK_OK) rc = A.alloc(&E->pts, (size_t)std::max(n, 1));
    if (rc == BTK_OK && cudaStreamSynchronize(nullptr) != cudaSuccess) rc = BTK_ERR_CUDA;
    if (rc != BTK_OK) {
      E->key.clear();  // never matches: rebuilt on the next call
      return rc;
    }
  }
  BTK_CUDA(launch_gather(n, E->T.d_perm, x, y, dim == 3 ? z : nullptr, q, E->pts, st));
  BTK_TRY(run_upward(E->T, E->pts, psw, st));
  BTK_CUDA(cudaStreamSynchronize(st));
  return BTK_OK;
}

template <class PanelT>
btk_status interactions_dropin(int dim, int kind, const btk_run_config* cfg, const double* xt, const double* yt,
                               const double* zt, const double* xs, const double* ys, const double* zs, const double* q,
                               Ptr4 out, const int* inside_s, const int* inside_t, const double* psw, Ptr4 ptw,
                               const btk_interact_pair* const dl[4], const PanelT* panels_s, const PanelT* panels_t,
                               int nt, int ns, int Pt, int Ps, cudaStream_t st) {
  BTK_TRY(validate_cfg(cfg, dim));
  BTK_CHECK(nt >= 0 && ns >= 0 && xt && yt && xs && ys && q && psw && inside_s && inside_t && (dim == 2 || (zt && zs)),
            BTK_ERR_INVALID_ARGUMENT, "interactions: null argument");
  BTK_CHECK(Pt > 0 && Ps > 0 && panels_s && panels_t, BTK_ERR_INVALID_ARGUMENT, "interactions: bad panel arrays");
  const int counts[4] = {cfg->fmm_pp_count, cfg->fmm_pc_count, cfg->fmm_cp_count, cfg->fmm_cc_count};
  for (int t = 0; t < 4; ++t)
    BTK_CHECK(counts[t] >= 0 && (counts[t] == 0 || dl[t]), BTK_ERR_INVALID_ARGUMENT, "interactions: null list");
  const size_t thresh = (size_t)cfg->fmm_cluster_thresh;
  std::lock_guard<std::mutex> lock(g_dropin_mu);
  const DropinKey key =
      key_of(1, dim, cfg, {kind, (long long)(uintptr_t)panels_t, (long long)(uintptr_t)panels_s,
                           (long long)(uintptr_t)inside_t, (long long)(uintptr_t)inside_s,
                           (long long)(uintptr_t)dl[0], (long long)(uintptr_t)dl[1], (long long)(uintptr_t)dl[2],
                           (long long)(uintptr_t)dl[3], counts[0], counts[1], counts[2], counts[3], nt, ns, Pt, Ps});
  std::vector<DevBuf> bufs = {{panels_t, sizeof(PanelT) * Pt}, {inside_t, sizeof(int) * thresh * Pt}};
  if ((const void*)panels_s != (const void*)panels_t) bufs.push_back({panels_s, sizeof(PanelT) * Ps});
  if (inside_s != inside_t) bufs.push_back({inside_s, sizeof(int) * thresh * Ps});
  for (int t = 0; t < 4; ++t) bufs.push_back({dl[t], sizeof(btk_interact_pair) * counts[t]});
  std::vector<unsigned long long> fp;
  BTK_TRY(fingerprints(bufs, fp, st));
  bool fresh = false;
  DropinEntry* E = dropin_lookup(key, fp, fresh);
  if (fresh) {
    auto build = [&]() -> btk_status {
      std::vector<PanelT> hpt, hps;
      std::vector<btk_interact_pair> hl[4];
      BTK_TRY(fetch_panels(panels_t, Pt, hpt, st));
      BTK_TRY(fetch_panels(panels_s, Ps, hps, st));
      for (int t = 0; t < 4; ++t) BTK_TRY(fetch(dl[t], counts[t], hl[t], st));
      BTK_CUDA(cudaStreamSynchronize(st));
      Side &T = E->T, &S = E->S;
      BTK_CHECK(host_tree_from_panels_nolevels(dim, hpt.data(), Pt, T.h), BTK_ERR_INVALID_ARGUMENT,
                "target panels are not in level order");
      BTK_TRY(side_layout(T, nt, cfg->interp_degree));
      BTK_CHECK(host_tree_from_panels_nolevels(dim, hps.data(), Ps, S.h), BTK_ERR_INVALID_ARGUMENT,
                "source panels are not in level order");
      BTK_TRY(side_layout(S, ns, cfg->interp_degree));
      E->arena.reset(new Arena(nullptr));
      Arena& A = *E->arena;
      BTK_TRY(side_upload(T, A, nullptr, inside_t, cfg->fmm_cluster_thresh));
      BTK_TRY(side_upload(S, A, nullptr, inside_s, cfg->fmm_cluster_thresh));
      const int ipc = S.ipc;
      const int nct = (int)T.clusters.size(), ncs = (int)S.clusters.size();
      BTK_TRY(A.alloc(&E->S4, (size_t)ns + (size_t)ncs * ipc + 1));
      BTK_TRY(A.alloc(&E->T4, (size_t)nt + (size_t)nct * ipc + 1));
      BTK_TRY(A.alloc(&E->T_out, (size_t)nt + (size_t)nct * ipc + 1));
      const btk_interact_pair* hlp[4] = {hl[0].data(), hl[1].data(), hl[2].data(), hl[3].data()};
      const bool guard = cfg->ker_eps * cfg->ker_eps < 1.1754943508222875e-38;
      const int slots = num_sms() * std::max(1, interact_blocks_per_sm(dim, kind, BTK_PREC_FP64, guard, kTile));
      WorkLists W;
      BTK_TRY(build_work(T, S, hlp, counts, slots, W));
      InteractCtx& C = E->ctx;
      C.dim = dim;
      C.kind = kind;
      C.precision = BTK_PREC_FP64;
      C.eps = cfg->ker_eps;
      C.n_items = (int)W.items.size();
      BTK_TRY(A.upload(&C.d_items, W.items));
      BTK_TRY(A.upload(&C.d_entries, W.entries));
      BTK_TRY(A.alloc(&C.d_ticket_status, 3));
      BTK_CUDA(cudaMemsetAsync(C.d_ticket_status, 0, 3 * sizeof(int), nullptr));
      BTK_CUDA(cudaStreamSynchronize(nullptr));  // the uploads read host vectors that go out of scope
      return BTK_OK;
    };
    const btk_status rc = build();
    if (rc != BTK_OK) {
      E->key.clear();
      return rc;
    }
  }
  const Side &T = E->T, &S = E->S;
  const int nct = (int)T.clusters.size(), ncs = (int)S.clusters.size();
  // Per call: sources (sorted points + cluster proxies carrying this call's
  // modified charges) and targets (sorted points + cluster proxy points).
  BTK_CUDA(launch_gather(ns, S.d_perm, xs, ys, dim == 3 ? zs : nullptr, q, E->S4, st));
  BTK_CUDA(launch_src_proxies(dim, S.degree, ncs, S.d_clusters, S.d_nodes_shift, psw, E->S4 + ns, st));
  BTK_CUDA(launch_gather(nt, T.d_perm, xt, yt, dim == 3 ? zt : nullptr, nullptr, E->T4, st));
  if (nt) BTK_CUDA(cudaMemcpyAsync(E->T_out, T.d_perm, sizeof(int) * nt, cudaMemcpyDeviceToDevice, st));
  BTK_CUDA(launch_tgt_proxies(dim, T.degree, nct, T.d_clusters, T.d_nodes_shift, E->T4 + nt, E->T_out + nt, st));
  BTK_CUDA(cudaMemsetAsync(E->ctx.d_ticket_status + 1, 0, sizeof(int), st));
  BTK_TRY(run_interactions(E->ctx, E->S4, E->T4, E->T_out, out, ptw, st));
  return check_status_word(E->ctx.d_ticket_status + 1, st);
}

template <class PanelT>
btk_status downward_dropin(int dim, int ncomp, const btk_run_config* cfg, const btk_tree_info* info, const double* x,
                           const double* y, const double* z, Ptr4 out, const PanelT* panels, Ptr4 ptw,
                           const int* inside, int n, cudaStream_t st) {
  BTK_TRY(validate_cfg(cfg, dim));
  BTK_CHECK(info && info->level_start && info->panel_count > 0 && info->levels > 0, BTK_ERR_INVALID_ARGUMENT,
            "downward_pass: bad tree_info");
  BTK_CHECK(n >= 0 && x && y && inside && panels && (dim == 2 || z), BTK_ERR_INVALID_ARGUMENT,
            "downward_pass: null argument");
  std::lock_guard<std::mutex> lock(g_dropin_mu);
  DropinKey key = key_of(2, dim, cfg, {(long long)(uintptr_t)panels, info->panel_count, info->levels,
                                       (long long)(uintptr_t)inside, n});
  key.insert(key.end(), info->level_start, info->level_start + info->levels + 1);
  std::vector<unsigned long long> fp;
  BTK_TRY(fingerprints({{panels, sizeof(PanelT) * info->panel_count},
                        {inside, sizeof(int) * (size_t)cfg->fmm_cluster_thresh * info->panel_count}},
                       fp, st));
  bool fresh = false;
  DropinEntry* E = dropin_lookup(key, fp, fresh);
  if (fresh) {
    auto build = [&]() -> btk_status {
      std::vector<PanelT> hp;
      BTK_TRY(fetch_panels(panels, info->panel_count, hp, st));
      BTK_CUDA(cudaStreamSynchronize(st));
      Side& T = E->T;
      host_tree_from_panels(dim, hp.data(), info->panel_count, info->level_start, info->levels, T.h);
      BTK_TRY(side_layout(T, n, cfg->interp_degree));
      E->arena.reset(new Arena(nullptr));
      BTK_TRY(side_upload(T, *E->arena, nullptr, inside, cfg->fmm_cluster_thresh));
      BTK_TRY(E->arena->alloc(&E->pts, (size_t)std::max(n, 1)));
      BTK_CUDA(cudaStreamSynchronize(nullptr));
      return BTK_OK;
    };
    const btk_status rc = build();
    if (rc != BTK_OK) {
      E->key.clear();
      return rc;
    }
  }
  BTK_CUDA(launch_gather(n, E->T.d_perm, x, y, dim == 3 ? z : nullptr, nullptr, E->pts, st));
  BTK_TRY(run_downward(E->T, ncomp, E->pts, ptw, out, st));
  BTK_CUDA(cudaStreamSynchronize(st));
  return BTK_OK;
}

}  // namespace
}  // namespace btk

extern "C" {

btk_status btk_dropin_cache_clear(void) {
  std::lock_guard<std::mutex> lock(btk::g_dropin_mu);
  if (!btk::g_dropin.empty()) {
    BTK_CUDA(cudaDeviceSynchronize());  // work issued by earlier calls may still read the entries
    btk::g_dropin.clear();
    BTK_CUDA(cudaDeviceSynchronize());
  }
  return BTK_OK;
}

btk_status btk_upward_pass_2d(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                              const double* ycos, const double* charges, const btk_panel_2d* blfmm_panels,
                              double* proxy_source_weights, const int* point_leaf_panel, int point_count,
                              btk_stream_t stream) {
  return upward_dropin(2, cfg, info, xcos, ycos, nullptr, charges, blfmm_panels, proxy_source_weights,
                       point_leaf_panel, point_count, (cudaStream_t)stream);
}

btk_status btk_upward_pass_3d(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                              const double* ycos, const double* zcos, const double* charges,
                              const btk_panel_3d* blfmm_panels, double* proxy_source_weights,
                              const int* point_leaf_panel, int point_count, btk_stream_t stream) {
  return upward_dropin(3, cfg, info, xcos, ycos, zcos, charges, blfmm_panels, proxy_source_weights, point_leaf_panel,
                       point_count, (cudaStream_t)stream);
}

btk_status btk_poisson_fmm_interactions_2d(const btk_run_config* cfg, const double* xcos_t, const double* ycos_t,
                                           const double* xcos_s, const double* ycos_s, const double* charges,
                                           double* soln, const int* panel_points_inside_source,
                                           const int* panel_points_inside_target, const double* proxy_source_weights,
                                           double* proxy_target_weights, const btk_interact_pair* pp_ints,
                                           const btk_interact_pair* pc_ints, const btk_interact_pair* cp_ints,
                                           const btk_interact_pair* cc_ints, const btk_panel_2d* blfmm_panels_source,
                                           const btk_panel_2d* blfmm_panels_target, int point_count_target,
                                           int point_count_source, int panel_count_target, int panel_count_source,
                                           btk_stream_t stream) {
  BTK_CHECK(soln && proxy_target_weights, BTK_ERR_INVALID_ARGUMENT, "interactions: null output");
  Ptr4 o{{soln}}, w{{proxy_target_weights}};
  const btk_interact_pair* dl[4] = {pp_ints, pc_ints, cp_ints, cc_ints};
  return interactions_dropin(2, BTK_KIND_POT, cfg, xcos_t, ycos_t, nullptr, xcos_s, ycos_s, nullptr, charges, o,
                             panel_points_inside_source, panel_points_inside_target, proxy_source_weights, w, dl,
                             blfmm_panels_source, blfmm_panels_target, point_count_target, point_count_source,
                             panel_count_target, panel_count_source, (cudaStream_t)stream);
}

btk_status btk_poisson_fmm_interactions_3d(const btk_run_config* cfg, const double* xcos_t, const double* ycos_t,
                                           const double* zcos_t, const double* xcos_s, const double* ycos_s,
                                           const double* zcos_s, const double* charges, double* soln,
                                           const int* panel_points_inside_source,
                                           const int* panel_points_inside_target, const double* proxy_source_weights,
                                           double* proxy_target_weights, const btk_interact_pair* pp_ints,
                                           const btk_interact_pair* pc_ints, const btk_interact_pair* cp_ints,
                                           const btk_interact_pair* cc_ints, const btk_panel_3d* blfmm_panels_source,
                                           const btk_panel_3d* blfmm_panels_target, int point_count_target,
                                           int point_count_source, int panel_count_target, int panel_count_source,
                                           btk_stream_t stream) {
  BTK_CHECK(soln && proxy_target_weights, BTK_ERR_INVALID_ARGUMENT, "interactions: null output");
  Ptr4 o{{soln}}, w{{proxy_target_weights}};
  const btk_interact_pair* dl[4] = {pp_ints, pc_ints, cp_ints, cc_ints};
  return interactions_dropin(3, BTK_KIND_POT, cfg, xcos_t, ycos_t, zcos_t, xcos_s, ycos_s, zcos_s, charges, o,
                             panel_points_inside_source, panel_points_inside_target, proxy_source_weights, w, dl,
                             blfmm_panels_source, blfmm_panels_target, point_count_target, point_count_source,
                             panel_count_target, panel_count_source, (cudaStream_t)stream);
}

btk_status btk_poisson_vel_fmm_interactions_3d(
    const btk_run_config* cfg, const double* xcos_t, const double* ycos_t, const double* zcos_t, const double* xcos_s,
    const double* ycos_s, const double* zcos_s, const double* charges, double* vel_x, double* vel_y, double* vel_z,
    const int* panel_points_inside_source, const int* panel_points_inside_target, const double* proxy_source_weights,
    double* proxy_target_weights_x, double* proxy_target_weights_y, double* proxy_target_weights_z,
    const btk_interact_pair* pp_ints, const btk_interact_pair* pc_ints, const btk_interact_pair* cp_ints,
    const btk_interact_pair* cc_ints, const btk_panel_3d* blfmm_panels_source, const btk_panel_3d* blfmm_panels_target,
    int point_count_target, int point_count_source, int panel_count_target, int panel_count_source,
    btk_stream_t stream) {
  BTK_CHECK(vel_x && vel_y && vel_z && proxy_target_weights_x && proxy_target_weights_y && proxy_target_weights_z,
            BTK_ERR_INVALID_ARGUMENT, "vel interactions: null output");
  Ptr4 o{{vel_x, vel_y, vel_z}}, w{{proxy_target_weights_x, proxy_target_weights_y, proxy_target_weights_z}};
  const btk_interact_pair* dl[4] = {pp_ints, pc_ints, cp_ints, cc_ints};
  return interactions_dropin(3, BTK_KIND_VEL, cfg, xcos_t, ycos_t, zcos_t, xcos_s, ycos_s, zcos_s, charges, o,
                             panel_points_inside_source, panel_points_inside_target, proxy_source_weights, w, dl,
                             blfmm_panels_source, blfmm_panels_target, point_count_target, point_count_source,
                             panel_count_target, panel_count_source, (cudaStream_t)stream);
}

btk_status btk_downward_pass_2d(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                                const double* ycos, double* soln, const btk_panel_2d* blfmm_panels,
                                double* proxy_target_weights, const int* panel_points_inside, int point_count,
                                btk_stream_t stream) {
  BTK_CHECK(soln && proxy_target_weights, BTK_ERR_INVALID_ARGUMENT, "downward_pass: null output");
  Ptr4 o{{soln}}, w{{proxy_target_weights}};
  return downward_dropin(2, 1, cfg, info, xcos, ycos, nullptr, o, blfmm_panels, w, panel_points_inside, point_count,
                         (cudaStream_t)stream);
}

btk_status btk_downward_pass_3d(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                                const double* ycos, const double* zcos, double* soln,
                                const btk_panel_3d* blfmm_panels, double* proxy_target_weights,
                                const int* panel_points_inside, int point_count, btk_stream_t stream) {
  BTK_CHECK(soln && proxy_target_weights, BTK_ERR_INVALID_ARGUMENT, "downward_pass: null output");
  Ptr4 o{{soln}}, w{{proxy_target_weights}};
  return downward_dropin(3, 1, cfg, info, xcos, ycos, zcos, o, blfmm_panels, w, panel_points_inside, point_count,
                         (cudaStream_t)stream);
}

btk_status btk_downward_pass_3d_3(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                                  const double* ycos, const double* zcos, double* vel_x, double* vel_y, double* vel_z,
                                  const btk_panel_3d* blfmm_panels, double* proxy_target_weights_x,
                                  double* proxy_target_weights_y, double* proxy_target_weights_z,
                                  const int* panel_points_inside, int point_count, btk_stream_t stream) {
  BTK_CHECK(vel_x && vel_y && vel_z && proxy_target_weights_x && proxy_target_weights_y && proxy_target_weights_z,
            BTK_ERR_INVALID_ARGUMENT, "downward_pass_3d_3: null output");
  Ptr4 o{{vel_x, vel_y, vel_z}}, w{{proxy_target_weights_x, proxy_target_weights_y, proxy_target_weights_z}};
  return downward_dropin(3, 3, cfg, info, xcos, ycos, zcos, o, blfmm_panels, w, panel_points_inside, point_count,
                         (cudaStream_t)stream);
}

btk_status btk_direct_sum(int dim, int kind, double eps, int nt, const double* xt, const double* yt, const double* zt,
                          int ns, const double* xs, const double* ys, const double* zs, const double* charges,
                          double* out, btk_stream_t stream) {
  BTK_CHECK(dim == 2 || dim == 3, BTK_ERR_INVALID_ARGUMENT, "dim must be 2 or 3");
  BTK_CHECK(!(kind == BTK_KIND_VEL && dim != 3) && kind >= 0 && kind <= 2, BTK_ERR_INVALID_ARGUMENT, "bad kind");
  BTK_CHECK(nt >= 0 && ns >= 0 && xt && yt && xs && ys && charges && out && (dim == 2 || (zt && zs)),
            BTK_ERR_INVALID_ARGUMENT, "direct_sum: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  Arena A(st);
  double4* src = nullptr;
  int* iota = nullptr;
  BTK_TRY(A.alloc(&src, (size_t)std::max(ns, 1)));
  std::vector<int> id(ns);
  std::iota(id.begin(), id.end(), 0);
  BTK_TRY(A.upload(&iota, id));
  BTK_CUDA(launch_gather(ns, iota, xs, ys, dim == 3 ? zs : nullptr, charges, src, st));
  BTK_CUDA(launch_direct(dim, kind, eps, nt, xt, yt, dim == 3 ? zt : nullptr, ns, src, out, st));
  BTK_CUDA(cudaStreamSynchronize(st));
  return BTK_OK;
}

}  // extern "C"
