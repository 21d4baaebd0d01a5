// TEST INFRASTRUCTURE ONLY — the parity checker and the timed CPU baseline.
//
// A C-ABI driver around BarytreeK's own, unmodified host/Kokkos sources
// (compiled from the reference tree against oracle/kokkos_shim by
// oracle/Makefile into oracle/_ref/libbtkref.so). It does what the reference's
// example drivers do (examples/example_poisson_3d.cpp:70-165,
// examples/example_poisson_vel_3d.cpp, examples/example_poisson_2d_split.cpp):
// build the tree and interaction lists, run the upward pass, the interaction
// phase and the downward pass, and the direct sum, all through the reference's
// own functions and functors. It adds four things the examples do not have:
//
//  * explicit inputs (seeded points instead of std::random_device) and access
//    to every intermediate array, so that tests can compare phase by phase;
//  * an optional "fixed" downward pass for trees whose leaves are not all on
//    the last level. The reference's downward_pass_* (src/downward_pass.cpp:7-41)
//    runs parent_to_child_* over every panel of levels 0..L-2, leaves included
//    (a leaf's child ids are -1: out-of-bounds), and leaf_to_point_* over the
//    last level only, so shallower leaves never receive the far field. The
//    fixed variant calls the reference's own functors
//    (src/downward_pass_impl.hpp:109-237, :239-379) on non-leaf parents only and
//    on every leaf. Nothing under the reference tree is edited;
//  * strided, timed samples of each phase for the CPU baseline;
//  * a solve restricted to the targets of sampled leaves (full upward pass,
//    the pairs of those leaves and their ancestors, the downward pass along
//    them) for parity checks at full workload sizes.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <Kokkos_Core.hpp>

#include "barytreek-config.h"
#include "structs.hpp"
#include "read_namelist.hpp"
#include "tree_construction.hpp"
#include "interaction_list.hpp"
#include "upward_pass.hpp"
#include "upward_pass_impl.hpp"
#include "downward_pass.hpp"
#include "downward_pass_impl.hpp"
#include "fmm_interactions/poisson_fmm.hpp"
#include "fmm_interactions/poisson_fmm_impl.hpp"
#include "fmm_interactions/poisson_vel_fmm.hpp"
#include "fmm_interactions/poisson_vel_fmm_impl.hpp"
#include "direct_sum_impl.hpp"
#include "general_utils_impl.hpp"

namespace {

// Host views feed the reference's host tree code; the "device" views (the
// same host memory space under the shim) are deep copies handed to the
// device-side functions, exactly as the examples deep_copy before solving.
struct Tree {
  TreeInfo info{};
  int n = 0;
  view_real_host hx, hy, hz;
  view_panel_2d_host hp2;
  view_panel_3d_host hp3;
  view_int_host hleaf;
  view_intt_host hinside;
  view_real x, y, z;
  view_panel_2d p2;
  view_panel_3d p3;
  view_int leaf_of;
  view_intt inside;
  ~Tree() { free(info.level_start); }
};

struct Handle {
  RunConfig cfg{};
  bool split = false;
  Tree tgt, src;  // src unused when !split
  view_interact_host all, pp, pc, cp, cc;
  view_interact dpp, dpc, dcp, dcc;
  Tree& source() { return split ? src : tgt; }
};

template <class V = view_real>
V make_view(const char* label, int n, const double* v) {
  V out(label, n);
  if (v) std::memcpy(out.data(), v, sizeof(double) * n);
  return out;
}

template <class D, class H>
D device_copy(const char* label, const H& h) {
  D d(label, h.extent(0), h.extent(1));
  Kokkos::deep_copy(d, h);
  return d;
}

void build_tree(Handle& h, Tree& t, int n, const double* x, const double* y, const double* z) {
  t.n = n;
  t.hx = make_view<view_real_host>("x", n, x);
  t.hy = make_view<view_real_host>("y", n, y);
  t.hz = make_view<view_real_host>("z", n, h.cfg.dim == 3 ? z : nullptr);
  t.hleaf = view_int_host("leaf", n);
  t.hinside = view_intt_host("inside", 1, 1);
  if (h.cfg.dim == 2) {
    t.hp2 = view_panel_2d_host("panels", 1);
    blfmm_tree_construction_2d(h.cfg, t.info, t.hx, t.hy, t.hp2, t.hleaf, t.hinside);
    t.p2 = device_copy<view_panel_2d>("panels", t.hp2);
  } else {
    t.hp3 = view_panel_3d_host("panels", 1);
    blfmm_tree_construction_3d(h.cfg, t.info, t.hx, t.hy, t.hz, t.hp3, t.hleaf, t.hinside);
    t.p3 = device_copy<view_panel_3d>("panels", t.hp3);
  }
  t.x = device_copy<view_real>("x", t.hx);
  t.y = device_copy<view_real>("y", t.hy);
  t.z = device_copy<view_real>("z", t.hz);
  t.leaf_of = device_copy<view_int>("leaf", t.hleaf);
  t.inside = device_copy<view_intt>("inside", t.hinside);
}

// Follows src/read_namelist.cpp:24-38 field by field (degree clamp, point count,
// cluster_size <= 0 rule, theta, kernel_eps).
void set_config(RunConfig& c, int dim, int degree, int cluster_size, double theta, double eps) {
  c.dim = dim;
  c.interp_degree = degree > max_degree ? max_degree : degree;
  c.interp_point_count = (int)std::pow(c.interp_degree + 1, dim);
  c.fmm_cluster_thresh = cluster_size;
  if (c.fmm_cluster_thresh <= 0) c.fmm_cluster_thresh = (int)std::pow(2, dim) * c.interp_point_count;
  c.fmm_theta = theta;
  c.ker_eps = eps;
  c.mpi_p = 1;
  c.mpi_id = 0;
}

bool is_leaf_panel(const Handle& h, const Tree& t, int i) {
  return h.cfg.dim == 2 ? t.p2(i).is_leaf : t.p3(i).is_leaf;
}
int panel_count(const Tree& t) { return t.info.panel_count; }
int point_count_of(const Handle& h, const Tree& t, int i) {
  return h.cfg.dim == 2 ? t.p2(i).point_count : t.p3(i).point_count;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

extern "C" {

void btkref_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : omp_get_num_procs());
#else
  (void)n;
#endif
}

int btkref_max_threads(void) { return Kokkos::num_threads(); }

int btkref_sizeof(int which) {
  switch (which) {
    case 0: return (int)sizeof(RunConfig);
    case 1: return (int)sizeof(TreeInfo);
    case 2: return (int)sizeof(TreePanel_2d);
    case 3: return (int)sizeof(TreePanel_3d);
    case 4: return (int)sizeof(interact_pair);
  }
  return -1;
}

// Parses a namelist file with the reference's read_run_config and returns the
// resulting RunConfig bytes (dim must be preset, as the examples do).
int btkref_read_namelist(const char* path, int dim, void* out_cfg) {
  RunConfig c;
  c.dim = dim;
  try {
    read_run_config(std::string(path), c);
  } catch (...) {
    return 1;
  }
  std::memcpy(out_cfg, &c, sizeof(RunConfig));
  return 0;
}

void* btkref_create(int dim, int nt, const double* tx, const double* ty, const double* tz, int ns,
                    const double* sx, const double* sy, const double* sz, int degree, int cluster_size,
                    double theta, double eps) {
  Handle* h = new Handle();
  set_config(h->cfg, dim, degree, cluster_size, theta, eps);
  h->split = (sx != nullptr);
  build_tree(*h, h->tgt, nt, tx, ty, tz);
  if (h->split) build_tree(*h, h->src, ns, sx, sy, sz);
  h->all = view_interact_host("interactions", 1);
  if (dim == 2)
    dual_tree_traversal_2d(h->cfg, h->tgt.hp2, h->source().hp2, h->all);
  else
    dual_tree_traversal_3d(h->cfg, h->tgt.hp3, h->source().hp3, h->all);
  h->pp = view_interact_host("pp", h->cfg.fmm_pp_count);
  h->pc = view_interact_host("pc", h->cfg.fmm_pc_count);
  h->cp = view_interact_host("cp", h->cfg.fmm_cp_count);
  h->cc = view_interact_host("cc", h->cfg.fmm_cc_count);
  split_interactions(h->all, h->pp, h->pc, h->cp, h->cc);
  h->dpp = device_copy<view_interact>("pp", h->pp);
  h->dpc = device_copy<view_interact>("pc", h->pc);
  h->dcp = device_copy<view_interact>("cp", h->cp);
  h->dcc = device_copy<view_interact>("cc", h->cc);
  return h;
}

void btkref_destroy(void* p) { delete static_cast<Handle*>(p); }

// info: [0] dim [1] target panels [2] target levels [3] source panels
// [4] source levels [5..8] pp/pc/cp/cc counts [9] interaction count
// [10] interp_point_count [11] cluster thresh [12] degree
void btkref_info(void* p, int* info) {
  Handle& h = *static_cast<Handle*>(p);
  info[0] = h.cfg.dim;
  info[1] = h.tgt.info.panel_count;
  info[2] = h.tgt.info.levels;
  info[3] = h.source().info.panel_count;
  info[4] = h.source().info.levels;
  info[5] = h.cfg.fmm_pp_count;
  info[6] = h.cfg.fmm_pc_count;
  info[7] = h.cfg.fmm_cp_count;
  info[8] = h.cfg.fmm_cc_count;
  info[9] = h.cfg.fmm_interaction_count;
  info[10] = h.cfg.interp_point_count;
  info[11] = h.cfg.fmm_cluster_thresh;
  info[12] = h.cfg.interp_degree;
}

void btkref_get_config(void* p, void* out_cfg) {
  std::memcpy(out_cfg, &static_cast<Handle*>(p)->cfg, sizeof(RunConfig));
}

// which: 0 = target tree, 1 = source tree. Any output pointer may be null.
void btkref_get_tree(void* p, int which, void* panels, int* level_start, int* leaf_of, int* inside) {
  Handle& h = *static_cast<Handle*>(p);
  Tree& t = which == 0 ? h.tgt : h.source();
  int P = t.info.panel_count;
  if (panels) {
    if (h.cfg.dim == 2)
      std::memcpy(panels, t.hp2.data(), sizeof(TreePanel_2d) * P);
    else
      std::memcpy(panels, t.hp3.data(), sizeof(TreePanel_3d) * P);
  }
  if (level_start) std::memcpy(level_start, t.info.level_start, sizeof(int) * (t.info.levels + 1));
  if (leaf_of) std::memcpy(leaf_of, t.hleaf.data(), sizeof(int) * t.n);
  if (inside) std::memcpy(inside, t.hinside.data(), sizeof(int) * t.hinside.size());
}

void btkref_get_lists(void* p, void* all, void* pp, void* pc, void* cp, void* cc) {
  Handle& h = *static_cast<Handle*>(p);
  auto cpy = [](void* dst, const view_interact_host& v) {
    if (dst && v.extent(0) > 0) std::memcpy(dst, v.data(), sizeof(interact_pair) * v.extent(0));
  };
  if (all && h.cfg.fmm_interaction_count > 0)
    std::memcpy(all, h.all.data(), sizeof(interact_pair) * h.cfg.fmm_interaction_count);
  cpy(pp, h.pp);
  cpy(pc, h.pc);
  cpy(cp, h.cp);
  cpy(cc, h.cc);
}

}  // extern "C"

// Fixed downward pass (see file header): the reference's functors, called on
// non-leaf parents only (levels 0..L-2, one parallel_for per level, as the
// reference's downward pass launches them) and on every leaf (one
// parallel_for).
template <class P2C, class L2P>
static void fixed_downward(Handle& h, const P2C& p2c, const L2P& l2p) {
  Tree& t = h.tgt;
  const int nchild = h.cfg.dim == 2 ? 4 : 8;
  for (int lev = 0; lev < t.info.levels - 1; ++lev) {
    std::vector<int> parents;
    for (int i = t.info.level_start[lev]; i < t.info.level_start[lev + 1]; ++i)
      if (!is_leaf_panel(h, t, i)) parents.push_back(i);
    Kokkos::parallel_for((int)parents.size() * nchild, [&](int k) { p2c(parents[k / nchild], k % nchild); });
  }
  std::vector<int> leaves;
  for (int i = 0; i < t.info.panel_count; ++i)
    if (is_leaf_panel(h, t, i)) leaves.push_back(i);
  Kokkos::parallel_for((int)leaves.size(), [&](int k) { l2p(leaves[k]); });
}

extern "C" {

// kind 0: potential (poisson_fmm_interactions_* + downward_pass_*);
// kind 1: 3-D "velocity" (poisson_vel_fmm_interactions_3d + downward_pass_3d_3).
// Outputs (any may be null): psw = proxy source weights after the upward pass
// [Ps x ipc]; ptw = proxy target weights after the interactions and before the
// downward pass [ncomp x Pt x ipc]; mid = per-target result after the
// interactions only [ncomp x nt]; out = final result [ncomp x nt].
int btkref_solve(void* p, int kind, int fixed, const double* charges, double* psw, double* ptw, double* mid,
                 double* out) {
  Handle& h = *static_cast<Handle*>(p);
  RunConfig& c = h.cfg;
  Tree& T = h.tgt;
  Tree& S = h.source();
  if (kind == 1 && c.dim != 3) return 2;
  const int ipc = c.interp_point_count;
  const int ncomp = kind == 1 ? 3 : 1;
  view_real q = make_view("charges", S.n, charges);
  view_reall w_src("psw", S.info.panel_count, ipc);
  std::vector<view_reall> w_tgt;
  std::vector<view_real> sol;
  for (int k = 0; k < ncomp; ++k) {
    w_tgt.emplace_back("ptw", T.info.panel_count, ipc);
    sol.emplace_back("sol", T.n);
  }
  if (c.dim == 2)
    upward_pass_2d(c, S.info, S.x, S.y, q, S.p2, w_src, S.leaf_of);
  else
    upward_pass_3d(c, S.info, S.x, S.y, S.z, q, S.p3, w_src, S.leaf_of);
  if (psw) std::memcpy(psw, w_src.data(), sizeof(double) * w_src.size());

  if (c.dim == 2) {
    poisson_fmm_interactions_2d(c, T.x, T.y, S.x, S.y, q, sol[0], S.inside, T.inside, w_src, w_tgt[0], h.dpp, h.dpc, h.dcp,
                                h.dcc, S.p2, T.p2);
  } else if (kind == 0) {
    poisson_fmm_interactions_3d(c, T.x, T.y, T.z, S.x, S.y, S.z, q, sol[0], S.inside, T.inside, w_src, w_tgt[0], h.dpp,
                                h.dpc, h.dcp, h.dcc, S.p3, T.p3);
  } else {
    poisson_vel_fmm_interactions_3d(c, T.x, T.y, T.z, S.x, S.y, S.z, q, sol[0], sol[1], sol[2], S.inside, T.inside,
                                    w_src, w_tgt[0], w_tgt[1], w_tgt[2], h.dpp, h.dpc, h.dcp, h.dcc, S.p3, T.p3);
  }
  for (int k = 0; k < ncomp; ++k) {
    if (ptw) std::memcpy(ptw + (size_t)k * w_tgt[k].size(), w_tgt[k].data(), sizeof(double) * w_tgt[k].size());
    if (mid) std::memcpy(mid + (size_t)k * T.n, sol[k].data(), sizeof(double) * T.n);
  }

  const int deg = c.interp_degree;
  if (!fixed) {
    if (c.dim == 2)
      downward_pass_2d(c, T.info, T.x, T.y, sol[0], T.p2, w_tgt[0], T.inside);
    else if (kind == 0)
      downward_pass_3d(c, T.info, T.x, T.y, T.z, sol[0], T.p3, w_tgt[0], T.inside);
    else
      downward_pass_3d_3(c, T.info, T.x, T.y, T.z, sol[0], sol[1], sol[2], T.p3, w_tgt[0], w_tgt[1], w_tgt[2],
                         T.inside);
  } else if (c.dim == 2) {
    fixed_downward(h, parent_to_child_2d(T.p2, w_tgt[0], deg),
                   leaf_to_point_2d(T.x, T.y, sol[0], w_tgt[0], T.p2, T.inside, deg));
  } else if (kind == 0) {
    fixed_downward(h, parent_to_child_3d(T.p3, w_tgt[0], deg),
                   leaf_to_point_3d(T.x, T.y, T.z, sol[0], w_tgt[0], T.p3, T.inside, deg));
  } else {
    fixed_downward(h, parent_to_child_3d_3(T.p3, w_tgt[0], w_tgt[1], w_tgt[2], deg),
                   leaf_to_point_3d_3(T.x, T.y, T.z, sol[0], sol[1], sol[2], w_tgt[0], w_tgt[1], w_tgt[2], T.p3,
                                      T.inside, deg));
  }
  for (int k = 0; k < ncomp; ++k)
    if (out) std::memcpy(out + (size_t)k * T.n, sol[k].data(), sizeof(double) * T.n);
  return 0;
}

// The same solve restricted to the targets of a few sampled leaves, for
// parity checks at sizes where a whole reference solve takes too long. The
// upward pass runs in full (the reference's upward_pass_2d/3d). Then:
//   * needed target panels = the sampled leaves and all their ancestors;
//   * each interaction list keeps the pairs whose target panel is needed, in
//     list order, and the reference's own poisson_fmm_interactions_* /
//     poisson_vel_fmm_interactions_3d runs on those sub-lists (the counts in a
//     copy of the RunConfig are set to the sub-list lengths);
//   * the fixed downward pass runs parent_to_child on (non-leaf parent, child)
//     pairs whose child is needed, level by level, and leaf_to_point on the
//     sampled leaves only.
// Every needed panel then holds exactly what the full solve gives it, so the
// output at the sampled leaves' targets equals the full (fixed) solve's. Other
// targets hold partial sums; callers read the sampled leaves' targets only.
// kind 0 potential, 1 3-D velocity; out [ncomp x nt].
int btkref_solve_leaves(void* p, int kind, const double* charges, int n_leaves, const int* leaves, double* out) {
  Handle& h = *static_cast<Handle*>(p);
  RunConfig c = h.cfg;
  Tree& T = h.tgt;
  Tree& S = h.source();
  if (kind == 1 && c.dim != 3) return 2;
  const int Pt = T.info.panel_count;
  std::vector<char> needed(Pt, 0), sampled(Pt, 0);
  for (int k = 0; k < n_leaves; ++k) {
    int i = leaves[k];
    if (i < 0 || i >= Pt || !is_leaf_panel(h, T, i)) return 3;
    sampled[i] = 1;
    while (i >= 0 && !needed[i]) {
      needed[i] = 1;
      i = c.dim == 2 ? T.hp2(i).parent_id : T.hp3(i).parent_id;
    }
  }
  auto filter = [&](const view_interact_host& L, const char* label, int& count) {
    std::vector<interact_pair> keep;
    for (int i = 0; i < (int)L.extent(0); ++i)
      if (needed[L(i).target_panel]) keep.push_back(L(i));
    count = (int)keep.size();
    view_interact d(label, std::max<size_t>(keep.size(), 1));
    if (!keep.empty()) std::memcpy(d.data(), keep.data(), sizeof(interact_pair) * keep.size());
    return d;
  };
  view_interact fpp = filter(h.pp, "pp", c.fmm_pp_count), fpc = filter(h.pc, "pc", c.fmm_pc_count);
  view_interact fcp = filter(h.cp, "cp", c.fmm_cp_count), fcc = filter(h.cc, "cc", c.fmm_cc_count);
  c.fmm_interaction_count = c.fmm_pp_count + c.fmm_pc_count + c.fmm_cp_count + c.fmm_cc_count;

  const int ipc = c.interp_point_count;
  const int ncomp = kind == 1 ? 3 : 1;
  view_real q = make_view("charges", S.n, charges);
  view_reall w_src("psw", S.info.panel_count, ipc);
  std::vector<view_reall> w_tgt;
  std::vector<view_real> sol;
  for (int k = 0; k < ncomp; ++k) {
    w_tgt.emplace_back("ptw", Pt, ipc);
    sol.emplace_back("sol", T.n);
  }
  if (c.dim == 2)
    upward_pass_2d(c, S.info, S.x, S.y, q, S.p2, w_src, S.leaf_of);
  else
    upward_pass_3d(c, S.info, S.x, S.y, S.z, q, S.p3, w_src, S.leaf_of);
  if (c.dim == 2)
    poisson_fmm_interactions_2d(c, T.x, T.y, S.x, S.y, q, sol[0], S.inside, T.inside, w_src, w_tgt[0], fpp, fpc, fcp,
                                fcc, S.p2, T.p2);
  else if (kind == 0)
    poisson_fmm_interactions_3d(c, T.x, T.y, T.z, S.x, S.y, S.z, q, sol[0], S.inside, T.inside, w_src, w_tgt[0], fpp,
                                fpc, fcp, fcc, S.p3, T.p3);
  else
    poisson_vel_fmm_interactions_3d(c, T.x, T.y, T.z, S.x, S.y, S.z, q, sol[0], sol[1], sol[2], S.inside, T.inside,
                                    w_src, w_tgt[0], w_tgt[1], w_tgt[2], fpp, fpc, fcp, fcc, S.p3, T.p3);

  const int deg = c.interp_degree;
  const int nchild = c.dim == 2 ? 4 : 8;
  auto child_of = [&](int i, int j) {
    if (c.dim == 2) {
      const TreePanel_2d& P = T.hp2(i);
      const int ch[4] = {P.child1, P.child2, P.child3, P.child4};
      return ch[j];
    }
    const TreePanel_3d& P = T.hp3(i);
    const int ch[8] = {P.child1, P.child2, P.child3, P.child4, P.child5, P.child6, P.child7, P.child8};
    return ch[j];
  };
  // One parallel_for per level (a level's children are distinct panels), as
  // the reference's downward pass launches its functors.
  auto down = [&](const auto& p2c, const auto& l2p) {
    for (int lev = 0; lev < T.info.levels - 1; ++lev) {
      std::vector<int> ij;
      for (int i = T.info.level_start[lev]; i < T.info.level_start[lev + 1]; ++i)
        if (needed[i] && !is_leaf_panel(h, T, i))
          for (int j = 0; j < nchild; ++j)
            if (needed[child_of(i, j)]) ij.push_back(i * nchild + j);
      Kokkos::parallel_for((int)ij.size(), [&](int k) { p2c(ij[k] / nchild, ij[k] % nchild); });
    }
    std::vector<int> ls;
    for (int i = 0; i < Pt; ++i)
      if (sampled[i]) ls.push_back(i);
    Kokkos::parallel_for((int)ls.size(), [&](int k) { l2p(ls[k]); });
  };
  if (c.dim == 2)
    down(parent_to_child_2d(T.p2, w_tgt[0], deg), leaf_to_point_2d(T.x, T.y, sol[0], w_tgt[0], T.p2, T.inside, deg));
  else if (kind == 0)
    down(parent_to_child_3d(T.p3, w_tgt[0], deg),
         leaf_to_point_3d(T.x, T.y, T.z, sol[0], w_tgt[0], T.p3, T.inside, deg));
  else
    down(parent_to_child_3d_3(T.p3, w_tgt[0], w_tgt[1], w_tgt[2], deg),
         leaf_to_point_3d_3(T.x, T.y, T.z, sol[0], sol[1], sol[2], w_tgt[0], w_tgt[1], w_tgt[2], T.p3, T.inside,
                            deg));
  for (int k = 0; k < ncomp; ++k) std::memcpy(out + (size_t)k * T.n, sol[k].data(), sizeof(double) * T.n);
  return 0;
}

// Direct sum with the reference's functors (src/direct_sum_impl.hpp), over
// all nt x ns pairs through an MDRangePolicy, as the examples do
// (examples/example_poisson_3d.cpp:165). kind 0 = potential, 1 = 3-D velocity.
int btkref_direct(int dim, int kind, int nt, const double* tx, const double* ty, const double* tz, int ns,
                  const double* sx, const double* sy, const double* sz, const double* charges, double eps,
                  double* out) {
  view_real txv = make_view("tx", nt, tx), tyv = make_view("ty", nt, ty);
  view_real sxv = make_view("sx", ns, sx), syv = make_view("sy", ns, sy);
  view_real q = make_view("q", ns, charges);
  view_real o0("o0", nt), o1("o1", nt), o2("o2", nt);
  if (dim == 2) {
    Kokkos::parallel_for(Kokkos::MDRangePolicy({0, 0}, {nt, ns}), poisson_2d_dir_sum(txv, tyv, sxv, syv, q, o0, eps));
  } else {
    view_real tzv = make_view("tz", nt, tz), szv = make_view("sz", ns, sz);
    if (kind == 0)
      Kokkos::parallel_for(Kokkos::MDRangePolicy({0, 0}, {nt, ns}),
                           poisson_3d_dir_sum(txv, tyv, tzv, sxv, syv, szv, q, o0, eps));
    else
      Kokkos::parallel_for(Kokkos::MDRangePolicy({0, 0}, {nt, ns}),
                           poisson_vel_3d_dir_sum(txv, tyv, tzv, sxv, syv, szv, q, o0, o1, o2, eps));
  }
  std::memcpy(out, o0.data(), sizeof(double) * nt);
  if (kind == 1) {
    std::memcpy(out + nt, o1.data(), sizeof(double) * nt);
    std::memcpy(out + 2 * (size_t)nt, o2.data(), sizeof(double) * nt);
  }
  return 0;
}

// Timed, strided samples of each phase of a 3-D solve (kind 0 potential,
// 1 velocity), for the CPU baseline. Every `stride`-th work item of each
// phase (denser for phases with fewer than 8 items per thread per stride) is
// run through the reference's own functor, under the OpenMP parallel_for of
// the shim. Per phase p (0 base_pots, 1 child_to_parent,
// 2 pp, 3 pc, 4 cp, 5 cc, 6 parent_to_child, 7 leaf_to_point):
//   sec[p]   = wall seconds of the sample,
//   scale[p] = full-phase work / sampled work (kernel evaluations for 2..5,
//              work items otherwise), so sec[p]*scale[p] estimates the phase.
// evals[0] = kernel evaluations in the sampled interaction items,
// evals[1] = kernel evaluations of the full interaction phase.
int btkref_time_sample_3d(void* p, int kind, int stride, const double* charges, double* sec, double* scale,
                          double* evals) {
  Handle& h = *static_cast<Handle*>(p);
  RunConfig& c = h.cfg;
  if (c.dim != 3 || stride < 1) return 2;
  Tree& T = h.tgt;
  Tree& S = h.source();
  const int ipc = c.interp_point_count, deg = c.interp_degree;
  view_real q = make_view("charges", S.n, charges);
  view_reall w_src("psw", S.info.panel_count, ipc);
  view_reall wx("ptw", T.info.panel_count, ipc), wy("ptwy", T.info.panel_count, ipc), wz("ptwz", T.info.panel_count, ipc);
  view_real s0("s0", T.n), s1("s1", T.n), s2("s2", T.n);
  double eps = c.ker_eps;
  // A phase with few work items is sampled more densely (at least 8 items
  // per thread, or all of them), so the sample keeps every thread busy as
  // the full phase does; scale[] follows the items actually run.
  const int min_items = 8 * Kokkos::num_threads();
  auto stride_of = [&](int count) { return std::max(1, std::min(stride, count / std::max(1, min_items))); };
  auto strided = [&](int count, auto&& f, double& sampled) {
    const int st = stride_of(count);
    int m = (count + st - 1) / st;
    sampled = m;
    auto t0 = std::chrono::steady_clock::now();
    Kokkos::parallel_for(m, [&](int k) { f(k * st); });
    return seconds_since(t0);
  };
  double sampled = 0;
  // 0: base_pots over points
  sec[0] = strided(S.n, base_pots_3d(S.x, S.y, S.z, q, S.p3, w_src, S.leaf_of, deg), sampled);
  scale[0] = S.n / sampled;
  // 1: child_to_parent over panels of levels 1..L-1
  {
    int lo = S.info.level_start[1 < S.info.levels ? 1 : 0], hi = S.info.panel_count;
    child_to_parent_3d f(S.p3, w_src, deg);
    sec[1] = strided(hi - lo, [&](int i) { f(lo + i); }, sampled);
    scale[1] = (hi - lo) / (sampled > 0 ? sampled : 1);
  }
  auto pair_evals = [&](const view_interact_host& L, int type, int i) -> double {
    int tp = L(i).target_panel, sp = L(i).source_panel;
    double mt = type >= 2 ? ipc : T.p3(tp).point_count;
    double ms = (type == 1 || type == 3) ? ipc : S.p3(sp).point_count;
    return mt * ms;
  };
  const view_interact_host* lists[4] = {&h.pp, &h.pc, &h.cp, &h.cc};
  const view_interact* dlists[4] = {&h.dpp, &h.dpc, &h.dcp, &h.dcc};
  double total_evals = 0, sampled_evals = 0;
  for (int type = 0; type < 4; ++type) {
    const view_interact_host& L = *lists[type];
    int count = L.extent_int(0);
    double full = 0, part = 0;
    const int st = stride_of(count);
    for (int i = 0; i < count; ++i) {
      double e = pair_evals(L, type, i);
      full += e;
      if (i % st == 0) part += e;
    }
    view_interact dL = *dlists[type];
    double sec_t = 0;
    if (kind == 0) {
      if (type == 0) sec_t = strided(count, poisson_pp_interaction_3d(T.x, T.y, T.z, S.x, S.y, S.z, q, s0, T.inside, S.inside, dL, T.p3, S.p3, eps), sampled);
      if (type == 1) sec_t = strided(count, poisson_pc_interaction_3d(T.x, T.y, T.z, s0, T.inside, w_src, dL, T.p3, S.p3, eps, deg), sampled);
      if (type == 2) sec_t = strided(count, poisson_cp_interaction_3d(S.x, S.y, S.z, q, S.inside, wx, dL, T.p3, S.p3, eps, deg), sampled);
      if (type == 3) sec_t = strided(count, poisson_cc_interaction_3d(wx, w_src, dL, T.p3, S.p3, eps, deg), sampled);
    } else {
      if (type == 0) sec_t = strided(count, poisson_vel_pp_interaction_3d(T.x, T.y, T.z, S.x, S.y, S.z, q, s0, s1, s2, T.inside, S.inside, dL, T.p3, S.p3, eps), sampled);
      if (type == 1) sec_t = strided(count, poisson_vel_pc_interaction_3d(T.x, T.y, T.z, s0, s1, s2, T.inside, w_src, dL, T.p3, S.p3, eps, deg), sampled);
      if (type == 2) sec_t = strided(count, poisson_vel_cp_interaction_3d(S.x, S.y, S.z, q, S.inside, wx, wy, wz, dL, T.p3, S.p3, eps, deg), sampled);
      if (type == 3) sec_t = strided(count, poisson_vel_cc_interaction_3d(wx, wy, wz, w_src, dL, T.p3, S.p3, eps, deg), sampled);
    }
    sec[2 + type] = sec_t;
    scale[2 + type] = part > 0 ? full / part : 0;
    total_evals += full;
    sampled_evals += part;
  }
  // 6: parent_to_child over (non-leaf parent, child) pairs
  {
    std::vector<int> parents;
    for (int i = 0; i < T.info.panel_count; ++i)
      if (!T.p3(i).is_leaf) parents.push_back(i);
    int m = (int)parents.size() * 8;
    if (kind == 0) {
      parent_to_child_3d f(T.p3, wx, deg);
      sec[6] = strided(m, [&](int k) { f(parents[k / 8], k % 8); }, sampled);
    } else {
      parent_to_child_3d_3 f(T.p3, wx, wy, wz, deg);
      sec[6] = strided(m, [&](int k) { f(parents[k / 8], k % 8); }, sampled);
    }
    scale[6] = m / (sampled > 0 ? sampled : 1);
  }
  // 7: leaf_to_point over leaves
  {
    std::vector<int> leaves;
    for (int i = 0; i < T.info.panel_count; ++i)
      if (T.p3(i).is_leaf) leaves.push_back(i);
    int m = (int)leaves.size();
    if (kind == 0) {
      leaf_to_point_3d f(T.x, T.y, T.z, s0, wx, T.p3, T.inside, deg);
      sec[7] = strided(m, [&](int k) { f(leaves[k]); }, sampled);
    } else {
      leaf_to_point_3d_3 f(T.x, T.y, T.z, s0, s1, s2, wx, wy, wz, T.p3, T.inside, deg);
      sec[7] = strided(m, [&](int k) { f(leaves[k]); }, sampled);
    }
    scale[7] = m / (sampled > 0 ? sampled : 1);
  }
  evals[0] = sampled_evals;
  evals[1] = total_evals;
  return 0;
}

}  // extern "C"
