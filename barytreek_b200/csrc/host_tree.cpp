// Host tree functions: namelist, tree construction, dual-tree traversal and
// list split. Their outputs are bit-identical to the reference's host C++
// (src/read_namelist.cpp, src/tree_construction.cpp, src/interaction_list.cpp):
// same panel order (breadth-first, children appended in the reference's child
// order), same floating-point expressions in the same evaluation order, same
// leaf point order (ascending original index) and same pair order. This file is
// compiled with -ffp-contract=off so no expression is fused differently.
//
// Deliberate difference: a panel holding more than cluster_size coincident
// points makes the reference refine forever; here refinement past depth 60
// returns BTK_ERR_INVALID_ARGUMENT instead.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "btk_internal.h"

namespace btk {

namespace {
thread_local std::string g_last_error;
std::uint64_t g_launches = 0;
}  // namespace

btk_status set_error(btk_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

btk_status cuda_error(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? BTK_ERR_OUT_OF_MEMORY : BTK_ERR_CUDA;
}

void count_launch(int n) { __atomic_fetch_add(&g_launches, (std::uint64_t)n, __ATOMIC_RELAXED); }

namespace {

// Dimension-generic view of the reference panel records.
template <int D> struct PanelT;
template <> struct PanelT<2> { using type = btk_panel_2d; };
template <> struct PanelT<3> { using type = btk_panel_3d; };

inline int* child_slot(btk_panel_2d& p, int c) { return &p.child1 + c; }
inline int* child_slot(btk_panel_3d& p, int c) { return &p.child1 + c; }
inline int child_of(const btk_panel_2d& p, int c) { return (&p.child1)[c]; }
inline int child_of(const btk_panel_3d& p, int c) { return (&p.child1)[c]; }

inline void set_box(btk_panel_2d& p, const double* lo, const double* hi) {
  p.min_x = lo[0]; p.max_x = hi[0]; p.min_y = lo[1]; p.max_y = hi[1];
}
inline void set_box(btk_panel_3d& p, const double* lo, const double* hi) {
  p.min_x = lo[0]; p.max_x = hi[0]; p.min_y = lo[1]; p.max_y = hi[1]; p.min_z = lo[2]; p.max_z = hi[2];
}
inline void get_box(const btk_panel_2d& p, double* lo, double* hi) {
  lo[0] = p.min_x; hi[0] = p.max_x; lo[1] = p.min_y; hi[1] = p.max_y;
}
inline void get_box(const btk_panel_3d& p, double* lo, double* hi) {
  lo[0] = p.min_x; hi[0] = p.max_x; lo[1] = p.min_y; hi[1] = p.max_y; lo[2] = p.min_z; hi[2] = p.max_z;
}

template <class P>
P fresh_panel() {
  P p;
  std::memset(&p, 0, sizeof(P));
  p.parent_id = -1;
  int nc = sizeof(P) == sizeof(btk_panel_2d) ? 4 : 8;
  for (int c = 0; c < nc; ++c) *child_slot(p, c) = -1;
  p.is_leaf = true;
  p.point_count = 0;
  return p;
}

// Child boxes in the reference's child order (tree_construction.cpp:51-54 for
// 2-D, :187-194 for 3-D): upper/lower z halves, each in the order
// (hi x, hi y), (lo x, hi y), (lo x, lo y), (hi x, lo y).
template <int D>
void child_box(int c, const double* lo, const double* mid, const double* hi, double* clo, double* chi) {
  static const int hx[4] = {1, 0, 0, 1}, hy[4] = {1, 1, 0, 0};
  int q = c & 3;
  clo[0] = hx[q] ? mid[0] : lo[0]; chi[0] = hx[q] ? hi[0] : mid[0];
  clo[1] = hy[q] ? mid[1] : lo[1]; chi[1] = hy[q] ? hi[1] : mid[1];
  if (D == 3) {
    bool upper = c < 4;
    clo[2] = upper ? mid[2] : lo[2];
    chi[2] = upper ? hi[2] : mid[2];
  }
}

// Which child a point falls in; ties (== midpoint) go to the lower half
// (tree_construction.cpp:81-93, :240-268).
template <int D>
int which_child(const double* pt, const double* mid) {
  int q = (pt[0] > mid[0]) ? ((pt[1] > mid[1]) ? 0 : 3) : ((pt[1] > mid[1]) ? 1 : 2);
  if (D == 3 && !(pt[2] > mid[2])) q += 4;
  return q;
}

template <int D>
btk_status build_tree(const btk_run_config* cfg, btk_tree_info* info, const double* const* xyz, int n,
                      typename PanelT<D>::type** panels_out, int* leaf_of, int** inside_out) {
  using P = typename PanelT<D>::type;
  constexpr int NC = 1 << D;
  BTK_CHECK(cfg && info && panels_out && inside_out && (n == 0 || leaf_of), BTK_ERR_INVALID_ARGUMENT,
            "tree_construction: null argument");
  BTK_CHECK(n >= 0, BTK_ERR_INVALID_ARGUMENT, "tree_construction: negative point count");
  for (int d = 0; d < D; ++d) BTK_CHECK(n == 0 || xyz[d], BTK_ERR_INVALID_ARGUMENT, "tree_construction: null coordinates");
  const int thresh = cfg->fmm_cluster_thresh;
  BTK_CHECK(thresh > 0, BTK_ERR_INVALID_ARGUMENT, "tree_construction: fmm_cluster_thresh must be positive");

  std::vector<P> panels(1, fresh_panel<P>());
  // Points of each panel as a range of `order`; children partition their
  // parent's range stably, so every leaf lists ascending original indices.
  std::vector<int> order(n), begin(1, 0), count(1, n), scratch(n);
  for (int i = 0; i < n; ++i) order[i] = i;

  // Root box (tree_construction.cpp:145-167). The reference starts every max
  // at numeric_limits<real>::min() (the smallest positive double); kept.
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int d = 0; d < D; ++d) {
    lo[d] = std::numeric_limits<double>::max();
    hi[d] = std::numeric_limits<double>::min();
  }
  for (int i = 0; i < n; ++i) {
    leaf_of[i] = 0;
    for (int d = 0; d < D; ++d) {
      lo[d] = std::min(lo[d], xyz[d][i]);
      hi[d] = std::max(hi[d], xyz[d][i]);
    }
  }
  panels[0].id = 0;
  panels[0].level = 0;
  panels[0].point_count = n;
  panels[0].is_leaf = true;
  set_box(panels[0], lo, hi);

  for (size_t i = 0; i < panels.size(); ++i) {
    if (!(panels[i].point_count > thresh && panels[i].is_leaf)) continue;
    BTK_CHECK(panels[i].level < 60, BTK_ERR_INVALID_ARGUMENT,
              "tree_construction: more than fmm_cluster_thresh coincident points (refinement does not terminate)");
    panels[i].is_leaf = false;
    const int base = (int)panels.size();
    const int lev = panels[i].level;
    double plo[3], phi[3], mid[3];
    get_box(panels[i], plo, phi);
    for (int d = 0; d < D; ++d) mid[d] = 0.5 * (plo[d] + phi[d]);
    for (int c = 0; c < NC; ++c) {
      P ch = fresh_panel<P>();
      double clo[3], chi[3];
      child_box<D>(c, plo, mid, phi, clo, chi);
      set_box(ch, clo, chi);
      ch.parent_id = (int)i;
      ch.level = lev + 1;
      ch.id = base + c;
      *child_slot(panels[i], c) = ch.id;
      panels.push_back(ch);
      begin.push_back(0);
      count.push_back(0);
    }
    // Stable partition of the parent's point range into the children.
    const int b = begin[i], m = count[i];
    int cnt[NC] = {0};
    std::vector<int> which(m);
    for (int j = 0; j < m; ++j) {
      int idx = order[b + j];
      double pt[3] = {xyz[0][idx], xyz[1][idx], D == 3 ? xyz[2][idx] : 0.0};
      which[j] = which_child<D>(pt, mid);
      cnt[which[j]]++;
    }
    int off[NC];
    int acc = b;
    for (int c = 0; c < NC; ++c) {
      off[c] = acc;
      begin[base + c] = acc;
      count[base + c] = cnt[c];
      panels[base + c].point_count = cnt[c];
      acc += cnt[c];
    }
    for (int j = 0; j < m; ++j) scratch[off[which[j]]++] = order[b + j];
    for (int j = 0; j < m; ++j) {
      order[b + j] = scratch[b + j];
    }
    for (int c = 0; c < NC; ++c)
      for (int j = 0; j < cnt[c]; ++j) leaf_of[order[begin[base + c] + j]] = base + c;
  }

  // Finalise (tree_construction.cpp:278-305): radius, level_start, leaf lists.
  const int P_count = (int)panels.size();
  const int levels = panels.back().level + 1;
  info->panel_count = P_count;
  info->levels = levels;
  info->level_start = (int*)std::malloc(sizeof(int) * (levels + 1));
  int* inside = (int*)std::calloc((size_t)P_count * thresh, sizeof(int));
  P* out = (P*)std::malloc(sizeof(P) * P_count);
  if (!info->level_start || !inside || !out) {
    std::free(info->level_start);
    std::free(inside);
    std::free(out);
    info->level_start = nullptr;
    return set_error(BTK_ERR_OUT_OF_MEMORY, "tree_construction: host allocation failed");
  }
  info->level_start[0] = 0;
  int target_level = 1;
  for (int i = 0; i < P_count; ++i) {
    P& p = panels[i];
    if (p.is_leaf)
      for (int j = 0; j < p.point_count; ++j) inside[(size_t)i * thresh + j] = order[begin[i] + j];
    double plo[3], phi[3];
    get_box(p, plo, phi);
    double x_ex = phi[0] - plo[0], y_ex = phi[1] - plo[1];
    if (D == 2) {
      p.radius = 0.5 * std::sqrt(x_ex * x_ex + y_ex * y_ex);
    } else {
      double z_ex = phi[2] - plo[2];
      p.radius = 0.5 * std::sqrt(x_ex * x_ex + y_ex * y_ex + z_ex * z_ex);
    }
    if (p.level == target_level) {
      info->level_start[target_level] = i;
      target_level += 1;
    }
    out[i] = p;
  }
  info->level_start[levels] = P_count;
  *panels_out = out;
  *inside_out = inside;
  return BTK_OK;
}

// Dual-tree traversal (interaction_list.cpp:5-117 / :119-250): breadth-first
// over (target, source) pairs starting at the roots; MAC
// (r_T + r_S) / dist < theta; classification by point_count > thresh.
template <int D>
btk_status traverse(btk_run_config* cfg, const typename PanelT<D>::type* T, const typename PanelT<D>::type* S,
                    btk_interact_pair** list_out) {
  constexpr int NC = 1 << D;
  BTK_CHECK(cfg && T && S && list_out, BTK_ERR_INVALID_ARGUMENT, "dual_tree_traversal: null argument");
  std::vector<btk_interact_pair> list;
  int counts[4] = {0, 0, 0, 0};
  std::vector<int> qt{0}, qs{0};  // FIFO as vectors with a read cursor
  size_t head = 0;
  const double theta = cfg->fmm_theta;
  const int thresh = cfg->fmm_cluster_thresh;
  while (head < qt.size()) {
    int it = qt[head], is = qs[head];
    ++head;
    double tlo[3], thi[3], slo[3], shi[3];
    get_box(T[it], tlo, thi);
    get_box(S[is], slo, shi);
    double c1[3], c2[3];
    for (int d = 0; d < D; ++d) {
      c1[d] = 0.5 * (tlo[d] + thi[d]);
      c2[d] = 0.5 * (slo[d] + shi[d]);
    }
    double x_ex = c2[0] - c1[0], y_ex = c2[1] - c1[1];
    double dist;
    if (D == 2) {
      dist = std::sqrt(x_ex * x_ex + y_ex * y_ex);
    } else {
      double z_ex = c2[2] - c1[2];
      dist = std::sqrt(x_ex * x_ex + y_ex * y_ex + z_ex * z_ex);
    }
    double separation = 100;
    if (dist > 0) separation = (T[it].radius + S[is].radius) / dist;
    if (separation < theta) {
      int type = 0;
      if (T[it].point_count > thresh) type += 2;
      if (S[is].point_count > thresh) type += 1;
      counts[type]++;
      list.push_back({it, is, type});
    } else {
      bool t_leaf = T[it].is_leaf, s_leaf = S[is].is_leaf;
      bool refine_target = false, refine_source = false;
      if (t_leaf && s_leaf) {
        list.push_back({it, is, 0});
        counts[0]++;
      } else if (t_leaf) {
        refine_source = true;
      } else if (s_leaf) {
        refine_target = true;
      } else if (T[it].point_count > S[is].point_count) {
        refine_target = true;
      } else {
        refine_source = true;
      }
      if (refine_target) {
        for (int c = 0; c < NC; ++c) {
          qt.push_back(child_of(T[it], c));
          qs.push_back(is);
        }
      } else if (refine_source) {
        for (int c = 0; c < NC; ++c) {
          qt.push_back(it);
          qs.push_back(child_of(S[is], c));
        }
      }
    }
    // The queue only grows; drop the consumed prefix now and then.
    if (head > (1u << 20) && head * 2 > qt.size()) {
      qt.erase(qt.begin(), qt.begin() + head);
      qs.erase(qs.begin(), qs.begin() + head);
      head = 0;
    }
  }
  cfg->fmm_interaction_count = (int)list.size();
  cfg->fmm_pp_count = counts[0];
  cfg->fmm_pc_count = counts[1];
  cfg->fmm_cp_count = counts[2];
  cfg->fmm_cc_count = counts[3];
  btk_interact_pair* out = (btk_interact_pair*)std::malloc(sizeof(btk_interact_pair) * (list.size() ? list.size() : 1));
  BTK_CHECK(out, BTK_ERR_OUT_OF_MEMORY, "dual_tree_traversal: host allocation failed");
  if (!list.empty()) std::memcpy(out, list.data(), sizeof(btk_interact_pair) * list.size());
  *list_out = out;
  return BTK_OK;
}

}  // namespace

void host_tree_from_panels(int dim, const void* panels, int panel_count, const int* level_start, int levels,
                           HostTree& t) {
  t.dim = dim;
  t.panel_count = panel_count;
  t.levels = levels;
  t.level_start.assign(level_start, level_start + levels + 1);
  const int nc = 1 << dim;
  t.geom.resize(panel_count);
  t.parent.resize(panel_count);
  t.level.resize(panel_count);
  t.is_leaf.resize(panel_count);
  t.point_count.resize(panel_count);
  t.child.assign((size_t)panel_count * nc, -1);
  for (int i = 0; i < panel_count; ++i) {
    if (dim == 2) {
      const btk_panel_2d& p = static_cast<const btk_panel_2d*>(panels)[i];
      get_box(p, t.geom[i].lo, t.geom[i].hi);
      t.geom[i].lo[2] = t.geom[i].hi[2] = 0;
      t.parent[i] = p.parent_id;
      t.level[i] = p.level;
      t.is_leaf[i] = p.is_leaf;
      t.point_count[i] = p.point_count;
      for (int c = 0; c < 4; ++c) t.child[(size_t)i * nc + c] = child_of(p, c);
    } else {
      const btk_panel_3d& p = static_cast<const btk_panel_3d*>(panels)[i];
      get_box(p, t.geom[i].lo, t.geom[i].hi);
      t.parent[i] = p.parent_id;
      t.level[i] = p.level;
      t.is_leaf[i] = p.is_leaf;
      t.point_count[i] = p.point_count;
      for (int c = 0; c < 8; ++c) t.child[(size_t)i * nc + c] = child_of(p, c);
    }
  }
}

// Rebuilds level_start from the panels' level fields (panels are stored in
// level order by construction), for callers that only hold the panel array.
bool host_tree_from_panels_nolevels(int dim, const void* panels, int panel_count, HostTree& t) {
  std::vector<int> ls{0};
  int cur = 0;
  for (int i = 0; i < panel_count; ++i) {
    int lev = dim == 2 ? static_cast<const btk_panel_2d*>(panels)[i].level
                       : static_cast<const btk_panel_3d*>(panels)[i].level;
    if (lev < cur) return false;
    while (lev > cur) {
      ls.push_back(i);
      ++cur;
    }
  }
  ls.push_back(panel_count);
  host_tree_from_panels(dim, panels, panel_count, ls.data(), (int)ls.size() - 1, t);
  return true;
}

}  // namespace btk

using namespace btk;

extern "C" {

const char* btk_last_error(void) { return g_last_error.c_str(); }
const char* btk_version(void) { return "barytreek_b200 0.1"; }
uint64_t btk_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }
int btk_max_degree(void) { return kMaxDegree; }
void btk_free(void* p) { std::free(p); }

btk_status btk_read_run_config(const char* file_name, btk_run_config* cfg) {
  BTK_CHECK(file_name && cfg, BTK_ERR_INVALID_ARGUMENT, "read_run_config: null argument");
  std::ifstream f(file_name);
  if (f.fail()) return set_error(BTK_ERR_IO, std::string("namelist not found: ") + file_name);
  // Key/value lines until the first key that is not one of the four
  // (read_namelist.cpp:19-42); "end" terminates by convention. End of file
  // also terminates: the reference re-parses its last line forever when the
  // file ends without a newline and without a terminating key (a failed
  // getline leaves `line` unchanged), which is not reproduced.
  std::string line, key, value;
  try {
    while (true) {
      if (!std::getline(f, line)) return BTK_OK;
      std::stringstream ss(line);
      std::getline(ss, key, '=');
      std::getline(ss, value);
      if (key == "interp_degree") {
        cfg->interp_degree = std::stoi(value);
        if (cfg->interp_degree > 10) cfg->interp_degree = 10;  // max_degree, barytreek-config.h.in:20
        cfg->interp_point_count = (int)std::pow(cfg->interp_degree + 1, cfg->dim);
      } else if (key == "cluster_size") {
        cfg->fmm_cluster_thresh = std::stoi(value);
        if (cfg->fmm_cluster_thresh <= 0)
          cfg->fmm_cluster_thresh = (int)(std::pow(2, cfg->dim) * cfg->interp_point_count);
      } else if (key == "theta") {
        cfg->fmm_theta = std::stod(value);
      } else if (key == "kernel_eps") {
        cfg->ker_eps = std::stod(value);
      } else {
        return BTK_OK;
      }
    }
  } catch (const std::exception& e) {
    return set_error(BTK_ERR_INVALID_ARGUMENT, std::string("read_run_config: bad value for ") + key);
  }
}

btk_status btk_tree_construction_2d(const btk_run_config* cfg, btk_tree_info* info, const double* xcos,
                                    const double* ycos, int point_count, btk_panel_2d** panels,
                                    int* point_leaf_panel, int** panel_points_inside) {
  const double* xyz[3] = {xcos, ycos, nullptr};
  return build_tree<2>(cfg, info, xyz, point_count, panels, point_leaf_panel, panel_points_inside);
}

btk_status btk_tree_construction_3d(const btk_run_config* cfg, btk_tree_info* info, const double* xcos,
                                    const double* ycos, const double* zcos, int point_count, btk_panel_3d** panels,
                                    int* point_leaf_panel, int** panel_points_inside) {
  const double* xyz[3] = {xcos, ycos, zcos};
  return build_tree<3>(cfg, info, xyz, point_count, panels, point_leaf_panel, panel_points_inside);
}

btk_status btk_dual_tree_traversal_2d(btk_run_config* cfg, const btk_panel_2d* panels_target,
                                      const btk_panel_2d* panels_source, btk_interact_pair** interaction_list) {
  return traverse<2>(cfg, panels_target, panels_source, interaction_list);
}

btk_status btk_dual_tree_traversal_3d(btk_run_config* cfg, const btk_panel_3d* panels_target,
                                      const btk_panel_3d* panels_source, btk_interact_pair** interaction_list) {
  return traverse<3>(cfg, panels_target, panels_source, interaction_list);
}

btk_status btk_split_interactions(const btk_interact_pair* list, int count, btk_interact_pair* pp,
                                  btk_interact_pair* pc, btk_interact_pair* cp, btk_interact_pair* cc) {
  BTK_CHECK(count == 0 || list, BTK_ERR_INVALID_ARGUMENT, "split_interactions: null list");
  btk_interact_pair* dst[4] = {pp, pc, cp, cc};
  int loc[4] = {0, 0, 0, 0};
  for (int i = 0; i < count; ++i) {
    int t = list[i].interact_type;
    BTK_CHECK(t >= 0 && t < 4, BTK_ERR_INVALID_ARGUMENT, "split_interactions: bad interact_type");
    BTK_CHECK(dst[t], BTK_ERR_INVALID_ARGUMENT, "split_interactions: null output list");
    dst[t][loc[t]++] = list[i];
  }
  return BTK_OK;
}

}  // extern "C"
