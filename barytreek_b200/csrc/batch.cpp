// Batches of independent treecode problems as one forest plan.
//
// Each problem's tree, traversal and split come from the host tree functions
// (bit-identical to the reference's host code, with the problem's own leaf
// size); host threads build the problems in parallel. The trees are then
// renumbered level-major into one panel array, so every per-level pass of the
// plan (upward child-to-parent, downward parent-to-child) and the single
// persistent interaction launch cover all problems at once; the lists never
// pair panels of different problems, so the problems stay independent. The
// solve is captured into a CUDA graph once and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "btk_internal.h"

namespace btk {
namespace {

int& child_ref(btk_panel_3d& p, int c) {
  switch (c) {
    case 0: return p.child1;
    case 1: return p.child2;
    case 2: return p.child3;
    case 3: return p.child4;
    case 4: return p.child5;
    case 5: return p.child6;
    case 6: return p.child7;
    default: return p.child8;
  }
}
int& child_ref(btk_panel_2d& p, int c) {
  switch (c) {
    case 0: return p.child1;
    case 1: return p.child2;
    case 2: return p.child3;
    default: return p.child4;
  }
}

// One problem's host tree and lists.
template <class Panel>
struct ProblemTree {
  btk_status status = BTK_OK;
  std::string error;
  btk_run_config cfg{};
  btk_tree_info info{};
  Panel* panels = nullptr;
  int* inside = nullptr;
  std::vector<int> leaf_of;
  std::vector<btk_interact_pair> lists[4];
  ~ProblemTree() {
    std::free(panels);
    std::free(inside);
    std::free(info.level_start);
  }
};

template <class Panel>
void build_problem(const btk_forest_desc& D, int b, const double* x, const double* y, const double* z,
                   ProblemTree<Panel>& P) {
  const int off = D.point_offset[b], n = D.point_offset[b + 1] - off;
  btk_run_config& c = P.cfg;
  c.dim = D.dim;
  c.interp_degree = D.degree;
  c.interp_point_count = D.dim == 3 ? (D.degree + 1) * (D.degree + 1) * (D.degree + 1) : (D.degree + 1) * (D.degree + 1);
  c.fmm_theta = D.theta;
  c.fmm_cluster_thresh = D.cluster_size[b];
  c.ker_eps = D.eps;
  c.mpi_p = 1;
  c.mpi_id = 0;
  P.leaf_of.assign(std::max(n, 1), 0);
  btk_status s;
  if (D.dim == 3)
    s = btk_tree_construction_3d(&c, &P.info, x + off, y + off, z + off, n, reinterpret_cast<btk_panel_3d**>(&P.panels),
                                 P.leaf_of.data(), &P.inside);
  else
    s = btk_tree_construction_2d(&c, &P.info, x + off, y + off, n, reinterpret_cast<btk_panel_2d**>(&P.panels),
                                 P.leaf_of.data(), &P.inside);
  btk_interact_pair* all = nullptr;
  if (s == BTK_OK)
    s = D.dim == 3 ? btk_dual_tree_traversal_3d(&c, reinterpret_cast<btk_panel_3d*>(P.panels),
                                                reinterpret_cast<btk_panel_3d*>(P.panels), &all)
                   : btk_dual_tree_traversal_2d(&c, reinterpret_cast<btk_panel_2d*>(P.panels),
                                                reinterpret_cast<btk_panel_2d*>(P.panels), &all);
  if (s == BTK_OK) {
    P.lists[0].resize(c.fmm_pp_count);
    P.lists[1].resize(c.fmm_pc_count);
    P.lists[2].resize(c.fmm_cp_count);
    P.lists[3].resize(c.fmm_cc_count);
    s = btk_split_interactions(all, c.fmm_interaction_count, P.lists[0].data(), P.lists[1].data(), P.lists[2].data(),
                               P.lists[3].data());
  }
  std::free(all);
  std::free(P.inside);  // the forest orders leaves from point_leaf_panel
  P.inside = nullptr;
  if (s != BTK_OK) {
    P.status = s;
    P.error = "problem " + std::to_string(b) + ": " + btk_last_error();
  }
}

template <class Panel>
btk_status forest_build(const btk_forest_desc& D, const double* x, const double* y, const double* z, btk_forest& F) {
  const int B = D.n_problems;
  std::vector<ProblemTree<Panel>> probs(B);
  {
    std::atomic<int> next{0};
    const int nthreads = std::max(1, std::min<int>(B, (int)std::thread::hardware_concurrency()));
    auto work = [&] {
      for (int b = next++; b < B; b = next++) build_problem(D, b, x, y, z, probs[b]);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; ++t) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
  }
  for (int b = 0; b < B; ++b)
    if (probs[b].status != BTK_OK) return set_error(probs[b].status, probs[b].error);

  // Level-major renumbering.
  int levels = 0;
  int64_t total_panels = 0;
  for (auto& p : probs) {
    levels = std::max(levels, p.info.levels);
    total_panels += p.info.panel_count;
  }
  BTK_CHECK(total_panels < (1ll << 31), BTK_ERR_UNSUPPORTED, "forest: too many panels");
  const int np = (int)total_panels;
  std::vector<std::vector<int>> new_of(B);
  for (int b = 0; b < B; ++b) new_of[b].assign(probs[b].info.panel_count, -1);
  std::vector<int> level_start{0}, panel_problem(np), panel_local(np);
  int idx = 0;
  for (int l = 0; l < levels; ++l) {
    for (int b = 0; b < B; ++b) {
      const ProblemTree<Panel>& p = probs[b];
      if (l >= p.info.levels) continue;
      for (int i = p.info.level_start[l]; i < p.info.level_start[l + 1]; ++i) {
        panel_problem[idx] = b;
        panel_local[idx] = i;
        new_of[b][i] = idx++;
      }
    }
    level_start.push_back(idx);
  }
  BTK_CHECK(idx == np, BTK_ERR_INTERNAL, "forest: level ranges do not cover every panel");

  const int nc = D.dim == 3 ? 8 : 4;
  const int64_t n_points = D.point_offset[B];
  Panel* panels = static_cast<Panel*>(std::malloc(sizeof(Panel) * std::max(np, 1)));
  int* ls = static_cast<int*>(std::malloc(sizeof(int) * level_start.size()));
  int* leaf_of = static_cast<int*>(std::malloc(sizeof(int) * std::max<int64_t>(n_points, 1)));
  int* pprob = static_cast<int*>(std::malloc(sizeof(int) * std::max(np, 1)));
  int* ploc = static_cast<int*>(std::malloc(sizeof(int) * std::max(np, 1)));
  int counts[4] = {0, 0, 0, 0};
  for (auto& p : probs)
    for (int t = 0; t < 4; ++t) counts[t] += (int)p.lists[t].size();
  btk_interact_pair* lists[4];
  for (int t = 0; t < 4; ++t) lists[t] = static_cast<btk_interact_pair*>(std::malloc(sizeof(btk_interact_pair) * std::max(counts[t], 1)));
  if (!panels || !ls || !leaf_of || !pprob || !ploc || !lists[0] || !lists[1] || !lists[2] || !lists[3]) {
    std::free(panels);
    std::free(ls);
    std::free(leaf_of);
    std::free(pprob);
    std::free(ploc);
    for (auto* l : lists) std::free(l);
    return set_error(BTK_ERR_OUT_OF_MEMORY, "forest: host allocation failed");
  }
  std::copy(level_start.begin(), level_start.end(), ls);
  std::copy(panel_problem.begin(), panel_problem.end(), pprob);
  std::copy(panel_local.begin(), panel_local.end(), ploc);
  int thresh = 1;
  int cur[4] = {0, 0, 0, 0};
  for (int b = 0; b < B; ++b) {
    const ProblemTree<Panel>& p = probs[b];
    const std::vector<int>& m = new_of[b];
    thresh = std::max(thresh, D.cluster_size[b]);
    for (int i = 0; i < p.info.panel_count; ++i) {
      Panel q = p.panels[i];
      q.id = m[i];
      q.parent_id = q.parent_id >= 0 ? m[q.parent_id] : -1;
      for (int c = 0; c < nc; ++c) {
        int& ch = child_ref(q, c);
        if (ch >= 0) ch = m[ch];
      }
      panels[m[i]] = q;
    }
    const int off = D.point_offset[b], n = D.point_offset[b + 1] - off;
    for (int k = 0; k < n; ++k) leaf_of[off + k] = m[p.leaf_of[k]];
    for (int t = 0; t < 4; ++t)
      for (const btk_interact_pair& pr : p.lists[t])
        lists[t][cur[t]++] = btk_interact_pair{m[pr.target_panel], m[pr.source_panel], pr.interact_type};
  }
  std::memset(&F, 0, sizeof(F));
  btk_run_config& c = F.cfg;
  c.dim = D.dim;
  c.interp_degree = D.degree;
  c.interp_point_count = D.dim == 3 ? (D.degree + 1) * (D.degree + 1) * (D.degree + 1) : (D.degree + 1) * (D.degree + 1);
  c.fmm_theta = D.theta;
  c.fmm_cluster_thresh = thresh;
  c.ker_eps = D.eps;
  c.mpi_p = 1;
  c.fmm_pp_count = counts[0];
  c.fmm_pc_count = counts[1];
  c.fmm_cp_count = counts[2];
  c.fmm_cc_count = counts[3];
  c.fmm_interaction_count = counts[0] + counts[1] + counts[2] + counts[3];
  F.info.panel_count = np;
  F.info.levels = levels;
  F.info.level_start = ls;
  F.panels = panels;
  F.point_leaf_panel = leaf_of;
  F.panel_problem = pprob;
  F.panel_local = ploc;
  F.pp_list = lists[0];
  F.pc_list = lists[1];
  F.cp_list = lists[2];
  F.cc_list = lists[3];
  return BTK_OK;
}

btk_status check_forest_desc(const btk_forest_desc* D) {
  BTK_CHECK(D, BTK_ERR_INVALID_ARGUMENT, "forest: null descriptor");
  BTK_CHECK(D->dim == 2 || D->dim == 3, BTK_ERR_INVALID_ARGUMENT, "forest: dim must be 2 or 3");
  BTK_CHECK(D->degree >= 1 && D->degree <= kMaxDegree, BTK_ERR_UNSUPPORTED, "forest: degree outside 1..12");
  BTK_CHECK(D->n_problems >= 1 && D->point_offset && D->cluster_size, BTK_ERR_INVALID_ARGUMENT,
            "forest: need at least one problem, point offsets and leaf sizes");
  BTK_CHECK(D->point_offset[0] == 0, BTK_ERR_INVALID_ARGUMENT, "forest: point_offset[0] must be 0");
  for (int b = 0; b < D->n_problems; ++b) {
    BTK_CHECK(D->point_offset[b + 1] >= D->point_offset[b], BTK_ERR_INVALID_ARGUMENT,
              "forest: point offsets must not decrease");
    BTK_CHECK(D->cluster_size[b] > 0, BTK_ERR_INVALID_ARGUMENT, "forest: leaf sizes must be positive");
  }
  return BTK_OK;
}

}  // namespace
}  // namespace btk

using namespace btk;

struct btk_batch {
  int dim = 3, ncomp = 1, n_problems = 0;
  int64_t n_points = 0;
  btk_forest forest{};
  btk_plan* plan = nullptr;
  double *d_xyz = nullptr, *d_q = nullptr, *d_out = nullptr;
  cudaStream_t cap = nullptr;  // capture stream
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  int graph_kernels = 0, graph_nodes = 0;
  bool timed = false;
};

extern "C" {

btk_status btk_forest_build(const btk_forest_desc* desc, const double* x, const double* y, const double* z,
                            btk_forest* forest) {
  BTK_TRY(check_forest_desc(desc));
  BTK_CHECK(forest && x && y && (desc->dim == 2 || z), BTK_ERR_INVALID_ARGUMENT, "forest: null argument");
  if (desc->dim == 3) return forest_build<btk_panel_3d>(*desc, x, y, z, *forest);
  return forest_build<btk_panel_2d>(*desc, x, y, nullptr, *forest);
}

void btk_forest_free(btk_forest* f) {
  if (!f) return;
  std::free(f->panels);
  std::free(f->info.level_start);
  std::free(f->point_leaf_panel);
  std::free(f->panel_problem);
  std::free(f->panel_local);
  std::free(f->pp_list);
  std::free(f->pc_list);
  std::free(f->cp_list);
  std::free(f->cc_list);
  std::memset(f, 0, sizeof(*f));
}

btk_status btk_batch_destroy(btk_batch* b) {
  if (!b) return BTK_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->cap) cudaStreamDestroy(b->cap);
  if (b->plan) btk_plan_destroy(b->plan);
  cudaFree(b->d_xyz);
  cudaFree(b->d_q);
  cudaFree(b->d_out);
  btk_forest_free(&b->forest);
  delete b;
  return BTK_OK;
}

btk_status btk_batch_create(btk_batch** out, const btk_batch_desc* desc, const double* x, const double* y,
                            const double* z, btk_stream_t stream) {
  BTK_CHECK(out && desc, BTK_ERR_INVALID_ARGUMENT, "btk_batch_create: null argument");
  *out = nullptr;
  const btk_forest_desc& F = desc->forest;
  BTK_CHECK(desc->kind >= 0 && desc->kind <= 2 && !(desc->kind == BTK_KIND_VEL && F.dim != 3),
            BTK_ERR_INVALID_ARGUMENT, "btk_batch_create: bad kind");
  btk_batch* b = new btk_batch();
  auto fail = [&](btk_status s) {
    std::string msg = btk_last_error();
    btk_batch_destroy(b);
    return set_error(s, msg);
  };
  btk_status s = btk_forest_build(&F, x, y, z, &b->forest);
  if (s != BTK_OK) return fail(s);
  b->dim = F.dim;
  b->n_problems = F.n_problems;
  b->ncomp = F.dim == 2 ? (desc->kind == BTK_KIND_FIELD ? 3 : 1)
                        : (desc->kind == BTK_KIND_POT ? 1 : (desc->kind == BTK_KIND_VEL ? 3 : 4));
  b->n_points = F.point_offset[F.n_problems];
  if (b->n_points >= (1ll << 31)) return fail(set_error(BTK_ERR_UNSUPPORTED, "batch: more than 2^31 points"));
  btk_plan_desc pd;
  std::memset(&pd, 0, sizeof(pd));
  pd.cfg = b->forest.cfg;
  pd.point_count_target = pd.point_count_source = (int)b->n_points;
  pd.tree_target = &b->forest.info;
  pd.panels_target = b->forest.panels;
  pd.panel_points_inside_target = nullptr;
  pd.point_leaf_panel_source = b->forest.point_leaf_panel;
  pd.pp_list = b->forest.pp_list;
  pd.pc_list = b->forest.pc_list;
  pd.cp_list = b->forest.cp_list;
  pd.cc_list = b->forest.cc_list;
  pd.kind = desc->kind;
  pd.precision = desc->precision;
  pd.degree_mode = BTK_DEGREE_FIXED;
  pd.work_split = desc->work_split;
  pd.tile_targets = desc->tile_targets;
  s = btk_plan_create(&b->plan, &pd, stream);
  if (s != BTK_OK) return fail(s);
  const size_t n = (size_t)std::max<int64_t>(b->n_points, 1);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMalloc(&b->d_xyz, sizeof(double) * n * F.dim);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_q, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_out, sizeof(double) * n * b->ncomp);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_q, 0, sizeof(double) * n, st);
  const double* src[3] = {x, y, z};
  for (int d = 0; d < F.dim && e == cudaSuccess; ++d)
    e = cudaMemcpyAsync(b->d_xyz + (size_t)d * n, src[d], sizeof(double) * b->n_points, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
  for (auto& ev : b->ev)
    if (e == cudaSuccess) e = cudaEventCreate(&ev);
  if (e != cudaSuccess) return fail(cuda_error(e, "btk_batch_create"));
  *out = b;
  return BTK_OK;
}

btk_status btk_batch_execute(btk_batch* b, const double* charges, double* out, btk_stream_t stream) {
  BTK_CHECK(b && charges && out, BTK_ERR_INVALID_ARGUMENT, "btk_batch_execute: null argument");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)std::max<int64_t>(b->n_points, 1);
  const double* X = b->d_xyz;
  const double* Y = b->d_xyz + n;
  const double* Z = b->dim == 3 ? b->d_xyz + 2 * n : nullptr;
  if (!b->exec) {
    // One eager solve first (loads every kernel's module), then the capture.
    BTK_TRY(btk_plan_execute(b->plan, X, Y, Z, X, Y, Z, b->d_q, b->d_out, (btk_stream_t)b->cap));
    BTK_CUDA(cudaStreamSynchronize(b->cap));
    BTK_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    btk_status s = btk_plan_execute(b->plan, X, Y, Z, X, Y, Z, b->d_q, b->d_out, (btk_stream_t)b->cap);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->cap, &g);
    if (s != BTK_OK) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    BTK_CUDA(e);
    b->graph = g;
    BTK_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    size_t nn = 0;
    BTK_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    BTK_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
    int kernels = 0;
    for (auto& nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
    }
    b->graph_nodes = (int)nn;
    b->graph_kernels = kernels;
  }
  if (charges != b->d_q)
    BTK_CUDA(cudaMemcpyAsync(b->d_q, charges, sizeof(double) * b->n_points, cudaMemcpyDefault, st));
  BTK_CUDA(cudaEventRecord(b->ev[0], st));
  BTK_CUDA(cudaGraphLaunch(b->exec, st));
  count_launch(b->graph_kernels);
  BTK_CUDA(cudaEventRecord(b->ev[1], st));
  if (out != b->d_out)
    BTK_CUDA(cudaMemcpyAsync(out, b->d_out, sizeof(double) * b->n_points * b->ncomp, cudaMemcpyDefault, st));
  b->timed = true;
  return BTK_OK;
}

btk_status btk_batch_stats_get(btk_batch* b, btk_batch_stats* s) {
  BTK_CHECK(b && s, BTK_ERR_INVALID_ARGUMENT, "btk_batch_stats_get: null argument");
  std::memset(s, 0, sizeof(*s));
  btk_plan_stats ps;
  BTK_TRY(btk_plan_stats_get(b->plan, &ps));
  s->n_problems = b->n_problems;
  s->total_points = b->n_points;
  s->panel_count = b->forest.info.panel_count;
  s->levels = b->forest.info.levels;
  s->evals_pp = ps.evals_pp;
  s->evals_pc = ps.evals_pc;
  s->evals_cp = ps.evals_cp;
  s->evals_cc = ps.evals_cc;
  s->work_items = ps.work_items;
  s->graph_kernel_nodes = b->graph_kernels;
  s->graph_nodes = b->graph_nodes;
  if (b->timed) {
    BTK_CUDA(cudaEventSynchronize(b->ev[1]));
    BTK_CUDA(cudaEventElapsedTime(&s->last_ms, b->ev[0], b->ev[1]));
  }
  return BTK_OK;
}

}  // extern "C"
