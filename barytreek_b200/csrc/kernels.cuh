// Kernel declarations and the device-side data layout shared by the
// translation units.
//
// Device layout of one tree side (targets or sources):
//   sorted points      : double4 {x, y, z, w}, leaves contiguous in panel order,
//                        points of a leaf in ascending original index
//                        (the order of panel_points_inside rows);
//   perm[k]            : original index of sorted point k;
//   leaf_begin[panel]  : first sorted point of a leaf (-1 for non-leaves);
//   nodes_shift        : [panel][3][kMaxNodes] Chebyshev points
//                        cos(pi/n*i)*r + c (src/bli_impl.hpp:66-77) — proxy
//                        point coordinates;
//   nodes_interp       : [panel][3][kMaxNodes] cos(pi*i/n)*r + c — the node set
//                        interp_vals_bli evaluates with (src/bli_impl.hpp:25);
//   xfer               : [panel][3][kMaxNodes][kMaxNodes]
//                        xfer[c][d][i][a] = L^{parent(c)}_a(node_shift^c_{d,i}),
//                        the 1-D factors of child->parent anterpolation and
//                        parent->child interpolation.
// Proxy weights: [panel][ipc] row-major, proxy index ((a*m)+b)*m+c with x
// slowest (src/upward_pass_impl.hpp:161-168).
#pragma once

#include "btk_internal.h"

namespace btk {

constexpr int kNodeStride = kMaxNodes;                     // per-axis stride
constexpr int kPanelNodes = 3 * kNodeStride;               // doubles per panel
constexpr int kPanelXfer = 3 * kMaxNodes * kMaxNodes;      // doubles per panel

struct DevPanel {  // compact device copy of what kernels need per panel
  double lo[3], hi[3];
  int parent, is_leaf, point_count, level;
};

// ---- interaction work lists -----------------------------------------------
struct WorkItem {
  int t_begin;         // first target in the T4 array
  int t_count;         // targets in this tile
  int e_begin, e_end;  // entry range
  int s_total;         // sources over the entries
  int flags;           // kItemProxyTargets | kItemAtomic | kItemAudit
  int near_total;      // the first near_total sources are PP (near-field) points
  float hx;            // half widths of the target box (mixed: a near source farther than
  double cx, cy, cz;   //   max(hx, hy, hz) from the box takes the FP32 path); FP64 centre of
  float hy, hz;        //   the target panel (mixed precision origin)
};
static_assert(sizeof(WorkItem) == 64, "WorkItem is one 64-byte record");
constexpr int kItemProxyTargets = 1;  // outputs go to proxy target weights
constexpr int kItemAtomic = 2;        // another item shares these targets
constexpr int kItemAudit = 4;         // FP64 direct-sum audit: targets T4a[t_begin + i], outputs aout[c][t_begin + i]

struct Entry {
  int s_begin;  // first source in the S4 array
  int s_count;
};

struct Ptr4 {
  double* p[4];
};

struct InteractParams {
  const WorkItem* items;
  int n_items;
  const Entry* entries;
  const double4* S4;
  const double4* T4;
  const int* T_out;
  double* out[4];  // point-target outputs, one per component
  double* ptw[4];  // proxy-target outputs, one per component
  const double4* T4a;  // audit targets (kItemAudit items)
  double* aout[4];     // audit outputs, one per component
  double eps2;
  double scale[4];
  int* ticket;
  int* status;
  // Polls of a chunk's mbarrier before the block gives up (sets *status to
  // BTK_ERR_DEVICE_TIMEOUT and leaves); 0 gives up at the first wait (tests
  // of the error path). In-flight copies are always drained with kDrainLimit.
  uint32_t wait_limit;
  // FP64 audit items (kItemAudit) items[n_items, n_items + n_audit_items),
  // handed out by their own counter *audit_ticket. Blocks [0, audit_blocks)
  // start on the audit items and the others on the rest; a block whose queue
  // runs dry moves to the other one, so the audit shares the SMs with the
  // solve from the start (its FP64 work runs beside FP32 work) and neither
  // queue leaves SMs idle at its end.
  int n_audit_items;
  int audit_blocks;
  int* audit_ticket;
};
constexpr uint32_t kWaitLimitDefault = 1u << 22;
constexpr uint32_t kDrainLimit = 1u << 22;

// Work items hold at most kTile targets; a plan's items are tiles of `tile`
// targets (256 or 128), run by interaction blocks of tile / 2 threads (two
// targets per thread, 64 per warp).
constexpr int kTargetsPerThread = 2;
constexpr int kTile = 256;

// ---- launchers (return cudaGetLastError of the launch) -----------------------
cudaError_t launch_panel_geometry(int dim, int degree, int P, const DevPanel* panels, const double* ucos_shift,
                                  const double* ucos_interp, double* nodes_shift, double* nodes_interp, double* xfer,
                                  cudaStream_t s);
cudaError_t launch_perm_from_inside(int n_leaves, const int* leaves, const int* leaf_begin, const int* point_count,
                                    const int* inside, int thresh, int* perm, cudaStream_t s);
cudaError_t launch_gather(int n, const int* perm, const double* x, const double* y, const double* z,
                          const double* w, double4* out, cudaStream_t s);
cudaError_t launch_leaf_moments(int dim, int degree, int n_leaves, const int* leaves, const int* leaf_begin,
                                const int* point_count, const double4* pts, const double* nodes_interp, double* psw,
                                cudaStream_t s);
cudaError_t launch_c2p(int dim, int degree, int n_parents, const int* parents, const int* child,
                       const double* xfer, double* psw, cudaStream_t s);
cudaError_t launch_src_proxies(int dim, int degree, int n_clusters, const int* cluster_panels,
                               const double* nodes_shift, const double* psw, double4* out, cudaStream_t s);
cudaError_t launch_tgt_proxies(int dim, int degree, int n_clusters, const int* cluster_panels,
                               const double* nodes_shift, double4* out, int* out_index, cudaStream_t s);
cudaError_t launch_p2c(int dim, int degree, int ncomp, int n_children, const int* children, const int* parent_of,
                       const double* xfer, Ptr4 ptw, int ptw_stride, cudaStream_t s);
cudaError_t launch_l2p(int dim, int degree, int ncomp, int n_leaves, const int* leaves, const int* leaf_begin,
                       const int* point_count, const double4* pts, const int* perm, const double* nodes_interp,
                       Ptr4 ptw, Ptr4 out, cudaStream_t s);
cudaError_t launch_interact(int dim, int kind, int precision, bool guard, const InteractParams& p, int grid,
                            cudaStream_t s, int tile);
int interact_blocks_per_sm(int dim, int kind, int precision, bool guard, int tile);
cudaError_t launch_direct(int dim, int kind, double eps, int nt, const double* xt, const double* yt,
                          const double* zt, int ns, const double4* src, double* out, cudaStream_t s);

// ---- CC pairs as shared kernel matrices (cc_operators.cu) ---------------------
struct CcTask {
  int tp, sp;            // the group's first pair: its panels give G's geometry
  int p_begin, p_count;  // pairs [p_begin, p_begin + p_count) of the pair array
};
struct CcPair {
  int t_row, s_row;  // target panel (row of the proxy target weights), source panel (row of psw)
};
struct CcParams {
  const CcTask* tasks;
  const CcPair* pairs;
  const double* nodes_t;  // target side nodes_shift
  const double* nodes_s;  // source side nodes_shift
  const double* psw;      // [source panels][ipc]
  Ptr4 ptw;               // per component [target panels][ipc]
  double eps2;
  double scale[4];
  int m, ipc;
};
int cc_pairs_per_task(int dim, int kind);
// f32: G and the products in FP32 (partial sums per source slab folded into
// FP64), for mixed-precision plans; otherwise FP64 throughout.
cudaError_t launch_cc_groups(int dim, int kind, bool guard, bool f32, const CcParams& p, const int* bucket_end,
                             cudaStream_t s);
bool cc_group_pairs(const HostTree& T, const HostTree& S, const btk_interact_pair* cc, int n_cc,
                    std::vector<int>& group_of, int& n_groups);
void cc_build_tasks(const btk_interact_pair* cc, int n_cc, const std::vector<int>& group_of, int n_groups, int pt,
                    std::vector<CcTask>& tasks, std::vector<CcPair>& pairs, int bucket_end[3]);

// ---- learned selector (selector.cu) -------------------------------------------
// Inputs of the training-sample generator (see btk_plan_error_samples).
struct SampleArgs {
  int dim, kind, ncomp, K, n_deg, deg_lo, n;
  double eps2;
  const int* pair_index;  // [n] into the plan's pair list
  const int* ptype;       // per pair: 1 PC, 2 CP, 3 CC
  const int* ptgt;        // per pair target panel
  const int* psrc;        // per pair source panel
  const double* xt;
  const double* yt;
  const double* zt;
  const int* tgt_orig;  // [n][K] original target indices
  const int* src_leaf_csr;
  const int* src_leaves;  // leaf panels under each sample's source
  const int* leaf_begin_s;
  const int* count_s;
  const double4* S4;       // sorted source points then source slots
  const long long* s_slot_off;
  const int* s_slot_begin;  // per source cluster slot index
  const int* cluster_slot_s;
  const double4* T4;  // target slots after the points
  const long long* t_slot_off;
  const int* t_slot_begin;
  const int* cluster_slot_t;
  long long ns, nt;
  const DevPanel* pt;
  int slot_d_lo;
  double* exact;   // [n][K][ncomp]
  double* approx;  // [n][n_deg][K][ncomp]
  const double* ref;  // optional [ncomp][nt] total solution: errors relative to it
};
cudaError_t launch_error_samples(const SampleArgs& a, float* log10_err, cudaStream_t s);
int selector_param_count();
cudaError_t launch_panel_desc(int dim, int n, int P, const double* psw, float* desc, cudaStream_t s);
cudaError_t launch_pair_features(int n_pairs, const int* ptype, const int* ptgt, const int* psrc, const DevPanel* pt,
                                 const DevPanel* ps, double root_radius, double eps, const float* desc_s,
                                 int n_points, const double4* pts, double* gsum, float* feat, cudaStream_t s);
cudaError_t launch_mlp_infer(int n, const void* w_bf16, const float* norm, const float* feat, float* out,
                             int* status, cudaStream_t s);  // status: optional device word, set on a timeout
// Pairs [conv0, n_pc) of the PC block are leaf pairs that may stay direct
// (degree 0); pc_direct[2 i], [2 i + 1]: their source leaf's first point and
// point count.
cudaError_t launch_choose_degrees_cost(int n, int dim, int n_pc, int n_cp, int conv0, const float* pred,
                                       float log10_target, int lo, int hi, const int* pc_tcount, const int* cp_scount,
                                       const int* pc_direct, const int* weight, float inv_cbar, float inv_wbar,
                                       int* deg, cudaStream_t s);
cudaError_t launch_choose_degrees(int n, const float* pred, float log10_target, int lo, int hi, int dim, int conv0,
                                  int n_pc, const int* pc_direct, int* deg, cudaStream_t s);
// The form of each leaf pair k < n (direct, PC entry pc0 + k, or for k < n_cc
// CC entry cc0 + k) and its degree; cost_rule as BTK_DEGREE_RULE_COST.
cudaError_t launch_choose_leaf_pairs(int n, int n_cc, int dim, int pc0, int cc0, const float* pred, float log10_target,
                                     int lo, int hi, int cost_rule, const int* pc_tcount, const int* pc_direct,
                                     const int* weight, float inv_cbar, float inv_wbar, int* deg, cudaStream_t s);
// PC pairs with a large target leaf or CP pairs with a large source leaf,
// k < n: their own form (entry idx[k], cost coef[k] (d+1)^dim, degree
// off_first when not taken) or the CC form (entry cc0 + k) and its degree.
cudaError_t launch_choose_two_forms(int n, int dim, const int* idx, const int* coef, int off_first, int cc0,
                                   const float* pred, float log10_target, int lo, int hi, int cost_rule,
                                   const int* weight, float inv_cbar, float inv_wbar, int* deg, cudaStream_t s);
// Far-field evaluations at the chosen degrees (summed into evals[0]), direct
// evaluations of the leaf pairs kept direct (evals[1]) and the histogram of
// the degrees (hist[0..12], added to; bin 0: leaf pairs kept direct). Leaf
// pairs: PC entries [conv0, conv0 + n_conv), the first n_conv_cc with CC
// entries, the last n_conv_cc of the CC block.
cudaError_t launch_far_evals(int dim, int n_pc, int n_cp, int n_cc, int conv0, int n_conv, int n_conv_cc,
                             const int* deg, const int* pc_tcount, const int* cp_scount, const int* pc_direct,
                             unsigned long long* evals, int* hist, cudaStream_t s);
cudaError_t launch_audit_compare(int n, int ncomp, int nt, const int* audit_sorted, const int* perm,
                                 const double* out, const double* audit_out, double* sums, cudaStream_t s);
cudaError_t launch_fill_int(int n, int value, int* dst, cudaStream_t s);

// ---- per-pair degrees (kernels_degree.cu) -------------------------------------
cudaError_t launch_src_slots(int dim, int n, int n_slots, const int* slot_cluster_panel, const int* slot_degree,
                             const long long* slot_offset, const DevPanel* panels, const double* psw,
                             const double* amat, const int* amat_off, const double* ucos_all, const int* ucos_off,
                             const int* used, double4* S4, cudaStream_t s);  // used: per slot, 0 = skip (NULL: all)
cudaError_t launch_tgt_slots(int dim, int n_slots, const int* slot_cluster_panel, const int* slot_degree,
                             const long long* slot_offset, const DevPanel* panels, const double* ucos_all,
                             const int* ucos_off, double4* T4, int* T_out, long long t4_base, cudaStream_t s);
cudaError_t launch_promote(int dim, int n, int ncomp, int n_clusters, const int* cluster_panel,
                           const int* cluster_slot_begin, const int* slot_degree, const long long* slot_offset,
                           const double* amat, const int* amat_off, Ptr4 ptwm, Ptr4 ptw, cudaStream_t s);
cudaError_t launch_resolve(int dim, int n_pc, const int* pc_entry, const int* pc_src_cluster, const int* deg_pc,
                           const int* pc_direct, int n_far, int tiles_max, const int* far_type, const int* far_tgt_cluster,
                           const int* far_src, const int* deg_far, const long long* src_slot_offset,
                           const int* cluster_slot_begin_s, const long long* tgt_slot_offset,
                           const int* cluster_slot_begin_t, int slot_d_lo, long long t4_base, long long s4_base,
                           const double* tgt_centre, int n_point_items, WorkItem* items, Entry* entries,
                           int far_item0, int far_entry0, int* slot_used, int tile,
                           cudaStream_t s);  // marks the source slots read

}  // namespace btk
