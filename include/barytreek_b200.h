/*
 * barytreek_b200 — B200-native evaluation path of BarytreeK's barycentric
 * Lagrange dual-tree treecode, exposed as a plain C ABI.
 *
 * Three layers, all extern "C", no torch or Kokkos types:
 *
 *  1. Host tree functions, bit-identical to the reference's host C++
 *     (read_run_config, blfmm_tree_construction_2d/3d, dual_tree_traversal_2d/3d,
 *     split_interactions). Outputs the reference's struct layouts.
 *  2. Drop-in device entry points with the reference's names and argument
 *     order (upward_pass_*, poisson_fmm_interactions_*,
 *     poisson_vel_fmm_interactions_3d, downward_pass_*). Every array argument is
 *     a DEVICE pointer laid out like the corresponding Kokkos::View
 *     (LayoutRight, row = panel); extents a View would carry are appended
 *     before the stream. Results accumulate (+=) like the reference's
 *     atomic_add; proxy arrays must be zeroed by the caller as the reference's
 *     drivers do (examples/example_poisson_3d.cpp:133-135).
 *  3. A plan API (btk_plan_*) that keeps the tree, the target-grouped work
 *     lists and all derived device data resident across solves, adds the
 *     extensions (field/gradient outputs, mixed precision) and a one-call
 *     host-buffer solve (btk_solve_host).
 *
 * Every function returns btk_status (0 = success); btk_last_error() gives a
 * thread-local message for the last failure on the calling thread. Launches are
 * asynchronous on the given stream unless stated otherwise.
 */
#ifndef BARYTREEK_B200_H
#define BARYTREEK_B200_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Same handle type as cudaStream_t (a CUstream); NULL = legacy default stream. */
typedef struct CUstream_st* btk_stream_t;

typedef enum {
  BTK_OK = 0,
  BTK_ERR_INVALID_ARGUMENT = 1,
  BTK_ERR_CUDA = 2,
  BTK_ERR_UNSUPPORTED = 3,
  BTK_ERR_OUT_OF_MEMORY = 4,
  BTK_ERR_DEVICE_TIMEOUT = 5, /* a bounded device-side wait gave up */
  BTK_ERR_IO = 6,
  BTK_ERR_INTERNAL = 7
} btk_status;

/* ---- Reference layouts (src/structs.hpp:6-75), byte-for-byte ---------- */

/* RunConfig, src/structs.hpp:6-22 (64 bytes). */
typedef struct {
  int dim;
  int interp_degree;
  int interp_point_count;
  double fmm_theta;
  int fmm_cluster_thresh;
  int fmm_interaction_count;
  int fmm_pp_count;
  int fmm_pc_count;
  int fmm_cp_count;
  int fmm_cc_count;
  double ker_eps;
  int mpi_p;
  int mpi_id;
} btk_run_config;

/* TreeInfo, src/structs.hpp:24-28 (16 bytes). level_start has levels+1
 * entries and lives in HOST memory (the reference's upward/downward loops read
 * it on the host: src/upward_pass.cpp:12-16). */
typedef struct {
  int panel_count;
  int levels;
  int* level_start;
} btk_tree_info;

/* TreePanel_2d, src/structs.hpp:30-45 (80 bytes). */
typedef struct {
  int id, level, parent_id;
  int child1, child2, child3, child4;
  bool is_leaf;
  double max_x, min_x, max_y, min_y;
  double radius;
  int point_count;
} btk_panel_2d;

/* TreePanel_3d, src/structs.hpp:47-66 (112 bytes; min_z precedes max_z). */
typedef struct {
  int id, level, parent_id;
  int child1, child2, child3, child4, child5, child6, child7, child8;
  bool is_leaf;
  double max_x, min_x, max_y, min_y, min_z, max_z;
  double radius;
  int point_count;
} btk_panel_3d;

/* interact_pair, src/structs.hpp:71-75 (12 bytes). type 0 pp, 1 pc, 2 cp, 3 cc. */
typedef struct {
  int target_panel;
  int source_panel;
  int interact_type;
} btk_interact_pair;

/* ---- Library ---------------------------------------------------------- */

const char* btk_last_error(void);
const char* btk_version(void);
/* Number of CUDA kernels this library has launched in this process. */
uint64_t btk_launch_count(void);
/* Highest polynomial degree the device kernels accept. */
int btk_max_degree(void);
void btk_free(void* p); /* frees arrays the host tree functions allocate */

/* ---- 1. Host tree functions (bit-identical to the reference) ----------- */

/* src/read_namelist.cpp:10-43. cfg->dim must be set first, as the reference's
 * drivers do. Parsing stops at the first unknown key. BTK_ERR_IO when the file
 * cannot be opened (the reference throws "namelist not found"). The degree is
 * clamped to 10, the reference's max_degree (barytreek-config.h.in:20). */
btk_status btk_read_run_config(const char* file_name, btk_run_config* cfg);

/* src/tree_construction.cpp:5-129 / :131-306. Inputs are host arrays of
 * point_count coordinates. Outputs, allocated by the library (btk_free):
 * *panels (info->panel_count records), info->level_start (levels+1 ints),
 * *panel_points_inside (panel_count x cfg->fmm_cluster_thresh ints, row-major;
 * rows of non-leaf panels are zero). point_leaf_panel[point_count] is caller
 * storage. */
btk_status btk_tree_construction_2d(const btk_run_config* cfg, btk_tree_info* info, const double* xcos,
                                    const double* ycos, int point_count, btk_panel_2d** panels,
                                    int* point_leaf_panel, int** panel_points_inside);
btk_status btk_tree_construction_3d(const btk_run_config* cfg, btk_tree_info* info, const double* xcos,
                                    const double* ycos, const double* zcos, int point_count, btk_panel_3d** panels,
                                    int* point_leaf_panel, int** panel_points_inside);

/* The same trees as btk_tree_construction_2d/3d (every panel field, the level
 * starts and point_leaf_panel bit-identical), built from DEVICE coordinates:
 * the point work (root box reduction, the stable per-level partition of the
 * points into children) runs on the GPU, the per-panel bookkeeping on the
 * host. Outputs: *panels and info->level_start host arrays allocated by the
 * library (btk_free); point_leaf_panel[point_count] DEVICE; leaf_order
 * (DEVICE, point_count ints, may be NULL): the point indices leaf by leaf in
 * panel order, each leaf ascending -- the rows of panel_points_inside
 * concatenated without the padding. Synchronises the stream once per tree
 * level. No counterpart in the reference (whose construction is host code). */
btk_status btk_tree_construction_2d_device(const btk_run_config* cfg, btk_tree_info* info, const double* xcos,
                                           const double* ycos, int point_count, btk_panel_2d** panels,
                                           int* point_leaf_panel, int* leaf_order, btk_stream_t stream);
btk_status btk_tree_construction_3d_device(const btk_run_config* cfg, btk_tree_info* info, const double* xcos,
                                           const double* ycos, const double* zcos, int point_count,
                                           btk_panel_3d** panels, int* point_leaf_panel, int* leaf_order,
                                           btk_stream_t stream);

/* src/interaction_list.cpp:5-117 / :119-250. Updates cfg's interaction
 * counts; *interaction_list (cfg->fmm_interaction_count pairs) is allocated
 * by the library (btk_free). */
btk_status btk_dual_tree_traversal_2d(btk_run_config* cfg, const btk_panel_2d* panels_target,
                                      const btk_panel_2d* panels_source, btk_interact_pair** interaction_list);
btk_status btk_dual_tree_traversal_3d(btk_run_config* cfg, const btk_panel_3d* panels_target,
                                      const btk_panel_3d* panels_source, btk_interact_pair** interaction_list);

/* The same interaction lists as btk_dual_tree_traversal_2d/3d (same pairs,
 * same order, same counts in cfg), computed on the GPU one breadth-first
 * generation of (target, source) pairs at a time. Panels are HOST arrays of
 * the given counts (targets = sources when both pointers and counts agree);
 * *interaction_list is a host array allocated by the library (btk_free).
 * Synchronises the stream once per generation. No counterpart in the
 * reference (whose traversal is host code). */
btk_status btk_dual_tree_traversal_2d_device(btk_run_config* cfg, const btk_panel_2d* panels_target,
                                             int target_panel_count, const btk_panel_2d* panels_source,
                                             int source_panel_count, btk_interact_pair** interaction_list,
                                             btk_stream_t stream);
btk_status btk_dual_tree_traversal_3d_device(btk_run_config* cfg, const btk_panel_3d* panels_target,
                                             int target_panel_count, const btk_panel_3d* panels_source,
                                             int source_panel_count, btk_interact_pair** interaction_list,
                                             btk_stream_t stream);

/* src/interaction_list.cpp:252-277. Output arrays are caller storage sized by
 * the counts in the traversal's config. */
btk_status btk_split_interactions(const btk_interact_pair* interaction_list, int interaction_count,
                                  btk_interact_pair* pp_list, btk_interact_pair* pc_list, btk_interact_pair* cp_list,
                                  btk_interact_pair* cc_list);

/* ---- 2. Drop-in device entry points (reference names and argument order) --
 *
 * Differences from the reference, by design:
 *  - parent-to-child runs only from non-leaf panels and leaf-to-point runs on
 *    every leaf (the reference skips leaves above the last level and reads
 *    child index -1 for them: src/downward_pass.cpp:9-16);
 *  - each call synchronises `stream` once to read the (small) panel and list
 *    metadata into host memory for planning; point data stays on the device;
 *  - degrees above btk_max_degree() are rejected (the reference clamps the
 *    namelist value to 10 before any call). */

/* The drop-in entry points below keep what they derive from the caller's
 * tree, leaf rows and interaction lists (the host tree, the device-side tree
 * arrays, the interaction work lists and their buffers) between calls, keyed
 * by those device buffers' addresses, the counts and the run configuration,
 * and checked on every call against a fingerprint of the buffers' contents
 * (computed on the device), so a tree rebuilt into the same buffers is noticed
 * and rebuilt. Calls are serialised by one process-wide lock. The cache holds
 * device memory until btk_dropin_cache_clear (no reference counterpart),
 * which frees it. */
btk_status btk_dropin_cache_clear(void);

/* src/upward_pass.hpp:7 */
btk_status btk_upward_pass_2d(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                              const double* ycos, const double* charges, const btk_panel_2d* blfmm_panels,
                              double* proxy_source_weights, const int* point_leaf_panel, int point_count,
                              btk_stream_t stream);
/* src/upward_pass.hpp:9 */
btk_status btk_upward_pass_3d(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                              const double* ycos, const double* zcos, const double* charges,
                              const btk_panel_3d* blfmm_panels, double* proxy_source_weights,
                              const int* point_leaf_panel, int point_count, btk_stream_t stream);

/* src/fmm_interactions/poisson_fmm.hpp:9-11 */
btk_status btk_poisson_fmm_interactions_2d(const btk_run_config* cfg, const double* xcos_t, const double* ycos_t,
                                           const double* xcos_s, const double* ycos_s, const double* charges,
                                           double* soln, const int* panel_points_inside_source,
                                           const int* panel_points_inside_target, const double* proxy_source_weights,
                                           double* proxy_target_weights, const btk_interact_pair* pp_ints,
                                           const btk_interact_pair* pc_ints, const btk_interact_pair* cp_ints,
                                           const btk_interact_pair* cc_ints, const btk_panel_2d* blfmm_panels_source,
                                           const btk_panel_2d* blfmm_panels_target, int point_count_target,
                                           int point_count_source, int panel_count_target, int panel_count_source,
                                           btk_stream_t stream);
/* src/fmm_interactions/poisson_fmm.hpp:13-15 */
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
                                           btk_stream_t stream);
/* src/fmm_interactions/poisson_vel_fmm.hpp:9-11 */
btk_status btk_poisson_vel_fmm_interactions_3d(
    const btk_run_config* cfg, const double* xcos_t, const double* ycos_t, const double* zcos_t, const double* xcos_s,
    const double* ycos_s, const double* zcos_s, const double* charges, double* vel_x, double* vel_y, double* vel_z,
    const int* panel_points_inside_source, const int* panel_points_inside_target, const double* proxy_source_weights,
    double* proxy_target_weights_x, double* proxy_target_weights_y, double* proxy_target_weights_z,
    const btk_interact_pair* pp_ints, const btk_interact_pair* pc_ints, const btk_interact_pair* cp_ints,
    const btk_interact_pair* cc_ints, const btk_panel_3d* blfmm_panels_source, const btk_panel_3d* blfmm_panels_target,
    int point_count_target, int point_count_source, int panel_count_target, int panel_count_source,
    btk_stream_t stream);

/* src/downward_pass.hpp:7 */
btk_status btk_downward_pass_2d(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                                const double* ycos, double* soln, const btk_panel_2d* blfmm_panels,
                                double* proxy_target_weights, const int* panel_points_inside, int point_count,
                                btk_stream_t stream);
/* src/downward_pass.hpp:9 */
btk_status btk_downward_pass_3d(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                                const double* ycos, const double* zcos, double* soln,
                                const btk_panel_3d* blfmm_panels, double* proxy_target_weights,
                                const int* panel_points_inside, int point_count, btk_stream_t stream);
/* src/downward_pass.hpp:11 */
btk_status btk_downward_pass_3d_3(const btk_run_config* cfg, const btk_tree_info* info, const double* xcos,
                                  const double* ycos, const double* zcos, double* vel_x, double* vel_y, double* vel_z,
                                  const btk_panel_3d* blfmm_panels, double* proxy_target_weights_x,
                                  double* proxy_target_weights_y, double* proxy_target_weights_z,
                                  const int* panel_points_inside, int point_count, btk_stream_t stream);

/* Direct sums (src/direct_sum_impl.hpp:9-94), FP64 on the device: every
 * (target, source) pair, target == source included. out[ncomp][nt] is
 * OVERWRITTEN (ncomp per kernel kind, below). Targets may be a subset. */
btk_status btk_direct_sum(int dim, int kind, double eps, int nt, const double* xt, const double* yt,
                          const double* zt, int ns, const double* xs, const double* ys, const double* zs,
                          const double* charges, double* out, btk_stream_t stream);

/* btk_direct_sum without any device allocation. No counterpart in the
 * reference. Same arguments and bit-identical results; its scratch (the
 * packed sources) lives in a static device array, so ns is limited to
 * 262,144 (BTK_ERR_INVALID_ARGUMENT above that). For callers that cannot
 * allocate during the call: a host whose caching allocator has reserved the
 * device memory, or a time-stepping loop that cannot pay an allocation every
 * step. Returns once the work is enqueued on `stream` (on the current
 * device). One scratch per device: overlapping calls on one device (threads,
 * or streams not ordered against each other) race. The first call on a
 * device looks up the scratch address (cudaGetSymbolAddress); make it before
 * any stream capture begins on that device. The address is kept for the
 * process: do not call this again on a device after cudaDeviceReset there. */
btk_status btk_direct_sum_noalloc(int dim, int kind, double eps, int nt, const double* xt, const double* yt,
                                  const double* zt, int ns, const double* xs, const double* ys, const double* zs,
                                  const double* charges, double* out, btk_stream_t stream);

/* ---- 3. Plan API ------------------------------------------------------ */

/* Kernel kinds. POT is the reference potential (2-D +(1/4pi)log(r^2+eps^2),
 * 3-D -1/(4pi sqrt(r^2+eps^2))). VEL is the reference's 3-D "velocity"
 * kernel -(1/4pi) q (t-s)/(r^2+eps^2) (poisson_vel_fmm_impl.hpp:81-84).
 * FIELD is the potential plus the field -grad_t phi of the regularised
 * potential (2-D -(1/2pi) q (t-s)/(r^2+eps^2), 3-D -(1/4pi) q (t-s)/(r^2+eps^2)^1.5);
 * FIELD has no reference counterpart. Output components: POT 1, VEL 3,
 * FIELD 1+dim (potential first). */
typedef enum { BTK_KIND_POT = 0, BTK_KIND_VEL = 1, BTK_KIND_FIELD = 2 } btk_kind;

/* Arithmetic of the interaction kernels. FP64 is the reference method.
 * MIXED evaluates in FP32 on coordinates relative to each tile's FP64 centre
 * and keeps compensated per-target sums, with FP64 interpolation weights,
 * near-node branch, centres and final sums. */
typedef enum { BTK_PREC_FP64 = 0, BTK_PREC_MIXED = 1 } btk_precision;

typedef struct btk_plan btk_plan;

/* Everything a plan is built from. Arrays are HOST memory and are copied;
 * the source_* fields may be NULL for targets = sources (one tree). */
typedef struct {
  btk_run_config cfg; /* dim, degree, thresh, eps and the four counts */
  int point_count_target, point_count_source;
  const btk_tree_info* tree_target;
  const btk_tree_info* tree_source; /* NULL: same tree */
  const void* panels_target;        /* btk_panel_2d[] or btk_panel_3d[] */
  const void* panels_source;        /* NULL: same tree */
  const int* panel_points_inside_target; /* NULL (one tree only): leaf order from point_leaf_panel_source */
  const int* panel_points_inside_source; /* NULL: same tree */
  const int* point_leaf_panel_source;
  const btk_interact_pair* pp_list;
  const btk_interact_pair* pc_list;
  const btk_interact_pair* cp_list;
  const btk_interact_pair* cc_list;
  int kind;      /* btk_kind */
  int precision; /* btk_precision */
  /* BTK_DEGREE_FIXED: every interaction at cfg.interp_degree (the reference
   * method). BTK_DEGREE_PER_PAIR: each PC/CP/CC pair at its own degree in
   * [degree_min, cfg.interp_degree], set with btk_plan_set_degrees or chosen by
   * the learned selector; the upward/downward passes stay at
   * cfg.interp_degree (exact anterpolation/promotion between degrees). */
  int degree_mode;
  int degree_min;
  /* Work items per persistent-grid slot the interaction scheduler aims at
   * (source lists of costlier items are cut into pieces); 0 = 8. */
  int work_split;
  /* 1: CC pairs are applied as shared kernel matrices (no reference
   * counterpart; a change of evaluation order, not of the method). The boxes
   * of one level are translates of each other, so pairs with equal target
   * level, source level and lattice offset share the proxy-to-proxy matrix G:
   * each such group becomes one FP64 matrix product, G evaluated once per
   * block for up to 16 pairs (32 for the potential; btk_cc_operator_groups
   * gives the grouping).
   * Used by BTK_DEGREE_FIXED plans whose trees are midpoint subdivisions of
   * one root box (one tree, or two trees over bitwise-equal root boxes);
   * ignored otherwise (btk_plan_stats.cc_groups = 0). 0: pairwise, as the
   * reference. */
  int cc_operators;
  /* BTK_DEGREE_PER_PAIR plans only (no reference counterpart). 1: the
   * learned degree choice also decides well-separated PP pairs, which the
   * reference always evaluates directly (both leaves hold at most
   * fmm_cluster_thresh points, a cost rule made for proxies at the plan
   * degree). Each such pair is evaluated directly, as target points x
   * source-leaf proxies at a chosen degree, or, where the target leaf holds
   * more points than the plan degree's proxies, as proxies x proxies; the PC
   * pairs of such target leaves and the CP pairs of source leaves larger than
   * that choose between their own form and proxies x proxies. Under the cost
   * rule the direct form costs n_t n_s with no error; under the threshold rule
   * it is taken when no approximation meets the pair tolerance or costs less.
   * Leaf pairs are direct until btk_plan_set_leaf_forms sets their forms;
   * btk_plan_set_degrees leaves those forms as they are. btk_plan_execute
   * uses the degrees and forms set by those two calls (a learned solve does
   * not change them), and the learned solve's fallback evaluates every leaf
   * pair directly and the other pairs at the plan degree, as the reference.
   * 0: PP pairs are always direct. */
  int leaf_far_pairs;
  /* The separation bound of those pairs: non-touching leaf pairs with
   * (r_t + r_s) / |c_t - c_s| < leaf_far_theta (r: half diagonals) join the
   * choice. <= 0: max(fmm_theta, 0.8), the largest MAC parameter the shipped
   * selector was trained on. */
  double leaf_far_theta;
  /* Targets per interaction work item (no reference counterpart): 256
   * (blocks of 128 threads) or 128 (blocks of 64 threads; fewer idle warps on
   * leaves and proxy sets that fill a 256-target tile only partly); 0: 256. */
  int tile_targets;
} btk_plan_desc;

enum { BTK_DEGREE_FIXED = 0, BTK_DEGREE_PER_PAIR = 1 };

/* Per-pair degrees (host arrays, one entry per pair of the plan's PC, CP and
 * CC lists, in list order; NULL keeps a class at its current degrees). Only for
 * BTK_DEGREE_PER_PAIR plans; values outside [degree_min, interp_degree] are
 * rejected. */
btk_status btk_plan_set_degrees(btk_plan* plan, const int* deg_pc, const int* deg_cp, const int* deg_cc);

/* Leaf pairs of a plan with leaf_far_pairs (the PP pairs the learned choice
 * may approximate): their count, how many of them (the first) also have the
 * proxies x proxies form, and (pp_index non-NULL) their indices in the PP list,
 * in plan order. */
btk_status btk_plan_leaf_pairs(const btk_plan* plan, int* n_pairs, int* n_with_cc, int* pp_index);
/* Sets the leaf pairs' forms for btk_plan_execute (host arrays in plan order):
 * form 0 direct, 1 target points x source-leaf proxies, 2 proxies x proxies
 * (first n_with_cc pairs only), each at degree[k] in [degree_min,
 * interp_degree] (ignored for form 0). The other pairs keep their degrees. */
btk_status btk_plan_set_leaf_forms(btk_plan* plan, const int* form, const int* degree);

btk_status btk_plan_create(btk_plan** plan, const btk_plan_desc* desc, btk_stream_t stream);
btk_status btk_plan_destroy(btk_plan* plan);

/* Work and memory figures of a plan. */
typedef struct {
  int64_t evals_pp, evals_pc, evals_cp, evals_cc; /* kernel evaluations per class */
  int64_t work_items;                             /* interaction work items */
  int64_t device_bytes;                           /* device memory the plan holds */
  int levels_target, levels_source;
  float build_ms_total; /* host wall time of btk_plan_create */
  float build_ms_work;  /* of which the work-list builder (grouping, near/far split, items) */
  int cc_groups;        /* CC pair groups applied as shared matrices (0: pairwise CC) */
  int cc_tasks;         /* tasks of the CC-group launches (groups cut into pieces of <= 16 or 32 pairs) */
  int leaf_far_pairs;   /* PP pairs the degree choice may approximate (btk_plan_desc.leaf_far_pairs) */
} btk_plan_stats;
btk_status btk_plan_stats_get(const btk_plan* plan, btk_plan_stats* stats);

/* Host-only grouping behind btk_plan_desc.cc_operators: pairs of the CC list
 * whose target level, source level and box-centre offset (in lattice units of
 * the finest level) agree get the same group id, groups numbered in key
 * order (target level, source level, offset x, y, z). panels_source NULL (or
 * equal to panels_target): one tree. When the trees are not midpoint
 * subdivisions of one common root box, *n_groups = 0 and every
 * group_of_pair[i] = -1. Panels must be in breadth-first level order. */
btk_status btk_cc_operator_groups(int dim, const void* panels_target, int n_target, const void* panels_source,
                                  int n_source, const btk_interact_pair* cc_list, int n_cc, int* group_of_pair,
                                  int* n_groups);

/* One solve on device-resident inputs: gathers points and charges into leaf
 * order, runs the upward pass, the interactions and the downward pass, and
 * writes out[ncomp][point_count_target] (OVERWRITTEN, original point order).
 * x/y/z_* and charges are device arrays in the caller's order; z may be NULL
 * in 2-D; target pointers may equal source pointers. */
btk_status btk_plan_execute(btk_plan* plan, const double* xt, const double* yt, const double* zt,
                            const double* xs, const double* ys, const double* zs, const double* charges,
                            double* out, btk_stream_t stream);

/* Phase timing of the last btk_plan_execute on this plan (CUDA events on the
 * execute stream; the call synchronises on them and reports a device-side
 * timeout as BTK_ERR_DEVICE_TIMEOUT). ms[0] upward, [1] interaction phase,
 * [2] downward, [3] total, [4] the interaction kernel alone. */
btk_status btk_plan_last_timing(btk_plan* plan, float* ms);

/* Polls of each shared-memory chunk's mbarrier the interaction kernels make
 * before giving up (no reference counterpart). A block that gives up waits
 * for its copies still in flight, stops taking work and sets the plan's
 * device status, which the next btk_plan_last_timing (or the learned solve
 * itself) returns as BTK_ERR_DEVICE_TIMEOUT; the solve's results are then
 * incomplete. 0 gives up at the first wait (to exercise that path);
 * polls < 0 restores the default (2^22). Each solve clears the status. */
btk_status btk_plan_set_wait_limit(btk_plan* plan, long long polls);

/* The targets the learned solve's audit checks (a fixed, seeded 1% of the
 * targets, at least one): their count, and (orig non-NULL, host) their
 * original indices in the order the audit evaluates them. */
btk_status btk_plan_audit_targets(const btk_plan* plan, int* n, int* orig);

/* One call from host buffers: builds the tree and lists with the host tree
 * functions, creates a plan, copies inputs to the device, solves, copies
 * out[ncomp][n] back (host) and destroys the plan. Sources = targets. */
btk_status btk_solve_host(int dim, int kind, int precision, int degree, int cluster_size, double theta,
                          double eps, int n, const double* x, const double* y, const double* z,
                          const double* charges, double* out, btk_stream_t stream);

/* ---- Learned degree selector (no reference counterpart) ------------------
 *
 * An MLP 16 -> 64 -> 64 -> 9 (ReLU) with BF16 weights and FP32 accumulation
 * predicts, for every far-field pair (PC, CP, CC) of a BTK_DEGREE_PER_PAIR
 * plan, log10 of the pair's relative error at degrees 4..12 from 16 features
 * (geometry ratios, point counts, class, eps/distance, Chebyshev-moment band
 * energies of the source's modified charges). Parameter layout (FP32, 5833):
 * W1[64][16], b1[64], W2[64][64], b2[64], W3[9][64], b3[9]. norm[34]: feature
 * means[16], feature std[16], target mean, target std (the network sees
 * normalised inputs and predicts normalised targets). */
typedef struct btk_selector btk_selector;
int btk_selector_param_count(void);
btk_status btk_selector_create(btk_selector** sel, const float* params, const float* norm);
btk_status btk_selector_destroy(btk_selector* sel);
const void* btk_selector_weights(const btk_selector* sel); /* device BF16 parameters */
/* The network on raw features: out[i][o] = predicted log10 error at degree
 * 4 + o (device arrays features[n][16], out[n][9]). Runs on the tensor cores
 * (BF16 operands, FP32 accumulation; normalised inputs and hidden activations
 * rounded to BF16). */
btk_status btk_selector_predict(const btk_selector* sel, int n, const float* features, float* out,
                                btk_stream_t stream);

/* Far-field pairs of a per-pair plan (PC, then CP, then CC, list order; with
 * leaf_far_pairs the leaf pairs follow the PC list). */
btk_status btk_plan_pair_count(const btk_plan* plan, int* n_pairs);
/* Runs the upward pass for these sources/charges and writes the features of
 * every far-field pair: device float features[n_pairs][16]. */
btk_status btk_plan_pair_features(btk_plan* plan, const double* xs, const double* ys, const double* zs,
                                  const double* charges, float* features, btk_stream_t stream);

typedef struct {
  double audit_rel_l2; /* treecode vs FP64 direct sum over the audited targets */
  int audit_targets;   /* 1% of the targets (fixed, seeded sample) */
  int fell_back;       /* 1: audit above tol, the fixed-degree FP64 result was returned */
  int64_t evals_near;  /* PP evaluations (approximated leaf pairs excluded) */
  int64_t evals_far;   /* PC + CP + CC evaluations at the chosen degrees */
  float ms_select;     /* upward pass + features + network + degree choice */
  float ms_solve;      /* interactions + promotion + downward at the chosen degrees */
  float ms_total;      /* everything, audit and fallback included */
  int degree_hist[13]; /* far-field pairs per chosen degree ([0]: leaf pairs kept direct) */
  float ms_kernel;     /* the interaction kernel of the learned solve (audit items included) */
  double pair_tol;     /* the per-pair tolerance this solve used */
} btk_learned_report;

/* Learned-degree solve: upward pass, features, network, per-pair degree =
 * the smallest d in [max(degree_lo, degree_min), interp_degree] whose
 * predicted error is <= pair_tol, interactions at those degrees (the plan's
 * precision), downward pass; then an FP64 direct-sum audit of 1% of the
 * targets (btk_plan_audit_targets), evaluated as FP64 work items of the
 * solve's own interaction launch whatever the plan's precision.
 * When the audit's relative L2 exceeds tol, the fixed-degree FP64 result is
 * computed and returned instead (report->fell_back = 1). Synchronises the
 * stream once (to read the audit). out as btk_plan_execute.
 * pair_tol <= 0 selects the plan's adaptive per-pair tolerance: it starts at
 * 0.05 tol, and after every such solve it is scaled by (tol/2) / audit
 * (clamped to [0.5, 2]), so repeated solves on one plan settle where the
 * audit reads about half the requested tolerance. */
btk_status btk_plan_execute_learned(btk_plan* plan, const btk_selector* sel, double tol, double pair_tol,
                                    int degree_lo, const double* xt, const double* yt, const double* zt,
                                    const double* xs, const double* ys, const double* zs, const double* charges,
                                    double* out, btk_learned_report* report, btk_stream_t stream);

/* How a learned solve turns predicted errors into degrees.
 * THRESHOLD: per pair the smallest degree whose predicted error <= pair_tol.
 * COST: per pair the degree minimising cost(d)/mean cost + (w/mean w) *
 * (err(d)/pair_tol)^2, with cost(d) the pair's evaluations at degree d and w
 * the points under its target panel: fewest evaluations for a given sum of
 * squared errors over the targets. COST is the default: at equal audited
 * error it needs 3-9 % fewer far-field evaluations than THRESHOLD. */
enum { BTK_DEGREE_RULE_THRESHOLD = 0, BTK_DEGREE_RULE_COST = 1 };
btk_status btk_plan_set_degree_rule(btk_plan* plan, int rule);

/* Training samples, generated by the treecode itself: for n sampled far-field
 * pairs (pair_index into the plan's pair list), the relative L2 error of the
 * pair's contribution at K target points (target_orig: original indices,
 * [n][K]) computed through the pair's degree-d proxies, for every degree
 * d = degree_min..interp_degree, against the FP64 direct sum over the points
 * under the pair's source panel (src_leaf_csr[n+1] / src_leaves: the leaf
 * panels under each source). Coordinates and charges are device arrays as in
 * btk_plan_execute. ref (optional, device [ncomp][point_count_target], original
 * order): when given, each error is relative to the L2 norm of ref at the
 * sample's targets (the total solution there) instead of to the pair's own
 * contribution. log10_err: host float [n][interp_degree - degree_min + 1]. */
btk_status btk_plan_error_samples(btk_plan* plan, const double* xt, const double* yt, const double* zt,
                                  const double* xs, const double* ys, const double* zs, const double* charges, int n,
                                  const int* pair_index, int K, const int* target_orig, const int* src_leaf_csr,
                                  const int* src_leaves, const double* ref, float* log10_err, btk_stream_t stream);

/* Training kernels (device arrays). Inputs xn are normalised features
 * [n][16], targets tn normalised [n][9], mask [n][9] (0/1). */
btk_status btk_mlp_forward(const void* w_bf16, int n, const float* xn, float* yn, btk_stream_t stream);
/* Masked mean-squared error L = sum mask (y - t)^2 / (9 n) and dL/dparams
 * (FP32, 5833 entries). work: 4*64*n + 9*n floats. */
btk_status btk_mlp_gradient(const void* w_bf16, int n, const float* xn, const float* tn, const float* mask,
                            float* grad, float* loss, float* work, btk_stream_t stream);
/* One Adam step (beta 0.9/0.999) on FP32 master parameters; refreshes the
 * BF16 copy the network runs with. step counts from 1. */
btk_status btk_mlp_adam(float* master, void* w_bf16, const float* grad, float* m, float* v, int step, float lr,
                        btk_stream_t stream);

/* Benchmark infrastructure (no reference counterpart): the sustained
 * fused-multiply-add rate of this GPU's FP64 (which = 0) or FP32 (which = 1)
 * CUDA-core pipe in TFLOP/s (2 flops per FMA), measured by a probe kernel with
 * independent FMA chains on every SM; the measured roofline denominator of
 * the pairwise interaction kernels. */
btk_status btk_measure_pipe_peak(int which, double* tflops, btk_stream_t stream);

/* ---- 5. Batches of independent problems ---------------------------------
 *
 * No counterpart in the reference (which solves one problem per call). Many
 * independent problems (targets = sources each) are solved as ONE plan over a
 * forest: each problem's tree and interaction lists come from the host tree
 * functions above (bit-identical to the reference's, with that problem's own
 * leaf size), and the trees are renumbered level by level into one panel
 * array (all level-0 roots, then all level-1 panels, ...), so the upward
 * pass, one persistent interaction launch and the downward pass cover every
 * problem at once. Interaction lists never cross problems. */

typedef struct {
  int dim, degree;
  double theta, eps;
  int n_problems;
  const int* point_offset; /* n_problems + 1: problem b owns points [off[b], off[b+1]) */
  const int* cluster_size; /* n_problems: leaf size of each problem's tree */
} btk_forest_desc;

/* A forest in the reference's layouts. Arrays are allocated by the library
 * (btk_forest_free). Point indices are global (concatenated order). */
typedef struct {
  btk_run_config cfg;        /* dim, degree, theta, eps, thresh = max leaf size, the four list counts */
  btk_tree_info info;        /* panel_count, levels, level_start[levels + 1] */
  void* panels;              /* btk_panel_2d / btk_panel_3d [panel_count]; id, parent and children renumbered */
  int* point_leaf_panel;     /* [total points] forest leaf of each point */
  int* panel_problem;        /* [panel_count] problem of each panel */
  int* panel_local;          /* [panel_count] index of the panel in its problem's own tree */
  btk_interact_pair* pp_list; /* per class: every problem's pairs, problem by problem, renumbered */
  btk_interact_pair* pc_list;
  btk_interact_pair* cp_list;
  btk_interact_pair* cc_list;
} btk_forest;

/* Builds every problem's tree and lists (host threads in parallel) and the
 * forest. x, y (, z) are HOST arrays of all points, concatenated. */
btk_status btk_forest_build(const btk_forest_desc* desc, const double* x, const double* y, const double* z,
                            btk_forest* forest);
void btk_forest_free(btk_forest* forest);

typedef struct btk_batch btk_batch;

typedef struct {
  btk_forest_desc forest;
  int kind;       /* btk_kind */
  int precision;  /* btk_precision */
  int work_split; /* work items per persistent-grid slot (0 = 8) */
  int tile_targets; /* targets per interaction work item: 256 or 128 (0 = 256) */
} btk_batch_desc;

/* Builds the forest and its plan and uploads the coordinates (HOST arrays,
 * concatenated). The geometry is fixed for the batch's life. */
btk_status btk_batch_create(btk_batch** batch, const btk_batch_desc* desc, const double* x, const double* y,
                            const double* z, btk_stream_t stream);
btk_status btk_batch_destroy(btk_batch* batch);

/* One solve of every problem. charges: DEVICE [total points]; out: DEVICE
 * [ncomp][total points] (OVERWRITTEN), both in the concatenated order. The
 * whole solve (gathers, upward pass, the persistent interaction launch,
 * downward pass) is one CUDA graph, captured on the first call (on a stream of
 * the batch's own) and replayed on `stream` after that; the charges are copied
 * into the batch's buffer and the result out of it inside the same stream
 * order. Asynchronous. */
btk_status btk_batch_execute(btk_batch* batch, const double* charges, double* out, btk_stream_t stream);

typedef struct {
  int n_problems;
  int64_t total_points;
  int panel_count, levels;
  int64_t evals_pp, evals_pc, evals_cp, evals_cc;
  int64_t work_items;
  int graph_kernel_nodes; /* kernels in the captured solve graph (0 before the first execute) */
  int graph_nodes;        /* all nodes of that graph */
  float last_ms;          /* device time of the last btk_batch_execute (graph launch only) */
} btk_batch_stats;
btk_status btk_batch_stats_get(btk_batch* batch, btk_batch_stats* stats);

#ifdef __cplusplus
}
#endif
#endif
