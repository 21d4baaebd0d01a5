/* TEST INFRASTRUCTURE ONLY — the CPU oracle for the treecode evaluation path.
 *
 * A plain-C, serial, FP64 restatement of BarytreeK's evaluation path
 * (upward pass, PP/PC/CP/CC interactions, downward pass, direct sum), used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker. The product (barytreek_b200/) never links or calls it.
 *
 * Pinning: every function here is compared in tests/ with the reference's own
 * code compiled from its sources (oracle/_ref/libbtkref.so, see Makefile) and
 * with golden fixtures generated from that library (tests/golden/).
 *
 * Panel records use the reference's exact byte layouts (src/structs.hpp:24-64).
 */
#ifndef BTK_ORACLE_H
#define BTK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* src/structs.hpp:24-39 (80 bytes) */
typedef struct {
  int id, level, parent_id, child[4];
  unsigned char is_leaf;
  double max_x, min_x, max_y, min_y, radius;
  int point_count;
} bto_panel2;

/* src/structs.hpp:41-64 (112 bytes; note min_z precedes max_z) */
typedef struct {
  int id, level, parent_id, child[8];
  unsigned char is_leaf;
  double max_x, min_x, max_y, min_y, min_z, max_z, radius;
  int point_count;
} bto_panel3;

/* src/structs.hpp:71-75 (12 bytes) */
typedef struct {
  int target_panel, source_panel, interact_type;
} bto_pair;

/* Kernel kinds shared with the product:
 *   0 POT   : 2-D  (1/4pi) log(r^2+eps^2)        (poisson_fmm_impl.hpp:38,47)
 *             3-D -(1/4pi) / sqrt(r^2+eps^2)     (poisson_fmm_impl.hpp:241,252)
 *   1 VEL   : 3-D -(1/4pi) q (t-s) / (r^2+eps^2) (poisson_vel_fmm_impl.hpp:42,53-56)
 *   2 FIELD : potential plus the field -grad_t phi of the regularised
 *             potential (no reference counterpart):
 *             2-D -(1/2pi) q (t-s) / (r^2+eps^2),
 *             3-D -(1/4pi) q (t-s) / (r^2+eps^2)^{3/2}.
 * Component counts: POT 1, VEL 3, FIELD 1+dim (potential first). */
enum { BTO_POT = 0, BTO_VEL = 1, BTO_FIELD = 2 };

int bto_ncomp(int dim, int kind);

/* Barycentric Lagrange basis on Chebyshev points of the 2nd kind
 * (src/bli_impl.hpp:9-63). out[0..n]. */
void bto_interp_basis(double* out, double x, double lo, double hi, int n);
/* Chebyshev points mapped to [lo,hi] (src/bli_impl.hpp:66-77). */
void bto_nodes(double* out, double lo, double hi, int n);

/* Upward pass (src/upward_pass.cpp:7-28): psw[panel_count x (n+1)^dim] is
 * zeroed, then filled by base_pots + child_to_parent. */
int bto_upward(int dim, int degree, int n_src, const double* x, const double* y, const double* z,
               const double* q, int panel_count, const void* panels, const int* level_start, int levels,
               const int* leaf_of, double* psw);

/* Interaction phase (src/fmm_interactions/poisson_fmm.cpp:8-26,
 * poisson_vel_fmm.cpp:8-17). Accumulates into out[ncomp][n_tgt] and
 * ptw[ncomp][panel_count_t x ipc] (callers zero them first, as the reference's
 * callers do). */
int bto_interactions(int dim, int kind, int degree, double eps, int thresh,
                     int n_tgt, const double* tx, const double* ty, const double* tz,
                     int n_src, const double* sx, const double* sy, const double* sz, const double* q,
                     const void* panels_t, const int* inside_t, const void* panels_s, const int* inside_s,
                     const bto_pair* pp, int n_pp, const bto_pair* pc, int n_pc,
                     const bto_pair* cp, int n_cp, const bto_pair* cc, int n_cc,
                     const double* psw, int panel_count_t, double* ptw, double* out);

/* Downward pass with the two-site fix for leaves above the last level:
 * parent_to_child only from non-leaf panels (levels 0..L-2), leaf_to_point on
 * every leaf (src/downward_pass.cpp:7-41, downward_pass_impl.hpp). Accumulates
 * into out[ncomp][n_tgt]; ptw is updated in place. */
int bto_downward(int dim, int ncomp, int degree, int thresh, int n_tgt, const double* tx, const double* ty,
                 const double* tz, int panel_count, const void* panels, const int* level_start, int levels,
                 const int* inside, double* ptw, double* out);

/* Treecode with a degree per far-field pair (the learned-degree extension; no
 * reference counterpart). PP as the reference; every PC/CP/CC pair (T, S) at
 * its own degree d is evaluated straight at the target points:
 *   Q^d_S  = modified charges of all points under S at degree d
 *            (base_pots at degree d on S's box),
 *   PC     : phi(t) += sum_k G(t, x^d_k(S)) Q^d_S[k]      for t in leaf T,
 *   CP, CC : Phi^d_T[j] = sum over S's points (CP) or proxies (CC) of
 *            G(x^d_j(T), s) w_s, then phi(t) += sum_j Phi^d_T[j] L^d_j(t) for
 *            every point t under T.
 * This equals the tree's anterpolate/transfer/promote/downward chain exactly
 * in exact arithmetic (polynomial reproduction). out[ncomp][n_tgt] is
 * overwritten. deg_* may be NULL (then `degree` is used for that class). */
int bto_solve_degrees(int dim, int kind, int degree, double eps, int thresh, int n_tgt, const double* tx,
                      const double* ty, const double* tz, int n_src, const double* sx, const double* sy,
                      const double* sz, const double* q, const void* panels_t, int panel_count_t,
                      const int* inside_t, const void* panels_s, int panel_count_s, const int* inside_s,
                      const bto_pair* pp, int n_pp, const bto_pair* pc, int n_pc, const int* deg_pc,
                      const bto_pair* cp, int n_cp, const int* deg_cp, const bto_pair* cc, int n_cc,
                      const int* deg_cc, double* out);

/* O(nt*ns) direct sum including i==j (src/direct_sum_impl.hpp:9-94).
 * out[ncomp][nt] is overwritten. */
int bto_direct(int dim, int kind, double eps, int nt, const double* tx, const double* ty, const double* tz,
               int ns, const double* sx, const double* sy, const double* sz, const double* q, double* out);

#ifdef __cplusplus
}
#endif
#endif
