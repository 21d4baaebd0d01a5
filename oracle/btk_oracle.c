/* TEST INFRASTRUCTURE ONLY — see btk_oracle.h. Serial FP64 restatement of the
 * reference's evaluation path; each function names the reference lines it
 * follows. Written for clarity, not speed: tests keep its inputs small. */
#include "btk_oracle.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

_Static_assert(sizeof(bto_panel2) == 80, "TreePanel_2d layout");
_Static_assert(sizeof(bto_panel3) == 112, "TreePanel_3d layout");
_Static_assert(offsetof(bto_panel3, min_z) == 80, "TreePanel_3d min_z offset");
_Static_assert(offsetof(bto_panel3, radius) == 96, "TreePanel_3d radius offset");
_Static_assert(offsetof(bto_panel3, point_count) == 104, "TreePanel_3d point_count offset");
_Static_assert(offsetof(bto_panel2, point_count) == 72, "TreePanel_2d point_count offset");
_Static_assert(sizeof(bto_pair) == 12, "interact_pair layout");

#define MAXD 16 /* stack arrays: degree <= 15 */
static const double PI = 3.14159265358979323846;

typedef struct {
  double lo[3], hi[3];
  int leaf, count, parent, nchild;
  int child[8];
} pnl;

static pnl get_panel(int dim, const void* panels, int i) {
  pnl p;
  memset(&p, 0, sizeof(p));
  if (dim == 2) {
    const bto_panel2* s = (const bto_panel2*)panels + i;
    p.lo[0] = s->min_x; p.hi[0] = s->max_x;
    p.lo[1] = s->min_y; p.hi[1] = s->max_y;
    p.leaf = s->is_leaf; p.count = s->point_count; p.parent = s->parent_id; p.nchild = 4;
    for (int c = 0; c < 4; ++c) p.child[c] = s->child[c];
  } else {
    const bto_panel3* s = (const bto_panel3*)panels + i;
    p.lo[0] = s->min_x; p.hi[0] = s->max_x;
    p.lo[1] = s->min_y; p.hi[1] = s->max_y;
    p.lo[2] = s->min_z; p.hi[2] = s->max_z;
    p.leaf = s->is_leaf; p.count = s->point_count; p.parent = s->parent_id; p.nchild = 8;
    for (int c = 0; c < 8; ++c) p.child[c] = s->child[c];
  }
  return p;
}

int bto_ncomp(int dim, int kind) {
  if (kind == BTO_POT) return 1;
  if (kind == BTO_VEL) return 3;
  return 1 + dim;
}

/* src/bli_impl.hpp:9-63. Nodes cos(pi*i/n) on [lo,hi]; weights 1/2, (-1)^i,
 * (-1)^n/2; absolute near-node test |x - x_i| < DBL_EPSILON. */
void bto_interp_basis(double* out, double x, double lo, double hi, int n) {
  double range = 0.5 * (hi - lo), mid = 0.5 * (hi + lo);
  double node[MAXD], wt[MAXD];
  if (n == 0) {
    out[0] = 1.0;
    return;
  }
  for (int i = 0; i <= n; ++i) {
    node[i] = cos(PI * i / n) * range + mid;
    wt[i] = (i % 2 == 0) ? 1.0 : -1.0;
    if (i == 0 || i == n) wt[i] *= 0.5;
  }
  for (int i = 0; i <= n; ++i) {
    if (fabs(x - node[i]) < 2.220446049250313e-16) {
      for (int j = 0; j <= n; ++j) out[j] = 0.0;
      out[i] = 1.0;
      return;
    }
  }
  double denom = 0.0;
  for (int i = 0; i <= n; ++i) {
    out[i] = wt[i] / (x - node[i]);
    denom += out[i];
  }
  for (int i = 0; i <= n; ++i) out[i] /= denom;
}

/* src/bli_impl.hpp:66-77 (note the cos(pi/n*i) evaluation order). */
void bto_nodes(double* out, double lo, double hi, int n) {
  double range = 0.5 * (hi - lo), mid = 0.5 * (hi + lo);
  if (n == 0) {
    out[0] = mid;
    return;
  }
  for (int i = 0; i <= n; ++i) out[i] = cos(PI / n * i) * range + mid;
}

static int ipow(int b, int e) {
  int r = 1;
  while (e-- > 0) r *= b;
  return r;
}

/* One kernel evaluation, accumulated into acc[]. POT follows
 * poisson_fmm_impl.hpp:47 (2-D) and :252 (3-D); VEL follows
 * poisson_vel_fmm_impl.hpp:81-84; FIELD is the regularised -grad_t phi. */
static void eval(int dim, int kind, double eps2, const double* t, const double* s, double w, double* acc) {
  double dx = t[0] - s[0], dy = t[1] - s[1], dz = dim == 3 ? t[2] - s[2] : 0.0;
  double r2 = dx * dx + dy * dy + dz * dz + eps2;
  if (dim == 2) {
    if (kind == BTO_POT) {
      acc[0] += (1.0 / (4.0 * PI)) * log(r2) * w;
    } else {
      acc[0] += (1.0 / (4.0 * PI)) * log(r2) * w;
      double g = -w / (2.0 * PI * r2);
      acc[1] += dx * g;
      acc[2] += dy * g;
    }
    return;
  }
  if (kind == BTO_POT) {
    acc[0] += (-1.0 / (4.0 * PI)) / sqrt(r2) * w;
  } else if (kind == BTO_VEL) {
    double g = w * (-1.0 / (4.0 * PI)) / r2;
    acc[0] += dx * g;
    acc[1] += dy * g;
    acc[2] += dz * g;
  } else {
    double rinv = 1.0 / sqrt(r2);
    acc[0] += (-1.0 / (4.0 * PI)) * rinv * w;
    double g = (-1.0 / (4.0 * PI)) * rinv * rinv * rinv * w;
    acc[1] += dx * g;
    acc[2] += dy * g;
    acc[3] += dz * g;
  }
}

/* Proxy point k of a panel in tensor order (x slowest, then y, then z), as the
 * reference's nested j/k/l loops index it (e.g. upward_pass_impl.hpp:161-168). */
static void proxy_point(int dim, int n, const double nodes[3][MAXD], int k, double* out) {
  int m = n + 1;
  if (dim == 2) {
    out[0] = nodes[0][k / m];
    out[1] = nodes[1][k % m];
  } else {
    out[0] = nodes[0][k / (m * m)];
    out[1] = nodes[1][(k / m) % m];
    out[2] = nodes[2][k % m];
  }
}

static void panel_nodes(int dim, int n, const pnl* p, double nodes[3][MAXD]) {
  for (int d = 0; d < dim; ++d) bto_nodes(nodes[d], p->lo[d], p->hi[d], n);
}

/* Tensor-product basis value for proxy index k given per-axis basis rows. */
static double basis_prod(int dim, int n, const double b[3][MAXD], int k) {
  int m = n + 1;
  if (dim == 2) return b[0][k / m] * b[1][k % m];
  return b[0][k / (m * m)] * b[1][(k / m) % m] * b[2][k % m];
}

/* src/upward_pass.cpp:7-28 with base_pots (upward_pass_impl.hpp:9-44,
 * 90-132) and child_to_parent (:46-88, 134-188) for levels L-1..1. */
int bto_upward(int dim, int degree, int n_src, const double* x, const double* y, const double* z,
               const double* q, int panel_count, const void* panels, const int* level_start, int levels,
               const int* leaf_of, double* psw) {
  int n = degree, ipc = ipow(n + 1, dim);
  memset(psw, 0, sizeof(double) * (size_t)panel_count * ipc);
  for (int i = 0; i < n_src; ++i) {
    pnl p = get_panel(dim, panels, leaf_of[i]);
    double pt[3] = {x[i], y[i], dim == 3 ? z[i] : 0.0};
    double b[3][MAXD];
    for (int d = 0; d < dim; ++d) bto_interp_basis(b[d], pt[d], p.lo[d], p.hi[d], n);
    for (int k = 0; k < ipc; ++k) psw[(size_t)leaf_of[i] * ipc + k] += basis_prod(dim, n, b, k) * q[i];
  }
  for (int lev = levels - 1; lev > 0; --lev) {
    for (int i = level_start[lev]; i < level_start[lev + 1]; ++i) {
      pnl c = get_panel(dim, panels, i);
      if (c.parent < 0) continue;
      pnl par = get_panel(dim, panels, c.parent);
      double cn[3][MAXD];
      panel_nodes(dim, n, &c, cn);
      for (int k1 = 0; k1 < ipc; ++k1) {
        double cpt[3], b[3][MAXD];
        proxy_point(dim, n, cn, k1, cpt);
        for (int d = 0; d < dim; ++d) bto_interp_basis(b[d], cpt[d], par.lo[d], par.hi[d], n);
        double w = psw[(size_t)i * ipc + k1];
        for (int k2 = 0; k2 < ipc; ++k2) psw[(size_t)c.parent * ipc + k2] += basis_prod(dim, n, b, k2) * w;
      }
    }
  }
  return 0;
}

int bto_interactions(int dim, int kind, int degree, double eps, int thresh,
                     int n_tgt, const double* tx, const double* ty, const double* tz,
                     int n_src, const double* sx, const double* sy, const double* sz, const double* q,
                     const void* panels_t, const int* inside_t, const void* panels_s, const int* inside_s,
                     const bto_pair* pp, int n_pp, const bto_pair* pc, int n_pc,
                     const bto_pair* cp, int n_cp, const bto_pair* cc, int n_cc,
                     const double* psw, int panel_count_t, double* ptw, double* out) {
  (void)n_src;
  int n = degree, ipc = ipow(n + 1, dim), nc = bto_ncomp(dim, kind);
  double eps2 = eps * eps;
  size_t ptw_stride = (size_t)panel_count_t * ipc;
  double acc[4];
  /* PP: poisson_fmm_impl.hpp:31-51 (2-D), :234-256 (3-D) */
  for (int e = 0; e < n_pp; ++e) {
    pnl T = get_panel(dim, panels_t, pp[e].target_panel), S = get_panel(dim, panels_s, pp[e].source_panel);
    for (int j = 0; j < T.count; ++j) {
      int it = inside_t[(size_t)pp[e].target_panel * thresh + j];
      double t[3] = {tx[it], ty[it], dim == 3 ? tz[it] : 0.0};
      memset(acc, 0, sizeof(acc));
      for (int k = 0; k < S.count; ++k) {
        int is = inside_s[(size_t)pp[e].source_panel * thresh + k];
        double s[3] = {sx[is], sy[is], dim == 3 ? sz[is] : 0.0};
        eval(dim, kind, eps2, t, s, q[is], acc);
      }
      for (int c = 0; c < nc; ++c) out[(size_t)c * n_tgt + it] += acc[c];
    }
  }
  /* PC: poisson_fmm_impl.hpp:73-102, :279-315 */
  for (int e = 0; e < n_pc; ++e) {
    pnl T = get_panel(dim, panels_t, pc[e].target_panel), S = get_panel(dim, panels_s, pc[e].source_panel);
    double sn[3][MAXD];
    panel_nodes(dim, n, &S, sn);
    for (int j = 0; j < T.count; ++j) {
      int it = inside_t[(size_t)pc[e].target_panel * thresh + j];
      double t[3] = {tx[it], ty[it], dim == 3 ? tz[it] : 0.0};
      memset(acc, 0, sizeof(acc));
      for (int k = 0; k < ipc; ++k) {
        double s[3];
        proxy_point(dim, n, sn, k, s);
        eval(dim, kind, eps2, t, s, psw[(size_t)pc[e].source_panel * ipc + k], acc);
      }
      for (int c = 0; c < nc; ++c) out[(size_t)c * n_tgt + it] += acc[c];
    }
  }
  /* CP: poisson_fmm_impl.hpp:124-152, :338-373 */
  for (int e = 0; e < n_cp; ++e) {
    pnl T = get_panel(dim, panels_t, cp[e].target_panel), S = get_panel(dim, panels_s, cp[e].source_panel);
    double tn[3][MAXD];
    panel_nodes(dim, n, &T, tn);
    for (int k = 0; k < ipc; ++k) {
      double t[3];
      proxy_point(dim, n, tn, k, t);
      memset(acc, 0, sizeof(acc));
      for (int j = 0; j < S.count; ++j) {
        int is = inside_s[(size_t)cp[e].source_panel * thresh + j];
        double s[3] = {sx[is], sy[is], dim == 3 ? sz[is] : 0.0};
        eval(dim, kind, eps2, t, s, q[is], acc);
      }
      for (int c = 0; c < nc; ++c) ptw[c * ptw_stride + (size_t)cp[e].target_panel * ipc + k] += acc[c];
    }
  }
  /* CC: poisson_fmm_impl.hpp:170-208, :391-441 */
  for (int e = 0; e < n_cc; ++e) {
    pnl T = get_panel(dim, panels_t, cc[e].target_panel), S = get_panel(dim, panels_s, cc[e].source_panel);
    double tn[3][MAXD], sn[3][MAXD];
    panel_nodes(dim, n, &T, tn);
    panel_nodes(dim, n, &S, sn);
    for (int k = 0; k < ipc; ++k) {
      double t[3];
      proxy_point(dim, n, tn, k, t);
      memset(acc, 0, sizeof(acc));
      for (int j = 0; j < ipc; ++j) {
        double s[3];
        proxy_point(dim, n, sn, j, s);
        eval(dim, kind, eps2, t, s, psw[(size_t)cc[e].source_panel * ipc + j], acc);
      }
      for (int c = 0; c < nc; ++c) ptw[c * ptw_stride + (size_t)cc[e].target_panel * ipc + k] += acc[c];
    }
  }
  return 0;
}

/* Downward pass: parent_to_child (downward_pass_impl.hpp:9-68, 109-191,
 * 239-325) from non-leaf panels of levels 0..L-2 in level order, then
 * leaf_to_point (:70-107, 193-237, 327-379) on every leaf. */
int bto_downward(int dim, int ncomp, int degree, int thresh, int n_tgt, const double* tx, const double* ty,
                 const double* tz, int panel_count, const void* panels, const int* level_start, int levels,
                 const int* inside, double* ptw, double* out) {
  int n = degree, ipc = ipow(n + 1, dim);
  size_t stride = (size_t)panel_count * ipc;
  for (int lev = 0; lev < levels - 1; ++lev) {
    for (int i = level_start[lev]; i < level_start[lev + 1]; ++i) {
      pnl par = get_panel(dim, panels, i);
      if (par.leaf) continue;
      for (int ch = 0; ch < par.nchild; ++ch) {
        int cid = par.child[ch];
        pnl c = get_panel(dim, panels, cid);
        double cn[3][MAXD];
        panel_nodes(dim, n, &c, cn);
        for (int k1 = 0; k1 < ipc; ++k1) {
          double cpt[3], b[3][MAXD];
          proxy_point(dim, n, cn, k1, cpt);
          for (int d = 0; d < dim; ++d) bto_interp_basis(b[d], cpt[d], par.lo[d], par.hi[d], n);
          for (int comp = 0; comp < ncomp; ++comp) {
            double s = 0.0;
            for (int k2 = 0; k2 < ipc; ++k2) s += basis_prod(dim, n, b, k2) * ptw[comp * stride + (size_t)i * ipc + k2];
            ptw[comp * stride + (size_t)cid * ipc + k1] += s;
          }
        }
      }
    }
  }
  for (int i = 0; i < panel_count; ++i) {
    pnl p = get_panel(dim, panels, i);
    if (!p.leaf) continue;
    for (int j = 0; j < p.count; ++j) {
      int it = inside[(size_t)i * thresh + j];
      double t[3] = {tx[it], ty[it], dim == 3 ? tz[it] : 0.0};
      double b[3][MAXD];
      for (int d = 0; d < dim; ++d) bto_interp_basis(b[d], t[d], p.lo[d], p.hi[d], n);
      for (int comp = 0; comp < ncomp; ++comp) {
        double s = 0.0;
        for (int k = 0; k < ipc; ++k) s += ptw[comp * stride + (size_t)i * ipc + k] * basis_prod(dim, n, b, k);
        out[(size_t)comp * n_tgt + it] += s;
      }
    }
  }
  return 0;
}

/* src/direct_sum_impl.hpp:9-94: every (i, j) pair, i == j included. */
int bto_direct(int dim, int kind, double eps, int nt, const double* tx, const double* ty, const double* tz,
               int ns, const double* sx, const double* sy, const double* sz, const double* q, double* out) {
  int nc = bto_ncomp(dim, kind);
  for (int i = 0; i < nt; ++i) {
    double t[3] = {tx[i], ty[i], dim == 3 ? tz[i] : 0.0};
    double acc[4] = {0, 0, 0, 0};
    for (int j = 0; j < ns; ++j) {
      double s[3] = {sx[j], sy[j], dim == 3 ? sz[j] : 0.0};
      eval(dim, kind, eps * eps, t, s, q[j], acc);
    }
    for (int c = 0; c < nc; ++c) out[(size_t)c * nt + i] = acc[c];
  }
  return 0;
}

/* ---- per-pair degrees (learned-degree extension) ------------------------- */

/* Appends the points under panel p (all leaves of its subtree) to buf. */
static void subtree_points(int dim, const void* panels, const int* inside, int thresh, int p, int* buf, int* n) {
  pnl P = get_panel(dim, panels, p);
  if (P.leaf) {
    for (int j = 0; j < P.count; ++j) buf[(*n)++] = inside[(size_t)p * thresh + j];
    return;
  }
  for (int c = 0; c < P.nchild; ++c) subtree_points(dim, panels, inside, thresh, P.child[c], buf, n);
}

/* Modified charges at degree d of the given points on panel S's box. */
static void charges_at_degree(int dim, int d, const pnl* S, const int* idx, int n, const double* sx, const double* sy,
                              const double* sz, const double* q, double* Q) {
  int ipc = ipow(d + 1, dim);
  memset(Q, 0, sizeof(double) * ipc);
  for (int i = 0; i < n; ++i) {
    int s = idx[i];
    double pt[3] = {sx[s], sy[s], dim == 3 ? sz[s] : 0.0};
    double b[3][MAXD];
    for (int a = 0; a < dim; ++a) bto_interp_basis(b[a], pt[a], S->lo[a], S->hi[a], d);
    for (int k = 0; k < ipc; ++k) Q[k] += basis_prod(dim, d, b, k) * q[s];
  }
}

int bto_solve_degrees(int dim, int kind, int degree, double eps, int thresh, int n_tgt, const double* tx,
                      const double* ty, const double* tz, int n_src, const double* sx, const double* sy,
                      const double* sz, const double* q, const void* panels_t, int panel_count_t,
                      const int* inside_t, const void* panels_s, int panel_count_s, const int* inside_s,
                      const bto_pair* pp, int n_pp, const bto_pair* pc, int n_pc, const int* deg_pc,
                      const bto_pair* cp, int n_cp, const int* deg_cp, const bto_pair* cc, int n_cc,
                      const int* deg_cc, double* out) {
  (void)panel_count_t;
  (void)panel_count_s;
  const int nc = bto_ncomp(dim, kind);
  const double eps2 = eps * eps;
  const int maxipc = ipow(MAXD, dim);
  int* tbuf = (int*)malloc(sizeof(int) * (n_tgt > 0 ? n_tgt : 1));
  int* sbuf = (int*)malloc(sizeof(int) * (n_src > 0 ? n_src : 1));
  double* Q = (double*)malloc(sizeof(double) * maxipc);
  double* Phi = (double*)malloc(sizeof(double) * maxipc * 4);
  if (!tbuf || !sbuf || !Q || !Phi) return 1;
  memset(out, 0, sizeof(double) * (size_t)nc * n_tgt);
  double acc[4];
  /* PP exactly as the reference */
  for (int e = 0; e < n_pp; ++e) {
    pnl T = get_panel(dim, panels_t, pp[e].target_panel), S = get_panel(dim, panels_s, pp[e].source_panel);
    for (int j = 0; j < T.count; ++j) {
      int it = inside_t[(size_t)pp[e].target_panel * thresh + j];
      double t[3] = {tx[it], ty[it], dim == 3 ? tz[it] : 0.0};
      memset(acc, 0, sizeof(acc));
      for (int k = 0; k < S.count; ++k) {
        int is = inside_s[(size_t)pp[e].source_panel * thresh + k];
        double s[3] = {sx[is], sy[is], dim == 3 ? sz[is] : 0.0};
        eval(dim, kind, eps2, t, s, q[is], acc);
      }
      for (int c = 0; c < nc; ++c) out[(size_t)c * n_tgt + it] += acc[c];
    }
  }
  const bto_pair* lists[3] = {pc, cp, cc};
  const int counts[3] = {n_pc, n_cp, n_cc};
  const int* degs[3] = {deg_pc, deg_cp, deg_cc};
  for (int L = 0; L < 3; ++L) {
    for (int e = 0; e < counts[L]; ++e) {
      const bto_pair pr = lists[L][e];
      const int d = degs[L] ? degs[L][e] : degree;
      const int ipc = ipow(d + 1, dim);
      pnl T = get_panel(dim, panels_t, pr.target_panel), S = get_panel(dim, panels_s, pr.source_panel);
      double tn[3][MAXD], sn[3][MAXD];
      panel_nodes(dim, d, &T, tn);
      panel_nodes(dim, d, &S, sn);
      int ns_ = 0, nt_ = 0;
      subtree_points(dim, panels_s, inside_s, thresh, pr.source_panel, sbuf, &ns_);
      subtree_points(dim, panels_t, inside_t, thresh, pr.target_panel, tbuf, &nt_);
      if (L == 0) { /* PC */
        charges_at_degree(dim, d, &S, sbuf, ns_, sx, sy, sz, q, Q);
        for (int j = 0; j < nt_; ++j) {
          int it = tbuf[j];
          double t[3] = {tx[it], ty[it], dim == 3 ? tz[it] : 0.0};
          memset(acc, 0, sizeof(acc));
          for (int k = 0; k < ipc; ++k) {
            double s[3];
            proxy_point(dim, d, sn, k, s);
            eval(dim, kind, eps2, t, s, Q[k], acc);
          }
          for (int c = 0; c < nc; ++c) out[(size_t)c * n_tgt + it] += acc[c];
        }
        continue;
      }
      if (L == 2) charges_at_degree(dim, d, &S, sbuf, ns_, sx, sy, sz, q, Q);
      for (int jj = 0; jj < ipc; ++jj) {
        double t[3];
        proxy_point(dim, d, tn, jj, t);
        memset(acc, 0, sizeof(acc));
        if (L == 1) { /* CP: S is a leaf, its own points */
          for (int k = 0; k < ns_; ++k) {
            int is = sbuf[k];
            double s[3] = {sx[is], sy[is], dim == 3 ? sz[is] : 0.0};
            eval(dim, kind, eps2, t, s, q[is], acc);
          }
        } else { /* CC */
          for (int k = 0; k < ipc; ++k) {
            double s[3];
            proxy_point(dim, d, sn, k, s);
            eval(dim, kind, eps2, t, s, Q[k], acc);
          }
        }
        for (int c = 0; c < nc; ++c) Phi[(size_t)c * ipc + jj] = acc[c];
      }
      for (int j = 0; j < nt_; ++j) {
        int it = tbuf[j];
        double t[3] = {tx[it], ty[it], dim == 3 ? tz[it] : 0.0};
        double b[3][MAXD];
        for (int a = 0; a < dim; ++a) bto_interp_basis(b[a], t[a], T.lo[a], T.hi[a], d);
        for (int c = 0; c < nc; ++c) {
          double s = 0.0;
          for (int k = 0; k < ipc; ++k) s += Phi[(size_t)c * ipc + k] * basis_prod(dim, d, b, k);
          out[(size_t)c * n_tgt + it] += s;
        }
      }
    }
  }
  free(tbuf);
  free(sbuf);
  free(Q);
  free(Phi);
  return 0;
}
