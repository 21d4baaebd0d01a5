// Upward and downward passes, gathers and proxy materialisation (FP64).
//
// These kernels follow the reference's functors (src/upward_pass_impl.hpp,
// src/downward_pass_impl.hpp) but are gather-shaped: each output row (a leaf's
// modified charges, a parent's anterpolated charges, a child's interpolated
// potentials, a target's value) is produced by one thread block, so no atomics
// are needed and results are bit-reproducible. The (n+1)^d x (n+1)^d
// child<->parent transfers are applied as d one-dimensional (n+1)x(n+1)
// contractions (the tensor-product basis factorises), which is the same linear
// map as the reference's nested loops with (n+1)^d fewer operations.
#include "device_math.cuh"
#include "kernels.cuh"

namespace btk {

namespace {

constexpr double kDblEps = 2.220446049250313e-16;  // numeric_limits<double>::epsilon()

// Barycentric weights 1/2, (-1)^i, (-1)^n/2 (src/bli_impl.hpp:26-32).
template <int M>
__device__ __forceinline__ double bary_weight(int i) {
  double w = (i & 1) ? -1.0 : 1.0;
  return (i == 0 || i == M - 1) ? 0.5 * w : w;
}

// interp_vals_bli (src/bli_impl.hpp:9-63) on precomputed nodes:
// the absolute near-node test, then w_i/(x-x_i) normalised by their sum.
template <int M>
__device__ __forceinline__ void bary_basis(double (&L)[M], double x, const double* node) {
  int hit = -1;
#pragma unroll
  for (int i = 0; i < M; ++i)
    if (hit < 0 && fabs(x - node[i]) < kDblEps) hit = i;
  if (hit >= 0) {
#pragma unroll
    for (int i = 0; i < M; ++i) L[i] = (i == hit) ? 1.0 : 0.0;
    return;
  }
  double denom = 0.0;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    L[i] = bary_weight<M>(i) / (x - node[i]);
    denom += L[i];
  }
#pragma unroll
  for (int i = 0; i < M; ++i) L[i] = L[i] / denom;
}

template <int M, int DIM>
__host__ __device__ constexpr int ipow_c() {
  return DIM == 2 ? M * M : M * M * M;
}

// ---- per-panel geometry ---------------------------------------------------
// One thread per (panel, axis, node): nodes_shift/nodes_interp, then (second
// kernel) the transfer rows L^{parent}_a(node_shift^child_i).
__global__ void k_panel_nodes(int dim, int m, int P, const DevPanel* panels, const double* ucos_shift,
                              const double* ucos_interp, double* nodes_shift, double* nodes_interp) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int total = P * dim * m;
  if (t >= total) return;
  int i = t % m, d = (t / m) % dim, p = t / (m * dim);
  double lo = panels[p].lo[d], hi = panels[p].hi[d];
  double range = __dmul_rn(0.5, __dsub_rn(hi, lo));
  double mid = __dmul_rn(0.5, __dadd_rn(hi, lo));
  nodes_shift[(size_t)p * kPanelNodes + d * kNodeStride + i] = __dadd_rn(__dmul_rn(ucos_shift[i], range), mid);
  nodes_interp[(size_t)p * kPanelNodes + d * kNodeStride + i] = __dadd_rn(__dmul_rn(ucos_interp[i], range), mid);
}

template <int M>
__global__ void k_panel_xfer(int dim, int P, const DevPanel* panels, const double* nodes_shift,
                             const double* nodes_interp, double* xfer) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int total = P * dim * M;
  if (t >= total) return;
  int i = t % M, d = (t / M) % dim, c = t / (M * dim);
  int par = panels[c].parent;
  double* row = xfer + (size_t)c * kPanelXfer + (d * kMaxNodes + i) * kMaxNodes;
  if (par < 0) {
    for (int a = 0; a < M; ++a) row[a] = 0.0;
    return;
  }
  double L[M];
  bary_basis<M>(L, nodes_shift[(size_t)c * kPanelNodes + d * kNodeStride + i],
                nodes_interp + (size_t)par * kPanelNodes + d * kNodeStride);
#pragma unroll
  for (int a = 0; a < M; ++a) row[a] = L[a];
}

// ---- gathers ---------------------------------------------------------------
__global__ void k_perm_from_inside(const int* leaves, const int* leaf_begin, const int* point_count,
                                   const int* inside, int thresh, int* perm) {
  int L = leaves[blockIdx.x];
  int b = leaf_begin[L], n = point_count[L];
  for (int j = threadIdx.x; j < n; j += blockDim.x) perm[b + j] = inside[(size_t)L * thresh + j];
}

__global__ void k_gather(int n, const int* perm, const double* x, const double* y, const double* z,
                         const double* w, double4* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int i = perm[k];
  out[k] = make_double4(x[i], y[i], z ? z[i] : 0.0, w ? w[i] : 0.0);
}

// ---- upward pass -----------------------------------------------------------
// base_pots (src/upward_pass_impl.hpp:90-132): a leaf's modified charges
// W[a,b,c] = sum_p q_p Lx_a(x_p) Ly_b(y_p) Lz_c(z_p), one block per leaf.
template <int DIM, int M>
__global__ void __launch_bounds__(256) k_leaf_moments(const int* leaves, const int* leaf_begin, const int* point_count,
                                                      const double4* pts, const double* nodes_interp, double* psw) {
  constexpr int IPC = ipow_c<M, DIM>();
  constexpr int PCH = 32;
  constexpr int PER = (IPC + 255) / 256;
  __shared__ double sb[3][PCH][M];
  __shared__ double snode[3][kMaxNodes];
  const int L = leaves[blockIdx.x];
  const int b = leaf_begin[L], cnt = point_count[L];
  if (threadIdx.x < 3 * kMaxNodes)
    snode[threadIdx.x / kMaxNodes][threadIdx.x % kMaxNodes] =
        nodes_interp[(size_t)L * kPanelNodes + threadIdx.x];
  double acc[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) acc[k] = 0.0;
  __syncthreads();
  for (int p0 = 0; p0 < cnt; p0 += PCH) {
    const int t = threadIdx.x;
    if (t < PCH * DIM) {
      int pp = t / DIM, d = t % DIM;
      if (p0 + pp < cnt) {
        double4 pt = pts[b + p0 + pp];
        double x = d == 0 ? pt.x : (d == 1 ? pt.y : pt.z);
        double Lv[M];
        bary_basis<M>(Lv, x, snode[d]);
        // The reference multiplies the basis product by the charge last
        // (upward_pass_impl.hpp:164); folding q into the x factor first
        // changes only the last bit.
#pragma unroll
        for (int a = 0; a < M; ++a) sb[d][pp][a] = d == 0 ? Lv[a] * pt.w : Lv[a];
      } else {
#pragma unroll
        for (int a = 0; a < M; ++a) sb[d][pp][a] = 0.0;
      }
    }
    __syncthreads();
    const int np = min(PCH, cnt - p0);
#pragma unroll
    for (int k = 0; k < PER; ++k) {
      int o = threadIdx.x + k * 256;
      if (o < IPC) {
        int a, bb, c = 0;
        if (DIM == 2) {
          a = o / M;
          bb = o % M;
        } else {
          a = o / (M * M);
          bb = (o / M) % M;
          c = o % M;
        }
        double s = acc[k];
        for (int pp = 0; pp < np; ++pp) {
          double v = sb[0][pp][a] * sb[1][pp][bb];
          s = DIM == 2 ? s + v : fma(v, sb[2][pp][c], s);
        }
        acc[k] = s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    int o = threadIdx.x + k * 256;
    if (o < IPC) psw[(size_t)L * IPC + o] += acc[k];
  }
}

// 3-D base_pots with register tiles: thread (a, b) of a group of M^2 threads
// keeps W[a][b][0..M-1]; G groups take every G-th point of a chunk and their
// partial sums are added at the end. Per point a thread reads Lx_a q, Ly_b and
// the M values Lz_c (shared-memory broadcasts) for M + 1 FP64 operations.
template <int M>
__global__ void __launch_bounds__(256) k_leaf_moments3(const int* leaves, const int* leaf_begin, const int* point_count,
                                                       const double4* pts, const double* nodes_interp, double* psw) {
  constexpr int IPC = M * M * M;
  constexpr int PCH = 32;
  constexpr int G = 256 / (M * M) > 0 ? 256 / (M * M) : 1;
  constexpr int RED_ROWS = G > 1 ? G - 1 : 1;
  constexpr int RED_COLS = G > 1 ? IPC : 1;
  __shared__ double sb[3][PCH][M];
  __shared__ double snode[3][kMaxNodes];
  __shared__ double red[RED_ROWS][RED_COLS];
  const int L = leaves[blockIdx.x];
  const int b = leaf_begin[L], cnt = point_count[L];
  const int t = threadIdx.x;
  const int grp = t / (M * M), ab = t % (M * M);
  const bool active = grp < G;
  const int a = ab / M, bb = ab % M;
  if (t < 3 * kMaxNodes) snode[t / kMaxNodes][t % kMaxNodes] = nodes_interp[(size_t)L * kPanelNodes + t];
  double acc[M];
#pragma unroll
  for (int c = 0; c < M; ++c) acc[c] = 0.0;
  __syncthreads();
  for (int p0 = 0; p0 < cnt; p0 += PCH) {
    if (t < PCH * 3) {
      const int pp = t / 3, d = t % 3;
      if (p0 + pp < cnt) {
        const double4 pt = pts[b + p0 + pp];
        const double x = d == 0 ? pt.x : (d == 1 ? pt.y : pt.z);
        double Lv[M];
        bary_basis<M>(Lv, x, snode[d]);
        // the charge is folded into the x factor (changes only the last bit
        // against the reference's product order, upward_pass_impl.hpp:164)
#pragma unroll
        for (int i = 0; i < M; ++i) sb[d][pp][i] = d == 0 ? Lv[i] * pt.w : Lv[i];
      } else {
#pragma unroll
        for (int i = 0; i < M; ++i) sb[d][pp][i] = 0.0;
      }
    }
    __syncthreads();
    if (active) {
      const int np = min(PCH, cnt - p0);
      for (int pp = grp; pp < np; pp += G) {
        const double v = sb[0][pp][a] * sb[1][pp][bb];
#pragma unroll
        for (int c = 0; c < M; ++c) acc[c] = fma(v, sb[2][pp][c], acc[c]);
      }
    }
    __syncthreads();
  }
  if (G > 1 && active && grp > 0) {
#pragma unroll
    for (int c = 0; c < M; ++c) red[grp - 1][ab * M + c] = acc[c];
  }
  __syncthreads();
  if (active && grp == 0) {
#pragma unroll
    for (int c = 0; c < M; ++c) {
      double v = acc[c];
      for (int g = 1; g < G; ++g) v += red[g - 1][ab * M + c];
      psw[(size_t)L * IPC + ab * M + c] += v;
    }
  }
}

// Applies one 1-D factor along axis `ax` of a tensor in tensor order:
// out[..i..] = sum_j A(i, j) in[..j..], A(i,j) = T ? X[j][i] : X[i][j].
template <int DIM, int M, int AX, bool T>
__device__ __forceinline__ void apply_axis(const double* in, double* out, const double* X) {
  constexpr int IPC = ipow_c<M, DIM>();
  constexpr int STR = (DIM == 2) ? (AX == 0 ? M : 1) : (AX == 0 ? M * M : (AX == 1 ? M : 1));
  for (int o = threadIdx.x; o < IPC; o += blockDim.x) {
    int i = (o / STR) % M;
    int base = o - i * STR;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < M; ++j) {
      double a = T ? X[j * kMaxNodes + i] : X[i * kMaxNodes + j];
      s = fma(a, in[base + j * STR], s);
    }
    out[o] = s;
  }
}

// child_to_parent (src/upward_pass_impl.hpp:134-188): one block per parent,
// W_parent[a,b,c] += sum_children sum_{i,j,k} X[i][a] Y[j][b] Z[k][c] W_child[i,j,k].
template <int DIM, int M>
__global__ void __launch_bounds__(256) k_c2p(const int* parents, const int* child, const double* xfer, double* psw) {
  constexpr int IPC = ipow_c<M, DIM>();
  constexpr int NCH = 1 << DIM;
  extern __shared__ double c2p_smem[];  // bufA, bufB, acc [IPC] each, then sX
  double* bufA = c2p_smem;
  double* bufB = bufA + IPC;
  double* acc = bufB + IPC;
  double* sX = acc + IPC;
  const int p = parents[blockIdx.x];
  for (int o = threadIdx.x; o < IPC; o += blockDim.x) acc[o] = 0.0;
  for (int ch = 0; ch < NCH; ++ch) {
    const int c = child[(size_t)p * NCH + ch];
    __syncthreads();
    for (int o = threadIdx.x; o < IPC; o += blockDim.x) bufA[o] = psw[(size_t)c * IPC + o];
    for (int o = threadIdx.x; o < DIM * kMaxNodes * kMaxNodes; o += blockDim.x)
      sX[o] = xfer[(size_t)c * kPanelXfer + o];
    __syncthreads();
    apply_axis<DIM, M, 0, true>(bufA, bufB, sX);
    __syncthreads();
    if (DIM == 2) {
      apply_axis<DIM, M, 1, true>(bufB, bufA, sX + kMaxNodes * kMaxNodes);
      __syncthreads();
      for (int o = threadIdx.x; o < IPC; o += blockDim.x) acc[o] += bufA[o];
    } else {
      apply_axis<DIM, M, 1, true>(bufB, bufA, sX + kMaxNodes * kMaxNodes);
      __syncthreads();
      apply_axis<DIM, M, 2, true>(bufA, bufB, sX + 2 * kMaxNodes * kMaxNodes);
      __syncthreads();
      for (int o = threadIdx.x; o < IPC; o += blockDim.x) acc[o] += bufB[o];
    }
  }
  __syncthreads();
  for (int o = threadIdx.x; o < IPC; o += blockDim.x) psw[(size_t)p * IPC + o] += acc[o];
}

// Source proxies as point sources: {node_x[a], node_y[b], node_z[c], W[k]}.
template <int DIM, int M>
__global__ void k_src_proxies(const int* cluster_panels, const double* nodes_shift, const double* psw, double4* out) {
  constexpr int IPC = ipow_c<M, DIM>();
  const int P = cluster_panels[blockIdx.x];
  const double* nd = nodes_shift + (size_t)P * kPanelNodes;
  for (int k = threadIdx.x; k < IPC; k += blockDim.x) {
    int a, b, c = 0;
    if (DIM == 2) {
      a = k / M;
      b = k % M;
    } else {
      a = k / (M * M);
      b = (k / M) % M;
      c = k % M;
    }
    out[(size_t)blockIdx.x * IPC + k] =
        make_double4(nd[a], nd[kNodeStride + b], DIM == 3 ? nd[2 * kNodeStride + c] : 0.0, psw[(size_t)P * IPC + k]);
  }
}

template <int DIM, int M>
__global__ void k_tgt_proxies(const int* cluster_panels, const double* nodes_shift, double4* out, int* out_index) {
  constexpr int IPC = ipow_c<M, DIM>();
  const int P = cluster_panels[blockIdx.x];
  const double* nd = nodes_shift + (size_t)P * kPanelNodes;
  for (int k = threadIdx.x; k < IPC; k += blockDim.x) {
    int a, b, c = 0;
    if (DIM == 2) {
      a = k / M;
      b = k % M;
    } else {
      a = k / (M * M);
      b = (k / M) % M;
      c = k % M;
    }
    out[(size_t)blockIdx.x * IPC + k] =
        make_double4(nd[a], nd[kNodeStride + b], DIM == 3 ? nd[2 * kNodeStride + c] : 0.0, 0.0);
    out_index[(size_t)blockIdx.x * IPC + k] = P * IPC + k;
  }
}

// ---- downward pass ---------------------------------------------------------
// parent_to_child (src/downward_pass_impl.hpp:109-191): one block per child,
// Phi_child[i,j,k] += sum_{a,b,c} X[i][a] Y[j][b] Z[k][c] Phi_parent[a,b,c].
template <int DIM, int M>
__global__ void __launch_bounds__(256) k_p2c(int ncomp, const int* children, const int* parent_of, const double* xfer,
                                             Ptr4 ptw) {
  constexpr int IPC = ipow_c<M, DIM>();
  __shared__ double bufA[IPC], bufB[IPC];
  __shared__ double sX[3 * kMaxNodes * kMaxNodes];
  const int c = children[blockIdx.x];
  const int p = parent_of[c];
  for (int o = threadIdx.x; o < DIM * kMaxNodes * kMaxNodes; o += blockDim.x) sX[o] = xfer[(size_t)c * kPanelXfer + o];
  for (int comp = 0; comp < ncomp; ++comp) {
    double* W = ptw.p[comp];
    __syncthreads();
    for (int o = threadIdx.x; o < IPC; o += blockDim.x) bufA[o] = W[(size_t)p * IPC + o];
    __syncthreads();
    apply_axis<DIM, M, 0, false>(bufA, bufB, sX);
    __syncthreads();
    if (DIM == 2) {
      apply_axis<DIM, M, 1, false>(bufB, bufA, sX + kMaxNodes * kMaxNodes);
      __syncthreads();
      for (int o = threadIdx.x; o < IPC; o += blockDim.x) W[(size_t)c * IPC + o] += bufA[o];
    } else {
      apply_axis<DIM, M, 1, false>(bufB, bufA, sX + kMaxNodes * kMaxNodes);
      __syncthreads();
      apply_axis<DIM, M, 2, false>(bufA, bufB, sX + 2 * kMaxNodes * kMaxNodes);
      __syncthreads();
      for (int o = threadIdx.x; o < IPC; o += blockDim.x) W[(size_t)c * IPC + o] += bufB[o];
    }
  }
}

// leaf_to_point (src/downward_pass_impl.hpp:193-237, 327-379) on every leaf:
// out[t] += sum_{a,b,c} Phi[a,b,c] Lx_a(x) Ly_b(y) Lz_c(z), one block per leaf.
template <int DIM, int M>
__global__ void __launch_bounds__(128) k_l2p(int ncomp, const int* leaves, const int* leaf_begin, const int* point_count,
                                             const double4* pts, const int* perm, const double* nodes_interp, Ptr4 ptw,
                                             Ptr4 out) {
  constexpr int IPC = ipow_c<M, DIM>();
  extern __shared__ double sP[];  // [ncomp][IPC]
  __shared__ double snode[3][kMaxNodes];
  const int L = leaves[blockIdx.x];
  const int b = leaf_begin[L], cnt = point_count[L];
  for (int comp = 0; comp < ncomp; ++comp)
    for (int o = threadIdx.x; o < IPC; o += blockDim.x) sP[comp * IPC + o] = ptw.p[comp][(size_t)L * IPC + o];
  if (threadIdx.x < 3 * kMaxNodes)
    snode[threadIdx.x / kMaxNodes][threadIdx.x % kMaxNodes] = nodes_interp[(size_t)L * kPanelNodes + threadIdx.x];
  __syncthreads();
  for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
    double4 pt = pts[b + j];
    double Lx[M], Ly[M], Lz[M];
    bary_basis<M>(Lx, pt.x, snode[0]);
    bary_basis<M>(Ly, pt.y, snode[1]);
    if (DIM == 3) bary_basis<M>(Lz, pt.z, snode[2]);
    const int orig = perm[b + j];
    for (int comp = 0; comp < ncomp; ++comp) {
      const double* P = sP + comp * IPC;
      double phi = 0.0;
#pragma unroll
      for (int a = 0; a < M; ++a) {
        double ta = 0.0;
#pragma unroll
        for (int bb = 0; bb < M; ++bb) {
          double v;
          if (DIM == 2) {
            v = P[a * M + bb];
          } else {
            v = 0.0;
#pragma unroll
            for (int c = 0; c < M; ++c) v = fma(P[(a * M + bb) * M + c], Lz[c], v);
          }
          ta = fma(Ly[bb], v, ta);
        }
        phi = fma(Lx[a], ta, phi);
      }
      out.p[comp][orig] += phi;
    }
  }
}

}  // namespace

#define BTK_DISPATCH_M(degree, ...)         \
  switch (degree) {                          \
    case 1: { constexpr int M = 2; __VA_ARGS__; } break;   \
    case 2: { constexpr int M = 3; __VA_ARGS__; } break;   \
    case 3: { constexpr int M = 4; __VA_ARGS__; } break;   \
    case 4: { constexpr int M = 5; __VA_ARGS__; } break;   \
    case 5: { constexpr int M = 6; __VA_ARGS__; } break;   \
    case 6: { constexpr int M = 7; __VA_ARGS__; } break;   \
    case 7: { constexpr int M = 8; __VA_ARGS__; } break;   \
    case 8: { constexpr int M = 9; __VA_ARGS__; } break;   \
    case 9: { constexpr int M = 10; __VA_ARGS__; } break;  \
    case 10: { constexpr int M = 11; __VA_ARGS__; } break; \
    case 11: { constexpr int M = 12; __VA_ARGS__; } break; \
    case 12: { constexpr int M = 13; __VA_ARGS__; } break; \
    default: return cudaErrorInvalidValue;   \
  }

static inline int blocks_for(long long n, int t) { return (int)((n + t - 1) / t); }

cudaError_t launch_panel_geometry(int dim, int degree, int P, const DevPanel* panels, const double* ucos_shift,
                                  const double* ucos_interp, double* nodes_shift, double* nodes_interp, double* xfer,
                                  cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  const int m = degree + 1;
  k_panel_nodes<<<blocks_for((long long)P * dim * m, 256), 256, 0, s>>>(dim, m, P, panels, ucos_shift, ucos_interp,
                                                                        nodes_shift, nodes_interp);
  count_launch();
  BTK_DISPATCH_M(degree, k_panel_xfer<M><<<blocks_for((long long)P * dim * M, 128), 128, 0, s>>>(
                             dim, P, panels, nodes_shift, nodes_interp, xfer));
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_perm_from_inside(int n_leaves, const int* leaves, const int* leaf_begin, const int* point_count,
                                    const int* inside, int thresh, int* perm, cudaStream_t s) {
  if (n_leaves <= 0) return cudaSuccess;
  k_perm_from_inside<<<n_leaves, 128, 0, s>>>(leaves, leaf_begin, point_count, inside, thresh, perm);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_gather(int n, const int* perm, const double* x, const double* y, const double* z,
                          const double* w, double4* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_gather<<<blocks_for(n, 256), 256, 0, s>>>(n, perm, x, y, z, w, out);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_leaf_moments(int dim, int degree, int n_leaves, const int* leaves, const int* leaf_begin,
                                const int* point_count, const double4* pts, const double* nodes_interp, double* psw,
                                cudaStream_t s) {
  if (n_leaves <= 0) return cudaSuccess;
  if (dim == 2) {
    BTK_DISPATCH_M(degree, k_leaf_moments<2, M><<<n_leaves, 256, 0, s>>>(leaves, leaf_begin, point_count, pts,
                                                                         nodes_interp, psw));
  } else {
    BTK_DISPATCH_M(degree, k_leaf_moments3<M><<<n_leaves, 256, 0, s>>>(leaves, leaf_begin, point_count, pts,
                                                                       nodes_interp, psw));
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_c2p(int dim, int degree, int n_parents, const int* parents, const int* child, const double* xfer,
                       double* psw, cudaStream_t s) {
  if (n_parents <= 0) return cudaSuccess;
  const int m = degree + 1;
  const int ipc = dim == 2 ? m * m : m * m * m;
  const size_t shm = sizeof(double) * (3 * ipc + 3 * kMaxNodes * kMaxNodes);
  if (dim == 2) {
    BTK_DISPATCH_M(degree, {
      cudaFuncSetAttribute(k_c2p<2, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
      k_c2p<2, M><<<n_parents, 256, shm, s>>>(parents, child, xfer, psw);
    });
  } else {
    BTK_DISPATCH_M(degree, {
      cudaFuncSetAttribute(k_c2p<3, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
      k_c2p<3, M><<<n_parents, 256, shm, s>>>(parents, child, xfer, psw);
    });
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_src_proxies(int dim, int degree, int n_clusters, const int* cluster_panels,
                               const double* nodes_shift, const double* psw, double4* out, cudaStream_t s) {
  if (n_clusters <= 0) return cudaSuccess;
  if (dim == 2) {
    BTK_DISPATCH_M(degree, k_src_proxies<2, M><<<n_clusters, 256, 0, s>>>(cluster_panels, nodes_shift, psw, out));
  } else {
    BTK_DISPATCH_M(degree, k_src_proxies<3, M><<<n_clusters, 256, 0, s>>>(cluster_panels, nodes_shift, psw, out));
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_tgt_proxies(int dim, int degree, int n_clusters, const int* cluster_panels,
                               const double* nodes_shift, double4* out, int* out_index, cudaStream_t s) {
  if (n_clusters <= 0) return cudaSuccess;
  if (dim == 2) {
    BTK_DISPATCH_M(degree, k_tgt_proxies<2, M><<<n_clusters, 256, 0, s>>>(cluster_panels, nodes_shift, out, out_index));
  } else {
    BTK_DISPATCH_M(degree, k_tgt_proxies<3, M><<<n_clusters, 256, 0, s>>>(cluster_panels, nodes_shift, out, out_index));
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_p2c(int dim, int degree, int ncomp, int n_children, const int* children, const int* parent_of,
                       const double* xfer, Ptr4 ptw, int /*ptw_stride*/, cudaStream_t s) {
  if (n_children <= 0) return cudaSuccess;
  if (dim == 2) {
    BTK_DISPATCH_M(degree, k_p2c<2, M><<<n_children, 256, 0, s>>>(ncomp, children, parent_of, xfer, ptw));
  } else {
    BTK_DISPATCH_M(degree, k_p2c<3, M><<<n_children, 256, 0, s>>>(ncomp, children, parent_of, xfer, ptw));
  }
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_l2p(int dim, int degree, int ncomp, int n_leaves, const int* leaves, const int* leaf_begin,
                       const int* point_count, const double4* pts, const int* perm, const double* nodes_interp,
                       Ptr4 ptw, Ptr4 out, cudaStream_t s) {
  if (n_leaves <= 0) return cudaSuccess;
  const int m = degree + 1;
  const int ipc = dim == 2 ? m * m : m * m * m;
  const size_t shm = sizeof(double) * ncomp * ipc;
  if (dim == 2) {
    BTK_DISPATCH_M(degree, {
      cudaFuncSetAttribute(k_l2p<2, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
      k_l2p<2, M><<<n_leaves, 128, shm, s>>>(ncomp, leaves, leaf_begin, point_count, pts, perm, nodes_interp, ptw, out);
    });
  } else {
    BTK_DISPATCH_M(degree, {
      cudaFuncSetAttribute(k_l2p<3, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
      k_l2p<3, M><<<n_leaves, 128, shm, s>>>(ncomp, leaves, leaf_begin, point_count, pts, perm, nodes_interp, ptw, out);
    });
  }
  count_launch();
  return cudaGetLastError();
}

}  // namespace btk
