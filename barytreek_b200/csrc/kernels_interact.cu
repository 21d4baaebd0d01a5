// The interaction phase: PP, PC, CP and CC (src/fmm_interactions/poisson_fmm_impl.hpp,
// poisson_vel_fmm_impl.hpp) as one persistent, gather-shaped kernel.
//
// Every interaction class is "targets x sources" once proxy points are treated
// as points: PP = leaf points x leaf points, PC = leaf points x cluster proxies
// (weights = modified charges), CP = cluster proxies x leaf points, CC =
// proxies x proxies. The host groups the pairs by target panel, cuts each
// target panel into tiles of kTile targets, and lists each tile's sources as
// entries (contiguous ranges of the S4 array). Work items are sorted by cost,
// largest first, and a persistent grid pulls them from a ticket counter
// (longest-processing-time-first scheduling).
//
// Per item, thread 0 streams the item's sources through a STAGES-deep ring of
// shared-memory chunks with TMA bulk copies (cp.async.bulk, completion on an
// mbarrier); all 128 threads evaluate their 2 targets against every source of a
// chunk (broadcast shared-memory reads) and keep the sums in registers. Each
// target's sum is written once at the end of its item, so results need no
// atomics unless the host split a long source list (kItemAtomic).
#include "device_math.cuh"
#include "kernels.cuh"

namespace btk {

namespace {

constexpr int kChunk = 256;     // sources per shared-memory chunk (8 KB of double4)
constexpr int kStages = 3;      // ring depth
constexpr uint32_t kWaitLimit = 1u << 22;  // polls of try_wait before giving up

template <int DIM, int KIND>
struct KernelTraits {
  // components: POT 1, VEL 3, FIELD 1 + DIM
  static constexpr int NC = KIND == BTK_KIND_POT ? 1 : (KIND == BTK_KIND_VEL ? 3 : 1 + DIM);
};

// One source against one target, FP64. Sums are kept without the kernel's
// constant factor (applied once per target at the end):
//   POT  3-D: sum w / R            2-D: sum w log(R^2)
//   VEL  3-D: sum w (t-s) / R^2
//   FIELD 3-D: sum w / R, sum w (t-s) / R^3;  2-D: sum w log R^2, sum w (t-s)/R^2
// with R^2 = |t-s|^2 + eps^2.
template <int DIM, int KIND, bool GUARD>
__device__ __forceinline__ void eval_fp64(double tx, double ty, double tz, const double4& s, double eps2,
                                          double* acc) {
  const double dx = tx - s.x, dy = ty - s.y;
  if (DIM == 2) {
    const double r2 = fma(dx, dx, fma(dy, dy, eps2));
    acc[0] = fma(s.w, log(r2), acc[0]);
    if (KIND == BTK_KIND_FIELD) {
      const double g = s.w * (GUARD ? rcp_fp64_pos_guarded(r2) : rcp_fp64_pos(r2));
      acc[1] = fma(dx, g, acc[1]);
      acc[2] = fma(dy, g, acc[2]);
    }
  } else {
    const double dz = tz - s.z;
    const double r2 = fma(dx, dx, fma(dy, dy, fma(dz, dz, eps2)));
    if (KIND == BTK_KIND_VEL) {
      const double g = s.w * (GUARD ? rcp_fp64_pos_guarded(r2) : rcp_fp64_pos(r2));
      acc[0] = fma(dx, g, acc[0]);
      acc[1] = fma(dy, g, acc[1]);
      acc[2] = fma(dz, g, acc[2]);
    } else {
      const double ri = GUARD ? rsqrt_fp64_guarded(r2) : rsqrt_fp64(r2);
      if (KIND == BTK_KIND_POT) {
        acc[0] = fma(s.w, ri, acc[0]);
      } else {
        const double wr = s.w * ri;
        acc[0] += wr;
        const double g = wr * (ri * ri);
        acc[1] = fma(dx, g, acc[1]);
        acc[2] = fma(dy, g, acc[2]);
        acc[3] = fma(dz, g, acc[3]);
      }
    }
  }
}

template <int DIM, int KIND, bool GUARD>
__global__ void __launch_bounds__(kInteractThreads, 4) k_interact_fp64(InteractParams p) {
  constexpr int NC = KernelTraits<DIM, KIND>::NC;
  constexpr int TPT = kTargetsPerThread;
  __shared__ __align__(128) double4 sbuf[kStages][kChunk];
  __shared__ __align__(8) uint64_t bars[kStages];
  __shared__ int s_item, s_abort;
  __shared__ uint32_t s_fail_chunk;

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    s_abort = 0;
  }
  __syncthreads();

  uint32_t g = 0;  // chunks this block has consumed so far (uniform)
  // Producer cursor (meaningful in thread 0 only).
  int pe = 0, poff = 0;
  uint32_t issued = 0;  // global chunk index of the next issue (thread 0)

  while (true) {
    __syncthreads();  // every thread has read the previous ticket
    if (tid == 0) s_item = atomicAdd(p.ticket, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= p.n_items || s_abort) break;
    const WorkItem w = p.items[it];
    if (w.t_count <= 0 || w.s_total <= 0) continue;  // unused tile of a per-pair-degree item block
    const int n_chunks = (w.s_total + kChunk - 1) / kChunk;

    auto issue = [&](int c) {  // thread 0 only: fill chunk c of this item
      const int stage = (g + c) % kStages;
      const int need = min(kChunk, w.s_total - c * kChunk);
      mbar_arrive_expect_tx(&bars[stage], (uint32_t)need * sizeof(double4));
      int filled = 0;
      while (filled < need) {
        const Entry e = p.entries[pe];
        const int take = min(need - filled, e.s_count - poff);
        bulk_copy_g2s(&sbuf[stage][filled], p.S4 + e.s_begin + poff, (uint32_t)take * sizeof(double4), &bars[stage]);
        filled += take;
        poff += take;
        if (poff == e.s_count) {
          ++pe;
          poff = 0;
        }
      }
      ++issued;
    };
    if (tid == 0) {
      pe = w.e_begin;
      poff = 0;
      for (int c = 0; c < min(kStages, n_chunks); ++c) issue(c);
    }

    double tx[TPT], ty[TPT], tz[TPT], acc[TPT][NC];
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int i = min(tid + u * kInteractThreads, w.t_count - 1);
      const double4 t = p.T4[w.t_begin + i];
      tx[u] = t.x;
      ty[u] = t.y;
      tz[u] = t.z;
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[u][c] = 0.0;
    }

    for (int c = 0; c < n_chunks; ++c) {
      const int stage = (g + c) % kStages;
      const uint32_t parity = ((g + c) / kStages) & 1u;
      if (!mbar_wait_bounded(&bars[stage], parity, kWaitLimit)) {
        s_abort = 1;
        s_fail_chunk = g + c;
        atomicCAS(p.status, 0, (int)BTK_ERR_DEVICE_TIMEOUT);
      }
      __syncthreads();
      if (s_abort) break;
      const int cnt = min(kChunk, w.s_total - c * kChunk);
      const double4* sb = sbuf[stage];
#pragma unroll 2
      for (int j = 0; j < cnt; ++j) {
        const double4 s = sb[j];
#pragma unroll
        for (int u = 0; u < TPT; ++u) eval_fp64<DIM, KIND, GUARD>(tx[u], ty[u], tz[u], s, p.eps2, acc[u]);
      }
      __syncthreads();
      if (tid == 0 && c + kStages < n_chunks) issue(c + kStages);
    }
    if (s_abort) break;
    g += n_chunks;

#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int i = tid + u * kInteractThreads;
      if (i < w.t_count) {
        const int idx = p.T_out[w.t_begin + i];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double* dst = ((w.flags & kItemProxyTargets) ? p.ptw[c] : p.out[c]) + idx;
          const double v = acc[u][c] * p.scale[c];
          if (w.flags & kItemAtomic)
            atomicAdd(dst, v);
          else
            *dst += v;
        }
      }
    }
  }

  // On a timed-out wait, drain (bounded) whatever copies thread 0 still has in
  // flight before the block's shared memory is released.
  if (s_abort && tid == 0) {
    for (uint32_t k = s_fail_chunk; k < issued; ++k)
      mbar_wait_bounded(&bars[k % kStages], (k / kStages) & 1u, kWaitLimit);
  }
}

// ---------------------------------------------------------------------------
// Mixed precision: the same pipeline, but every chunk of FP64 sources is
// rewritten in shared memory as FP32 coordinates relative to the item's FP64
// target-panel centre (one FP64 subtraction per source per item), and the
// pairwise arithmetic runs in FP32 with the MUFU approximations. Per target,
// FP32 partial sums over kFold sources are folded into an FP64 accumulator
// with a compensated (two-sum) addition, so the final per-target sum carries
// FP64 precision; the constant factor is applied in FP64 at the end.
// ---------------------------------------------------------------------------
constexpr int kFold = 128;

// NEAR: coordinates carry an FP32 low part (x = hi + lo, both relative to the
// item's centre), and the difference is formed as (t_hi - s_hi) + (t_lo - s_lo)
// so near-field pairs (PP) keep their separation to ~1e-14 relative to the
// centre distance, not FP32's 6e-8.
template <int DIM, int KIND, bool NEAR>
__device__ __forceinline__ void eval_fp32(float tx, float ty, float tz, float lx, float ly, float lz, const float4& s,
                                          const float4& sl, float eps2, float* acc) {
  const float dx = NEAR ? (tx - s.x) + (lx - sl.x) : tx - s.x;
  const float dy = NEAR ? (ty - s.y) + (ly - sl.y) : ty - s.y;
  if (DIM == 2) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, eps2));
    acc[0] = fmaf(s.w, __logf(r2), acc[0]);
    if (KIND == BTK_KIND_FIELD) {
      const float g = s.w * rcp_fp32(r2);
      acc[1] = fmaf(dx, g, acc[1]);
      acc[2] = fmaf(dy, g, acc[2]);
    }
  } else {
    const float dz = NEAR ? (tz - s.z) + (lz - sl.z) : tz - s.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
    if (KIND == BTK_KIND_VEL) {
      const float g = s.w * rcp_fp32(r2);
      acc[0] = fmaf(dx, g, acc[0]);
      acc[1] = fmaf(dy, g, acc[1]);
      acc[2] = fmaf(dz, g, acc[2]);
    } else {
      const float ri = rsqrt_fp32(r2);
      if (KIND == BTK_KIND_POT) {
        acc[0] = fmaf(s.w, ri, acc[0]);
      } else {
        const float wr = s.w * ri;
        acc[0] += wr;
        const float g = wr * (ri * ri);
        acc[1] = fmaf(dx, g, acc[1]);
        acc[2] = fmaf(dy, g, acc[2]);
        acc[3] = fmaf(dz, g, acc[3]);
      }
    }
  }
}

// x - c split into FP32 hi + lo (hi = x - c rounded, lo = the FP32-rounded rest).
__device__ __forceinline__ void split_rel(double x, double c, float& hi, float& lo) {
  const double r = x - c;
  hi = (float)r;
  lo = (float)(r - (double)hi);
}

// Knuth's two-sum: s + e == a + b exactly; the error term is kept in `comp`.
__device__ __forceinline__ void two_sum_add(double& sum, double& comp, double b) {
  const double s = sum + b;
  const double bp = s - sum;
  const double e = (sum - (s - bp)) + (b - bp);
  sum = s;
  comp += e;
}

template <int DIM, int KIND>
__global__ void __launch_bounds__(kInteractThreads, 6) k_interact_mixed(InteractParams p) {
  constexpr int NC = KernelTraits<DIM, KIND>::NC;
  constexpr int TPT = kTargetsPerThread;
  __shared__ __align__(128) double4 sbuf[kStages][kChunk];
  __shared__ __align__(16) float4 fbuf[kChunk], fbuf_lo[kChunk];
  __shared__ __align__(8) uint64_t bars[kStages];
  __shared__ int s_item, s_abort;
  __shared__ uint32_t s_fail_chunk;

  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    s_abort = 0;
  }
  __syncthreads();
  const float eps2 = (float)p.eps2;

  uint32_t g = 0;
  int pe = 0, poff = 0;
  uint32_t issued = 0;

  while (true) {
    __syncthreads();  // every thread has read the previous ticket
    if (tid == 0) s_item = atomicAdd(p.ticket, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= p.n_items || s_abort) break;
    const WorkItem w = p.items[it];
    if (w.t_count <= 0 || w.s_total <= 0) continue;  // unused tile of a per-pair-degree item block
    const int n_chunks = (w.s_total + kChunk - 1) / kChunk;

    auto issue = [&](int c) {
      const int stage = (g + c) % kStages;
      const int need = min(kChunk, w.s_total - c * kChunk);
      mbar_arrive_expect_tx(&bars[stage], (uint32_t)need * sizeof(double4));
      int filled = 0;
      while (filled < need) {
        const Entry e = p.entries[pe];
        const int take = min(need - filled, e.s_count - poff);
        bulk_copy_g2s(&sbuf[stage][filled], p.S4 + e.s_begin + poff, (uint32_t)take * sizeof(double4), &bars[stage]);
        filled += take;
        poff += take;
        if (poff == e.s_count) {
          ++pe;
          poff = 0;
        }
      }
      ++issued;
    };
    if (tid == 0) {
      pe = w.e_begin;
      poff = 0;
      for (int c = 0; c < min(kStages, n_chunks); ++c) issue(c);
    }

    float tx[TPT], ty[TPT], tz[TPT], lx[TPT], ly[TPT], lz[TPT];
    double acc[TPT][NC], comp[TPT][NC];
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int i = min(tid + u * kInteractThreads, w.t_count - 1);
      const double4 t = p.T4[w.t_begin + i];
      split_rel(t.x, w.cx, tx[u], lx[u]);
      split_rel(t.y, w.cy, ty[u], ly[u]);
      split_rel(t.z, w.cz, tz[u], lz[u]);
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[u][c] = comp[u][c] = 0.0;
    }

    for (int c = 0; c < n_chunks; ++c) {
      const int stage = (g + c) % kStages;
      const uint32_t parity = ((g + c) / kStages) & 1u;
      if (!mbar_wait_bounded(&bars[stage], parity, kWaitLimit)) {
        s_abort = 1;
        s_fail_chunk = g + c;
        atomicCAS(p.status, 0, (int)BTK_ERR_DEVICE_TIMEOUT);
      }
      __syncthreads();
      if (s_abort) break;
      const int cnt = min(kChunk, w.s_total - c * kChunk);
      const int near_end = min(cnt, max(0, w.near_total - c * kChunk));  // near sources of this chunk
      for (int j = tid; j < cnt; j += kInteractThreads) {
        const double4 s = sbuf[stage][j];
        float4 h, l;
        split_rel(s.x, w.cx, h.x, l.x);
        split_rel(s.y, w.cy, h.y, l.y);
        split_rel(s.z, w.cz, h.z, l.z);
        h.w = (float)s.w;
        l.w = 0.f;
        fbuf[j] = h;
        fbuf_lo[j] = l;
      }
      __syncthreads();
      // The FP64 stage is free again: refill it while this chunk is evaluated.
      if (tid == 0 && c + kStages < n_chunks) issue(c + kStages);
      for (int f0 = 0; f0 < cnt; f0 += kFold) {
        const int f1 = min(cnt, f0 + kFold);
        float part[TPT][NC];
#pragma unroll
        for (int u = 0; u < TPT; ++u)
#pragma unroll
          for (int k = 0; k < NC; ++k) part[u][k] = 0.f;
        const int fn = min(f1, max(f0, near_end));
#pragma unroll 2
        for (int j = f0; j < fn; ++j) {
          const float4 s = fbuf[j], sl = fbuf_lo[j];
#pragma unroll
          for (int u = 0; u < TPT; ++u)
            eval_fp32<DIM, KIND, true>(tx[u], ty[u], tz[u], lx[u], ly[u], lz[u], s, sl, eps2, part[u]);
        }
#pragma unroll 4
        for (int j = fn; j < f1; ++j) {
          const float4 s = fbuf[j];
#pragma unroll
          for (int u = 0; u < TPT; ++u)
            eval_fp32<DIM, KIND, false>(tx[u], ty[u], tz[u], lx[u], ly[u], lz[u], s, s, eps2, part[u]);
        }
#pragma unroll
        for (int u = 0; u < TPT; ++u)
#pragma unroll
          for (int k = 0; k < NC; ++k) two_sum_add(acc[u][k], comp[u][k], (double)part[u][k]);
      }
      __syncthreads();
    }
    if (s_abort) break;
    g += n_chunks;

#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int i = tid + u * kInteractThreads;
      if (i < w.t_count) {
        const int idx = p.T_out[w.t_begin + i];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double* dst = ((w.flags & kItemProxyTargets) ? p.ptw[c] : p.out[c]) + idx;
          const double v = (acc[u][c] + comp[u][c]) * p.scale[c];
          if (w.flags & kItemAtomic)
            atomicAdd(dst, v);
          else
            *dst += v;
        }
      }
    }
  }
  if (s_abort && tid == 0) {
    for (uint32_t k = s_fail_chunk; k < issued; ++k)
      mbar_wait_bounded(&bars[k % kStages], (k / kStages) & 1u, kWaitLimit);
  }
}

template <int DIM, int KIND, bool GUARD>
cudaError_t launch_mixed(const InteractParams& p, int grid, cudaStream_t s) {
  k_interact_mixed<DIM, KIND><<<grid, kInteractThreads, 0, s>>>(p);
  return cudaGetLastError();
}

template <int DIM, int KIND, bool GUARD>
int occupancy_mixed() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_interact_mixed<DIM, KIND>, kInteractThreads, 0);
  return n;
}

template <int DIM, int KIND, bool GUARD>
cudaError_t launch_fp64(const InteractParams& p, int grid, cudaStream_t s) {
  k_interact_fp64<DIM, KIND, GUARD><<<grid, kInteractThreads, 0, s>>>(p);
  return cudaGetLastError();
}

template <int DIM, int KIND, bool GUARD>
int occupancy_fp64() {
  int n = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_interact_fp64<DIM, KIND, GUARD>, kInteractThreads, 0);
  return n;
}

}  // namespace

#define BTK_KIND_SWITCH(dim, kind, guard, F, ...)                                   \
  do {                                                                              \
    if (dim == 2) {                                                                 \
      if (kind == BTK_KIND_POT) return guard ? F<2, BTK_KIND_POT, true>(__VA_ARGS__) \
                                             : F<2, BTK_KIND_POT, false>(__VA_ARGS__); \
      if (kind == BTK_KIND_FIELD) return guard ? F<2, BTK_KIND_FIELD, true>(__VA_ARGS__) \
                                               : F<2, BTK_KIND_FIELD, false>(__VA_ARGS__); \
    } else {                                                                        \
      if (kind == BTK_KIND_POT) return guard ? F<3, BTK_KIND_POT, true>(__VA_ARGS__) \
                                             : F<3, BTK_KIND_POT, false>(__VA_ARGS__); \
      if (kind == BTK_KIND_VEL) return guard ? F<3, BTK_KIND_VEL, true>(__VA_ARGS__) \
                                             : F<3, BTK_KIND_VEL, false>(__VA_ARGS__); \
      if (kind == BTK_KIND_FIELD) return guard ? F<3, BTK_KIND_FIELD, true>(__VA_ARGS__) \
                                               : F<3, BTK_KIND_FIELD, false>(__VA_ARGS__); \
    }                                                                               \
  } while (0)

cudaError_t launch_interact(int dim, int kind, int precision, bool guard, const InteractParams& p, int grid,
                            cudaStream_t s) {
  if (p.n_items <= 0) return cudaSuccess;
  count_launch();
  if (precision == BTK_PREC_FP64) BTK_KIND_SWITCH(dim, kind, guard, launch_fp64, p, grid, s);
  if (precision == BTK_PREC_MIXED) BTK_KIND_SWITCH(dim, kind, false, launch_mixed, p, grid, s);
  return cudaErrorInvalidValue;
}

int interact_blocks_per_sm(int dim, int kind, int precision, bool guard) {
  if (precision == BTK_PREC_FP64) BTK_KIND_SWITCH(dim, kind, guard, occupancy_fp64);
  if (precision == BTK_PREC_MIXED) BTK_KIND_SWITCH(dim, kind, false, occupancy_mixed);
  return 0;
}

}  // namespace btk
