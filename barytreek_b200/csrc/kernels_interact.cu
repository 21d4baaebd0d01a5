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
// chunk (broadcast shared-memory reads) and keep the sums in registers. One
// block barrier per chunk. Warp w
// owns targets 32 w + lane and 32 w + THREADS + lane of a tile (a partly
// filled tile spreads over all warps first); warps whose targets lie past the
// tile's count skip the arithmetic. Each
// target's sum is written once at the end of its item, so results need no
// atomics unless the host split a long source list (kItemAtomic).
#include "device_math.cuh"
#include "kernels.cuh"

namespace btk {

namespace {

constexpr int kChunk = 256;     // sources per shared-memory chunk (8 KB of double4)
constexpr int kStages = 3;      // ring depth

// Next work item of a block (thread 0 only): from its own queue, else from
// the other one; -1 when both are empty. audit: the block's current queue.
__device__ __forceinline__ int next_item(const InteractParams& p, bool& audit, bool& moved) {
  for (;;) {
    if (audit) {
      const int t = p.n_audit_items > 0 ? atomicAdd(p.audit_ticket, 1) : p.n_audit_items;
      if (t < p.n_audit_items) return p.n_items + t;
    } else {
      const int t = atomicAdd(p.ticket, 1);
      if (t < p.n_items) return t;
    }
    if (moved) return -1;
    moved = true;
    audit = !audit;
  }
}

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

// THREADS = 128 (tiles of 256 targets) or 64 (tiles of 128): blocks of
// THREADS / 32 warps, 6 * 128 / THREADS blocks per SM (at most 85 registers;
// measured 143.7 -> 139.3 ms on the 1M potential + gradient solve against 4
// blocks per SM, no spills).
template <int DIM, int KIND, bool GUARD, int THREADS>
__global__ void __launch_bounds__(THREADS, 768 / THREADS) k_interact_fp64(InteractParams p) {
  constexpr int NC = KernelTraits<DIM, KIND>::NC;
  constexpr int TPT = kTargetsPerThread;
  static_assert(TPT == 2, "targets of warp w are 32 w + lane and 32 w + THREADS + lane");
  __shared__ __align__(128) double4 sbuf[kStages][kChunk];
  __shared__ __align__(8) uint64_t bars[kStages];
  __shared__ int s_item, s_abort;
  __shared__ uint32_t s_fail_chunk;

  const int tid = threadIdx.x;
  const int lane = tid & 31, tbase = (tid >> 5) * 32;
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

  bool audit_queue = (int)blockIdx.x < p.audit_blocks, moved = false;  // thread 0's queue state
  while (true) {
    __syncthreads();  // every thread has read the previous ticket
    if (tid == 0) s_item = next_item(p, audit_queue, moved);
    __syncthreads();
    const int it = s_item;
    if (it < 0 || s_abort) break;
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

    // This warp's targets: [tbase, tbase + 32) and [tbase + THREADS, tbase +
    // THREADS + 32) of the tile, nu of the two in use (warp-uniform). A tile
    // of up to THREADS targets gives every warp up to 32 of them, so a partly
    // filled tile keeps all of the block's warps busy: the warps of a block sit
    // on different SM sub-partitions, whose MUFU and FMA pipes are separate.
    const int nu = w.t_count > tbase + THREADS ? 2 : (w.t_count > tbase ? 1 : 0);
    double tx[TPT], ty[TPT], tz[TPT], acc[TPT][NC];
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int i = min(tbase + u * THREADS + lane, w.t_count - 1);
      const double4 t = ((w.flags & kItemAudit) ? p.T4a : p.T4)[w.t_begin + i];
      tx[u] = t.x;
      ty[u] = t.y;
      tz[u] = t.z;
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[u][c] = 0.0;
    }

    for (int c = 0; c < n_chunks; ++c) {
      const int stage = (g + c) % kStages;
      const uint32_t parity = ((g + c) / kStages) & 1u;
      if (!mbar_wait_bounded(&bars[stage], parity, p.wait_limit)) {
        s_abort = 1;
        s_fail_chunk = g + c;
        atomicCAS(p.status, 0, (int)BTK_ERR_DEVICE_TIMEOUT);
      }
      // One barrier per chunk: chunk c has landed for every thread, and every
      // thread has finished chunk c - 1, whose stage is refilled now.
      __syncthreads();
      if (s_abort) break;
      if (tid == 0 && c >= 1 && c - 1 + kStages < n_chunks) issue(c - 1 + kStages);
      const int cnt = min(kChunk, w.s_total - c * kChunk);
      const double4* sb = sbuf[stage];
      if (nu == 2) {
#pragma unroll 2
        for (int j = 0; j < cnt; ++j) {
          const double4 s = sb[j];
          eval_fp64<DIM, KIND, GUARD>(tx[0], ty[0], tz[0], s, p.eps2, acc[0]);
          eval_fp64<DIM, KIND, GUARD>(tx[1], ty[1], tz[1], s, p.eps2, acc[1]);
        }
      } else if (nu == 1) {
#pragma unroll 2
        for (int j = 0; j < cnt; ++j) eval_fp64<DIM, KIND, GUARD>(tx[0], ty[0], tz[0], sb[j], p.eps2, acc[0]);
      }
    }
    if (s_abort) break;
    g += n_chunks;

#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int i = tbase + u * THREADS + lane;
      if (i < w.t_count) {
        const bool audit = (w.flags & kItemAudit) != 0;
        const int idx = audit ? w.t_begin + i : p.T_out[w.t_begin + i];
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          double* dst = (audit ? p.aout[c] : (w.flags & kItemProxyTargets) ? p.ptw[c] : p.out[c]) + idx;
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
      mbar_wait_bounded(&bars[k % kStages], (k / kStages) & 1u, kDrainLimit);
  }
}

// ---------------------------------------------------------------------------
// Mixed precision: the same pipeline, but every chunk of FP64 sources is
// rewritten in shared memory as FP32 coordinates relative to the item's FP64
// target-panel centre (one FP64 subtraction per source per item), and the
// pairwise arithmetic runs in FP32 with the MUFU approximations. Sources are
// stored as PAIRS (even, odd) in packed float2 lanes, negated, so one sm_100
// f32x2 instruction (FADD2/FMUL2/FFMA2) evaluates a target against two
// sources: half the issue slots of scalar FP32 for the same work. Per target,
// FP32 partial sums over each 256-source chunk are folded into an FP64 accumulator
// with a compensated (two-sum) addition, so the final per-target sum carries
// FP64 precision; the constant factor is applied in FP64 at the end.
// ---------------------------------------------------------------------------
// Per block of THREADS threads: chunks of 2 * THREADS sources (one source
// pair converted per thread), folded into FP64 once per chunk.
// Padding source for an odd chunk: zero weight, placed 3e18 away (negated
// relative coordinate), so r^2 stays finite in FP32 and the term is exactly 0.
constexpr float kPadCoord = -3.0e18f;

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// One target, both lanes holding the same coordinate (hi relative to the
// item's centre, and its FP32 low part).
struct TargetPair {
  float2 x, y, z, lx, ly, lz;
};

// Target against a source pair. n* are the NEGATED source coordinates (hi and,
// for NEAR, lo). NEAR forms the difference as (t_hi - s_hi) + (t_lo - s_lo), so
// near-field pairs (touching PP sources) keep their separation to ~1e-14
// relative to the centre distance, not FP32's 6e-8.
template <int DIM, int KIND, bool NEAR>
__device__ __forceinline__ void eval_pair(const TargetPair& t, float2 nx, float2 ny, float2 nz, float2 w, float2 nlx,
                                          float2 nly, float2 nlz, float2 e2, float2* acc) {
  float2 dx = add2(t.x, nx), dy = add2(t.y, ny);
  if (NEAR) {
    dx = add2(dx, add2(t.lx, nlx));
    dy = add2(dy, add2(t.ly, nly));
  }
  if (DIM == 2) {
    const float2 r2 = fma2(dx, dx, fma2(dy, dy, e2));
    acc[0] = fma2(w, make_float2(__logf(r2.x), __logf(r2.y)), acc[0]);
    if (KIND == BTK_KIND_FIELD) {
      const float2 g = mul2(w, make_float2(rcp_fp32(r2.x), rcp_fp32(r2.y)));
      acc[1] = fma2(dx, g, acc[1]);
      acc[2] = fma2(dy, g, acc[2]);
    }
  } else {
    float2 dz = add2(t.z, nz);
    if (NEAR) dz = add2(dz, add2(t.lz, nlz));
    const float2 r2 = fma2(dx, dx, fma2(dy, dy, fma2(dz, dz, e2)));
    if (KIND == BTK_KIND_VEL) {
      const float2 g = mul2(w, make_float2(rcp_fp32(r2.x), rcp_fp32(r2.y)));
      acc[0] = fma2(dx, g, acc[0]);
      acc[1] = fma2(dy, g, acc[1]);
      acc[2] = fma2(dz, g, acc[2]);
    } else {
      const float2 ri = make_float2(rsqrt_fp32(r2.x), rsqrt_fp32(r2.y));
      if (KIND == BTK_KIND_POT) {
        acc[0] = fma2(w, ri, acc[0]);
      } else {
        const float2 wr = mul2(w, ri);
        acc[0] = add2(acc[0], wr);
        const float2 g = mul2(wr, mul2(ri, ri));
        acc[1] = fma2(dx, g, acc[1]);
        acc[2] = fma2(dy, g, acc[2]);
        acc[3] = fma2(dz, g, acc[3]);
      }
    }
  }
}

// Source pairs [j0, j1) of a converted chunk against NU targets.
template <int DIM, int KIND, bool NEAR, int NU, int NC>
__device__ __forceinline__ void pair_loop(const float4* fA, const float4* fB, const float4* fL, const float2* fLz,
                                          int j0, int j1, const TargetPair* T, float2 e2, float2 (*part)[NC]) {
  // Source pairs in flight per warp (measured, 128-thread blocks): one target
  // 4 (batch 269.3 -> 260.6 ms, learned 1M 40.9 -> 40.5 ms, 2M sphere vector
  // kernel 68.4 -> 67.8 ms, against 2); two targets 6 for potential +
  // gradient (1M mixed 60.6 -> 59.9 ms at 4, 59.6 ms at 6 or 8), 3 for the
  // potential (batch 260.6 -> 258.9 ms; 4 spills), 2 for the vector kernel
  // (its register budget at 5 blocks per SM). The FP64 kernel's one-target
  // loop measured slower at 4.
  constexpr int kUnroll =
      NU == 1 ? 4 : (KIND == BTK_KIND_FIELD ? 6 : (KIND == BTK_KIND_POT ? 3 : 2));
#pragma unroll kUnroll
  for (int j = j0; j < j1; ++j) {
    const float4 a = fA[j], b = fB[j];
    float4 l = make_float4(0.f, 0.f, 0.f, 0.f);
    float2 lz = make_float2(0.f, 0.f);
    if (NEAR) {
      l = fL[j];
      lz = fLz[j];
    }
#pragma unroll
    for (int u = 0; u < NU; ++u)
      eval_pair<DIM, KIND, NEAR>(T[u], make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y),
                                 make_float2(b.z, b.w), make_float2(l.x, l.y), make_float2(l.z, l.w), lz, e2, part[u]);
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

// Blocks per SM: potential + gradient 4 * 128 / THREADS (at most 128
// registers; at 5 blocks it spills); the vector kernel 5 * 128 / THREADS (96
// registers; 2M sphere learned solve 69.4 -> 68.3 ms against 4 blocks); the
// potential alone 7 * 128 / THREADS with a 2-stage ring (72 registers with a
// few bytes spilled, 30.8 KB of shared memory at 128 threads, so 7 blocks is
// also the shared-memory limit; measured on the 256-problem batch: 5 blocks
// with 3 stages 299 ms, 6 blocks 280 ms, 7 blocks 270 ms).
template <int DIM, int KIND, int THREADS, int STAGES = KIND == BTK_KIND_POT ? 2 : kStages,
          int MINB = KIND == BTK_KIND_POT ? 7 * 128 / THREADS : (KIND == BTK_KIND_VEL ? 5 : 4) * 128 / THREADS>
__global__ void __launch_bounds__(THREADS, MINB) k_interact_mixed(InteractParams p) {
  constexpr int NC = KernelTraits<DIM, KIND>::NC;
  constexpr int TPT = kTargetsPerThread;
  static_assert(TPT == 2, "targets of warp w are 32 w + lane and 32 w + THREADS + lane");
  constexpr int kChunk = 2 * THREADS;  // sources per chunk: one pair per thread
  constexpr int kPairs = THREADS;
  constexpr int kFoldPairs = kPairs;
  __shared__ __align__(128) double4 sbuf[STAGES][kChunk];
  // converted chunk, by source pair j = (2j, 2j+1): negated hi coordinates and
  // weights, negated lo coordinates
  // (double-buffered: chunk c is converted into buffer c & 1 while other warps
  // may still evaluate chunk c - 1 from the other buffer)
  __shared__ __align__(16) float4 fA[2][kPairs], fB[2][kPairs], fL[2][kPairs];
  __shared__ __align__(16) float2 fLz[2][kPairs];
  __shared__ __align__(8) uint64_t bars[STAGES];
  __shared__ int s_item, s_abort;
  __shared__ uint32_t s_fail_chunk;
  __shared__ int s_ncp[2][THREADS / 32];  // per warp region: pairs on the hi/lo path

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5, tbase = warp * 32;
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    s_abort = 0;
  }
  __syncthreads();
  const float2 e2 = make_float2((float)p.eps2, (float)p.eps2);

  uint32_t g = 0;
  int pe = 0, poff = 0;
  uint32_t issued = 0;

  bool audit_queue = (int)blockIdx.x < p.audit_blocks, moved = false;  // thread 0's queue state
  while (true) {
    __syncthreads();  // every thread has read the previous ticket
    if (tid == 0) s_item = next_item(p, audit_queue, moved);
    __syncthreads();
    const int it = s_item;
    if (it < 0 || s_abort) break;
    const WorkItem w = p.items[it];
    if (w.t_count <= 0 || w.s_total <= 0) continue;  // unused tile of a per-pair-degree item block
    const int n_chunks = (w.s_total + kChunk - 1) / kChunk;
    const float thr = fmaxf(w.hx, fmaxf(w.hy, w.hz));  // near sources at least this far from the box: FP32 path

    auto issue = [&](int c) {
      const int stage = (g + c) % STAGES;
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
      for (int c = 0; c < min(STAGES, n_chunks); ++c) issue(c);
    }

    // This warp's targets: [tbase, tbase + 32) and [tbase + THREADS, tbase +
    // THREADS + 32) of the tile, nu of the two in use (warp-uniform). A tile
    // of up to THREADS targets gives every warp up to 32 of them, so a partly
    // filled tile keeps all of the block's warps busy: the warps of a block sit
    // on different SM sub-partitions, whose MUFU and FMA pipes are separate.
    const int nu = w.t_count > tbase + THREADS ? 2 : (w.t_count > tbase ? 1 : 0);

    if (w.flags & kItemAudit) {
      // The audit's direct sum, in FP64 like the reference's
      // (src/direct_sum_impl.hpp:34-94): absolute coordinates, the FP64
      // reciprocal square root, FP64 sums. Sources are read from the FP64
      // stage itself, so a stage is refilled only after the next chunk's
      // barrier (every thread has finished it): chunk c - 1 + STAGES is
      // issued at chunk c, one barrier per chunk.
      double ax[TPT], ay[TPT], az[TPT], a64[TPT][NC];
#pragma unroll
      for (int u = 0; u < TPT; ++u) {
        const double4 t = p.T4a[w.t_begin + min(tbase + u * THREADS + lane, w.t_count - 1)];
        ax[u] = t.x;
        ay[u] = t.y;
        az[u] = t.z;
#pragma unroll
        for (int c = 0; c < NC; ++c) a64[u][c] = 0.0;
      }
      for (int c = 0; c < n_chunks; ++c) {
        const int stage = (g + c) % STAGES;
        const uint32_t parity = ((g + c) / STAGES) & 1u;
        if (!mbar_wait_bounded(&bars[stage], parity, p.wait_limit)) {
          s_abort = 1;
          s_fail_chunk = g + c;
          atomicCAS(p.status, 0, (int)BTK_ERR_DEVICE_TIMEOUT);
        }
        __syncthreads();
        if (s_abort) break;
        if (tid == 0 && c >= 1 && c - 1 + STAGES < n_chunks) issue(c - 1 + STAGES);
        const int cnt = min(kChunk, w.s_total - c * kChunk);
        const double4* sb = sbuf[stage];
        if (p.eps2 < 1.1754943508222875e-38) {  // r^2 may leave the FP32 normal range: guarded
          for (int j = 0; j < cnt; ++j)
            for (int u = 0; u < nu; ++u) eval_fp64<DIM, KIND, true>(ax[u], ay[u], az[u], sb[j], p.eps2, a64[u]);
        } else if (nu == 2) {
#pragma unroll 2
          for (int j = 0; j < cnt; ++j) {
            const double4 sj = sb[j];
            eval_fp64<DIM, KIND, false>(ax[0], ay[0], az[0], sj, p.eps2, a64[0]);
            eval_fp64<DIM, KIND, false>(ax[1], ay[1], az[1], sj, p.eps2, a64[1]);
          }
        } else if (nu == 1) {
#pragma unroll 2
          for (int j = 0; j < cnt; ++j)
            eval_fp64<DIM, KIND, false>(ax[0], ay[0], az[0], sb[j], p.eps2, a64[0]);
        }
      }
      if (s_abort) break;
      g += n_chunks;
#pragma unroll
      for (int u = 0; u < TPT; ++u) {
        const int i = tbase + u * THREADS + lane;
        if (i < w.t_count) {
#pragma unroll
          for (int c = 0; c < NC; ++c) atomicAdd(p.aout[c] + w.t_begin + i, a64[u][c] * p.scale[c]);
        }
      }
      continue;
    }

    TargetPair T[TPT];
    double acc[TPT][NC], comp[TPT][NC];
#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int i = min(tbase + u * THREADS + lane, w.t_count - 1);
      const double4 t = p.T4[w.t_begin + i];
      float h, l;
      split_rel(t.x, w.cx, h, l);
      T[u].x = make_float2(h, h);
      T[u].lx = make_float2(l, l);
      split_rel(t.y, w.cy, h, l);
      T[u].y = make_float2(h, h);
      T[u].ly = make_float2(l, l);
      split_rel(t.z, w.cz, h, l);
      T[u].z = make_float2(h, h);
      T[u].lz = make_float2(l, l);
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[u][c] = comp[u][c] = 0.0;
    }

    for (int c = 0; c < n_chunks; ++c) {
      const int stage = (g + c) % STAGES;
      const uint32_t parity = ((g + c) / STAGES) & 1u;
      if (!mbar_wait_bounded(&bars[stage], parity, p.wait_limit)) {
        s_abort = 1;
        s_fail_chunk = g + c;
        atomicCAS(p.status, 0, (int)BTK_ERR_DEVICE_TIMEOUT);
      }
      const int cnt = min(kChunk, w.s_total - c * kChunk);
      const int near_end = min(cnt, max(0, w.near_total - c * kChunk));  // near sources of this chunk
      const int b = c & 1;
      // A chunk with near-field sources is laid out per warp region (the 64
      // sources warp r converts fill pairs [32 r, 32 r + 32)): the near
      // sources closer to the target box than max(hx, hy, hz) first, on the
      // hi/lo path; the others after them, on the FP32 path (their separation
      // is at least as large as a non-touching leaf's).
      const bool split = near_end > 0;  // block-uniform
      {  // thread tid converts source pair tid into buffer b
        float hx[2], hy[2], hz[2], lx[2], ly[2], lz[2], ww[2];
        bool close[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int j = 2 * tid + k;
          if (j < cnt) {
            const double4 s = sbuf[stage][j];
            const double rx = s.x - w.cx, ry = s.y - w.cy, rz = s.z - w.cz;
            hx[k] = (float)rx;
            hy[k] = (float)ry;
            hz[k] = (float)rz;
            const float gap = fmaxf(fabsf(hx[k]) - w.hx,
                                    fmaxf(fabsf(hy[k]) - w.hy, DIM == 3 ? fabsf(hz[k]) - w.hz : -3.0e38f));
            close[k] = j < near_end && gap < thr;
            // Low parts only where the hi/lo path reads them (close sources;
            // a farther source sharing a hi/lo pair reads 0: its FP32 value);
            // the FP64 <-> FP32 conversions share the MUFU pipe.
            if (close[k]) {
              lx[k] = (float)(rx - (double)hx[k]);
              ly[k] = (float)(ry - (double)hy[k]);
              lz[k] = (float)(rz - (double)hz[k]);
            } else {
              lx[k] = ly[k] = lz[k] = 0.f;
            }
            hx[k] = -hx[k];
            hy[k] = -hy[k];
            hz[k] = -hz[k];
            lx[k] = -lx[k];
            ly[k] = -ly[k];
            lz[k] = -lz[k];
            ww[k] = (float)s.w;
          } else {
            hx[k] = hy[k] = hz[k] = kPadCoord;
            lx[k] = ly[k] = lz[k] = 0.f;
            ww[k] = 0.f;
            close[k] = false;
          }
        }
        if (!split) {
          fA[b][tid] = make_float4(hx[0], hx[1], hy[0], hy[1]);
          fB[b][tid] = make_float4(hz[0], hz[1], ww[0], ww[1]);
          fL[b][tid] = make_float4(lx[0], lx[1], ly[0], ly[1]);
          fLz[b][tid] = make_float2(lz[0], lz[1]);
        } else {
          // slot q of the warp's 64: close sources in (lane, k) order, then the
          // rest (padding last); source in slot q -> pair 32 warp + q / 2, lane q & 1
          const unsigned m0 = __ballot_sync(0xffffffffu, close[0]), m1 = __ballot_sync(0xffffffffu, close[1]);
          const unsigned lt = (1u << lane) - 1u;
          const int cb = __popc(m0 & lt) + __popc(m1 & lt), n_close = __popc(m0) + __popc(m1);
          const int fb = 2 * lane - cb;  // sources before this lane's two that are not close
          const int q[2] = {close[0] ? cb : n_close + fb,
                            close[1] ? cb + (close[0] ? 1 : 0) : n_close + fb + (close[0] ? 0 : 1)};
#pragma unroll
          for (int k = 0; k < 2; ++k) {
            const int pr = warp * 32 + (q[k] >> 1), h = q[k] & 1;
            float* a = reinterpret_cast<float*>(&fA[b][pr]);
            float* bb = reinterpret_cast<float*>(&fB[b][pr]);
            float* l = reinterpret_cast<float*>(&fL[b][pr]);
            float* lzp = reinterpret_cast<float*>(&fLz[b][pr]);
            a[h] = hx[k];
            a[2 + h] = hy[k];
            bb[h] = hz[k];
            bb[2 + h] = ww[k];
            l[h] = lx[k];
            l[2 + h] = ly[k];
            lzp[h] = lz[k];
          }
          if (lane == 0) s_ncp[b][warp] = (n_close + 1) >> 1;  // a pair with one close source takes hi/lo
        }
      }
      // One barrier per chunk: buffer b is complete, every thread has finished
      // chunk c - 1 (so buffer b ^ 1 may be overwritten next), and the FP64
      // stage has been read, so it is refilled while this chunk is evaluated.
      __syncthreads();
      if (s_abort) break;
      if (tid == 0 && c + STAGES < n_chunks) issue(c + STAGES);
      if (!split) {
        const int np = (cnt + 1) / 2, nnp = (near_end + 1) / 2;  // a pair with one near source is near
        for (int f0 = 0; f0 < np; f0 += kFoldPairs) {
          const int f1 = min(np, f0 + kFoldPairs);
          const int fn = min(f1, max(f0, nnp));
          float2 part[TPT][NC];
#pragma unroll
          for (int u = 0; u < TPT; ++u)
#pragma unroll
            for (int k = 0; k < NC; ++k) part[u][k] = make_float2(0.f, 0.f);
          if (nu == 2) {
            pair_loop<DIM, KIND, true, 2, NC>(fA[b], fB[b], fL[b], fLz[b], f0, fn, T, e2, part);
            pair_loop<DIM, KIND, false, 2, NC>(fA[b], fB[b], fL[b], fLz[b], fn, f1, T, e2, part);
          } else if (nu == 1) {
            pair_loop<DIM, KIND, true, 1, NC>(fA[b], fB[b], fL[b], fLz[b], f0, fn, T, e2, part);
            pair_loop<DIM, KIND, false, 1, NC>(fA[b], fB[b], fL[b], fLz[b], fn, f1, T, e2, part);
          }
#pragma unroll
          for (int u = 0; u < TPT; ++u)
            if (u < nu) {
#pragma unroll
              for (int k = 0; k < NC; ++k)
                two_sum_add(acc[u][k], comp[u][k], (double)(part[u][k].x + part[u][k].y));
            }
        }
      } else if (nu > 0) {
        static_assert(kFoldPairs == kPairs, "one fold per chunk");
        float2 part[TPT][NC];
#pragma unroll
        for (int u = 0; u < TPT; ++u)
#pragma unroll
          for (int k = 0; k < NC; ++k) part[u][k] = make_float2(0.f, 0.f);
#pragma unroll 1
        for (int r = 0; r < THREADS / 32; ++r) {
          const int p0 = r * 32, rp = (min(64, max(0, cnt - 64 * r)) + 1) / 2;  // pairs holding sources
          const int pn = p0 + min(s_ncp[b][r], rp);
          if (nu == 2) {
            pair_loop<DIM, KIND, true, 2, NC>(fA[b], fB[b], fL[b], fLz[b], p0, pn, T, e2, part);
            pair_loop<DIM, KIND, false, 2, NC>(fA[b], fB[b], fL[b], fLz[b], pn, p0 + rp, T, e2, part);
          } else {
            pair_loop<DIM, KIND, true, 1, NC>(fA[b], fB[b], fL[b], fLz[b], p0, pn, T, e2, part);
            pair_loop<DIM, KIND, false, 1, NC>(fA[b], fB[b], fL[b], fLz[b], pn, p0 + rp, T, e2, part);
          }
        }
#pragma unroll
        for (int u = 0; u < TPT; ++u)
          if (u < nu) {
#pragma unroll
            for (int k = 0; k < NC; ++k)
              two_sum_add(acc[u][k], comp[u][k], (double)(part[u][k].x + part[u][k].y));
          }
      }
    }
    if (s_abort) break;
    g += n_chunks;

#pragma unroll
    for (int u = 0; u < TPT; ++u) {
      const int i = tbase + u * THREADS + lane;
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
      mbar_wait_bounded(&bars[k % STAGES], (k / STAGES) & 1u, kDrainLimit);
  }
}

template <int DIM, int KIND, bool GUARD>
cudaError_t launch_mixed(const InteractParams& p, int grid, cudaStream_t s, int tile) {
  if (tile == 128)
    k_interact_mixed<DIM, KIND, 64><<<grid, 64, 0, s>>>(p);
  else
    k_interact_mixed<DIM, KIND, 128><<<grid, 128, 0, s>>>(p);
  return cudaGetLastError();
}

template <int DIM, int KIND, bool GUARD>
int occupancy_mixed(int tile) {
  int n = 0;
  if (tile == 128)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_interact_mixed<DIM, KIND, 64>, 64, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_interact_mixed<DIM, KIND, 128>, 128, 0);
  return n;
}

template <int DIM, int KIND, bool GUARD>
cudaError_t launch_fp64(const InteractParams& p, int grid, cudaStream_t s, int tile) {
  if (tile == 128)
    k_interact_fp64<DIM, KIND, GUARD, 64><<<grid, 64, 0, s>>>(p);
  else
    k_interact_fp64<DIM, KIND, GUARD, 128><<<grid, 128, 0, s>>>(p);
  return cudaGetLastError();
}

template <int DIM, int KIND, bool GUARD>
int occupancy_fp64(int tile) {
  int n = 0;
  if (tile == 128)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_interact_fp64<DIM, KIND, GUARD, 64>, 64, 0);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_interact_fp64<DIM, KIND, GUARD, 128>, 128, 0);
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
                            cudaStream_t s, int tile) {
  if (p.n_items + p.n_audit_items <= 0) return cudaSuccess;
  if (tile != 128 && tile != 256) return cudaErrorInvalidValue;
  count_launch();
  if (precision == BTK_PREC_FP64) BTK_KIND_SWITCH(dim, kind, guard, launch_fp64, p, grid, s, tile);
  if (precision == BTK_PREC_MIXED) BTK_KIND_SWITCH(dim, kind, false, launch_mixed, p, grid, s, tile);
  return cudaErrorInvalidValue;
}

int interact_blocks_per_sm(int dim, int kind, int precision, bool guard, int tile) {
  if (precision == BTK_PREC_FP64) BTK_KIND_SWITCH(dim, kind, guard, occupancy_fp64, tile);
  if (precision == BTK_PREC_MIXED) BTK_KIND_SWITCH(dim, kind, false, occupancy_mixed, tile);
  return 0;
}

}  // namespace btk
