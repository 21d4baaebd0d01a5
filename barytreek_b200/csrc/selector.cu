// Learned interpolation-degree selector (no reference counterpart).
//
// Per far-field pair (PC, CP, CC) a 16-feature vector describes the geometry
// (radii, separation ratios, point counts, interaction class, kernel
// regularisation) and the source cluster's modified charges (Chebyshev-moment
// band energies from a DCT-I of the degree-n modified charges, net-charge
// fraction). An MLP 16 -> 64 -> 64 -> 9 with ReLU, BF16 weights and FP32
// accumulation predicts log10 of the pair's relative far-field error at
// degrees 4..12; the smallest degree whose prediction meets the pair target is
// chosen on the device. Training uses error samples generated here: each
// sampled pair is evaluated at every degree through its proxies and compared
// with the direct sum over the source cluster's points, in FP64.
#include <atomic>

#include "device_math.cuh"
#include "kernels.cuh"

#include <cuda_bf16.h>

namespace btk {

namespace {

constexpr int kF = 16, kH = 64, kO = 9, kDegLo = 4;
constexpr int kW1 = 0, kB1 = kW1 + kH * kF, kW2 = kB1 + kH, kB2 = kW2 + kH * kH, kW3 = kB2 + kH, kB3 = kW3 + kO * kH;
constexpr int kParams = kB3 + kO;  // 5833
constexpr int kDescs = 6;          // per-panel charge descriptors

__device__ __forceinline__ float lg(double x) { return (float)log10(x > 1e-300 ? x : 1e-300); }

// ---- per-panel charge descriptors ------------------------------------------
// desc[0] = log10 sum|W|, desc[1] = log10(|sum W| / sum|W|), desc[2..5] =
// log10 of the Chebyshev-moment energy in bands max(i,j,k) in {1,2}, {3,4},
// {5,6}, {>=7}, each relative to sum|W|. Moments M = (C x C x C) W with
// C[i][a] = cos(pi i a / n): Chebyshev moments of the panel's charge
// distribution (exact through polynomial reproduction).
__global__ void __launch_bounds__(256) k_panel_desc(int dim, int n, int P, const double* psw, float* desc) {
  __shared__ double bufA[kMaxNodes * kMaxNodes * kMaxNodes], bufB[kMaxNodes * kMaxNodes * kMaxNodes];
  __shared__ double C[kMaxNodes * kMaxNodes];
  __shared__ double red[8][32];
  const int p = blockIdx.x;
  const int m = n + 1;
  const int ipc = dim == 3 ? m * m * m : m * m;
  const double pi = 3.141592653589793238462643383279502884;
  for (int o = threadIdx.x; o < m * m; o += blockDim.x) C[o] = cos(pi * (o / m) * (o % m) / n);
  double l1 = 0.0, s = 0.0;
  for (int o = threadIdx.x; o < ipc; o += blockDim.x) {
    const double w = psw[(size_t)p * ipc + o];
    bufA[o] = w;
    l1 += fabs(w);
    s += w;
  }
  __syncthreads();
  // separable DCT-I along each axis (same stride logic as the transfers)
  const int strides[3] = {dim == 3 ? m * m : m, dim == 3 ? m : 1, 1};
  double* in = bufA;
  double* out = bufB;
  for (int ax = 0; ax < dim; ++ax) {
    const int str = strides[ax];
    for (int o = threadIdx.x; o < ipc; o += blockDim.x) {
      const int i = (o / str) % m;
      const int base = o - i * str;
      double acc = 0.0;
      for (int a = 0; a < m; ++a) acc = fma(C[i * m + a], in[base + a * str], acc);
      out[o] = acc;
    }
    __syncthreads();
    double* t = in;
    in = out;
    out = t;
  }
  double band[4] = {0, 0, 0, 0};
  for (int o = threadIdx.x; o < ipc; o += blockDim.x) {
    int i, j, k = 0;
    if (dim == 2) {
      i = o / m;
      j = o % m;
    } else {
      i = o / (m * m);
      j = (o / m) % m;
      k = o % m;
    }
    const int mx = max(i, max(j, k));
    const double e = in[o] * in[o];
    if (mx >= 1) band[mx <= 2 ? 0 : (mx <= 4 ? 1 : (mx <= 6 ? 2 : 3))] += e;
  }
  double v[6] = {l1, s, band[0], band[1], band[2], band[3]};
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int q = 0; q < 6; ++q) {
    double x = v[q];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (lane == 0) red[wid][q] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[6] = {0, 0, 0, 0, 0, 0};
    for (int w = 0; w < (int)(blockDim.x / 32); ++w)
      for (int q = 0; q < 6; ++q) t[q] += red[w][q];
    const double L1 = t[0] > 1e-300 ? t[0] : 1e-300;
    float* d = desc + (size_t)p * kDescs;
    d[0] = lg(L1);
    d[1] = lg(fabs(t[1]) / L1 + 1e-16);
    for (int b = 0; b < 4; ++b) d[2 + b] = lg(sqrt(t[2 + b]) / L1 + 1e-16);
  }
}

// ---- per-pair features -------------------------------------------------------
// type: 1 PC, 2 CP, 3 CC. Pairs listed PC, then CP, then CC.
// Sum |q| and sum q over the sources (the global potential scale and net
// charge the features are normalised by).
__global__ void k_global_sums(int n, const double4* pts, double* sums) {
  double a = 0.0, b = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    a += fabs(pts[i].w);
    b += pts[i].w;
  }
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, off);
    b += __shfl_down_sync(0xffffffffu, b, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(sums, a);
    atomicAdd(sums + 1, b);
  }
}

// Features of pair i:
//  0 log10(r_T/R)  1 log10(r_S/R)  2 log10(d/(r_T+r_S))  3 log10(d/r_S)
//  4 log10(d/r_T)  5 log10(1+m_T)  6 log10(1+m_S)  7-9 class (PC, CP, CC)
// 10 log10(eps/d)  11 source net-charge fraction  12, 13 source Chebyshev-
// moment energy in bands 3-4 and >=7  14 log10((sum|W_S|/d) / (sum|q|/R)):
// the pair's potential scale against the global one  15 global net-charge
// fraction log10(|sum q| / sum |q|). R = root radius, d = centre distance.
__global__ void k_pair_features(int n_pairs, const int* ptype, const int* ptgt, const int* psrc,
                                const DevPanel* pt, const DevPanel* ps, double root_radius, double eps,
                                const float* desc_s, const double* gsum, float* feat) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_pairs) return;
  const DevPanel T = pt[ptgt[i]], S = ps[psrc[i]];
  double ct[3], cs[3], rt2 = 0, rs2 = 0, d2 = 0;
  for (int a = 0; a < 3; ++a) {
    ct[a] = 0.5 * (T.lo[a] + T.hi[a]);
    cs[a] = 0.5 * (S.lo[a] + S.hi[a]);
    rt2 += (T.hi[a] - T.lo[a]) * (T.hi[a] - T.lo[a]);
    rs2 += (S.hi[a] - S.lo[a]) * (S.hi[a] - S.lo[a]);
    d2 += (ct[a] - cs[a]) * (ct[a] - cs[a]);
  }
  const double rt = 0.5 * sqrt(rt2) + 1e-300, rs = 0.5 * sqrt(rs2) + 1e-300, dist = sqrt(d2) + 1e-300;
  float* f = feat + (size_t)i * kF;
  f[0] = lg(rt / root_radius);
  f[1] = lg(rs / root_radius);
  f[2] = lg(dist / (rt + rs));
  f[3] = lg(dist / rs);
  f[4] = lg(dist / rt);
  f[5] = lg(1.0 + T.point_count);
  f[6] = lg(1.0 + S.point_count);
  f[7] = ptype[i] == 1 ? 1.f : 0.f;
  f[8] = ptype[i] == 2 ? 1.f : 0.f;
  f[9] = ptype[i] == 3 ? 1.f : 0.f;
  f[10] = lg(eps / dist + 1e-12);
  const float* d = desc_s + (size_t)psrc[i] * kDescs;
  f[11] = d[1];
  f[12] = d[3];
  f[13] = d[5];
  const double g_abs = gsum[0] > 1e-300 ? gsum[0] : 1e-300;
  f[14] = d[0] - lg(dist) - lg(g_abs / root_radius);
  f[15] = lg(fabs(gsum[1]) / g_abs + 1e-16);
}

// ---- MLP ----------------------------------------------------------------------
// Parameters as BF16, loaded to shared FP32; inputs normalised on the fly.
struct MlpNorm {
  float xm[kF], xs[kF], ym, ys;
};

__device__ __forceinline__ void load_params(const __nv_bfloat16* w, float* sw) {
  for (int o = threadIdx.x; o < kParams; o += blockDim.x) sw[o] = __bfloat162float(w[o]);
}

// y[o] for one normalised input row; h1/h2 post-ReLU returned when non-null.
__device__ __forceinline__ void mlp_row(const float* sw, const float* x, float* y, float* h1o, float* h2o) {
  float h1[kH], h2[kH];
#pragma unroll 4
  for (int j = 0; j < kH; ++j) {
    float a = sw[kB1 + j];
#pragma unroll
    for (int i = 0; i < kF; ++i) a = fmaf(sw[kW1 + j * kF + i], x[i], a);
    h1[j] = fmaxf(a, 0.f);
  }
#pragma unroll 2
  for (int j = 0; j < kH; ++j) {
    float a = sw[kB2 + j];
#pragma unroll 8
    for (int i = 0; i < kH; ++i) a = fmaf(sw[kW2 + j * kH + i], h1[i], a);
    h2[j] = fmaxf(a, 0.f);
  }
#pragma unroll
  for (int o = 0; o < kO; ++o) {
    float a = sw[kB3 + o];
#pragma unroll 8
    for (int i = 0; i < kH; ++i) a = fmaf(sw[kW3 + o * kH + i], h2[i], a);
    y[o] = a;
  }
  if (h1o)
    for (int j = 0; j < kH; ++j) h1o[j] = h1[j];
  if (h2o)
    for (int j = 0; j < kH; ++j) h2o[j] = h2[j];
}

// Inference on raw features, out[i][o] = predicted log10 error at degree 4+o,
// on the 5th-generation tensor cores (tcgen05, kind::f16: BF16 operands, FP32
// accumulators in TMEM). A CTA of 128 threads owns tiles of 128 pairs (the MMA
// M; thread t's pair is TMEM lane t) and pushes each through the three layers:
//   layer 1: A = normalised features [128 x 16], B = W1 [64 x 16]  -> D1 [128 x 64]
//   layer 2: A = ReLU(D1 + b1) [128 x 64], B = W2 [64 x 64] (4 K steps) -> D2
//   layer 3: A = ReLU(D2 + b2), B = W3 [9 (padded to 16) x 64] -> D3 [128 x 16]
// One thread issues each layer's MMAs and commits them to an mbarrier; every
// thread then reads its lane's accumulators with tcgen05.ld, applies bias,
// ReLU and the BF16 rounding, and writes its row of the next layer's A tile
// (K-major, no swizzle). The weights are staged once per CTA. Normalised
// inputs and hidden activations are BF16 (the training kernels keep them in
// FP32; the difference is within the network's error). Waits are bounded: a
// CTA that gives up sets *status (when given), stops and frees its TMEM.
constexpr int kTcM = 128;          // pairs per tile (MMA M), one per thread
constexpr uint32_t kTmemCols = 128;  // D1/D2 in columns 0..63, D3 in 64..79
constexpr uint32_t kTcWaitLimit = 1u << 22;
struct TcSmem {
  alignas(1024) uint8_t a1[kTcM * kF * 2];  // layer-1 A, K = 16
  alignas(1024) uint8_t a2[kTcM * kH * 2];  // layer-2, then layer-3 A, K = 64 (4 K steps of 4096 B)
  alignas(1024) uint8_t w1[kH * kF * 2];    // N = 64, K = 16
  alignas(1024) uint8_t w2[kH * kH * 2];    // N = 64, K = 64 (4 K steps of 2048 B)
  alignas(1024) uint8_t w3[16 * kH * 2];    // N = 16, K = 64 (4 K steps of 512 B); rows 9..15 zero
  float b1[kH], b2[kH], b3[16];
  uint64_t bar;
  uint32_t tmem;
  int abort;
};
// At least this much dynamic shared memory per CTA, so at most 3 CTAs share an
// SM and their TMEM columns (3 x 128 <= 512) never run out.
constexpr size_t kTcSmemBytes = 64 * 1024;
static_assert(sizeof(TcSmem) + 1024 <= kTcSmemBytes, "tile buffers exceed the reserved shared memory");

// Byte offset of BF16 element (row, k) in a K-major, unswizzled tile of R rows:
// K steps of 16 elements are R x 32 bytes apart; within one, 8-row groups are
// 256 bytes apart (sbo) and the two 8-element halves 128 bytes apart (lbo).
__device__ __forceinline__ uint32_t kmaj_off(int row, int k, int R) {
  return (uint32_t)((k >> 4) * (R * 32) + (row >> 3) * 256 + ((k >> 3) & 1) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// 16 values of row `row` (columns k0..k0+15) into a K-major tile as BF16.
__device__ __forceinline__ void store_row16(uint8_t* tile, int row, int k0, int R, const float* v) {
  uint4 lo, hi;
  lo.x = pack_bf16x2(v[0], v[1]);
  lo.y = pack_bf16x2(v[2], v[3]);
  lo.z = pack_bf16x2(v[4], v[5]);
  lo.w = pack_bf16x2(v[6], v[7]);
  hi.x = pack_bf16x2(v[8], v[9]);
  hi.y = pack_bf16x2(v[10], v[11]);
  hi.z = pack_bf16x2(v[12], v[13]);
  hi.w = pack_bf16x2(v[14], v[15]);
  *reinterpret_cast<uint4*>(tile + kmaj_off(row, k0, R)) = lo;
  *reinterpret_cast<uint4*>(tile + kmaj_off(row, k0 + 8, R)) = hi;
}

__global__ void __launch_bounds__(kTcM) k_mlp_infer(int n, const __nv_bfloat16* w, MlpNorm nrm, const float* feat,
                                                   float* out, int* status) {
  extern __shared__ uint8_t dsm_raw[];
  TcSmem& sm = *reinterpret_cast<TcSmem*>(dsm_raw + ((1024u - (smem_addr(dsm_raw) & 1023u)) & 1023u));
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int o = tid; o < kH * kF; o += kTcM)
    *reinterpret_cast<__nv_bfloat16*>(sm.w1 + kmaj_off(o / kF, o % kF, kH)) = w[kW1 + o];
  for (int o = tid; o < kH * kH; o += kTcM)
    *reinterpret_cast<__nv_bfloat16*>(sm.w2 + kmaj_off(o / kH, o % kH, kH)) = w[kW2 + o];
  for (int o = tid; o < 16 * kH; o += kTcM)
    *reinterpret_cast<__nv_bfloat16*>(sm.w3 + kmaj_off(o / kH, o % kH, 16)) =
        o / kH < kO ? w[kW3 + o] : __float2bfloat16(0.f);
  for (int o = tid; o < kH; o += kTcM) {
    sm.b1[o] = __bfloat162float(w[kB1 + o]);
    sm.b2[o] = __bfloat162float(w[kB2 + o]);
  }
  if (tid < 16) sm.b3[tid] = tid < kO ? __bfloat162float(w[kB3 + tid]) : 0.f;
  if (tid == 0) {
    mbar_init(&sm.bar, 1);
    mbar_fence_init();
    sm.abort = 0;
  }
  if (warp == 0) {
    tmem_alloc(&sm.tmem, kTmemCols);
    tmem_relinquish();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = sm.tmem;
  const uint32_t taddr = tbase + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
  constexpr uint32_t id64 = umma_idesc_bf16_f32(kTcM, kH), id16 = umma_idesc_bf16_f32(kTcM, 16);
  uint32_t phase = 0, issued = 0, waited = 0;
  // Waits for the MMAs committed last; false (and the CTA stops) on timeout.
  auto wait_mma = [&]() {
    if (mbar_wait_bounded(&sm.bar, phase, kTcWaitLimit)) {
      phase ^= 1u;
      ++waited;
    } else {  // still in flight: the drain below waits for it
      sm.abort = 1;
      if (status) atomicCAS(status, 0, (int)BTK_ERR_DEVICE_TIMEOUT);
    }
    __syncthreads();
    tc_fence_after();
    return sm.abort == 0;
  };
  const int tiles = (n + kTcM - 1) / kTcM;
  for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const int row = tile * kTcM + tid;
    {  // layer-1 A: this thread's normalised features
      float x[kF];
#pragma unroll
      for (int c = 0; c < kF; ++c) x[c] = row < n ? (feat[(size_t)row * kF + c] - nrm.xm[c]) / nrm.xs[c] : 0.f;
      store_row16(sm.a1, tid, 0, kTcM, x);
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma_bf16(tbase, umma_desc_kmajor(sm.a1, 128, 256), umma_desc_kmajor(sm.w1, 128, 256), id64, 0);
      umma_commit(&sm.bar);
      ++issued;
    }
    if (!wait_mma()) break;
#pragma unroll 1
    for (int layer = 0; layer < 2; ++layer) {  // D1 -> layer-2 A, D2 -> layer-3 A
      const float* bias = layer == 0 ? sm.b1 : sm.b2;
#pragma unroll 1
      for (int c0 = 0; c0 < kH; c0 += 16) {
        float v[16];
        tmem_ld16(taddr + (uint32_t)c0, v);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = fmaxf(v[k] + bias[c0 + k], 0.f);
        store_row16(sm.a2, tid, c0, kTcM, v);
      }
      fence_proxy_async_smem();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        for (int ks = 0; ks < kH / 16; ++ks) {
          const uint64_t da = umma_desc_kmajor(sm.a2 + ks * (kTcM * 32), 128, 256);
          if (layer == 0)
            umma_bf16(tbase, da, umma_desc_kmajor(sm.w2 + ks * (kH * 32), 128, 256), id64, ks > 0);
          else
            umma_bf16(tbase + 64, da, umma_desc_kmajor(sm.w3 + ks * (16 * 32), 128, 256), id16, ks > 0);
        }
        umma_commit(&sm.bar);
        ++issued;
      }
      if (!wait_mma()) break;
    }
    if (sm.abort) break;
    float v[16];
    tmem_ld16(taddr + 64, v);
    if (row < n) {
#pragma unroll
      for (int o = 0; o < kO; ++o) out[(size_t)row * kO + o] = (v[o] + sm.b3[o]) * nrm.ys + nrm.ym;
    }
    tc_fence_before();
    __syncthreads();  // every lane's TMEM reads are done before the next tile's MMAs
    tc_fence_after();
  }
  // After a timeout, wait (bounded) for what thread 0 still has in flight
  // before the TMEM columns are released.
  if (tid == 0)
    for (; waited < issued; ++waited, phase ^= 1u) mbar_wait_bounded(&sm.bar, phase, kTcWaitLimit);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, kTmemCols);
  }
}

// Forward on normalised inputs (training/validation): yn[i][o].
__global__ void __launch_bounds__(128) k_mlp_forward_n(int n, const __nv_bfloat16* w, const float* xn, float* yn) {
  extern __shared__ float sw[];
  load_params(w, sw);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float y[kO];
  mlp_row(sw, xn + (size_t)i * kF, y, nullptr, nullptr);
  for (int o = 0; o < kO; ++o) yn[(size_t)i * kO + o] = y[o];
}

// Per-sample forward + backward of the masked mean-squared error
// L = sum_{i,o} mask (y - t)^2 / sum mask. Stores post-ReLU activations and
// pre-activation deltas for the weight-gradient reduction.
__global__ void __launch_bounds__(128) k_mlp_backprop(int n, const __nv_bfloat16* w, const float* xn, const float* tn,
                                                      const float* mask, float inv_count, float* h1s, float* h2s,
                                                      float* d1s, float* d2s, float* d3s, float* loss) {
  extern __shared__ float sw[];
  load_params(w, sw);
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float lsum = 0.f;
  if (i < n) {
    float y[kO], h1[kH], h2[kH], d3[kO], d2[kH];
    mlp_row(sw, xn + (size_t)i * kF, y, h1, h2);
    for (int o = 0; o < kO; ++o) {
      const float mk = mask[(size_t)i * kO + o];
      const float e = y[o] - tn[(size_t)i * kO + o];
      lsum += mk * e * e;
      d3[o] = 2.f * mk * e * inv_count;
      d3s[(size_t)i * kO + o] = d3[o];
    }
    for (int j = 0; j < kH; ++j) {
      float a = 0.f;
      for (int o = 0; o < kO; ++o) a = fmaf(sw[kW3 + o * kH + j], d3[o], a);
      d2[j] = h2[j] > 0.f ? a : 0.f;
      d2s[(size_t)i * kH + j] = d2[j];
      h1s[(size_t)i * kH + j] = h1[j];
      h2s[(size_t)i * kH + j] = h2[j];
    }
    for (int j = 0; j < kH; ++j) {
      float a = 0.f;
      for (int k = 0; k < kH; ++k) a = fmaf(sw[kW2 + k * kH + j], d2[k], a);
      d1s[(size_t)i * kH + j] = h1[j] > 0.f ? a : 0.f;
    }
  }
  for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
  if ((threadIdx.x & 31) == 0 && lsum != 0.f) atomicAdd(loss, lsum * inv_count);
}

// Weight gradients: one thread per parameter, summing over the batch.
__global__ void k_mlp_wgrad(int n, const float* xn, const float* h1s, const float* h2s, const float* d1s,
                            const float* d2s, const float* d3s, float* grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  float g = 0.f;
  if (p < kB1) {
    const int j = p / kF, k = p % kF;
    for (int i = 0; i < n; ++i) g = fmaf(d1s[(size_t)i * kH + j], xn[(size_t)i * kF + k], g);
  } else if (p < kW2) {
    const int j = p - kB1;
    for (int i = 0; i < n; ++i) g += d1s[(size_t)i * kH + j];
  } else if (p < kB2) {
    const int j = (p - kW2) / kH, k = (p - kW2) % kH;
    for (int i = 0; i < n; ++i) g = fmaf(d2s[(size_t)i * kH + j], h1s[(size_t)i * kH + k], g);
  } else if (p < kW3) {
    const int j = p - kB2;
    for (int i = 0; i < n; ++i) g += d2s[(size_t)i * kH + j];
  } else if (p < kB3) {
    const int o = (p - kW3) / kH, k = (p - kW3) % kH;
    for (int i = 0; i < n; ++i) g = fmaf(d3s[(size_t)i * kO + o], h2s[(size_t)i * kH + k], g);
  } else {
    const int o = p - kB3;
    for (int i = 0; i < n; ++i) g += d3s[(size_t)i * kO + o];
  }
  grad[p] = g;
}

// Adam on FP32 master weights; the BF16 copy is what the network runs with.
__global__ void k_adam(float* master, __nv_bfloat16* w, const float* grad, float* m, float* v, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  const float g = grad[p];
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  const float upd = lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  master[p] -= upd;
  w[p] = __float2bfloat16_rn(master[p]);
}

// Degree choice: the smallest d in [lo, hi] with prediction <= target, else hi.
// Leaf pairs [conv0, n_pc) also have the direct evaluation (degree 0): taken
// when no degree meets the target or when the source leaf has no more points
// than the chosen degree's proxies (pc_direct[2 i + 1]).
__global__ void k_choose_degrees(int n, const float* pred, float log10_target, int lo, int hi, int dim, int conv0,
                                 int n_pc, const int* pc_direct, int* deg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int d = hi;
  bool met = false;
  for (int c = max(lo, kDegLo); c <= hi && c < kDegLo + kO; ++c)
    if (pred[(size_t)i * kO + (c - kDegLo)] <= log10_target) {
      d = c;
      met = true;
      break;
    }
  if (i >= conv0 && i < n_pc) {
    const int m = d + 1, proxies = dim == 3 ? m * m * m : m * m;
    if (!met || proxies >= pc_direct[2 * i + 1]) d = 0;
  }
  deg[i] = d;
}

// Cost-aware choice: per pair the degree minimising
//   cost(d) / cbar + (w / wbar) * (err(d) / pair_tol)^2,
// cost(d) = evaluations at degree d ((d+1)^dim per target point for PC, per
// source point for CP, (d+1)^(2 dim) for CC), w = points under the target
// panel (how many targets carry the pair's error), err(d) = the predicted
// error. The Lagrangian of "fewest evaluations for a given sum of squared
// errors over the targets": expensive pairs accept a larger error, cheap ones
// a smaller one, where the uniform threshold gives every pair the same.
// Leaf pairs [conv0, n_pc) also have the direct evaluation (degree 0): cost
// target points x source points, no approximation error.
__global__ void k_choose_degrees_cost(int n, int dim, int n_pc, int n_cp, int conv0, const float* pred,
                                      float log10_target, int lo, int hi, const int* pc_tcount, const int* cp_scount,
                                      const int* pc_direct, const int* weight, float inv_cbar, float inv_wbar,
                                      int* deg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float wr = (float)weight[i] * inv_wbar;
  float best = 3.4e38f;
  int d_best = hi;
  if (i >= conv0 && i < n_pc) {
    best = (float)pc_tcount[i] * (float)pc_direct[2 * i + 1] * inv_cbar;
    d_best = 0;
  }
  for (int c = max(lo, kDegLo); c <= hi && c < kDegLo + kO; ++c) {
    const float m = (float)(c + 1);
    const float md = dim == 3 ? m * m * m : m * m;
    const float cost = i < n_pc ? md * (float)pc_tcount[i] : (i < n_pc + n_cp ? md * (float)cp_scount[i - n_pc] : md * md);
    const float e = exp10f(fminf(pred[(size_t)i * kO + (c - kDegLo)] - log10_target, 18.f));
    const float J = cost * inv_cbar + wr * e * e;
    if (J < best) {
      best = J;
      d_best = c;
    }
  }
  deg[i] = d_best;
}

// Leaf pairs k < n (the PP pairs the degree choice may approximate): one
// decision over the direct evaluation, target points x source-leaf proxies
// (PC entry pc0 + k) and, for k < n_cc (target leaves with more points than
// the plan degree's proxies), target-leaf proxies x source-leaf proxies (CC
// entry cc0 + k), each approximation at its own predicted errors. Cost rule:
// the least cost / mean cost + (w / mean w) (err / pair_tol)^2, direct at its
// cost and no error; threshold rule: the cheapest form meeting the pair
// tolerance (direct always does). Degrees written: direct = PC entry 0 (its
// entry is the source leaf's points), CC entry 0 (no items); PC form = PC
// entry d, CC entry 0; CC form = PC entry -1 (empty entry), CC entry d.
__global__ void k_choose_leaf_pairs(int n, int n_cc, int dim, int pc0, int cc0, const float* pred,
                                    float log10_target, int lo, int hi, int cost_rule, const int* pc_tcount,
                                    const int* pc_direct, const int* weight, float inv_cbar, float inv_wbar,
                                    int* deg) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = pc0 + k, j = cc0 + k;
  const bool has_cc = k < n_cc;
  const float nt = (float)pc_tcount[i], ns = (float)pc_direct[2 * i + 1];
  const float wr = (float)weight[i] * inv_wbar;
  float best = cost_rule ? nt * ns * inv_cbar : nt * ns;
  int form = 0, d_best = 0;
  for (int c = max(lo, kDegLo); c <= hi && c < kDegLo + kO; ++c) {
    const float m = (float)(c + 1);
    const float md = dim == 3 ? m * m * m : m * m;
    const float p_pc = pred[(size_t)i * kO + (c - kDegLo)];
    const float p_cc = has_cc ? pred[(size_t)j * kO + (c - kDegLo)] : 3.4e38f;
    float j_pc, j_cc = 3.4e38f;
    if (cost_rule) {
      const float e_pc = exp10f(fminf(p_pc - log10_target, 18.f));
      j_pc = nt * md * inv_cbar + wr * e_pc * e_pc;
      if (has_cc) {
        const float e_cc = exp10f(fminf(p_cc - log10_target, 18.f));
        j_cc = md * md * inv_cbar + wr * e_cc * e_cc;
      }
    } else {
      j_pc = p_pc <= log10_target ? nt * md : 3.4e38f;
      if (has_cc && p_cc <= log10_target) j_cc = md * md;
    }
    if (j_pc < best) {
      best = j_pc;
      form = 1;
      d_best = c;
    }
    if (j_cc < best) {
      best = j_cc;
      form = 2;
      d_best = c;
    }
  }
  deg[i] = form == 1 ? d_best : (form == 2 ? -1 : 0);
  if (has_cc) deg[j] = form == 2 ? d_best : 0;
}

// Pairs with two approximate forms, k < n: the form of entry idx[k] (PC:
// target leaf points x source proxies, coef[k] = the target leaf's points; CP:
// target proxies x source leaf points, coef[k] = the source leaf's points),
// costing coef (d+1)^dim, or proxies on both sides (CC entry cc0 + k),
// (d+1)^(2 dim); each at its own degrees, by the same rules as the other
// pairs (threshold rule with no form meeting the tolerance: the first form at
// hi). The form not taken gets degree off_first (its entry) or 0 (CC entry).
__global__ void k_choose_two_forms(int n, int dim, const int* idx, const int* coef, int off_first, int cc0,
                                   const float* pred, float log10_target, int lo, int hi, int cost_rule,
                                   const int* weight, float inv_cbar, float inv_wbar, int* deg) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int i = idx[k], j = cc0 + k;
  const float cf = (float)coef[k];
  const float wr = (float)weight[i] * inv_wbar;
  float best = 3.4e38f;
  int form = 1, d_best = hi;
  for (int c = max(lo, kDegLo); c <= hi && c < kDegLo + kO; ++c) {
    const float m = (float)(c + 1);
    const float md = dim == 3 ? m * m * m : m * m;
    const float p_1 = pred[(size_t)i * kO + (c - kDegLo)], p_cc = pred[(size_t)j * kO + (c - kDegLo)];
    float j_1, j_cc;
    if (cost_rule) {
      const float e_1 = exp10f(fminf(p_1 - log10_target, 18.f)), e_cc = exp10f(fminf(p_cc - log10_target, 18.f));
      j_1 = cf * md * inv_cbar + wr * e_1 * e_1;
      j_cc = md * md * inv_cbar + wr * e_cc * e_cc;
    } else {
      j_1 = p_1 <= log10_target ? cf * md : 3.4e38f;
      j_cc = p_cc <= log10_target ? md * md : 3.4e38f;
    }
    if (j_1 < best) {
      best = j_1;
      form = 1;
      d_best = c;
    }
    if (j_cc < best) {
      best = j_cc;
      form = 2;
      d_best = c;
    }
  }
  deg[i] = form == 1 ? d_best : off_first;
  deg[j] = form == 2 ? d_best : 0;
}

// Far-field evaluations at the chosen degrees (pairs PC, CP, CC in order) into
// evals[0]. Leaf pairs: PC entries [conv0, conv0 + n_conv), the first n_conv_cc
// of them with a CC entry among the last n_conv_cc of the CC block; a leaf pair
// kept direct (PC entry 0 and no CC form taken) adds its direct evaluations to
// evals[1] and counts in histogram bin 0; entries at degree <= 0 (forms not
// taken) count nowhere.
__global__ void k_far_evals(int dim, int n_pc, int n_cp, int n_cc, int conv0, int n_conv, int n_conv_cc,
                            const int* deg, const int* pc_tcount, const int* cp_scount, const int* pc_direct,
                            unsigned long long* evals, int* hist) {
  __shared__ int sh[kMaxDegree + 1];
  if (threadIdx.x <= kMaxDegree) sh[threadIdx.x] = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long v = 0, vd = 0;
  const int n = n_pc + n_cp + n_cc;
  const int cc_leaf0 = n - n_conv_cc;
  bool counted = i < n && deg[i] > 0 && deg[i] <= kMaxDegree;
  if (i < n && deg[i] == 0 && i >= conv0 && i < conv0 + n_conv &&
      (i - conv0 >= n_conv_cc || deg[cc_leaf0 + (i - conv0)] == 0)) {
    counted = true;  // leaf pair kept direct
    vd = (unsigned long long)pc_tcount[i] * (unsigned long long)pc_direct[2 * i + 1];
  }
  if (counted) atomicAdd(&sh[deg[i]], 1);
  if (i < n && deg[i] > 0) {
    const unsigned long long m = (unsigned long long)(deg[i] + 1);
    const unsigned long long s = dim == 3 ? m * m * m : m * m;
    if (i < n_pc)
      v = s * (unsigned long long)pc_tcount[i];
    else if (i < n_pc + n_cp)
      v = s * (unsigned long long)cp_scount[i - n_pc];
    else
      v = s * s;
  }
  for (int off = 16; off > 0; off >>= 1) {
    v += __shfl_down_sync(0xffffffffu, v, off);
    vd += __shfl_down_sync(0xffffffffu, vd, off);
  }
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(evals, v);
  if ((threadIdx.x & 31) == 0 && vd) atomicAdd(evals + 1, vd);
  __syncthreads();
  if (threadIdx.x <= kMaxDegree && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

// Audit: sums of |treecode - direct|^2 and |direct|^2 over the audited
// targets and all components.
__global__ void k_audit_compare(int n, int ncomp, int nt, const int* audit_sorted, const int* perm, const double* out,
                                const double* audit_out, double* sums) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, r = 0.0;
  if (i < n) {
    const int orig = perm ? perm[audit_sorted[i]] : audit_sorted[i];
    for (int c = 0; c < ncomp; ++c) {
      const double a = out[(size_t)c * nt + orig], b = audit_out[(size_t)c * n + i];
      e += (a - b) * (a - b);
      r += b * b;
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    e += __shfl_down_sync(0xffffffffu, e, off);
    r += __shfl_down_sync(0xffffffffu, r, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(sums, e);
    atomicAdd(sums + 1, r);
  }
}

// ---- training samples ----------------------------------------------------------
// Kernel value with its constant, FP64, into acc[c] (c < ncomp).
template <int DIM>
__device__ __forceinline__ void kval(int kind, double eps2, const double* t, const double4& s, double* acc) {
  const double dx = t[0] - s.x, dy = t[1] - s.y, dz = DIM == 3 ? t[2] - s.z : 0.0;
  const double r2 = dx * dx + dy * dy + dz * dz + eps2;
  const double pi = 3.141592653589793238462643383279502884;
  if (DIM == 2) {
    acc[0] += s.w * log(r2) / (4.0 * pi);
    if (kind == BTK_KIND_FIELD) {
      const double g = -s.w / (2.0 * pi * r2);
      acc[1] += dx * g;
      acc[2] += dy * g;
    }
    return;
  }
  if (kind == BTK_KIND_VEL) {
    const double g = -s.w / (4.0 * pi * r2);
    acc[0] += dx * g;
    acc[1] += dy * g;
    acc[2] += dz * g;
    return;
  }
  const double ri = 1.0 / sqrt(r2);
  acc[0] += -s.w * ri / (4.0 * pi);
  if (kind == BTK_KIND_FIELD) {
    const double g = -s.w * ri * ri * ri / (4.0 * pi);
    acc[1] += dx * g;
    acc[2] += dy * g;
    acc[3] += dz * g;
  }
}



__device__ __forceinline__ void target_point(const SampleArgs& a, int s, int k, double* t) {
  const int i = a.tgt_orig[(size_t)s * a.K + k];
  t[0] = a.xt[i];
  t[1] = a.yt[i];
  t[2] = a.dim == 3 ? a.zt[i] : 0.0;
}

// One block per sample: direct sum over every point under the source panel.
template <int DIM>
__global__ void __launch_bounds__(256) k_sample_exact(SampleArgs a) {
  __shared__ double red[256][4];
  const int s = blockIdx.x;
  const int lanes = blockDim.x / a.K;  // threads per target
  const int k = threadIdx.x / lanes, part = threadIdx.x % lanes;
  double acc[4] = {0, 0, 0, 0};
  if (k < a.K) {
    double t[3];
    target_point(a, s, k, t);
    for (int l = a.src_leaf_csr[s]; l < a.src_leaf_csr[s + 1]; ++l) {
      const int leaf = a.src_leaves[l];
      const int b = a.leaf_begin_s[leaf], c = a.count_s[leaf];
      for (int j = part; j < c; j += lanes) kval<DIM>(a.kind, a.eps2, t, a.S4[b + j], acc);
    }
  }
  for (int c = 0; c < 4; ++c) red[threadIdx.x][c] = acc[c];
  __syncthreads();
  if (k < a.K && part == 0) {
    for (int c = 0; c < a.ncomp; ++c) {
      double v = 0.0;
      for (int q = 0; q < lanes; ++q) v += red[threadIdx.x + q][c];
      a.exact[((size_t)s * a.K + k) * a.ncomp + c] = v;
    }
  }
}

// One block per (sample, degree): the pair's contribution at the sample's
// targets through its degree-d proxies.
template <int DIM>
__global__ void __launch_bounds__(256) k_sample_approx(SampleArgs a) {
  extern __shared__ double phi[];  // [ncomp][(d+1)^DIM]
  __shared__ double red[256][4];
  const int s = blockIdx.x / a.n_deg, di = blockIdx.x % a.n_deg;
  const int d = a.deg_lo + di, md = d + 1;
  const int ipc = DIM == 3 ? md * md * md : md * md;
  const int p = a.pair_index[s];
  const int type = a.ptype[p];
  const int tgt = a.ptgt[p], src = a.psrc[p];
  double* outp = a.approx + ((size_t)s * a.n_deg + di) * a.K * a.ncomp;
  // source slot of degree d (PC, CC) or the source leaf (CP)
  long long sb = 0;
  int sc = 0;
  if (type == 2) {
    sb = a.leaf_begin_s[src];
    sc = a.count_s[src];
  } else {
    const int slot = a.s_slot_begin[a.cluster_slot_s[src]] + (d - a.slot_d_lo);
    sb = a.ns + a.s_slot_off[slot];
    sc = ipc;
  }
  if (type == 1) {  // PC: targets against the degree-d source proxies
    const int lanes = blockDim.x / a.K;
    const int k = threadIdx.x / lanes, part = threadIdx.x % lanes;
    double acc[4] = {0, 0, 0, 0};
    if (k < a.K) {
      double t[3];
      target_point(a, s, k, t);
      for (int j = part; j < sc; j += lanes) kval<DIM>(a.kind, a.eps2, t, a.S4[sb + j], acc);
    }
    for (int c = 0; c < 4; ++c) red[threadIdx.x][c] = acc[c];
    __syncthreads();
    if (k < a.K && part == 0)
      for (int c = 0; c < a.ncomp; ++c) {
        double v = 0.0;
        for (int q = 0; q < lanes; ++q) v += red[threadIdx.x + q][c];
        outp[(size_t)k * a.ncomp + c] = v;
      }
    return;
  }
  // CP, CC: potentials at the target's degree-d proxies, then interpolation.
  const int tslot = a.t_slot_begin[a.cluster_slot_t[tgt]] + (d - a.slot_d_lo);
  const double4* tp = a.T4 + a.nt + a.t_slot_off[tslot];
  for (int j = threadIdx.x; j < ipc; j += blockDim.x) {
    const double4 tq = tp[j];
    const double t[3] = {tq.x, tq.y, tq.z};
    double acc[4] = {0, 0, 0, 0};
    for (int q = 0; q < sc; ++q) kval<DIM>(a.kind, a.eps2, t, a.S4[sb + q], acc);
    for (int c = 0; c < a.ncomp; ++c) phi[(size_t)c * ipc + j] = acc[c];
  }
  __syncthreads();
  const DevPanel T = a.pt[tgt];
  const double pi = 3.141592653589793238462643383279502884;
  for (int k = threadIdx.x; k < a.K; k += blockDim.x) {
    double t[3];
    target_point(a, s, k, t);
    double L[3][kMaxNodes];
    for (int ax = 0; ax < DIM; ++ax) {
      const double range = 0.5 * (T.hi[ax] - T.lo[ax]), mid = 0.5 * (T.hi[ax] + T.lo[ax]);
      int hit = -1;
      double den = 0.0;
      for (int i = 0; i < md; ++i) {
        const double node = cos(pi * i / d) * range + mid;
        const double diff = t[ax] - node;
        if (hit < 0 && fabs(diff) < 2.220446049250313e-16) hit = i;
        const double w = ((i & 1) ? -1.0 : 1.0) * ((i == 0 || i == d) ? 0.5 : 1.0);
        L[ax][i] = w / diff;
        den += L[ax][i];
      }
      for (int i = 0; i < md; ++i) L[ax][i] = hit >= 0 ? (i == hit ? 1.0 : 0.0) : L[ax][i] / den;
    }
    for (int c = 0; c < a.ncomp; ++c) {
      double v = 0.0;
      for (int j = 0; j < ipc; ++j) {
        const int i0 = DIM == 3 ? j / (md * md) : j / md, i1 = DIM == 3 ? (j / md) % md : j % md;
        double b = L[0][i0] * L[1][i1];
        if (DIM == 3) b *= L[2][j % md];
        v += phi[(size_t)c * ipc + j] * b;
      }
      outp[(size_t)k * a.ncomp + c] = v;
    }
  }
}

// log10 of each degree's L2 error at the sample's targets, relative to the L2
// norm of `ref` there (ref = [ncomp][nt] total solution in original order) or,
// without ref, to the pair's exact contribution.
__global__ void k_sample_errors(int n, int n_deg, int K, int ncomp, const double* exact, const double* approx,
                                const double* ref, int nt, const int* tgt_orig, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * n_deg) return;
  const int s = i / n_deg, di = i % n_deg;
  double e = 0.0, r = 0.0;
  for (int k = 0; k < K; ++k)
    for (int c = 0; c < ncomp; ++c) {
      const int q = k * ncomp + c;
      const double x = exact[(size_t)s * K * ncomp + q];
      const double y = approx[((size_t)s * n_deg + di) * K * ncomp + q];
      e += (x - y) * (x - y);
      const double rv = ref ? ref[(size_t)c * nt + tgt_orig[(size_t)s * K + k]] : x;
      r += rv * rv;
    }
  out[i] = (float)log10(sqrt(e / (r > 1e-300 ? r : 1e-300)) + 1e-30);
}

__global__ void k_fill_int(int n, int value, int* dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = value;
}

}  // namespace

// ---- launchers -----------------------------------------------------------------
int selector_param_count() { return kParams; }

cudaError_t launch_far_evals(int dim, int n_pc, int n_cp, int n_cc, int conv0, int n_conv, int n_conv_cc,
                             const int* deg, const int* pc_tcount, const int* cp_scount, const int* pc_direct,
                             unsigned long long* evals, int* hist, cudaStream_t s) {
  const int n = n_pc + n_cp + n_cc;
  if (n <= 0) return cudaSuccess;
  k_far_evals<<<(n + 255) / 256, 256, 0, s>>>(dim, n_pc, n_cp, n_cc, conv0, n_conv, n_conv_cc, deg, pc_tcount,
                                              cp_scount, pc_direct, evals, hist);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_audit_compare(int n, int ncomp, int nt, const int* audit_sorted, const int* perm,
                                 const double* out, const double* audit_out, double* sums, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_audit_compare<<<(n + 255) / 256, 256, 0, s>>>(n, ncomp, nt, audit_sorted, perm, out, audit_out, sums);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_error_samples(const SampleArgs& a, float* log10_err, cudaStream_t s) {
  if (a.n <= 0) return cudaSuccess;
  const int md = a.deg_lo + a.n_deg;  // highest degree + 1
  const size_t shm = sizeof(double) * a.ncomp * (a.dim == 3 ? md * md * md : md * md);
  if (a.dim == 2) {
    k_sample_exact<2><<<a.n, 256, 0, s>>>(a);
    cudaFuncSetAttribute(k_sample_approx<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    k_sample_approx<2><<<a.n * a.n_deg, 256, shm, s>>>(a);
  } else {
    k_sample_exact<3><<<a.n, 256, 0, s>>>(a);
    cudaFuncSetAttribute(k_sample_approx<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm);
    k_sample_approx<3><<<a.n * a.n_deg, 256, shm, s>>>(a);
  }
  const int m = a.n * a.n_deg;
  k_sample_errors<<<(m + 255) / 256, 256, 0, s>>>(a.n, a.n_deg, a.K, a.ncomp, a.exact, a.approx, a.ref, (int)a.nt,
                                                  a.tgt_orig, log10_err);
  count_launch(3);
  return cudaGetLastError();
}

cudaError_t launch_fill_int(int n, int value, int* dst, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_fill_int<<<(n + 255) / 256, 256, 0, s>>>(n, value, dst);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_panel_desc(int dim, int n, int P, const double* psw, float* desc, cudaStream_t s) {
  if (P <= 0) return cudaSuccess;
  k_panel_desc<<<P, 256, 0, s>>>(dim, n, P, psw, desc);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_pair_features(int n_pairs, const int* ptype, const int* ptgt, const int* psrc, const DevPanel* pt,
                                 const DevPanel* ps, double root_radius, double eps, const float* desc_s,
                                 int n_points, const double4* pts, double* gsum, float* feat, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(gsum, 0, 2 * sizeof(double), s);
  if (e != cudaSuccess) return e;
  if (n_points > 0) {
    k_global_sums<<<296, 256, 0, s>>>(n_points, pts, gsum);
    count_launch();
  }
  if (n_pairs <= 0) return cudaGetLastError();
  k_pair_features<<<(n_pairs + 127) / 128, 128, 0, s>>>(n_pairs, ptype, ptgt, psrc, pt, ps, root_radius, eps, desc_s,
                                                        gsum, feat);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_mlp_infer(int n, const void* w_bf16, const float* norm, const float* feat, float* out,
                             int* status, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  MlpNorm nrm;
  for (int k = 0; k < kF; ++k) {
    nrm.xm[k] = norm[k];
    nrm.xs[k] = norm[kF + k] > 0 ? norm[kF + k] : 1.f;
  }
  nrm.ym = norm[2 * kF];
  nrm.ys = norm[2 * kF + 1] > 0 ? norm[2 * kF + 1] : 1.f;
  // Tiles of 128 pairs; two CTAs per SM, each looping over its tiles (the
  // weights are staged once per CTA). The shared-memory opt-in is set once
  // per device.
  int dev = 0, sms = 148;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  static std::atomic<uint64_t> opted{0};
  const uint64_t bit = 1ull << (dev & 63);
  if (!(opted.load(std::memory_order_acquire) & bit)) {
    e = cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmemBytes);
    if (e != cudaSuccess) return e;
    opted.fetch_or(bit, std::memory_order_release);
  }
  const int tiles = (n + kTcM - 1) / kTcM;
  const int grid = std::max(1, std::min(tiles, 2 * sms));
  k_mlp_infer<<<grid, kTcM, kTcSmemBytes, s>>>(n, (const __nv_bfloat16*)w_bf16, nrm, feat, out, status);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_choose_leaf_pairs(int n, int n_cc, int dim, int pc0, int cc0, const float* pred, float log10_target,
                                     int lo, int hi, int cost_rule, const int* pc_tcount, const int* pc_direct,
                                     const int* weight, float inv_cbar, float inv_wbar, int* deg, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_choose_leaf_pairs<<<(n + 255) / 256, 256, 0, s>>>(n, n_cc, dim, pc0, cc0, pred, log10_target, lo, hi, cost_rule,
                                                      pc_tcount, pc_direct, weight, inv_cbar, inv_wbar, deg);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_choose_two_forms(int n, int dim, const int* idx, const int* coef, int off_first, int cc0,
                                   const float* pred, float log10_target, int lo, int hi, int cost_rule,
                                   const int* weight, float inv_cbar, float inv_wbar, int* deg, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_choose_two_forms<<<(n + 255) / 256, 256, 0, s>>>(n, dim, idx, coef, off_first, cc0, pred, log10_target, lo, hi,
                                                     cost_rule, weight, inv_cbar, inv_wbar, deg);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_choose_degrees(int n, const float* pred, float log10_target, int lo, int hi, int dim, int conv0,
                                  int n_pc, const int* pc_direct, int* deg, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_choose_degrees<<<(n + 255) / 256, 256, 0, s>>>(n, pred, log10_target, lo, hi, dim, conv0, n_pc, pc_direct, deg);
  count_launch();
  return cudaGetLastError();
}

cudaError_t launch_choose_degrees_cost(int n, int dim, int n_pc, int n_cp, int conv0, const float* pred,
                                       float log10_target, int lo, int hi, const int* pc_tcount, const int* cp_scount,
                                       const int* pc_direct, const int* weight, float inv_cbar, float inv_wbar,
                                       int* deg, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_choose_degrees_cost<<<(n + 255) / 256, 256, 0, s>>>(n, dim, n_pc, n_cp, conv0, pred, log10_target, lo, hi,
                                                        pc_tcount, cp_scount, pc_direct, weight, inv_cbar, inv_wbar,
                                                        deg);
  count_launch();
  return cudaGetLastError();
}

}  // namespace btk

using namespace btk;

extern "C" {

int btk_selector_param_count(void) { return kParams; }

btk_status btk_mlp_forward(const void* w_bf16, int n, const float* xn, float* yn, btk_stream_t stream) {
  BTK_CHECK(w_bf16 && n >= 0 && (n == 0 || (xn && yn)), BTK_ERR_INVALID_ARGUMENT, "btk_mlp_forward: bad argument");
  if (n == 0) return BTK_OK;
  const size_t shm = sizeof(float) * kParams;
  BTK_CUDA(cudaFuncSetAttribute(k_mlp_forward_n, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
  k_mlp_forward_n<<<(n + 127) / 128, 128, shm, (cudaStream_t)stream>>>(n, (const __nv_bfloat16*)w_bf16, xn, yn);
  count_launch();
  BTK_CUDA(cudaGetLastError());
  return BTK_OK;
}

btk_status btk_mlp_gradient(const void* w_bf16, int n, const float* xn, const float* tn, const float* mask,
                            float* grad, float* loss, float* work, btk_stream_t stream) {
  BTK_CHECK(w_bf16 && n > 0 && xn && tn && mask && grad && loss && work, BTK_ERR_INVALID_ARGUMENT,
            "btk_mlp_gradient: bad argument");
  cudaStream_t st = (cudaStream_t)stream;
  float* h1 = work;
  float* h2 = h1 + (size_t)n * kH;
  float* d1 = h2 + (size_t)n * kH;
  float* d2 = d1 + (size_t)n * kH;
  float* d3 = d2 + (size_t)n * kH;
  // normalisation of the loss: the number of unmasked targets is taken as
  // n * outputs (masked entries contribute zero).
  const float inv = 1.f / (float)((size_t)n * kO);
  BTK_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), st));
  const size_t shm = sizeof(float) * kParams;
  BTK_CUDA(cudaFuncSetAttribute(k_mlp_backprop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
  k_mlp_backprop<<<(n + 127) / 128, 128, shm, st>>>(n, (const __nv_bfloat16*)w_bf16, xn, tn, mask, inv, h1, h2, d1,
                                                    d2, d3, loss);
  count_launch();
  k_mlp_wgrad<<<(kParams + 127) / 128, 128, 0, st>>>(n, xn, h1, h2, d1, d2, d3, grad);
  count_launch();
  BTK_CUDA(cudaGetLastError());
  return BTK_OK;
}

btk_status btk_mlp_adam(float* master, void* w_bf16, const float* grad, float* m, float* v, int step, float lr,
                        btk_stream_t stream) {
  BTK_CHECK(master && w_bf16 && grad && m && v && step >= 1, BTK_ERR_INVALID_ARGUMENT, "btk_mlp_adam: bad argument");
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  k_adam<<<(kParams + 127) / 128, 128, 0, (cudaStream_t)stream>>>(master, (__nv_bfloat16*)w_bf16, grad, m, v, lr, b1,
                                                                  b2, 1e-8f, c1, c2);
  count_launch();
  BTK_CUDA(cudaGetLastError());
  return BTK_OK;
}

}  // extern "C"
