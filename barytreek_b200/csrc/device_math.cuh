// Device arithmetic and data-movement helpers for sm_100a.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace btk {

// ---------------------------------------------------------------------------
// FP64 reciprocal square root and reciprocal for the pairwise kernels.
//
// Seed: the FP32 approximation rsqrt.approx.f32 / rcp.approx.f32 (one MUFU op)
// of the FP32 number that shares x's exponent and top 23 mantissa bits. The
// FP32 bit pattern is built from x's two words by integer re-biasing of the
// exponent (11-bit bias 1023 -> 8-bit bias 127: a 3-bit funnel shift of the
// high word with the top bits of the low word, then + 128 << 23 in the 9-bit
// field the shift leaves), and the FP32 result is widened the same way in
// reverse. No floating-point conversion instruction is issued. The seed's
// relative error e0 is the truncation (<= 2^-23) plus the approximation's
// own (about 2^-23), so |e0| <~ 2.5e-7.
//
// Refinement: one Newton step, which squares the relative error:
//   rsqrt: e = 1 - x y^2, y' = y + (y/2) e   -> error 1.5 e0^2 <~ 1e-13 (4 FP64 ops;
//          forming y/2 from the seed with integer operations instead measured
//          2.5 % slower in the FP64 interaction kernel)
//   rcp:   e = 1 - x y,   y' = y + y e       -> error e0^2 <~ 7e-14     (2 FP64 ops)
// far below the 1e-12 agreement with the reference that the FP64 path keeps.
//
// Domain: x in the FP32 normal range [2^-126, 2^127]. The kernels guarantee it
// with eps^2 >= 2^-126; callers with smaller eps use the guarded variants.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fp32_seed_arg(double x) {
  return __int_as_float(__funnelshift_l(__double2loint(x), __double2hiint(x), 3) + 0x40000000);
}
__device__ __forceinline__ double fp64_from_seed(float yf) {
  const int yb = __float_as_int(yf);
  return __hiloint2double((yb >> 3) + 0x38000000, yb << 29);
}

__device__ __forceinline__ double rsqrt_fp64(double x) {
  float yf;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(fp32_seed_arg(x)));
  const double y = fp64_from_seed(yf);
  const double e = fma(-x, y * y, 1.0);
  return fma(0.5 * y, e, y);
}

// Same, extended to x = 0 (-> +inf, matching 1/sqrt(0)) and to x below the
// FP32 normal range (rare: only with eps^2 < 2^-126 and near-coincident points).
__device__ __forceinline__ double rsqrt_fp64_guarded(double x) {
  if (x < 1.1754943508222875e-38) return x == 0.0 ? __longlong_as_double(0x7ff0000000000000LL) : 1.0 / sqrt(x);
  return rsqrt_fp64(x);
}

// FP64 reciprocal of a positive x in the FP32 normal range (seed and Newton
// step as above).
__device__ __forceinline__ double rcp_fp64_pos(double x) {
  float yf;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(fp32_seed_arg(x)));
  const double y = fp64_from_seed(yf);
  return fma(y, fma(-x, y, 1.0), y);
}

__device__ __forceinline__ double rcp_fp64_pos_guarded(double x) {
  if (x < 1.1754943508222875e-38) return x == 0.0 ? __longlong_as_double(0x7ff0000000000000LL) : 1.0 / x;
  return rcp_fp64_pos(x);
}

// FP32 hardware approximations used by the mixed-precision kernels.
__device__ __forceinline__ float rsqrt_fp32(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_fp32(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ---------------------------------------------------------------------------
// mbarrier + TMA bulk copies (cp.async.bulk, no tensor map, no multicast).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each poll may itself suspend
// for a hardware-chosen interval) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Global -> shared bulk copy completing on `bar`. dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ---------------------------------------------------------------------------
// tcgen05 (5th-generation tensor cores): TMEM allocation, shared-memory
// operand descriptors, UMMA issue, completion and TMEM loads, cta_group::1.
// ---------------------------------------------------------------------------
// Allocates ncols TMEM columns (a power of two >= 32) for the CTA; the whole
// warp executes it and the base address lands in *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Orders this thread's generic-proxy shared-memory writes before the tensor
// cores (async proxy) read them.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Descriptor of a K-major operand tile in shared memory without swizzle: core
// matrices of 8 rows x 16 bytes (each row's 16 bytes contiguous), lbo = byte
// distance between the two 16-byte K halves of one 32-byte MMA K step, sbo =
// byte distance between consecutive groups of 8 rows; descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc_kmajor(const void* tile, uint32_t lbo, uint32_t sbo) {
  const uint32_t a = smem_addr(tile);
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with BF16 A and B (both K-major) and an
// FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// D[tmem] = A * B^T (+ D when accumulate), issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
  const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3)
      : "memory");
}

// The mbarrier receives one arrival when every MMA this thread issued before
// has completed (its shared-memory reads included).
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

// 16 consecutive 32-bit TMEM columns of this thread's lane (warp w reads lanes
// 32w..32w+31; taddr carries the lane in bits 31..16), then waits for them.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  // the registers pass through the wait, so no use of them is scheduled before it
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15])
               :
               : "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

}  // namespace btk
