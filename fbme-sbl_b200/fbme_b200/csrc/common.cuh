// Common device helpers for the FBME sm_100a kernels: complex arithmetic,
// deterministic reductions, mbarrier / bulk-copy / tcgen05 PTX wrappers.
//
// Every wait on an mbarrier is bounded by a clock deadline.  A wait that
// runs out records FBME_STATUS_TIMEOUT in the launch's status word and
// returns false; callers then skip the remaining work, drain what they
// issued and release tensor memory, so the context stays usable.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../../include/fbme_b200.h"

#define FBME_DEV __device__ __forceinline__

namespace fbme {

// SMs of the current device (persistent grids size to it).
static inline int sm_count() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1)
      n = 148;
  }
  return n;
}

// ---------------------------------------------------------------------------
// complex helpers (interleaved complex64 as float2)
// ---------------------------------------------------------------------------
FBME_DEV float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
FBME_DEV float2 cmulc(float2 a, float2 b) {  // conj(a) * b
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
FBME_DEV float abs2(float2 a) { return a.x * a.x + a.y * a.y; }
// |z|^2 computed as hypot(z)^2, the way ``z.abs().square()`` forms it.
FBME_DEV float abs_sq(float2 a) {
  float h = hypotf(a.x, a.y);
  return h * h;
}

// ---------------------------------------------------------------------------
// warp / block reductions (fixed order => bit-reproducible run to run)
// ---------------------------------------------------------------------------
template <typename T>
FBME_DEV T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
FBME_DEV float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum over the block of one double per thread; result valid in thread 0.
// ``scratch`` holds one double per warp.
FBME_DEV double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) r += scratch[w];
  }
  return r;
}

FBME_DEV void record_status(int* status, int code) {
  if (status) atomicOr(status, code);
}

// ---------------------------------------------------------------------------
// shared-memory address / mbarrier / bulk copy
// ---------------------------------------------------------------------------
FBME_DEV uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

FBME_DEV void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
FBME_DEV void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
FBME_DEV void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}"
               ::"r"(smem_u32(bar)) : "memory");
}
FBME_DEV void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}"
               ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
FBME_DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// Bounded wait: ~0.5 s of SM clock at most by default; launches may pass a
// shorter limit.
constexpr long long kWaitCycles = 1000000000LL;
FBME_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, int* status, long long limit = kWaitCycles) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) {
      record_status(status, FBME_STATUS_TIMEOUT);
      return false;
    }
  }
  return true;
}

// Untiled bulk copy global -> shared completing on an mbarrier.
FBME_DEV void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst_smem)), "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// Make this thread's generic-proxy shared-memory writes visible to the
// async proxy (tensor-core operand reads).
FBME_DEV void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---------------------------------------------------------------------------
// tcgen05 (5th-generation tensor core, tensor memory)
// ---------------------------------------------------------------------------
FBME_DEV void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               ::"r"(smem_u32(dst_smem)), "r"(ncols) : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
FBME_DEV void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
FBME_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
FBME_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, kind::f16 (bf16 inputs, f32 accumulate).
FBME_DEV void umma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate) : "memory");
}
// Arrive on an mbarrier once every tcgen05.mma issued so far by this thread
// has completed.
FBME_DEV void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(smem_u32(bar)) : "memory");
}

// 32 lanes x 32 bit, 16 consecutive columns per thread.
FBME_DEV void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Issue a 16-column TMEM load without waiting (pair with tmem_wait_ld).
FBME_DEV void tmem_ld16_async(uint32_t taddr, float* v) {
  uint32_t* r = reinterpret_cast<uint32_t*>(v);
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// Wait for outstanding TMEM loads; `v` (the destination of the last async
// load) is an in/out operand so no use of it can be scheduled earlier.
FBME_DEV void tmem_wait_ld(float* v) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+f"(v[0]), "+f"(v[1]), "+f"(v[2]), "+f"(v[3]), "+f"(v[4]), "+f"(v[5]),
                 "+f"(v[6]), "+f"(v[7]), "+f"(v[8]), "+f"(v[9]), "+f"(v[10]), "+f"(v[11]),
                 "+f"(v[12]), "+f"(v[13]), "+f"(v[14]), "+f"(v[15])
               :
               : "memory");
}

// Shared-memory matrix descriptor, K-major operand, 128-byte swizzle:
// 8-row x 128-byte swizzle atoms stacked at 1024-byte stride (SBO); the
// leading-byte offset is unused for this layout.  Version field = 1.
FBME_DEV uint64_t sw128_desc(uint32_t smem_addr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((smem_addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>(1u) << 16;                 // LBO (unused) = 16 B
  d |= static_cast<uint64_t>(1024u >> 4) << 32;         // SBO = 1024 B
  d |= static_cast<uint64_t>(1u) << 46;                 // descriptor version
  d |= static_cast<uint64_t>(2u) << 61;                 // SWIZZLE_128B
  return d;
}

// Instruction descriptor: bf16 x bf16 -> f32, both operands K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4)                                     // D format F32
         | (1u << 7)                                   // A format BF16
         | (1u << 10)                                  // B format BF16
         | (static_cast<uint32_t>(n >> 3) << 17)       // N / 8
         | (static_cast<uint32_t>(m >> 4) << 24);      // M / 16
}

// Byte offset of element (row, k) (bf16, k in [0, 64)) inside a K-major
// SW128 tile whose rows are 128 bytes: the 16-byte chunk index is XORed
// with (row mod 8).
__host__ __device__ inline uint32_t sw128_offset(uint32_t row, uint32_t k) {
  const uint32_t byte = k * 2u;
  return row * 128u + ((((byte >> 4) ^ (row & 7u)) & 7u) << 4) + (byte & 15u);
}

}  // namespace fbme
