// tc_common.cuh - sm_100a tensor-core plumbing shared by the tcgen05 kernels
// (private to libfastgpu): mbarrier waits with a time limit, tcgen05 fences,
// and the shared-memory / instruction descriptors of tcgen05.mma for
// K-major operands without swizzle.
//
// Canonical K-major, non-swizzled operand layout used throughout: the matrix
// is cut into core matrices of 8 rows x 16 bytes, each stored as 128
// contiguous bytes (row-major inside); the core matrices of one 8-row group
// follow each other along K (leading-dimension byte offset LBO = 128), and
// successive 8-row groups are SBO = (K bytes / 16) * 128 bytes apart.  One
// MMA consumes 32 bytes of K (16 BF16 or 8 TF32 values): two core matrices.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace fastgpu {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// true once the phase with this parity has completed, false after limit_ns
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const uint64_t t0 = gtimer();
  while (!mbar_try(bar, parity))
    if (gtimer() - t0 > limit_ns) return false;
  return true;
}

// arrive on the barrier and announce `bytes` of asynchronous transfer
__device__ __forceinline__ void mbar_arrive_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// untiled bulk copy global -> shared (both 16-byte aligned, bytes a multiple
// of 16), completion counted on the barrier; the source is this GPU's memory
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// shared-memory matrix descriptor, K-major, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100
  return d;                // base offset 0, absolute LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16 / kind::tf32: D FP32, A and B of the
// given type (0 F16, 1 BF16, 2 TF32), both K-major, M x N
__host__ __device__ constexpr uint32_t idesc(int M, int N, uint32_t ab_type) {
  return (1u << 4) | (ab_type << 7) | (ab_type << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
constexpr uint32_t kTypeBF16 = 1, kTypeTF32 = 2;

// one tcgen05.mma.cta_group::1 of the given kind; accumulate unless acc == 0
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t id, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(id), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// 32 lanes x 32 bits, 8 consecutive columns: thread t of the warp gets lane
// (warp's subpartition base + t), columns col..col+7
__device__ __forceinline__ void ld_32x32b_x8(uint32_t taddr, float v[8]) {
  uint32_t r0, r1, r2, r3, r4, r5, r6, r7;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3), "+r"(r4), "+r"(r5), "+r"(r6), "+r"(r7)::"memory");
  v[0] = __uint_as_float(r0); v[1] = __uint_as_float(r1); v[2] = __uint_as_float(r2); v[3] = __uint_as_float(r3);
  v[4] = __uint_as_float(r4); v[5] = __uint_as_float(r5); v[6] = __uint_as_float(r6); v[7] = __uint_as_float(r7);
}

// x (FP64) -> TF32 hi + TF32 lo with x ~ hi + lo to about 2^-22 relative
// (round-to-nearest TF32 conversion of the FP32 value, then of the remainder)
__device__ __forceinline__ void split_tf32(double x, uint32_t &hi, uint32_t &lo) {
  const float xf = (float)x;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(xf));
  const float rem = (float)(x - (double)__uint_as_float(hi));
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(rem));
}

// x (FP64) -> three TF32 parts, x ~ hi + lo + mid to about 2^-33 relative
// (each part the round-to-nearest TF32 conversion of what the earlier parts
// leave).  Of the nine partial products of x y the six down to 2^-22 |x y|
// (hi hi, hi lo, lo hi, lo lo, hi mid, mid hi) bring the product to FP32
// accuracy; the three dropped ones are below 2^-32 |x y|.
__device__ __forceinline__ void split3_tf32(double x, uint32_t &hi, uint32_t &lo, uint32_t &mid) {
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"((float)x));
  const double r1 = x - (double)__uint_as_float(hi);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"((float)r1));
  const double r2 = r1 - (double)__uint_as_float(lo);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(mid) : "f"((float)r2));
}

// The six partial products of the three-part split as (A part, B part)
// indices (0 hi, 1 lo, 2 mid), smallest first, so the accumulator takes the
// small terms before the large ones
constexpr int kSplitTerms = 6;
__device__ __forceinline__ void split_term(int t, int &pa, int &pb) {
  // (lo,lo) (hi,mid) (mid,hi) (hi,lo) (lo,hi) (hi,hi)
  constexpr int A[6] = {1, 0, 2, 0, 1, 0}, B[6] = {1, 2, 0, 1, 0, 0};
  pa = A[t];
  pb = B[t];
}

// bring the line holding p into L2 (no register result, nothing waits on it)
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// byte offset of element (row r, k) of a 4-byte K-major operand with kp
// columns in the canonical layout above
__device__ __forceinline__ uint32_t kmajor_off4(int r, int k, int kp) {
  return (uint32_t)(((r >> 3) * (kp >> 2) + (k >> 2)) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

}  // namespace tc
}  // namespace fastgpu
