// elem_tc.cu - element stiffness on the tensor cores for hex buckets, one
// launch per colour (the element itself is tc_hex_body.cuh: tcgen05.mma
// kind::tf32 on TF32 operands split in three, FP32 accumulators in tensor
// memory, sm_100a); the tensor-core stiffness of a whole mesh
// (launch_assemble_tc) and its element matrices.
//
// One CTA of 256 threads takes the elements of one colour in turn
// (grid-stride), with the bucket's Gauss tables brought in once.  Elements
// of a colour share no node, so the scatter needs no atomics and K is
// bit-identical from run to run.
#include <cstdint>

#include "elem_common.cuh"
#include "internal.h"
#include "tc_common.cuh"
#include "tc_hex_body.cuh"

namespace fastgpu {

// bsp_tc.cu
bool bsp_tc_supported(const int pd[3], int ngp);
cudaError_t launch_bsp_tc(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, float *K32);

namespace {

using tcb::kThreads;

// elements sharing one 128-row operand tile per pass: five hex8 or two hex20
template <int NN> constexpr int kEpt = 128 / (3 * NN);

template <int NN, int NG>
__global__ void __launch_bounds__(kThreads, 1) elem_tc_kernel(ElemArgs A, float *__restrict__ K32) {
  constexpr int EPT = kEpt<NN>;
  using S = tcb::TcHex<NN, NG, EPT>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t bars[2];   // [0] bulk copies, [1] MMAs
  __shared__ uint32_t tmem_sh;
  __shared__ int fail_sh;
  tcb::Cta c = tcb::cta_begin(S::TCOLS, bars, &tmem_sh, &fail_sh);
  bool ok = tcb::tc_hex_setup<NN, NG, EPT>(A, sm, c);
  // pass k of this CTA takes items (blockIdx.x + k gridDim.x) EPT .. + EPT-1
  for (int64_t it0 = (int64_t)blockIdx.x * EPT; ok && it0 < A.ne; it0 += (int64_t)gridDim.x * EPT) {
    const int nv = (int)(A.ne - it0 < EPT ? A.ne - it0 : EPT);
    int64_t its[EPT], es[EPT];
#pragma unroll
    for (int j = 0; j < EPT; j++) {
      its[j] = it0 + (j < nv ? j : 0);
      es[j] = A.index ? (int64_t)A.index[its[j]] : A.offset + its[j];
    }
    ok = tcb::tc_hex_elements<NN, NG, EPT>(A, K32, sm, c, its, es, nv);
  }
  tcb::cta_end(c, S::TCOLS, A.status);
}

template <int NN, int NG>
cudaError_t run_tc(Ctx &c, ElemArgs a, int64_t count, float *K32) {
  if (count <= 0) return cudaSuccess;
  using S = tcb::TcHex<NN, NG, kEpt<NN>>;
  auto kern = elem_tc_kernel<NN, NG>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, S::bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  // tensor-memory columns of the CTAs resident on one SM stay within its 512
  if (per_sm * S::TCOLS > 512) per_sm = 512 / S::TCOLS;
  per_sm = elem_per_sm(c, per_sm, a.ctas_per_sm);
  int64_t grid = (int64_t)per_sm * c.sm_count;
  const int64_t passes = (count + kEpt<NN> - 1) / kEpt<NN>;
  if (grid > passes) grid = passes;
  a.ne = count;
  kern<<<(unsigned)grid, kThreads, S::bytes, c.stream>>>(a, K32);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t dispatch_tc(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, float *K32) {
  if (B.type == FAST_ELEM_HEX8) {
    switch (B.ng) {
      case 1: return run_tc<8, 1>(c, a, count, K32);
      case 8: return run_tc<8, 8>(c, a, count, K32);
      case 27: return run_tc<8, 27>(c, a, count, K32);
      default: break;
    }
  } else if (B.type == FAST_ELEM_HEX20) {
    switch (B.ng) {
      case 8: return run_tc<20, 8>(c, a, count, K32);
      case 27: return run_tc<20, 27>(c, a, count, K32);
      case 64: return run_tc<20, 64>(c, a, count, K32);
      default: break;
    }
  }
  return cudaErrorNotSupported;
}

ElemArgs tc_args(Ctx &c, const Bucket &B) {
  ElemArgs a{};
  a.conn = B.d_conn;
  a.E = B.d_E;
  a.nu = B.d_nu;
  a.slot = B.d_slot;
  a.X = c.d_X;
  a.fix = c.d_fix;
  a.dN = B.d_dN;
  a.w = B.d_w;
  a.status = c.d_status;
  a.ctas_per_sm = B.tune_tc_ctas;
  return a;
}

__global__ void zero_fixed_identity32(int64_t nnode, const uint8_t *fix, const int32_t *diag, float *K) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  const uint8_t f = fix[n];
  if (!f) return;
  const int32_t d = diag[n];
  if (d < 0) return;
  for (int i = 0; i < 3; i++)
    if ((f >> i) & 1) K[(int64_t)d * 9 + 4 * i] = 1.0f;
}

}  // namespace

// Buckets the tensor-core stiffness supports: small-strain hex8 / hex20, and
// small-strain B-spline solids of degree (2,2,2) or (3,3,3) / (3,3,2)
// (bsp_tc.cu).
bool tc_supported(const Bucket &B) {
  if (B.tl) return false;
  if (B.type == FAST_ELEM_HEX8) return B.ng == 1 || B.ng == 8 || B.ng == 27;
  if (B.type == FAST_ELEM_HEX20) return B.ng == 8 || B.ng == 27 || B.ng == 64;
  if (B.type == FAST_ELEM_BSP_SOLID) return bsp_tc_supported(B.pd, B.ngp[0]);
  return false;
}

// The FP32 stiffness K32 [nnzb][3][3] of every bucket: zero, unit diagonal on
// fixed DOFs (the stiffness slot's convention), then one launch per colour;
// the elements touching a tied node keep their FP64 element matrices (the
// scratch buffer the element-by-element residual reuses) and are scattered
// into K32 by the tied-interface kernel.
cudaError_t launch_assemble_tc(Ctx &c, float *K32) {
  cudaError_t e = cudaSuccess;
  if (!c.use_first_touch()) {  // (with first-touch flags every block is stored by its first writer)
    e = cudaMemsetAsync(K32, 0, sizeof(float) * 9 * (size_t)c.nnzb, c.stream);
    if (e != cudaSuccess) return e;
    zero_fixed_identity32<<<(unsigned)((c.nnode + 255) / 256), 256, 0, c.stream>>>(c.nnode, c.d_fix, c.d_diag, K32);
    c.launches++;
  }
  if (c.persist_asm && persist_supported(c)) {
    // every bucket in one persistent launch
    e = launch_persist_elements(c, K32);
    if (e != cudaSuccess) return e;
    return launch_tied_assemble32(c, K32);
  }
  for (size_t b = 0; b < c.buckets.size(); b++) {
    const Bucket &B = c.buckets[b];
    if (!tc_supported(B)) return cudaErrorNotSupported;
    for (size_t k = 0; k + 1 < B.color_off.size(); k++) {
      ElemArgs a = tc_args(c, B);
      a.offset = B.color_off[k];
      if (c.use_first_touch()) {
        a.first = B.d_first;
        a.fw = first_words(B.nn);
      }
      const int64_t cnt = B.color_off[k + 1] - B.color_off[k];
      e = B.type == FAST_ELEM_BSP_SOLID ? launch_bsp_tc(c, B, a, cnt, K32) : dispatch_tc(c, B, a, cnt, K32);
      if (e != cudaSuccess) return e;
    }
  }
  // elements with a tied node: FP64 element matrices, scattered as T^T K_e T
  return launch_tied_assemble32(c, K32);
}

cudaError_t launch_assemble_tc_bucket(Ctx &c, size_t b, float *K32) {
  const Bucket &B = c.buckets[b];
  if (!tc_supported(B)) return cudaErrorNotSupported;
  for (size_t k = 0; k + 1 < B.color_off.size(); k++) {
    ElemArgs a = tc_args(c, B);
    a.offset = B.color_off[k];
    if (c.use_first_touch()) {
      a.first = B.d_first;
      a.fw = first_words(B.nn);
    }
    const int64_t cnt = B.color_off[k + 1] - B.color_off[k];
    cudaError_t e = B.type == FAST_ELEM_BSP_SOLID ? launch_bsp_tc(c, B, a, cnt, K32) : dispatch_tc(c, B, a, cnt, K32);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Element matrices of the tensor-core path, dense FP64 [count][3nn][3nn], for
// the colour-sorted positions packed as [count] int32 after the matrices.
cudaError_t launch_element_matrices_tc(Ctx &c, int bucket, int64_t count, double *d_out_and_index) {
  const Bucket &B = c.buckets[bucket];
  if (!tc_supported(B)) return cudaErrorNotSupported;
  const int nd = 3 * B.nn;
  ElemArgs a = tc_args(c, B);
  a.Ke_out = d_out_and_index;
  a.index = reinterpret_cast<const int32_t *>(d_out_and_index + (size_t)count * nd * nd);
  return B.type == FAST_ELEM_BSP_SOLID ? launch_bsp_tc(c, B, a, count, nullptr) : dispatch_tc(c, B, a, count, nullptr);
}

}  // namespace fastgpu
