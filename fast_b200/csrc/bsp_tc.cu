// bsp_tc.cu - B-spline / NURBS solid stiffness on the tensor cores, one
// launch per colour (the element itself is tc_bsp_body.cuh).  One CTA of 256
// threads takes the elements of one colour in turn (grid-stride).
#include <cstdint>

#include "elem_common.cuh"
#include "internal.h"
#include "tc_bsp_body.cuh"

namespace fastgpu {

namespace {

// two CTAs per SM where their shared memory fits (registers held to 128)
template <int PR, int PS, int PT, int NG1, int LPC>
__global__ void __launch_bounds__(tcb::kThreads, tcb::BspTc<PR, PS, PT, NG1, LPC>::bytes <= 116 * 1024 ? 2 : 1)
    bsp_tc_kernel(ElemArgs A, float *__restrict__ K32) {
  using S = tcb::BspTc<PR, PS, PT, NG1, LPC>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t bars[2];   // one per operand buffer
  __shared__ uint32_t tmem_sh;
  __shared__ int fail_sh;
  tcb::Cta c = tcb::cta_begin(S::TCOLS, bars, &tmem_sh, &fail_sh);
  tcb::tc_bsp_setup<PR, PS, PT, NG1, LPC>(sm);
  bool ok = true;
  // A.split (1, or S::MT: the element's two tiles on two CTAs) parts per element
  const int np = A.split > 1 ? S::MT : 1;
  for (int64_t w = blockIdx.x; ok && w < A.ne * np; w += gridDim.x) {
    const int64_t it = w / np;
    ok = tcb::tc_bsp_element<PR, PS, PT, NG1, LPC>(A, K32, sm, c, it, A.index ? (int64_t)A.index[it] : A.offset + it,
                                                  (int)(w - it * np), np);
  }
  tcb::cta_end(c, S::TCOLS, A.status);
}

template <int PR, int PS, int PT, int NG1, int LPC>
cudaError_t run_bsp_tc(Ctx &c, ElemArgs a, int64_t count, float *K32) {
  if (count <= 0) return cudaSuccess;
  using S = tcb::BspTc<PR, PS, PT, NG1, LPC>;
  auto kern = bsp_tc_kernel<PR, PS, PT, NG1, LPC>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, tcb::kThreads, S::bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (per_sm * S::TCOLS > 512) per_sm = 512 / S::TCOLS;
  per_sm = elem_per_sm(c, per_sm, a.ctas_per_sm);
  const int64_t slots = (int64_t)per_sm * c.sm_count;
  // two-tile elements go to two CTAs each when a colour does not fill the GPU
  a.split = (S::MT > 1 && count < slots) ? S::MT : 1;
  int64_t grid = slots;
  if (grid > count * a.split) grid = count * a.split;
  a.ne = count;
  kern<<<(unsigned)grid, tcb::kThreads, S::bytes, c.stream>>>(a, K32);
  c.launches++;
  return cudaGetLastError();
}

}  // namespace

bool bsp_tc_supported(const int pd[3], int ngp) {
  return (pd[0] == 2 && pd[1] == 2 && pd[2] == 2 && (ngp == 3 || ngp == 4)) ||
         (pd[0] == 3 && pd[1] == 3 && (pd[2] == 3 || pd[2] == 2) && ngp == 4);
}

// tensor-core stiffness of one colour of a B-spline bucket into the FP32
// blocks K32 (or, with K32 null, the element matrices into a.Ke_out)
cudaError_t launch_bsp_tc(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, float *K32) {
  a.span = B.d_span;
  for (int d = 0; d < 3; d++) a.bas[d] = B.d_bas + B.bas_off[d];
  a.wt = B.d_wt;
  a.rational = B.rational;
  const int ng = B.ngp[0];
  const int *p = B.pd;
  if (p[0] == 2 && p[1] == 2 && p[2] == 2 && ng == 3) return run_bsp_tc<2, 2, 2, 3, 3>(c, a, count, K32);
  if (p[0] == 2 && p[1] == 2 && p[2] == 2 && ng == 4) return run_bsp_tc<2, 2, 2, 4, 2>(c, a, count, K32);
  if (p[0] == 3 && p[1] == 3 && p[2] == 3 && ng == 4) return run_bsp_tc<3, 3, 3, 4, 1>(c, a, count, K32);
  if (p[0] == 3 && p[1] == 3 && p[2] == 2 && ng == 4) return run_bsp_tc<3, 3, 2, 4, 1>(c, a, count, K32);
  return cudaErrorNotSupported;
}

}  // namespace fastgpu
