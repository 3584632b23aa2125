// geom.cu - geometric stiffness at the current displacements, assembled on
// the device (launch_geom_stiffness): cControl::GeomStiffMatrix
// (ctrl/ctrl.cpp:1031-1063) over cElmParam::GeomStiff (elc/elmparam.cpp:
// 743-830) for small-strain hex buckets.  At each Gauss point the stress
// s = C B u_e (Voigt xx yy zz xy xz yz) forms the tensor sigma, and
//   G[3a+i][3b+j] += delta_ij w detJ dN_a^T sigma dN_b
// (Bnl^T S Bnl with cSolid::BnlMatrix / SMatrix, elc/anmodel.cpp:1514-1560):
// every 3x3 block is a multiple of the identity.
//
// One CTA per element, one thread per node pair (a, b); the Jacobian, the
// shape-function gradients and the stress of each Gauss point are formed
// once in shared memory.  Elements are launched colour by colour, so no two
// CTAs in flight touch the same block: the += into the target is race-free
// and the same every run.  Rows and columns of fixed DOFs stay 0.
#include <cstdint>

#include "internal.h"

namespace fastgpu {

namespace {

template <int NN, int NG>
__global__ void __launch_bounds__(NN *NN) geom_kernel(int64_t offset, const int32_t *__restrict__ conn,
                                                     const double *__restrict__ E, const double *__restrict__ nu,
                                                     const double *__restrict__ X, const double *__restrict__ U,
                                                     const double *__restrict__ dN, const double *__restrict__ w,
                                                     const int32_t *__restrict__ slot, const uint8_t *__restrict__ fix,
                                                     double sign, double *__restrict__ G, int32_t *__restrict__ status) {
  __shared__ double sx[NN][3], su[NN][3], sd[NN][3], sI[9], sS[9];
  __shared__ uint8_t sfix[NN];
  const int64_t e = offset + blockIdx.x;
  const int tid = threadIdx.x;
  if (tid < NN) {
    const int32_t n = conn[e * NN + tid];
    for (int k = 0; k < 3; k++) {
      sx[tid][k] = X[3 * (int64_t)n + k];
      su[tid][k] = U[4 * (int64_t)n + k];
    }
    sfix[tid] = fix[n];
  }
  __syncthreads();
  const int a = tid / NN, b = tid - a * NN;
  double g = 0.0;
  for (int gp = 0; gp < NG; gp++) {
    const double *d = dN + (int64_t)gp * NN * 3;
    if (tid == 0) {
      double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int k = 0; k < NN; k++)
        for (int p = 0; p < 3; p++)
          for (int q = 0; q < 3; q++) J[3 * p + q] = fma(d[3 * k + p], sx[k][q], J[3 * p + q]);
      const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                         J[2] * (J[3] * J[7] - J[4] * J[6]);
      if (!(det > 0.0)) atomicOr(status, 1);
      const double id = 1.0 / ((det != 0.0) ? det : 1.0);
      sI[0] = (J[4] * J[8] - J[5] * J[7]) * id;
      sI[1] = -(J[1] * J[8] - J[2] * J[7]) * id;
      sI[2] = (J[1] * J[5] - J[2] * J[4]) * id;
      sI[3] = -(J[3] * J[8] - J[5] * J[6]) * id;
      sI[4] = (J[0] * J[8] - J[2] * J[6]) * id;
      sI[5] = -(J[0] * J[5] - J[2] * J[3]) * id;
      sI[6] = (J[3] * J[7] - J[4] * J[6]) * id;
      sI[7] = -(J[0] * J[7] - J[1] * J[6]) * id;
      sI[8] = (J[0] * J[4] - J[1] * J[3]) * id;
      sS[0] = det * w[gp];  // the weight, until the stress replaces it
    }
    __syncthreads();
    if (tid < NN) {
      const double d0 = d[3 * tid], d1 = d[3 * tid + 1], d2 = d[3 * tid + 2];
      sd[tid][0] = sI[0] * d0 + sI[1] * d1 + sI[2] * d2;
      sd[tid][1] = sI[3] * d0 + sI[4] * d1 + sI[5] * d2;
      sd[tid][2] = sI[6] * d0 + sI[7] * d1 + sI[8] * d2;
    }
    __syncthreads();
    if (tid == 0) {
      double H[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // du_i / dx_j
      for (int k = 0; k < NN; k++)
        for (int i = 0; i < 3; i++)
          for (int j = 0; j < 3; j++) H[3 * i + j] = fma(su[k][i], sd[k][j], H[3 * i + j]);
      const double ev[6] = {H[0], H[4], H[8], H[1] + H[3], H[2] + H[6], H[5] + H[7]};
      const double En = E[e], v = nu[e];
      const double dd = (1.0 + v) * (1.0 - 2.0 * v);
      const double C00 = En * (1.0 - v) / dd, C01 = En * v / dd, Gs = 0.5 * En / (1.0 + v);
      const double s0 = C00 * ev[0] + C01 * (ev[1] + ev[2]);
      const double s1 = C00 * ev[1] + C01 * (ev[0] + ev[2]);
      const double s2 = C00 * ev[2] + C01 * (ev[0] + ev[1]);
      const double s3 = Gs * ev[3], s4 = Gs * ev[4], s5 = Gs * ev[5];
      const double c = sS[0];
      sS[0] = c * s0; sS[1] = c * s3; sS[2] = c * s4;
      sS[3] = c * s3; sS[4] = c * s1; sS[5] = c * s5;
      sS[6] = c * s4; sS[7] = c * s5; sS[8] = c * s2;
    }
    __syncthreads();
    double v = 0.0;
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const double t = sS[3 * p] * sd[b][0] + sS[3 * p + 1] * sd[b][1] + sS[3 * p + 2] * sd[b][2];
      v = fma(sd[a][p], t, v);
    }
    g += v;
    __syncthreads();  // sI, sd, sS are rewritten for the next point
  }
  const int64_t sl = (int64_t)slot[(e * NN + a) * NN + b] * 9;
  const uint8_t fa = sfix[a], fb = sfix[b];
#pragma unroll
  for (int i = 0; i < 3; i++)
    if (!((fa >> i) & 1) && !((fb >> i) & 1)) G[sl + 4 * i] += sign * g;
}

template <int NN, int NG>
cudaError_t run_geom(Ctx &c, const Bucket &B, double *G, double sign) {
  for (size_t k = 0; k + 1 < B.color_off.size(); k++) {
    const int64_t off = B.color_off[k], cnt = B.color_off[k + 1] - off;
    if (cnt <= 0) continue;
    geom_kernel<NN, NG><<<(unsigned)cnt, NN * NN, 0, c.stream>>>(off, B.d_conn, B.d_E, B.d_nu, c.d_X, c.d_disp, B.d_dN,
                                                                B.d_w, B.d_slot, c.d_fix, sign, G, c.d_status);
    c.launches++;
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_geom_stiffness(Ctx &c, double *G, double sign) {
  for (const Bucket &B : c.buckets) {
    cudaError_t e = cudaErrorInvalidValue;
    if (B.type == FAST_ELEM_HEX8 && B.ng == 8) e = run_geom<8, 8>(c, B, G, sign);
    else if (B.type == FAST_ELEM_HEX8 && B.ng == 27) e = run_geom<8, 27>(c, B, G, sign);
    else if (B.type == FAST_ELEM_HEX8 && B.ng == 1) e = run_geom<8, 1>(c, B, G, sign);
    else if (B.type == FAST_ELEM_HEX20 && B.ng == 27) e = run_geom<20, 27>(c, B, G, sign);
    else if (B.type == FAST_ELEM_HEX20 && B.ng == 8) e = run_geom<20, 8>(c, B, G, sign);
    else if (B.type == FAST_ELEM_HEX20 && B.ng == 64) e = run_geom<20, 64>(c, B, G, sign);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace fastgpu
