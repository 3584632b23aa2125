// stress.cu - Gauss-point strains and stresses at the current displacements
// (fast_gpu_gauss_stress): what cElmParam::IntPntStress (elc/elmparam.cpp:
// 859-935) returns for an isotropic small-strain solid, e = B u_e at each
// integration point (cSolid::BMatrix, elc/anmodel.cpp:1418-1447: Voigt xx yy
// zz xy xz yz, engineering shears) and s = C e (cSolid::QMatrix,
// elc/anmodel.cpp:1286-1298).  It is the per-point work FAST repeats on the
// CPU for every printed step (stress recovery).
//
// One thread per (element, Gauss point): the point's Jacobian from the
// element's coordinates, its inverse by cofactors, then the strain summed
// over the element's nodes; the threads of one element read the same nodes,
// which the L1 cache serves.
//
// fast_gpu_nodal_stress goes on to the printing step's nodal values: the
// element-nodal stresses extrapolated from the Gauss points
// (cElmParam::NodalStress with CompTRMatrix, elc/elmparam.cpp:1304-1312,
// 1444-1535) and their average at each node over the elements sharing it
// (cControl::PrintAvrNodalStress, ctrl/ctrl.cpp:2397-2440).
#include <cstdint>
#include <string>
#include <vector>

#include "internal.h"

using namespace fastgpu;

struct fast_gpu_ctx : public Ctx {};

namespace {

template <int NN, int NG>
__global__ void gauss_stress(int64_t count, const int32_t *__restrict__ index, const int32_t *__restrict__ conn,
                             const double *__restrict__ E, const double *__restrict__ nu,
                             const double *__restrict__ X, const double *__restrict__ U,
                             const double *__restrict__ dN, double *__restrict__ strain /* or NULL */,
                             double *__restrict__ stress, int32_t *__restrict__ status) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count * NG) return;
  const int64_t k = t / NG;
  const int g = (int)(t - k * NG);
  const int64_t e = index[k];
  const int32_t *en = conn + e * NN;
  const double *d = dN + (int64_t)g * NN * 3;
  double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < NN; a++) {
    const double *x = X + 3 * (int64_t)en[a];
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int q = 0; q < 3; q++) J[3 * p + q] = fma(d[3 * a + p], x[q], J[3 * p + q]);
  }
  const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                     J[2] * (J[3] * J[7] - J[4] * J[6]);
  if (!(det > 0.0)) atomicOr(status, 1);
  const double id = 1.0 / ((det != 0.0) ? det : 1.0);
  const double I[9] = {(J[4] * J[8] - J[5] * J[7]) * id,  -(J[1] * J[8] - J[2] * J[7]) * id,
                       (J[1] * J[5] - J[2] * J[4]) * id,  -(J[3] * J[8] - J[5] * J[6]) * id,
                       (J[0] * J[8] - J[2] * J[6]) * id,  -(J[0] * J[5] - J[2] * J[3]) * id,
                       (J[3] * J[7] - J[4] * J[6]) * id,  -(J[0] * J[7] - J[1] * J[6]) * id,
                       (J[0] * J[4] - J[1] * J[3]) * id};
  // displacement gradient G[i][j] = du_i/dx_j
  double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < NN; a++) {
    const double d0 = d[3 * a], d1 = d[3 * a + 1], d2 = d[3 * a + 2];
    const double gx = I[0] * d0 + I[1] * d1 + I[2] * d2;
    const double gy = I[3] * d0 + I[4] * d1 + I[5] * d2;
    const double gz = I[6] * d0 + I[7] * d1 + I[8] * d2;
    const double *u = U + 4 * (int64_t)en[a];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      G[3 * i] = fma(u[i], gx, G[3 * i]);
      G[3 * i + 1] = fma(u[i], gy, G[3 * i + 1]);
      G[3 * i + 2] = fma(u[i], gz, G[3 * i + 2]);
    }
  }
  const double ev[6] = {G[0], G[4], G[8], G[1] + G[3], G[2] + G[6], G[5] + G[7]};
  const double En = E[e], v = nu[e];
  const double dd = (1.0 + v) * (1.0 - 2.0 * v);
  const double C00 = En * (1.0 - v) / dd, C01 = En * v / dd, Gs = 0.5 * En / (1.0 + v);
  double *so = stress + t * 6;
  if (strain) {
    double *eo = strain + t * 6;
#pragma unroll
    for (int c = 0; c < 6; c++) eo[c] = ev[c];
  }
  so[0] = C00 * ev[0] + C01 * (ev[1] + ev[2]);
  so[1] = C00 * ev[1] + C01 * (ev[0] + ev[2]);
  so[2] = C00 * ev[2] + C01 * (ev[0] + ev[1]);
  so[3] = Gs * ev[3];
  so[4] = Gs * ev[4];
  so[5] = Gs * ev[5];
}

// B-spline / NURBS solids: the same per point, with the shape-function
// derivatives of the element's knot spans from the Bezier-extracted span
// tables (rational quotient N_a = B_a w_a / W as cShapeBspSolid), three
// passes over the nodes: W and dW, the Jacobian, the displacement gradient.
// A B-spline patch may be parametrised left-handed: only a zero or
// non-finite det J is flagged, as in the stiffness kernels.
template <int PR, int PS, int PT, int NG1>
__global__ void bsp_gauss_stress(int64_t count, const int32_t *__restrict__ index, const int32_t *__restrict__ conn,
                                 const double *__restrict__ E, const double *__restrict__ nu,
                                 const double *__restrict__ X, const double *__restrict__ U,
                                 const int32_t *__restrict__ span, const double *__restrict__ bas_r,
                                 const double *__restrict__ bas_s, const double *__restrict__ bas_t,
                                 const double *__restrict__ wt, int rational, double *__restrict__ strain,
                                 double *__restrict__ stress, int32_t *__restrict__ status) {
  constexpr int QR = PR + 1, QS = PS + 1, QT = PT + 1, NN = QR * QS * QT, NG = NG1 * NG1 * NG1;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= count * NG) return;
  const int64_t k = t / NG;
  const int g = (int)(t - k * NG);
  const int64_t e = index[k];
  const int gl = g % NG1, gj = (g / NG1) % NG1, gi = g / (NG1 * NG1);
  const double *br = bas_r + (size_t)span[4 * e] * NG1 * QR * 2 + gl * QR * 2;
  const double *bs = bas_s + (size_t)span[4 * e + 1] * NG1 * QS * 2 + gj * QS * 2;
  const double *bt = bas_t + (size_t)span[4 * e + 2] * NG1 * QT * 2 + gi * QT * 2;
  const int32_t *en = conn + e * NN;
  const bool rat = rational != 0;
  double W = 1.0, Wr = 0.0, Ws = 0.0, Wt = 0.0;
  if (rat) {
    W = 0.0;
    for (int a = 0; a < NN; a++) {
      const int ia = a % QR, ja = (a / QR) % QS, ka = a / (QR * QS);
      const double *fr = br + 2 * ia, *fs = bs + 2 * ja, *ft = bt + 2 * ka;
      const double w = wt ? wt[en[a]] : 1.0;
      W += fr[0] * fs[0] * ft[0] * w;
      Wr += fr[1] * fs[0] * ft[0] * w;
      Ws += fr[0] * fs[1] * ft[0] * w;
      Wt += fr[0] * fs[0] * ft[1] * w;
    }
  }
  auto dnat = [&](int a, double &d0, double &d1, double &d2) {
    const int ia = a % QR, ja = (a / QR) % QS, ka = a / (QR * QS);
    const double *fr = br + 2 * ia, *fs = bs + 2 * ja, *ft = bt + 2 * ka;
    d0 = fr[1] * fs[0] * ft[0];
    d1 = fr[0] * fs[1] * ft[0];
    d2 = fr[0] * fs[0] * ft[1];
    if (rat) {
      const double w = wt ? wt[en[a]] : 1.0;
      const double n = fr[0] * fs[0] * ft[0] * w / W;
      d0 = (d0 * w - n * Wr) / W;
      d1 = (d1 * w - n * Ws) / W;
      d2 = (d2 * w - n * Wt) / W;
    }
  };
  double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < NN; a++) {
    double d[3];
    dnat(a, d[0], d[1], d[2]);
    const double *x = X + 3 * (int64_t)en[a];
#pragma unroll
    for (int p = 0; p < 3; p++)
#pragma unroll
      for (int q = 0; q < 3; q++) J[3 * p + q] = fma(d[p], x[q], J[3 * p + q]);
  }
  const double det = J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
                     J[2] * (J[3] * J[7] - J[4] * J[6]);
  if (!(fabs(det) > 0.0) || !isfinite(det)) atomicOr(status, 1);
  const double id = 1.0 / ((det != 0.0) ? det : 1.0);
  const double I[9] = {(J[4] * J[8] - J[5] * J[7]) * id,  -(J[1] * J[8] - J[2] * J[7]) * id,
                       (J[1] * J[5] - J[2] * J[4]) * id,  -(J[3] * J[8] - J[5] * J[6]) * id,
                       (J[0] * J[8] - J[2] * J[6]) * id,  -(J[0] * J[5] - J[2] * J[3]) * id,
                       (J[3] * J[7] - J[4] * J[6]) * id,  -(J[0] * J[7] - J[1] * J[6]) * id,
                       (J[0] * J[4] - J[1] * J[3]) * id};
  double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < NN; a++) {
    double d0, d1, d2;
    dnat(a, d0, d1, d2);
    const double gx = I[0] * d0 + I[1] * d1 + I[2] * d2;
    const double gy = I[3] * d0 + I[4] * d1 + I[5] * d2;
    const double gz = I[6] * d0 + I[7] * d1 + I[8] * d2;
    const double *u = U + 4 * (int64_t)en[a];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      G[3 * i] = fma(u[i], gx, G[3 * i]);
      G[3 * i + 1] = fma(u[i], gy, G[3 * i + 1]);
      G[3 * i + 2] = fma(u[i], gz, G[3 * i + 2]);
    }
  }
  const double ev[6] = {G[0], G[4], G[8], G[1] + G[3], G[2] + G[6], G[5] + G[7]};
  const double En = E[e], v = nu[e];
  const double dd = (1.0 + v) * (1.0 - 2.0 * v);
  const double C00 = En * (1.0 - v) / dd, C01 = En * v / dd, Gs = 0.5 * En / (1.0 + v);
  double *so = stress + t * 6, *eo = strain + t * 6;
#pragma unroll
  for (int c = 0; c < 6; c++) eo[c] = ev[c];
  so[0] = C00 * ev[0] + C01 * (ev[1] + ev[2]);
  so[1] = C00 * ev[1] + C01 * (ev[0] + ev[2]);
  so[2] = C00 * ev[2] + C01 * (ev[0] + ev[1]);
  so[3] = Gs * ev[3];
  so[4] = Gs * ev[4];
  so[5] = Gs * ev[5];
}

template <int PR, int PS, int PT, int NG1>
cudaError_t run_bsp(Ctx &c, const Bucket &B, int64_t count, const int32_t *idx, double *st, double *ss) {
  constexpr int NG = NG1 * NG1 * NG1;
  const int64_t n = count * NG;
  bsp_gauss_stress<PR, PS, PT, NG1><<<(unsigned)((n + 127) / 128), 128, 0, c.stream>>>(
      count, idx, B.d_conn, B.d_E, B.d_nu, c.d_X, c.d_disp, B.d_span, B.d_bas + B.bas_off[0],
      B.d_bas + B.bas_off[1], B.d_bas + B.bas_off[2], B.d_wt, B.rational, st, ss, c.d_status);
  c.launches++;
  return cudaGetLastError();
}

template <int NN, int NG>
cudaError_t run(Ctx &c, const Bucket &B, int64_t count, const int32_t *idx, double *st, double *ss) {
  const int64_t n = count * NG;
  gauss_stress<NN, NG><<<(unsigned)((n + 127) / 128), 128, 0, c.stream>>>(count, idx, B.d_conn, B.d_E, B.d_nu, c.d_X,
                                                                          c.d_disp, B.d_dN, st, ss, c.d_status);
  c.launches++;
  return cudaGetLastError();
}

// element-nodal stresses [ne][NN][6] = TR [NN][NG] x Gauss-point stresses
// [ne][NG][6] (cElmParam::NodalStress, elc/elmparam.cpp:1304-1312): one
// thread per (element, local node)
template <int NN, int NG>
__global__ void extrapolate_to_nodes(int64_t ne, const double *__restrict__ TR, const double *__restrict__ Sg,
                                     double *__restrict__ Sn) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ne * NN) return;
  const int64_t k = t / NN;
  const int a = (int)(t - k * NN);
  const double *sg = Sg + k * NG * 6;
  const double *tr = TR + a * NG;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int g = 0; g < NG; g++) {
    const double w = tr[g];
#pragma unroll
    for (int c = 0; c < 6; c++) acc[c] = fma(w, sg[6 * g + c], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < 6; c++) Sn[t * 6 + c] = acc[c];
}

// averaged nodal stresses (cControl::PrintAvrNodalStress, ctrl/ctrl.cpp:
// 2397-2440): one thread per node gathers its (element, local node) entries
// in element order, so the sum is the reference's and the same every run
__global__ void average_at_nodes(int64_t nnode, const int64_t *__restrict__ ptr, const int64_t *__restrict__ ent,
                                 const double *__restrict__ Sn, double *__restrict__ out) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  const int64_t p0 = ptr[n], p1 = ptr[n + 1];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t p = p0; p < p1; p++) {
    const double *v = Sn + ent[p] * 6;
#pragma unroll
    for (int c = 0; c < 6; c++) acc[c] += v[c];
  }
  const double cnt = (double)(p1 - p0);
#pragma unroll
  for (int c = 0; c < 6; c++) out[n * 6 + c] = p1 > p0 ? acc[c] / cnt : 0.0;
}

// the same for any node and point count (B-spline buckets)
__global__ void extrapolate_to_nodes_n(int64_t ne, int nn, int ng, const double *__restrict__ TR,
                                       const double *__restrict__ Sg, double *__restrict__ Sn) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= ne * nn) return;
  const int64_t k = t / nn;
  const int a = (int)(t - k * nn);
  const double *sg = Sg + k * ng * 6;
  const double *tr = TR + (int64_t)a * ng;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int g = 0; g < ng; g++) {
    const double w = tr[g];
#pragma unroll
    for (int c = 0; c < 6; c++) acc[c] = fma(w, sg[6 * g + c], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < 6; c++) Sn[t * 6 + c] = acc[c];
}

// B-spline bucket: Gauss-point stresses (strains into scratch), extrapolated
// to the control points, averaged
template <int PR, int PS, int PT, int NG1>
cudaError_t run_nodal_bsp(Ctx &c, const Bucket &B, const int32_t *idx, double *Se, double *Sg, double *Sn,
                          double *avg) {
  constexpr int NG = NG1 * NG1 * NG1;
  const int64_t ne = B.ne;
  cudaError_t e = run_bsp<PR, PS, PT, NG1>(c, B, ne, idx, Se, Sg);
  if (e != cudaSuccess) return e;
  extrapolate_to_nodes_n<<<(unsigned)((ne * B.nn + 127) / 128), 128, 0, c.stream>>>(ne, B.nn, NG, B.d_tr, Sg, Sn);
  c.launches++;
  if (avg) {
    average_at_nodes<<<(unsigned)((c.nnode + 127) / 128), 128, 0, c.stream>>>(c.nnode, B.d_nptr, B.d_nent, Sn, avg);
    c.launches++;
  }
  return cudaGetLastError();
}

template <int NN, int NG>
cudaError_t run_nodal(Ctx &c, const Bucket &B, const int32_t *idx, double *Sg, double *Sn, double *avg) {
  const int64_t ne = B.ne;
  gauss_stress<NN, NG><<<(unsigned)((ne * NG + 127) / 128), 128, 0, c.stream>>>(
      ne, idx, B.d_conn, B.d_E, B.d_nu, c.d_X, c.d_disp, B.d_dN, nullptr, Sg, c.d_status);
  extrapolate_to_nodes<NN, NG><<<(unsigned)((ne * NN + 127) / 128), 128, 0, c.stream>>>(ne, B.d_tr, Sg, Sn);
  c.launches += 2;
  if (avg) {
    average_at_nodes<<<(unsigned)((c.nnode + 127) / 128), 128, 0, c.stream>>>(c.nnode, B.d_nptr, B.d_nent, Sn, avg);
    c.launches++;
  }
  return cudaGetLastError();
}

}  // namespace

#define SCK(call)                                                                 \
  do {                                                                            \
    cudaError_t _e = (call);                                                      \
    if (_e != cudaSuccess) {                                                      \
      c->err = std::string("gauss_stress: ") + #call + ": " + cudaGetErrorString(_e); \
      if (buf) cudaFree(buf);                                                     \
      return FAST_GPU_ECUDA;                                                      \
    }                                                                             \
  } while (0)

extern "C" int fast_gpu_gauss_stress(fast_gpu_ctx *c, int32_t b, int64_t first, int64_t count, double *strain,
                                     double *stress) {
  if (!c || b < 0 || b >= (int)c->buckets.size() || !strain || !stress) return FAST_GPU_EINVAL;
  const Bucket &B = c->buckets[b];
  if (first < 0 || count <= 0 || first + count > B.ne) return FAST_GPU_EINVAL;
  if (B.tl) {
    c->err = "gauss_stress: small-strain buckets only";
    return FAST_GPU_ENOTSUP;
  }
  const int ng = B.ng;
  const size_t vals = (size_t)count * ng * 6;
  double *buf = nullptr;
  SCK(cudaMalloc((void **)&buf, sizeof(double) * 2 * vals + sizeof(int32_t) * count + 16));
  std::vector<int32_t> idx(count);
  for (int64_t k = 0; k < count; k++) idx[k] = B.inv[first + k];
  int32_t *d_idx = reinterpret_cast<int32_t *>(buf + 2 * vals);
  SCK(cudaMemcpyAsync(d_idx, idx.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice, c->stream));
  SCK(cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream));
  cudaError_t e = cudaErrorInvalidValue;
  if (B.type == FAST_ELEM_HEX8 && ng == 8) e = run<8, 8>(*c, B, count, d_idx, buf, buf + vals);
  else if (B.type == FAST_ELEM_HEX8 && ng == 27) e = run<8, 27>(*c, B, count, d_idx, buf, buf + vals);
  else if (B.type == FAST_ELEM_HEX8 && ng == 1) e = run<8, 1>(*c, B, count, d_idx, buf, buf + vals);
  else if (B.type == FAST_ELEM_HEX20 && ng == 27) e = run<20, 27>(*c, B, count, d_idx, buf, buf + vals);
  else if (B.type == FAST_ELEM_HEX20 && ng == 8) e = run<20, 8>(*c, B, count, d_idx, buf, buf + vals);
  else if (B.type == FAST_ELEM_HEX20 && ng == 64) e = run<20, 64>(*c, B, count, d_idx, buf, buf + vals);
  else if (B.type == FAST_ELEM_BSP_SOLID) {
    const int *p = B.pd, g1 = B.ngp[0];
    if (p[0] == 2 && p[1] == 2 && p[2] == 2 && g1 == 3) e = run_bsp<2, 2, 2, 3>(*c, B, count, d_idx, buf, buf + vals);
    else if (p[0] == 2 && p[1] == 2 && p[2] == 2 && g1 == 4) e = run_bsp<2, 2, 2, 4>(*c, B, count, d_idx, buf, buf + vals);
    else if (p[0] == 3 && p[1] == 3 && p[2] == 3 && g1 == 4) e = run_bsp<3, 3, 3, 4>(*c, B, count, d_idx, buf, buf + vals);
    else if (p[0] == 3 && p[1] == 3 && p[2] == 2 && g1 == 4) e = run_bsp<3, 3, 2, 4>(*c, B, count, d_idx, buf, buf + vals);
    else if (p[0] == 4 && p[1] == 2 && p[2] == 4 && g1 == 5) e = run_bsp<4, 2, 4, 5>(*c, B, count, d_idx, buf, buf + vals);
    else if (p[0] == 4 && p[1] == 2 && p[2] == 2 && g1 == 5) e = run_bsp<4, 2, 2, 5>(*c, B, count, d_idx, buf, buf + vals);
    else if (p[0] == 5 && p[1] == 2 && p[2] == 5 && g1 == 6) e = run_bsp<5, 2, 5, 6>(*c, B, count, d_idx, buf, buf + vals);
  }
  SCK(e);
  SCK(cudaMemcpyAsync(strain, buf, sizeof(double) * vals, cudaMemcpyDeviceToHost, c->stream));
  SCK(cudaMemcpyAsync(stress, buf + vals, sizeof(double) * vals, cudaMemcpyDeviceToHost, c->stream));
  int32_t status = 0;
  SCK(cudaMemcpyAsync(&status, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  SCK(cudaStreamSynchronize(c->stream));
  cudaFree(buf);
  if (status) {
    c->err = "gauss_stress: non-positive Jacobian determinant in at least one element";
    return FAST_GPU_EDETJ;
  }
  return FAST_GPU_OK;
}

// Extrapolation matrix and node incidence of a bucket, built once.
static int nodal_tables(Ctx &c, Bucket &B) {
  if (B.d_tr) return FAST_GPU_OK;
  std::vector<double> TR;
  if (!extrapolation_matrix(B.type, B.ngp, TR, B.pd)) {
    c.err = "nodal_stress: no extrapolation for this element and rule";
    return FAST_GPU_ENOTSUP;
  }
  const int nn = B.nn;
  const int64_t ne = B.ne, nnode = c.nnode;
  std::vector<int64_t> ptr(nnode + 1, 0), ent((size_t)ne * nn);
  for (int64_t k = 0; k < ne; k++)
    for (int a = 0; a < nn; a++) ptr[B.h_conn[(size_t)B.inv[k] * nn + a] + 1]++;
  for (int64_t n = 0; n < nnode; n++) ptr[n + 1] += ptr[n];
  std::vector<int64_t> fill(ptr.begin(), ptr.end() - 1);
  for (int64_t k = 0; k < ne; k++)  // element order: each node's entries ascend in k
    for (int a = 0; a < nn; a++) ent[fill[B.h_conn[(size_t)B.inv[k] * nn + a]]++] = k * nn + a;
  cudaError_t e = cudaMalloc((void **)&B.d_tr, sizeof(double) * TR.size());
  if (e == cudaSuccess) e = cudaMalloc((void **)&B.d_nptr, sizeof(int64_t) * ptr.size());
  if (e == cudaSuccess) e = cudaMalloc((void **)&B.d_nent, sizeof(int64_t) * ent.size());
  if (e == cudaSuccess) e = cudaMemcpy(B.d_tr, TR.data(), sizeof(double) * TR.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B.d_nptr, ptr.data(), sizeof(int64_t) * ptr.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(B.d_nent, ent.data(), sizeof(int64_t) * ent.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    for (void *p : {(void *)B.d_tr, (void *)B.d_nptr, (void *)B.d_nent})
      if (p) cudaFree(p);
    B.d_tr = nullptr;
    B.d_nptr = B.d_nent = nullptr;
    c.err = std::string("nodal_stress: ") + cudaGetErrorString(e);
    return FAST_GPU_ECUDA;
  }
  return FAST_GPU_OK;
}

extern "C" int fast_gpu_nodal_stress(fast_gpu_ctx *c, int32_t b, double *elem_nodal, double *nodal) {
  if (!c || b < 0 || b >= (int)c->buckets.size() || (!elem_nodal && !nodal)) return FAST_GPU_EINVAL;
  Bucket &B = c->buckets[b];
  if (B.tl) {
    c->err = "nodal_stress: small-strain buckets only";
    return FAST_GPU_ENOTSUP;
  }
  const bool bsp = B.type == FAST_ELEM_BSP_SOLID;
  if (bsp && !(B.ngp[0] == B.ngp[1] && B.ngp[1] == B.ngp[2])) {
    c->err = "nodal_stress: B-spline buckets with the same Gauss rule in every direction only";
    return FAST_GPU_ENOTSUP;
  }
  if (!c->d_disp) {
    c->err = "nodal_stress: no displacement state";
    return FAST_GPU_ESTATE;
  }
  int rc = nodal_tables(*c, B);
  if (rc != FAST_GPU_OK) return rc;
  const int64_t ne = B.ne, nn = B.nn, ng = B.ng;
  const size_t nsg = (size_t)ne * ng * 6, nsn = (size_t)ne * nn * 6, nav = (size_t)c->nnode * 6;
  double *buf = nullptr;
  // (B-spline buckets: their Gauss-point strains go to a scratch block too)
  const size_t nse = bsp ? nsg : 0;
  SCK(cudaMalloc((void **)&buf, sizeof(double) * (nsg + nsn + nav + nse) + sizeof(int32_t) * ne + 16));
  double *Sg = buf, *Sn = buf + nsg, *avg = nodal ? buf + nsg + nsn : nullptr, *Se = buf + nsg + nsn + nav;
  int32_t *d_idx = reinterpret_cast<int32_t *>(buf + nsg + nsn + nav + nse);
  SCK(cudaMemcpyAsync(d_idx, B.inv.data(), sizeof(int32_t) * ne, cudaMemcpyHostToDevice, c->stream));
  SCK(cudaMemsetAsync(c->d_status, 0, sizeof(int32_t), c->stream));
  cudaError_t e = cudaErrorInvalidValue;
  if (B.type == FAST_ELEM_HEX8 && ng == 8) e = run_nodal<8, 8>(*c, B, d_idx, Sg, Sn, avg);
  else if (B.type == FAST_ELEM_HEX8 && ng == 27) e = run_nodal<8, 27>(*c, B, d_idx, Sg, Sn, avg);
  else if (B.type == FAST_ELEM_HEX8 && ng == 1) e = run_nodal<8, 1>(*c, B, d_idx, Sg, Sn, avg);
  else if (B.type == FAST_ELEM_HEX20 && ng == 27) e = run_nodal<20, 27>(*c, B, d_idx, Sg, Sn, avg);
  else if (B.type == FAST_ELEM_HEX20 && ng == 8) e = run_nodal<20, 8>(*c, B, d_idx, Sg, Sn, avg);
  else if (B.type == FAST_ELEM_HEX20 && ng == 64) e = run_nodal<20, 64>(*c, B, d_idx, Sg, Sn, avg);
  else if (bsp) {
    const int *p = B.pd, g1 = B.ngp[0];
    if (p[0] == 2 && p[1] == 2 && p[2] == 2 && g1 == 3) e = run_nodal_bsp<2, 2, 2, 3>(*c, B, d_idx, Se, Sg, Sn, avg);
    else if (p[0] == 2 && p[1] == 2 && p[2] == 2 && g1 == 4) e = run_nodal_bsp<2, 2, 2, 4>(*c, B, d_idx, Se, Sg, Sn, avg);
    else if (p[0] == 3 && p[1] == 3 && p[2] == 3 && g1 == 4) e = run_nodal_bsp<3, 3, 3, 4>(*c, B, d_idx, Se, Sg, Sn, avg);
    else if (p[0] == 3 && p[1] == 3 && p[2] == 2 && g1 == 4) e = run_nodal_bsp<3, 3, 2, 4>(*c, B, d_idx, Se, Sg, Sn, avg);
    else if (p[0] == 4 && p[1] == 2 && p[2] == 4 && g1 == 5) e = run_nodal_bsp<4, 2, 4, 5>(*c, B, d_idx, Se, Sg, Sn, avg);
    else if (p[0] == 4 && p[1] == 2 && p[2] == 2 && g1 == 5) e = run_nodal_bsp<4, 2, 2, 5>(*c, B, d_idx, Se, Sg, Sn, avg);
    else if (p[0] == 5 && p[1] == 2 && p[2] == 5 && g1 == 6) e = run_nodal_bsp<5, 2, 5, 6>(*c, B, d_idx, Se, Sg, Sn, avg);
  }
  SCK(e);
  if (elem_nodal) SCK(cudaMemcpyAsync(elem_nodal, Sn, sizeof(double) * nsn, cudaMemcpyDeviceToHost, c->stream));
  if (nodal) SCK(cudaMemcpyAsync(nodal, avg, sizeof(double) * nav, cudaMemcpyDeviceToHost, c->stream));
  int32_t status = 0;
  SCK(cudaMemcpyAsync(&status, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  SCK(cudaStreamSynchronize(c->stream));
  cudaFree(buf);
  if (status) {
    c->err = "nodal_stress: non-positive Jacobian determinant in at least one element";
    return FAST_GPU_EDETJ;
  }
  return FAST_GPU_OK;
}
