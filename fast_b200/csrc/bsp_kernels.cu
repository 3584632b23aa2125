// bsp_kernels.cu - Bezier-extracted B-spline / NURBS solid elements (sm_100a).
//
// Computes what cElmParam::StiffMat (elc/elmparam.cpp:539-597) computes for an
// element of %ELEMENT.BSPLINE.SOLID: the same Gauss loop and isotropic B^T C B
// as the hex kernels, on the shape functions of cShapeBspSolid
// (shp/shpbsp.cpp:928-1067):
//   B_a(g)   = Nr_i(r_g) Ns_j(s_g) Nt_k(t_g)     a = i + Qr j + Qr Qs k,  Qd = (degree in d) + 1
//   rational: N_a = B_a w_a / W,  W = sum_a B_a w_a,
//             dN_a/dxi = (dB_a/dxi w_a - N_a dW/dxi) / W
// where the univariate factors of the element's knot span are the Bezier-
// extracted tables built on the host (one table per direction, span and
// Gauss point; see bspline_gauss_tables).  For non-rational patches the plain
// tensor-product derivative is used: the reference's non-rational branch
// (shp/shpbsp.cpp:1015-1030) never advances its node index, so only its
// rational branch is a usable oracle, and with unit weights both agree.
//
// Layout per CTA (one element at a time, grid-stride over one colour):
//   sD  [NG][3][NN]  natural derivatives, overwritten in place by dN/dx
//   sB  [NG][NN]     rational numerators (rational patches only)
// Thread t owns node pairs t, t+NT, ...: M_ij = sum_g c_g dNa/dx_i dNb/dx_j,
// turned into the isotropic 3x3 block and added into K through the slot map
// (elements of one colour share no node, so the adds need no atomics and K
// is bit-identical from run to run).
#include <algorithm>
#include <cstdint>

#include "elem_common.cuh"
#include "internal.h"

namespace fastgpu {

template <int PR, int PS, int PT, int NG1>
struct BspSmem {
  static constexpr int QR = PR + 1, QS = PS + 1, QT = PT + 1;
  static constexpr int NN = QR * QS * QT;
  static constexpr int NG = NG1 * NG1 * NG1;
  static constexpr int NP = NN * (NN + 1) / 2;
  static constexpr int kX = NN * 3, kW = NN, kB = NG * NN, kD = NG * 3 * NN, kJ = NG * 9, kC = NG, kWg = NG * 4;
  static constexpr size_t doubles = kX + kW + kB + kD + kJ + kC + kWg;
  static constexpr size_t bytes = doubles * sizeof(double) + NP * 2 + NN + 16;
};

// split > 1: `split` CTAs share one element, each taking every split-th block
// of NT node pairs (they write disjoint blocks of K); the geometry is
// recomputed by each.  Fills the GPU when a colour holds few elements (a
// degree-3 patch needs 64 colours).
// MASS: the consistent mass instead (cElmParam::MassMat, elc/elmparam.cpp:
// 672-739, on the same Gauss points as the stiffness): block (a, b) =
// rho sum_g c_g N_a N_b I3 with the (rational) basis values N.
template <int PR, int PS, int PT, int NG1, int NT, bool MASS>
__global__ void __launch_bounds__(NT, 1) bsp_elem_kernel(ElemArgs A, int split) {
  using S = BspSmem<PR, PS, PT, NG1>;
  constexpr int QR = S::QR, QS = S::QS, QT = S::QT, NN = S::NN, NG = S::NG, NP = S::NP, ND = 3 * NN;
  extern __shared__ __align__(16) double sm[];
  double *sX = sm;
  double *sW = sX + S::kX;
  double *sB = sW + S::kW;
  double *sD = sB + S::kB;
  double *sJ = sD + S::kD;
  double *sc = sJ + S::kJ;
  double *sWg = sc + S::kC;
  uint8_t *spair = reinterpret_cast<uint8_t *>(sWg + S::kWg);
  uint8_t *sfix = spair + 2 * NP;
  const int tid = threadIdx.x;
  for (int q = tid; q < NP; q += NT) {
    int a, b;
    pair_of(q, NN, a, b);
    spair[2 * q] = (uint8_t)a;
    spair[2 * q + 1] = (uint8_t)b;
  }
  const double *__restrict__ gw = A.w;
  const bool rat = A.rational != 0;

  for (int64_t wi = blockIdx.x; wi < A.ne * split; wi += gridDim.x) {
    const int64_t it = wi / split;
    const int part = (int)(wi - it * split);
    const int64_t e = A.index ? (int64_t)A.index[it] : A.offset + it;
    __syncthreads();
    const int32_t *en = A.conn + e * NN;
    for (int i = tid; i < NN * 3; i += NT) sX[i] = A.X[3 * (int64_t)en[i / 3] + (i % 3)];
    for (int i = tid; i < NN; i += NT) {
      sfix[i] = A.fix[en[i]];
      sW[i] = (rat && A.wt) ? A.wt[en[i]] : 1.0;
    }
    const int sr = A.span[4 * e], ss = A.span[4 * e + 1], st = A.span[4 * e + 2];
    const double *br = A.bas[0] + (size_t)sr * NG1 * QR * 2;
    const double *bs = A.bas[1] + (size_t)ss * NG1 * QS * 2;
    const double *bt = A.bas[2] + (size_t)st * NG1 * QT * 2;
    __syncthreads();

    // tensor-product basis (cShapeBspSolid::DrvShpRST, shp/shpbsp.cpp:985-1067)
    for (int t = tid; t < NG * NN; t += NT) {
      const int g = t / NN, a = t - NN * g;
      const int gl = g % NG1, gj = (g / NG1) % NG1, gi = g / (NG1 * NG1);
      const int ia = a % QR, ja = (a / QR) % QS, ka = a / (QR * QS);
      const double *fr = br + (gl * QR + ia) * 2, *fs = bs + (gj * QS + ja) * 2, *ft = bt + (gi * QT + ka) * 2;
      double *D = sD + g * ND;
      if (rat) {
        const double w = sW[a];
        sB[g * NN + a] = fr[0] * fs[0] * ft[0] * w;
        D[a] = fr[1] * fs[0] * ft[0] * w;
        D[NN + a] = fr[0] * fs[1] * ft[0] * w;
        D[2 * NN + a] = fr[0] * fs[0] * ft[1] * w;
      } else {
        if (MASS) sB[g * NN + a] = fr[0] * fs[0] * ft[0];
        D[a] = fr[1] * fs[0] * ft[0];
        D[NN + a] = fr[0] * fs[1] * ft[0];
        D[2 * NN + a] = fr[0] * fs[0] * ft[1];
      }
    }
    constexpr int NW = NT / 32;
    const int lane = tid & 31, warp = tid >> 5;
    if (rat) {
      __syncthreads();
      // W and dW/dxi per Gauss point: one warp per point, lanes over the nodes
      // (consecutive addresses), then a fixed butterfly
      for (int g = warp; g < NG; g += NW) {
        const double *D = sD + g * ND;
        double w = 0.0, wr = 0.0, ws = 0.0, wt = 0.0;
        for (int a = lane; a < NN; a += 32) {
          w += sB[g * NN + a];
          wr += D[a];
          ws += D[NN + a];
          wt += D[2 * NN + a];
        }
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) {
          w += __shfl_xor_sync(0xffffffffu, w, m);
          wr += __shfl_xor_sync(0xffffffffu, wr, m);
          ws += __shfl_xor_sync(0xffffffffu, ws, m);
          wt += __shfl_xor_sync(0xffffffffu, wt, m);
        }
        if (lane == 0) {
          sWg[4 * g] = w;
          sWg[4 * g + 1] = wr;
          sWg[4 * g + 2] = ws;
          sWg[4 * g + 3] = wt;
        }
      }
      __syncthreads();
      for (int t = tid; t < NG * NN; t += NT) {
        const int g = t / NN, a = t - NN * g;
        const double *Wg = sWg + 4 * g;
        const double n = sB[g * NN + a] / Wg[0];
        double *D = sD + g * ND;
        D[a] = (D[a] - n * Wg[1]) / Wg[0];
        D[NN + a] = (D[NN + a] - n * Wg[2]) / Wg[0];
        D[2 * NN + a] = (D[2 * NN + a] - n * Wg[3]) / Wg[0];
      }
    }
    __syncthreads();

    // Jacobians J[g][p][q] = sum_a dN_a/dxi_p X_a,q (cShapeSolid::DrvShpXYZ, shp/shpsolid.cpp:58-126):
    // one warp per Gauss point, lanes over the nodes
    for (int g = warp; g < NG; g += NW) {
      const double *D = sD + g * ND;
      double j[9];
#pragma unroll
      for (int k = 0; k < 9; k++) j[k] = 0.0;
      for (int a = lane; a < NN; a += 32) {
        const double x0 = sX[3 * a], x1 = sX[3 * a + 1], x2 = sX[3 * a + 2];
#pragma unroll
        for (int p = 0; p < 3; p++) {
          const double d = D[p * NN + a];
          j[3 * p] = fma(d, x0, j[3 * p]);
          j[3 * p + 1] = fma(d, x1, j[3 * p + 1]);
          j[3 * p + 2] = fma(d, x2, j[3 * p + 2]);
        }
      }
#pragma unroll
      for (int k = 0; k < 9; k++)
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) j[k] += __shfl_xor_sync(0xffffffffu, j[k], m);
      if (lane < 9) {
        double v = j[0];
#pragma unroll
        for (int k = 1; k < 9; k++)
          if (lane == k) v = j[k];
        sJ[9 * g + lane] = v;
      }
    }
    __syncthreads();
    // determinant and inverse by cofactors (cShape::ShpMatInv, shp/shape.cpp:360-393)
    for (int g = tid; g < NG; g += NT) {
      double *J = sJ + 9 * g;
      const double j00 = J[0], j01 = J[1], j02 = J[2], j10 = J[3], j11 = J[4], j12 = J[5], j20 = J[6],
                   j21 = J[7], j22 = J[8];
      const double det = j00 * (j11 * j22 - j12 * j21) - j01 * (j10 * j22 - j12 * j20) + j02 * (j10 * j21 - j11 * j20);
      // a B-spline patch may be parametrised left-handed: the reference keeps the
      // signed determinant (and so a negative definite K and load); only a
      // vanishing or non-finite Jacobian is an error here
      if (!(fabs(det) > 0.0) || !isfinite(det)) atomicOr(A.status, 1);
      const double id = 1.0 / ((det != 0.0) ? det : 1.0);
      J[0] = (j11 * j22 - j12 * j21) * id;
      J[1] = -(j01 * j22 - j02 * j21) * id;
      J[2] = (j01 * j12 - j02 * j11) * id;
      J[3] = -(j10 * j22 - j12 * j20) * id;
      J[4] = (j00 * j22 - j02 * j20) * id;
      J[5] = -(j00 * j12 - j02 * j10) * id;
      J[6] = (j10 * j21 - j11 * j20) * id;
      J[7] = -(j00 * j21 - j01 * j20) * id;
      J[8] = (j00 * j11 - j01 * j10) * id;
      sc[g] = gw[g] * det;
    }
    __syncthreads();
    // dN/dx in place: each (g, a) reads and writes only its own three entries
    for (int t = tid; t < NG * NN; t += NT) {
      const int g = t / NN, a = t - NN * g;
      const double *J = sJ + 9 * g;
      double *D = sD + g * ND;
      const double d0 = D[a], d1 = D[NN + a], d2 = D[2 * NN + a];
      D[a] = J[0] * d0 + J[1] * d1 + J[2] * d2;
      D[NN + a] = J[3] * d0 + J[4] * d1 + J[5] * d2;
      D[2 * NN + a] = J[6] * d0 + J[7] * d1 + J[8] * d2;
    }
    __syncthreads();

    if (MASS && rat) {
      // the rational basis values N_a = B_a w_a / W
      for (int t = tid; t < NG * NN; t += NT) {
        const int g = t / NN;
        sB[t] = sB[t] / sWg[4 * g];
      }
      __syncthreads();
    }
    const double E = A.E[e], nu = A.nu[e];
    const double dd = (1.0 + nu) * (1.0 - 2.0 * nu);
    const double C00 = E * (1.0 - nu) / dd, C01 = E * nu / dd, G = 0.5 * E / (1.0 + nu);
    const double rho = (MASS && A.rho) ? A.rho[e] : 0.0;
    for (int q = tid + part * NT; q < NP; q += NT * split) {
      const int pa = spair[2 * q], pb = spair[2 * q + 1];
      // the pair's two K blocks are loaded before its Gauss-point sum, so the
      // read latency overlaps the arithmetic
      // (blocks this element writes first, by the first-touch flags, are not read)
      double *Kab = nullptr, *Kba = nullptr;
      double oab[9], oba[9];
      bool fab = false, fba = false;
      if (A.K) {
        Kab = A.K + (int64_t)A.slot[(e * NN + pa) * NN + pb] * 9;
        Kba = pa != pb ? A.K + (int64_t)A.slot[(e * NN + pb) * NN + pa] * 9 : nullptr;
        fab = first_touch(A, e, pa * NN + pb);
        fba = Kba && first_touch(A, e, pb * NN + pa);
        if (!fab) {
#pragma unroll
          for (int k = 0; k < 9; k++) oab[k] = Kab[k];
        }
        if (Kba && !fba) {
#pragma unroll
          for (int k = 0; k < 9; k++) oba[k] = Kba[k];
        }
      }
      double v[9];
      if (MASS) {
        double sm_ab = 0.0;
        for (int g = 0; g < NG; g++) sm_ab += sc[g] * sB[g * NN + pa] * sB[g * NN + pb];
        sm_ab *= rho;
#pragma unroll
        for (int k = 0; k < 9; k++) v[k] = (k % 4 == 0) ? sm_ab : 0.0;
      } else {
        double M[9];
#pragma unroll
        for (int k = 0; k < 9; k++) M[k] = 0.0;
        for (int g = 0; g < NG; g++) {
          const double *D = sD + g * ND;
          const double cg = sc[g];
          const double a0 = cg * D[pa], a1 = cg * D[NN + pa], a2 = cg * D[2 * NN + pa];
          const double b0 = D[pb], b1 = D[NN + pb], b2 = D[2 * NN + pb];
          M[0] = fma(a0, b0, M[0]); M[1] = fma(a0, b1, M[1]); M[2] = fma(a0, b2, M[2]);
          M[3] = fma(a1, b0, M[3]); M[4] = fma(a1, b1, M[4]); M[5] = fma(a1, b2, M[5]);
          M[6] = fma(a2, b0, M[6]); M[7] = fma(a2, b1, M[7]); M[8] = fma(a2, b2, M[8]);
        }
        // isotropic block (cSolid::QMatrix elc/anmodel.cpp:1286-1298, BMatrix :1418-1447)
        const double tr = M[0] + M[4] + M[8];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++)
            v[3 * i + j] = (i == j) ? C00 * M[4 * i] + G * (tr - M[4 * i]) : C01 * M[3 * i + j] + G * M[3 * j + i];
      }
      if (A.Ke_out) {
        double *Ko = A.Ke_out + it * ND * ND;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) {
            Ko[(3 * pa + i) * ND + 3 * pb + j] = v[3 * i + j];
            Ko[(3 * pb + j) * ND + 3 * pa + i] = v[3 * i + j];
          }
      }
      if (A.K) {
        const uint8_t fa = sfix[pa], fb = sfix[pb];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) {
            const bool fixed = ((fa >> i) & 1) || ((fb >> j) & 1);
            double out;
            if (entry_value(fab, fixed, pa == pb && i == j, fab ? 0.0 : oab[3 * i + j], v[3 * i + j], out))
              Kab[3 * i + j] = out;
            if (Kba && entry_value(fba, fixed, false, fba ? 0.0 : oba[3 * j + i], v[3 * i + j], out))
              Kba[3 * j + i] = out;
          }
      }
    }
  }
}

template <int PR, int PS, int PT, int NG1, int NT, bool MASS = false>
static cudaError_t run_bsp(Ctx &c, ElemArgs a, int64_t count) {
  if (count <= 0) return cudaSuccess;
  using S = BspSmem<PR, PS, PT, NG1>;
  auto kern = bsp_elem_kernel<PR, PS, PT, NG1, NT, MASS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, S::bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  per_sm = elem_per_sm(c, per_sm, a.ctas_per_sm);
  // as many CTAs per element as fit in one wave (a second, partial wave would
  // double the launch time), at most one per block of NT node pairs; a tuned
  // shape fixes the count instead
  const int64_t slots = (int64_t)per_sm * c.sm_count;
  const int smax = (S::NP + NT - 1) / NT;
  if (smax > c.elem_split_max) c.elem_split_max = smax;
  int split = (int)std::min<int64_t>(smax, std::max<int64_t>(1, slots / count));
  if (a.split > 0) split = std::min(a.split, smax);
  int64_t grid = std::min<int64_t>(slots, count * split);
  a.ne = count;
  kern<<<(unsigned)grid, NT, S::bytes, c.stream>>>(a, split);
  c.launches++;
  return cudaGetLastError();
}

// Higher degrees (the reference's (4,2,4) and (5,2,5) NURBS cylinders): the
// per-element tables of all Gauss points no longer fit in shared memory, so
// the points are taken one layer in t at a time (NG1 x NG1 points per chunk)
// and every thread keeps the 3x3 sums of its PPT node pairs in registers
// across the layers.  CTAs of one element split its pairs (blocks of
// NT * PPT); each recomputes the geometry.  Same arithmetic per point as
// bsp_elem_kernel.
template <int PR, int PS, int PT, int NG1>
struct BspBigSmem {
  static constexpr int QR = PR + 1, QS = PS + 1, QT = PT + 1;
  static constexpr int NN = QR * QS * QT;
  static constexpr int GC = NG1 * NG1;  // Gauss points per chunk
  static constexpr int NP = NN * (NN + 1) / 2;
  static constexpr int kX = NN * 3, kW = NN, kB = GC * NN, kD = GC * 3 * NN, kJ = GC * 9, kC = GC, kWg = GC * 4;
  static constexpr size_t doubles = kX + kW + kB + kD + kJ + kC + kWg;
  static constexpr size_t bytes = doubles * sizeof(double) + NP * 2 + NN + 16;
};

template <int PR, int PS, int PT, int NG1, int NT, int PPT>
__global__ void __launch_bounds__(NT, 1) bsp_big_kernel(ElemArgs A, int split) {
  using S = BspBigSmem<PR, PS, PT, NG1>;
  constexpr int QR = S::QR, QS = S::QS, QT = S::QT, NN = S::NN, GC = S::GC, NP = S::NP, ND = 3 * NN;
  extern __shared__ __align__(16) double sm[];
  double *sX = sm;
  double *sW = sX + S::kX;
  double *sB = sW + S::kW;
  double *sD = sB + S::kB;
  double *sJ = sD + S::kD;
  double *sc = sJ + S::kJ;
  double *sWg = sc + S::kC;
  uint8_t *spair = reinterpret_cast<uint8_t *>(sWg + S::kWg);
  uint8_t *sfix = spair + 2 * NP;
  const int tid = threadIdx.x;
  for (int q = tid; q < NP; q += NT) {
    int a, b;
    pair_of(q, NN, a, b);
    spair[2 * q] = (uint8_t)a;
    spair[2 * q + 1] = (uint8_t)b;
  }
  const double *__restrict__ gw = A.w;
  const bool rat = A.rational != 0;
  constexpr int NW = NT / 32;
  const int lane = tid & 31, warp = tid >> 5;

  for (int64_t wi = blockIdx.x; wi < A.ne * split; wi += gridDim.x) {
    const int64_t it = wi / split;
    const int part = (int)(wi - it * split);
    const int64_t e = A.index ? (int64_t)A.index[it] : A.offset + it;
    __syncthreads();
    const int32_t *en = A.conn + e * NN;
    for (int i = tid; i < NN * 3; i += NT) sX[i] = A.X[3 * (int64_t)en[i / 3] + (i % 3)];
    for (int i = tid; i < NN; i += NT) {
      sfix[i] = A.fix[en[i]];
      sW[i] = (rat && A.wt) ? A.wt[en[i]] : 1.0;
    }
    const int sr = A.span[4 * e], ss = A.span[4 * e + 1], st = A.span[4 * e + 2];
    const double *br = A.bas[0] + (size_t)sr * NG1 * QR * 2;
    const double *bs = A.bas[1] + (size_t)ss * NG1 * QS * 2;
    const double *bt = A.bas[2] + (size_t)st * NG1 * QT * 2;
    double M[PPT][9];
#pragma unroll
    for (int k = 0; k < PPT; k++)
#pragma unroll
      for (int m = 0; m < 9; m++) M[k][m] = 0.0;
    int pa[PPT], pb[PPT];
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      const int q = (part * PPT + k) * NT + tid;
      pa[k] = q < NP ? spair[2 * q] : -1;
      pb[k] = q < NP ? spair[2 * q + 1] : -1;
    }

    for (int gi = 0; gi < NG1; gi++) {  // one layer of Gauss points in t
      __syncthreads();
      for (int t = tid; t < GC * NN; t += NT) {
        const int g = t / NN, a = t - NN * g;
        const int gl = g % NG1, gj = g / NG1;
        const int ia = a % QR, ja = (a / QR) % QS, ka = a / (QR * QS);
        const double *fr = br + (gl * QR + ia) * 2, *fs = bs + (gj * QS + ja) * 2, *ft = bt + (gi * QT + ka) * 2;
        double *D = sD + g * ND;
        if (rat) {
          const double w = sW[a];
          sB[g * NN + a] = fr[0] * fs[0] * ft[0] * w;
          D[a] = fr[1] * fs[0] * ft[0] * w;
          D[NN + a] = fr[0] * fs[1] * ft[0] * w;
          D[2 * NN + a] = fr[0] * fs[0] * ft[1] * w;
        } else {
          D[a] = fr[1] * fs[0] * ft[0];
          D[NN + a] = fr[0] * fs[1] * ft[0];
          D[2 * NN + a] = fr[0] * fs[0] * ft[1];
        }
      }
      if (rat) {
        __syncthreads();
        for (int g = warp; g < GC; g += NW) {
          const double *D = sD + g * ND;
          double w = 0.0, wr = 0.0, ws = 0.0, wt = 0.0;
          for (int a = lane; a < NN; a += 32) {
            w += sB[g * NN + a];
            wr += D[a];
            ws += D[NN + a];
            wt += D[2 * NN + a];
          }
#pragma unroll
          for (int m = 16; m > 0; m >>= 1) {
            w += __shfl_xor_sync(0xffffffffu, w, m);
            wr += __shfl_xor_sync(0xffffffffu, wr, m);
            ws += __shfl_xor_sync(0xffffffffu, ws, m);
            wt += __shfl_xor_sync(0xffffffffu, wt, m);
          }
          if (lane == 0) {
            sWg[4 * g] = w;
            sWg[4 * g + 1] = wr;
            sWg[4 * g + 2] = ws;
            sWg[4 * g + 3] = wt;
          }
        }
        __syncthreads();
        for (int t = tid; t < GC * NN; t += NT) {
          const int g = t / NN, a = t - NN * g;
          const double *Wg = sWg + 4 * g;
          const double n = sB[g * NN + a] / Wg[0];
          double *D = sD + g * ND;
          D[a] = (D[a] - n * Wg[1]) / Wg[0];
          D[NN + a] = (D[NN + a] - n * Wg[2]) / Wg[0];
          D[2 * NN + a] = (D[2 * NN + a] - n * Wg[3]) / Wg[0];
        }
      }
      __syncthreads();
      for (int g = warp; g < GC; g += NW) {
        const double *D = sD + g * ND;
        double j[9];
#pragma unroll
        for (int k = 0; k < 9; k++) j[k] = 0.0;
        for (int a = lane; a < NN; a += 32) {
          const double x0 = sX[3 * a], x1 = sX[3 * a + 1], x2 = sX[3 * a + 2];
#pragma unroll
          for (int p = 0; p < 3; p++) {
            const double d = D[p * NN + a];
            j[3 * p] = fma(d, x0, j[3 * p]);
            j[3 * p + 1] = fma(d, x1, j[3 * p + 1]);
            j[3 * p + 2] = fma(d, x2, j[3 * p + 2]);
          }
        }
#pragma unroll
        for (int k = 0; k < 9; k++)
#pragma unroll
          for (int m = 16; m > 0; m >>= 1) j[k] += __shfl_xor_sync(0xffffffffu, j[k], m);
        if (lane < 9) {
          double v = j[0];
#pragma unroll
          for (int k = 1; k < 9; k++)
            if (lane == k) v = j[k];
          sJ[9 * g + lane] = v;
        }
      }
      __syncthreads();
      for (int g = tid; g < GC; g += NT) {
        double *J = sJ + 9 * g;
        const double j00 = J[0], j01 = J[1], j02 = J[2], j10 = J[3], j11 = J[4], j12 = J[5], j20 = J[6],
                     j21 = J[7], j22 = J[8];
        const double det =
            j00 * (j11 * j22 - j12 * j21) - j01 * (j10 * j22 - j12 * j20) + j02 * (j10 * j21 - j11 * j20);
        if (!(fabs(det) > 0.0) || !isfinite(det)) atomicOr(A.status, 1);
        const double id = 1.0 / ((det != 0.0) ? det : 1.0);
        J[0] = (j11 * j22 - j12 * j21) * id;
        J[1] = -(j01 * j22 - j02 * j21) * id;
        J[2] = (j01 * j12 - j02 * j11) * id;
        J[3] = -(j10 * j22 - j12 * j20) * id;
        J[4] = (j00 * j22 - j02 * j20) * id;
        J[5] = -(j00 * j12 - j02 * j10) * id;
        J[6] = (j10 * j21 - j11 * j20) * id;
        J[7] = -(j00 * j21 - j01 * j20) * id;
        J[8] = (j00 * j11 - j01 * j10) * id;
        sc[g] = gw[gi * GC + g] * det;
      }
      __syncthreads();
      for (int t = tid; t < GC * NN; t += NT) {
        const int g = t / NN, a = t - NN * g;
        const double *J = sJ + 9 * g;
        double *D = sD + g * ND;
        const double d0 = D[a], d1 = D[NN + a], d2 = D[2 * NN + a];
        D[a] = J[0] * d0 + J[1] * d1 + J[2] * d2;
        D[NN + a] = J[3] * d0 + J[4] * d1 + J[5] * d2;
        D[2 * NN + a] = J[6] * d0 + J[7] * d1 + J[8] * d2;
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < PPT; k++) {
        if (pa[k] < 0) continue;
        const int a = pa[k], b = pb[k];
        for (int g = 0; g < GC; g++) {
          const double *D = sD + g * ND;
          const double cg = sc[g];
          const double a0 = cg * D[a], a1 = cg * D[NN + a], a2 = cg * D[2 * NN + a];
          const double b0 = D[b], b1 = D[NN + b], b2 = D[2 * NN + b];
          M[k][0] = fma(a0, b0, M[k][0]); M[k][1] = fma(a0, b1, M[k][1]); M[k][2] = fma(a0, b2, M[k][2]);
          M[k][3] = fma(a1, b0, M[k][3]); M[k][4] = fma(a1, b1, M[k][4]); M[k][5] = fma(a1, b2, M[k][5]);
          M[k][6] = fma(a2, b0, M[k][6]); M[k][7] = fma(a2, b1, M[k][7]); M[k][8] = fma(a2, b2, M[k][8]);
        }
      }
    }

    const double E = A.E[e], nu = A.nu[e];
    const double dd = (1.0 + nu) * (1.0 - 2.0 * nu);
    const double C00 = E * (1.0 - nu) / dd, C01 = E * nu / dd, G = 0.5 * E / (1.0 + nu);
#pragma unroll
    for (int k = 0; k < PPT; k++) {
      if (pa[k] < 0) continue;
      const int a = pa[k], b = pb[k];
      double v[9];
      const double tr = M[k][0] + M[k][4] + M[k][8];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
          v[3 * i + j] = (i == j) ? C00 * M[k][4 * i] + G * (tr - M[k][4 * i]) : C01 * M[k][3 * i + j] + G * M[k][3 * j + i];
      if (A.Ke_out) {
        double *Ko = A.Ke_out + it * ND * ND;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) {
            Ko[(3 * a + i) * ND + 3 * b + j] = v[3 * i + j];
            Ko[(3 * b + j) * ND + 3 * a + i] = v[3 * i + j];
          }
      }
      if (A.K) {
        double *Kab = A.K + (int64_t)A.slot[(e * NN + a) * NN + b] * 9;
        double *Kba = a != b ? A.K + (int64_t)A.slot[(e * NN + b) * NN + a] * 9 : nullptr;
        const bool fab = first_touch(A, e, a * NN + b), fba = Kba && first_touch(A, e, b * NN + a);
        const uint8_t fa = sfix[a], fb = sfix[b];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) {
            // add where both DOFs have equations; a first write stores instead
            const bool fixed = ((fa >> i) & 1) || ((fb >> j) & 1);
            if (fab) Kab[3 * i + j] = fixed ? ((a == b && i == j) ? 1.0 : 0.0) : v[3 * i + j];
            else if (!fixed) Kab[3 * i + j] += v[3 * i + j];
            if (Kba) {
              if (fba) Kba[3 * j + i] = fixed ? 0.0 : v[3 * i + j];
              else if (!fixed) Kba[3 * j + i] += v[3 * i + j];
            }
          }
      }
    }
  }
}

template <int PR, int PS, int PT, int NG1, int NT, int PPT>
static cudaError_t run_bsp_big(Ctx &c, ElemArgs a, int64_t count) {
  if (count <= 0) return cudaSuccess;
  using S = BspBigSmem<PR, PS, PT, NG1>;
  auto kern = bsp_big_kernel<PR, PS, PT, NG1, NT, PPT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, S::bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  per_sm = elem_per_sm(c, per_sm, a.ctas_per_sm);
  const int split = (S::NP + NT * PPT - 1) / (NT * PPT);
  const int64_t slots = (int64_t)per_sm * c.sm_count;
  const int64_t grid = std::min<int64_t>(slots, count * split);
  a.ne = count;
  kern<<<(unsigned)grid, NT, S::bytes, c.stream>>>(a, split);
  c.launches++;
  return cudaGetLastError();
}

bool bsp_supported(const int pd[3], int ngp) {
  if (pd[0] == 2 && pd[1] == 2 && pd[2] == 2) return ngp == 3 || ngp == 4;
  if (pd[0] == 3 && pd[1] == 3 && (pd[2] == 3 || pd[2] == 2)) return ngp == 4;
  if (pd[0] == 4 && pd[1] == 2 && pd[2] == 4) return ngp == 5;
  if (pd[0] == 4 && pd[1] == 2 && pd[2] == 2) return ngp == 5;
  if (pd[0] == 5 && pd[1] == 2 && pd[2] == 5) return ngp == 6;
  return false;
}

cudaError_t launch_bsp_elements(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, bool mass) {
  a.span = B.d_span;
  for (int d = 0; d < 3; d++) a.bas[d] = B.d_bas + B.bas_off[d];
  a.wt = B.d_wt;
  a.rational = B.rational;
  const int ng = B.ngp[0];
  const int *p = B.pd;
  if (mass) {
    if (p[0] == 2 && p[1] == 2 && p[2] == 2 && ng == 3) return run_bsp<2, 2, 2, 3, 384, true>(c, a, count);
    if (p[0] == 2 && p[1] == 2 && p[2] == 2 && ng == 4) return run_bsp<2, 2, 2, 4, 384, true>(c, a, count);
    if (p[0] == 3 && p[1] == 3 && p[2] == 3 && ng == 4) return run_bsp<3, 3, 3, 4, 384, true>(c, a, count);
    if (p[0] == 3 && p[1] == 3 && p[2] == 2 && ng == 4) return run_bsp<3, 3, 2, 4, 384, true>(c, a, count);
    return cudaErrorNotSupported;
  }
  if (p[0] == 2 && p[1] == 2 && p[2] == 2 && ng == 3) return run_bsp<2, 2, 2, 3, 384>(c, a, count);
  if (p[0] == 2 && p[1] == 2 && p[2] == 2 && ng == 4) return run_bsp<2, 2, 2, 4, 384>(c, a, count);
  if (p[0] == 3 && p[1] == 3 && p[2] == 3 && ng == 4) return run_bsp<3, 3, 3, 4, 384>(c, a, count);
  if (p[0] == 3 && p[1] == 3 && p[2] == 2 && ng == 4) return run_bsp<3, 3, 2, 4, 384>(c, a, count);
  if (p[0] == 4 && p[1] == 2 && p[2] == 4 && ng == 5) return run_bsp_big<4, 2, 4, 5, 256, 2>(c, a, count);
  if (p[0] == 4 && p[1] == 2 && p[2] == 2 && ng == 5) return run_bsp_big<4, 2, 2, 5, 256, 2>(c, a, count);
  if (p[0] == 5 && p[1] == 2 && p[2] == 5 && ng == 6) return run_bsp_big<5, 2, 5, 6, 256, 2>(c, a, count);
  return cudaErrorInvalidValue;
}

}  // namespace fastgpu
