// bsp_tl.cu - total-Lagrangian tangent and internal force, and the
// small-strain internal force, of Bezier-extracted B-spline / NURBS solids
// (sm_100a): cElmParamTL::StiffMat / IntForce (elc/elmparam.cpp:1615-1807)
// and cElmParam::IntForce (:449-535) on the shape functions of
// cShapeBspSolid (shp/shpbsp.cpp:928-1067), e.g. %ELEMENT.BSPLINE.SOLIDTL.
//
// The per-point arithmetic is that of the hex kernel in tl_kernels.cu
// (F = I + H, E = (F^T F - I)/2, S = lambda tr(E) I + 2 mu E; per node pair
// K_ab = lambda P + mu P^T + mu Q + s I with P = sum c h_a h_b^T,
// h = F grad N, Q = sum c (grad N_a . grad N_b) F F^T, s = sum c grad N_a . S
// grad N_b; g_a = sum c F S grad N_a), and the basis and geometry are those of
// bsp_big_kernel in bsp_kernels.cu: the Gauss points are taken one t-layer at
// a time, each thread keeps the sums of its PPT node pairs (and thread a the
// force of node a) in registers across layers.  CTAs of one element split
// its pairs; only the first of them adds the nodal forces.  One launch per
// colour, so neither K nor the forces need atomics: same bits every run.
#include <algorithm>
#include <cstdint>

#include "elem_common.cuh"
#include "internal.h"

namespace fastgpu {

namespace {

template <int PR, int PS, int PT, int NG1>
struct BspTlSmem {
  static constexpr int QR = PR + 1, QS = PS + 1, QT = PT + 1;
  static constexpr int NN = QR * QS * QT;
  static constexpr int GC = NG1 * NG1;
  static constexpr int NP = NN * (NN + 1) / 2;
  static constexpr int kX = NN * 3, kU = NN * 3, kW = NN, kB = GC * NN, kD = GC * 3 * NN, kJ = GC * 9, kC = GC,
                       kWg = GC * 4, kF = GC * 9, kS = GC * 9, kFS = GC * 9, kFF = GC * 6;
  static constexpr size_t doubles = kX + kU + kW + kB + kD + kJ + kC + kWg + kF + kS + kFS + kFF;
  static constexpr size_t bytes = doubles * sizeof(double) + NP * 2 + NN + 16;
};

template <int PR, int PS, int PT, int NG1, int NT, int PPT, bool TL, bool WK, bool WG>
__global__ void __launch_bounds__(NT, 1) bsp_tl_kernel(ElemArgs A, int split) {
  using S_ = BspTlSmem<PR, PS, PT, NG1>;
  constexpr int QR = S_::QR, QS = S_::QS, QT = S_::QT, NN = S_::NN, GC = S_::GC, NP = S_::NP, ND = 3 * NN;
  static_assert(NN <= NT, "one thread per node for the forces");
  extern __shared__ __align__(16) double sm[];
  double *sX = sm;
  double *sU = sX + S_::kX;
  double *sW = sU + S_::kU;
  double *sB = sW + S_::kW;
  double *sD = sB + S_::kB;
  double *sJ = sD + S_::kD;
  double *sc = sJ + S_::kJ;
  double *sWg = sc + S_::kC;
  double *sF = sWg + S_::kWg;
  double *sS = sF + S_::kF;
  double *sFS = sS + S_::kS;
  double *sFF = sFS + S_::kFS;
  uint8_t *spair = reinterpret_cast<uint8_t *>(sFF + S_::kFF);
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

  if (A.skip && *A.skip) return;
  for (int64_t wi = blockIdx.x; wi < A.ne * split; wi += gridDim.x) {
    const int64_t it = wi / split;
    const int part = (int)(wi - it * split);
    const int64_t e = A.index ? (int64_t)A.index[it] : A.offset + it;
    __syncthreads();
    const int32_t *en = A.conn + e * NN;
    for (int i = tid; i < NN * 3; i += NT) {
      const int32_t n = en[i / 3];
      sX[i] = A.X[3 * (int64_t)n + (i % 3)];
      sU[i] = A.U[4 * (int64_t)n + (i % 3)];
    }
    for (int i = tid; i < NN; i += NT) {
      sfix[i] = A.fix[en[i]];
      sW[i] = (rat && A.wt) ? A.wt[en[i]] : 1.0;
    }
    const int sr = A.span[4 * e], ss = A.span[4 * e + 1], st = A.span[4 * e + 2];
    const double *br = A.bas[0] + (size_t)sr * NG1 * QR * 2;
    const double *bs = A.bas[1] + (size_t)ss * NG1 * QS * 2;
    const double *bt = A.bas[2] + (size_t)st * NG1 * QT * 2;
    const double Ey = A.E[e], nu = A.nu[e];
    const double lam = Ey * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = 0.5 * Ey / (1.0 + nu);
    double P[PPT][9], Q[PPT][6], sg[PPT];
    int pa[PPT], pb[PPT];
#pragma unroll
    for (int k = 0; k < PPT; k++) {
#pragma unroll
      for (int m = 0; m < 9; m++) P[k][m] = 0.0;
#pragma unroll
      for (int m = 0; m < 6; m++) Q[k][m] = 0.0;
      sg[k] = 0.0;
      const int q = (part * PPT + k) * NT + tid;
      pa[k] = (WK && q < NP) ? spair[2 * q] : -1;
      pb[k] = (WK && q < NP) ? spair[2 * q + 1] : -1;
    }
    const bool force = WG && part == 0 && tid < NN;
    double g0 = 0.0, g1 = 0.0, g2 = 0.0;

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
      // F = I + H, H_ij = sum_a u_a,i dN_a/dX_j
      for (int t = tid; t < GC * 9; t += NT) {
        const int g = t / 9, ij = t - 9 * g, i = ij / 3, j = ij - 3 * i;
        const double *D = sD + g * ND + j * NN;
        double s = 0.0;
        for (int a = 0; a < NN; a++) s += sU[3 * a + i] * D[a];
        sF[t] = s + (i == j ? 1.0 : 0.0);
      }
      __syncthreads();
      for (int g = tid; g < GC; g += NT) {
        const double *F = sF + 9 * g;
        double E[9];
        if (TL) {
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              E[3 * i + j] = 0.5 * (F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j] - (i == j ? 1.0 : 0.0));
        } else {
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) E[3 * i + j] = 0.5 * (F[3 * i + j] + F[3 * j + i]) - (i == j ? 1.0 : 0.0);
        }
        const double tr = E[0] + E[4] + E[8];
        double *S = sS + 9 * g;
#pragma unroll
        for (int k = 0; k < 9; k++) S[k] = 2.0 * mu * E[k] + ((k % 4 == 0) ? lam * tr : 0.0);
        double *FS = sFS + 9 * g;
        if (TL) {
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              FS[3 * i + j] = F[3 * i] * S[j] + F[3 * i + 1] * S[3 + j] + F[3 * i + 2] * S[6 + j];
          double *FF = sFF + 6 * g;
          FF[0] = F[0] * F[0] + F[1] * F[1] + F[2] * F[2];
          FF[1] = F[0] * F[3] + F[1] * F[4] + F[2] * F[5];
          FF[2] = F[0] * F[6] + F[1] * F[7] + F[2] * F[8];
          FF[3] = F[3] * F[3] + F[4] * F[4] + F[5] * F[5];
          FF[4] = F[3] * F[6] + F[4] * F[7] + F[5] * F[8];
          FF[5] = F[6] * F[6] + F[7] * F[7] + F[8] * F[8];
        } else {
#pragma unroll
          for (int k = 0; k < 9; k++) FS[k] = S[k];
        }
      }
      __syncthreads();
      if (WK && TL) {
#pragma unroll
        for (int k = 0; k < PPT; k++) {
          if (pa[k] < 0) continue;
          const int a = pa[k], b = pb[k];
          for (int g = 0; g < GC; g++) {
            const double cg = sc[g];
            const double *D = sD + g * ND, *F = sF + 9 * g, *S = sS + 9 * g, *FF = sFF + 6 * g;
            const double da0 = D[a], da1 = D[NN + a], da2 = D[2 * NN + a];
            const double db0 = D[b], db1 = D[NN + b], db2 = D[2 * NN + b];
            const double ha0 = cg * (F[0] * da0 + F[1] * da1 + F[2] * da2);
            const double ha1 = cg * (F[3] * da0 + F[4] * da1 + F[5] * da2);
            const double ha2 = cg * (F[6] * da0 + F[7] * da1 + F[8] * da2);
            const double hb0 = F[0] * db0 + F[1] * db1 + F[2] * db2;
            const double hb1 = F[3] * db0 + F[4] * db1 + F[5] * db2;
            const double hb2 = F[6] * db0 + F[7] * db1 + F[8] * db2;
            P[k][0] = fma(ha0, hb0, P[k][0]); P[k][1] = fma(ha0, hb1, P[k][1]); P[k][2] = fma(ha0, hb2, P[k][2]);
            P[k][3] = fma(ha1, hb0, P[k][3]); P[k][4] = fma(ha1, hb1, P[k][4]); P[k][5] = fma(ha1, hb2, P[k][5]);
            P[k][6] = fma(ha2, hb0, P[k][6]); P[k][7] = fma(ha2, hb1, P[k][7]); P[k][8] = fma(ha2, hb2, P[k][8]);
            const double gg = cg * (da0 * db0 + da1 * db1 + da2 * db2);
#pragma unroll
            for (int m = 0; m < 6; m++) Q[k][m] = fma(gg, FF[m], Q[k][m]);
            const double sb0 = S[0] * db0 + S[1] * db1 + S[2] * db2;
            const double sb1 = S[3] * db0 + S[4] * db1 + S[5] * db2;
            const double sb2 = S[6] * db0 + S[7] * db1 + S[8] * db2;
            sg[k] += cg * (da0 * sb0 + da1 * sb1 + da2 * sb2);
          }
        }
      }
      if (force) {
        const int a = tid;
        for (int g = 0; g < GC; g++) {
          const double cg = sc[g];
          const double *FS = sFS + 9 * g, *D = sD + g * ND;
          const double d0 = cg * D[a], d1 = cg * D[NN + a], d2 = cg * D[2 * NN + a];
          g0 += FS[0] * d0 + FS[1] * d1 + FS[2] * d2;
          g1 += FS[3] * d0 + FS[4] * d1 + FS[5] * d2;
          g2 += FS[6] * d0 + FS[7] * d1 + FS[8] * d2;
        }
      }
    }

    if (WK && TL) {
#pragma unroll
      for (int k = 0; k < PPT; k++) {
        if (pa[k] < 0) continue;
        const int a = pa[k], b = pb[k];
        const double Qf[9] = {Q[k][0], Q[k][1], Q[k][2], Q[k][1], Q[k][3], Q[k][4], Q[k][2], Q[k][4], Q[k][5]};
        double v[9];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++)
            v[3 * i + j] = lam * P[k][3 * i + j] + mu * P[k][3 * j + i] + mu * Qf[3 * i + j] + (i == j ? sg[k] : 0.0);
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
          const uint8_t fa = sfix[a], fb = sfix[b];
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              if (!((fa >> i) & 1) && !((fb >> j) & 1)) {
                Kab[3 * i + j] += v[3 * i + j];
                if (Kba) Kba[3 * j + i] += v[3 * i + j];
              }
        }
      }
    }
    if (force) {
      const int a = tid;
      if (A.G) {
        const uint8_t f = sfix[a];
        double *Gn = A.G + 4 * (int64_t)en[a];
        if (!(f & 1)) Gn[0] += g0;
        if (!(f & 2)) Gn[1] += g1;
        if (!(f & 4)) Gn[2] += g2;
      }
      if (A.Ke_out && !WK) {
        double *Go = A.Ke_out + it * ND;
        Go[3 * a] = g0;
        Go[3 * a + 1] = g1;
        Go[3 * a + 2] = g2;
      }
    }
  }
}

template <int PR, int PS, int PT, int NG1, bool TL, bool WK, bool WG>
cudaError_t run_bsp_tl(Ctx &c, ElemArgs a, int64_t count) {
  if (count <= 0) return cudaSuccess;
  constexpr int NT = 256, PPT = 2;
  using S_ = BspTlSmem<PR, PS, PT, NG1>;
  auto kern = bsp_tl_kernel<PR, PS, PT, NG1, NT, PPT, TL, WK, WG>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S_::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, S_::bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int split = WK ? (S_::NP + NT * PPT - 1) / (NT * PPT) : 1;
  const int64_t slots = (int64_t)per_sm * c.sm_count;
  const int64_t grid = std::min<int64_t>(slots, count * split);
  a.ne = count;
  kern<<<(unsigned)grid, NT, S_::bytes, c.stream>>>(a, split);
  c.launches++;
  return cudaGetLastError();
}

// mode: 0 tangent + internal force, 1 tangent only, 2 internal force only
template <int PR, int PS, int PT, int NG1>
cudaError_t dispatch_mode(Ctx &c, ElemArgs a, int64_t count, bool tl, int mode) {
  if (!tl) return mode == 2 ? run_bsp_tl<PR, PS, PT, NG1, false, false, true>(c, a, count) : cudaErrorInvalidValue;
  if (mode == 0) return run_bsp_tl<PR, PS, PT, NG1, true, true, true>(c, a, count);
  if (mode == 1) return run_bsp_tl<PR, PS, PT, NG1, true, true, false>(c, a, count);
  return run_bsp_tl<PR, PS, PT, NG1, true, false, true>(c, a, count);
}

}  // namespace

bool bsp_tl_supported(const int pd[3], int ngp) {
  if (pd[0] == 2 && pd[1] == 2 && pd[2] == 2) return ngp == 3 || ngp == 4;
  if (pd[0] == 3 && pd[1] == 3 && (pd[2] == 3 || pd[2] == 2)) return ngp == 4;
  if (pd[0] == 4 && pd[1] == 2 && pd[2] == 2) return ngp == 5;
  return false;
}

cudaError_t launch_bsp_tl(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, int mode) {
  a.span = B.d_span;
  for (int d = 0; d < 3; d++) a.bas[d] = B.d_bas + B.bas_off[d];
  a.wt = B.d_wt;
  a.rational = B.rational;
  const int ng = B.ngp[0];
  const int *p = B.pd;
  const bool tl = B.tl != 0;
  if (p[0] == 2 && p[1] == 2 && p[2] == 2 && ng == 3) return dispatch_mode<2, 2, 2, 3>(c, a, count, tl, mode);
  if (p[0] == 2 && p[1] == 2 && p[2] == 2 && ng == 4) return dispatch_mode<2, 2, 2, 4>(c, a, count, tl, mode);
  if (p[0] == 3 && p[1] == 3 && p[2] == 3 && ng == 4) return dispatch_mode<3, 3, 3, 4>(c, a, count, tl, mode);
  if (p[0] == 3 && p[1] == 3 && p[2] == 2 && ng == 4) return dispatch_mode<3, 3, 2, 4>(c, a, count, tl, mode);
  if (p[0] == 4 && p[1] == 2 && p[2] == 2 && ng == 5) return dispatch_mode<4, 2, 2, 5>(c, a, count, tl, mode);
  return cudaErrorNotSupported;
}

}  // namespace fastgpu
