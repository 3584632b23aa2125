// elem_warp.cu - FP64 hex element stiffness with one warp per element.
//
// The same element as elem_kernels.cu (cElmParam::StiffMat,
// elc/elmparam.cpp:539-597, in the factored form H = sum_g c_g dN dN^T and
// the isotropic 3x3 block per node pair; cSolid::QMatrix,
// elc/anmodel.cpp:1286-1298), scattered the same way (colour by colour, no
// atomics, first-touch stores), with another division of the work: the
// CTA-per-element kernel spends most of an element waiting at CTA barriers
// between its phases (gather, Jacobians, inverses, dN/dx, node pairs,
// scatter) with few threads busy in each, three elements in flight per SM.
// Here a warp takes an element through all phases with warp barriers only,
// and each SM keeps a dozen or more elements in flight (one per resident
// warp), so the latencies of one element overlap the work of the others:
//   * lanes gather the coordinates and fixity, copy the element's slot row
//     (and first-touch flags) into the warp's shared memory;
//   * Jacobians, inverses (cofactors / det, as cShape::ShpMatInv) and
//     D = sqrt(c_g) dN/dx in the warp's shared memory;
//   * lane l takes node pairs l, l+32, ...: it requests the pair's two K
//     blocks, forms M_ij = sum_g D_ia D_jb over the Gauss points (the loads
//     arrive meanwhile), the isotropic block, and writes both blocks back.
// Which of the two kernels serves a bucket is a launch shape the autotuner
// measures (Bucket::tune_kernel).
#include <cstdint>

#include "elem_common.cuh"
#include "internal.h"

namespace fastgpu {

namespace {

template <int NN, int NG>
struct WarpSmem {
  static constexpr int ND = 3 * NN;
  static constexpr int FW = (NN * NN + 127) / 128 * 4;   // first-touch flag words (first_words)
  static constexpr int kD = NG * ND;     // sqrt(c_g) dN/dx, [g][i*NN + a]
  static constexpr int kJ = NG * 9;      // Jacobians, then inverses
  static constexpr int kC = NG;          // w_g det J_g
  static constexpr int kX = NN * 3;
  static constexpr size_t doubles = kD + kJ + kC + kX;
  static constexpr size_t bytes = doubles * 8 + (NN * NN + FW) * 4 + ((NN + 15) / 16) * 16;  // + slots, flags, fixity
  static constexpr size_t stride = (bytes + 15) / 16 * 16;                                      // per warp
};

template <int NN, int NG, int WPC>
__global__ void __launch_bounds__(WPC * 32) elem_warp_kernel(ElemArgs A) {
  using S = WarpSmem<NN, NG>;
  constexpr int ND = S::ND, NP = NN * (NN + 1) / 2;
  extern __shared__ __align__(16) uint8_t smem_w[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t *base = smem_w + (size_t)warp * S::stride;
  double *sD = reinterpret_cast<double *>(base);
  double *sJ = sD + S::kD;
  double *sc = sJ + S::kJ;
  double *sX = sc + S::kC;
  int32_t *sSlot = reinterpret_cast<int32_t *>(sX + S::kX);
  uint32_t *sFirst = reinterpret_cast<uint32_t *>(sSlot + NN * NN);
  uint8_t *sfix = reinterpret_cast<uint8_t *>(sFirst + S::FW);
  const double *__restrict__ gdN = A.dN;
  const double *__restrict__ gw = A.w;
  const bool ft = A.first != nullptr;

  for (int64_t it = (int64_t)blockIdx.x * WPC + warp; it < A.ne; it += (int64_t)gridDim.x * WPC) {
    const int64_t e = A.index ? (int64_t)A.index[it] : A.offset + it;
    const int32_t *en = A.conn + e * NN;
    __syncwarp();
    for (int i = lane; i < NN * 3; i += 32) sX[i] = A.X[3 * (int64_t)en[i / 3] + (i % 3)];
    for (int i = lane; i < NN; i += 32) sfix[i] = A.fix[en[i]];
    const int32_t *es = A.slot + e * NN * NN;
    for (int q = lane; q < NN * NN; q += 32) sSlot[q] = es[q];
    if (ft)
      for (int w = lane; w < S::FW; w += 32) sFirst[w] = __ldg(A.first + e * S::FW + w);
    __syncwarp();
    // Jacobians J[g][p][q] = sum_a dN_a/dxi_p X_a,q (cShapeSolid::DrvShpXYZ, shp/shpsolid.cpp:58-126)
    for (int t = lane; t < NG * 9; t += 32) {
      const int g = t / 9, pq = t - 9 * g, p = pq / 3, q = pq - 3 * p;
      const double *d = gdN + g * NN * 3 + p;
      double s = 0.0;
#pragma unroll 4
      for (int a = 0; a < NN; a++) s += d[3 * a] * sX[3 * a + q];
      sJ[t] = s;
    }
    __syncwarp();
    // determinant and inverse by cofactors (cShape::ShpMatInv, shp/shape.cpp:360-393)
    for (int g = lane; g < NG; g += 32) {
      double *J = sJ + 9 * g;
      const double j00 = J[0], j01 = J[1], j02 = J[2], j10 = J[3], j11 = J[4], j12 = J[5], j20 = J[6],
                   j21 = J[7], j22 = J[8];
      const double det = j00 * (j11 * j22 - j12 * j21) - j01 * (j10 * j22 - j12 * j20) + j02 * (j10 * j21 - j11 * j20);
      if (!(det > 0.0)) atomicOr(A.status, 1);
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
    __syncwarp();
    // D[g][i*NN + a] = sqrt(c_g) dN_a/dx_i (detJ > 0 required, else EDETJ)
    for (int t = lane; t < NG * NN; t += 32) {
      const int g = t / NN, a = t - NN * g;
      const double *J = sJ + 9 * g;
      const double *dn = gdN + (g * NN + a) * 3;
      const double d0 = dn[0], d1 = dn[1], d2 = dn[2];
      const double sq = sqrt(sc[g]);
      double *D = sD + g * ND;
      D[a] = sq * (J[0] * d0 + J[1] * d1 + J[2] * d2);
      D[NN + a] = sq * (J[3] * d0 + J[4] * d1 + J[5] * d2);
      D[2 * NN + a] = sq * (J[6] * d0 + J[7] * d1 + J[8] * d2);
    }
    __syncwarp();
    const double E = A.E[e], nu = A.nu[e];
    const double dd = (1.0 + nu) * (1.0 - 2.0 * nu);
    const double C00 = E * (1.0 - nu) / dd, C01 = E * nu / dd, G = 0.5 * E / (1.0 + nu);
    for (int p = lane; p < NP; p += 32) {
      int pa, pb;
      pair_of(p, NN, pa, pb);
      // the pair's current blocks (none read at a first write), requested
      // before the Gauss-point sum so the loads overlap it
      double *Kab = A.K + (int64_t)sSlot[pa * NN + pb] * 9;
      double *Kba = pa != pb ? A.K + (int64_t)sSlot[pb * NN + pa] * 9 : nullptr;
      const int qab = pa * NN + pb, qba = pb * NN + pa;
      const bool fab = ft && ((sFirst[qab >> 5] >> (qab & 31)) & 1u);
      const bool fba = ft && Kba && ((sFirst[qba >> 5] >> (qba & 31)) & 1u);
      double oab[9], oba[9];
      if (!fab) {
#pragma unroll
        for (int k = 0; k < 9; k++) oab[k] = Kab[k];
      }
      if (Kba && !fba) {
#pragma unroll
        for (int k = 0; k < 9; k++) oba[k] = Kba[k];
      }
      double M[9];
#pragma unroll
      for (int k = 0; k < 9; k++) M[k] = 0.0;
#pragma unroll 3
      for (int g = 0; g < NG; g++) {
        const double *D = sD + g * ND;
        const double a0 = D[pa], a1 = D[NN + pa], a2 = D[2 * NN + pa];
        const double b0 = D[pb], b1 = D[NN + pb], b2 = D[2 * NN + pb];
        M[0] = fma(a0, b0, M[0]); M[1] = fma(a0, b1, M[1]); M[2] = fma(a0, b2, M[2]);
        M[3] = fma(a1, b0, M[3]); M[4] = fma(a1, b1, M[4]); M[5] = fma(a1, b2, M[5]);
        M[6] = fma(a2, b0, M[6]); M[7] = fma(a2, b1, M[7]); M[8] = fma(a2, b2, M[8]);
      }
      const double tr = M[0] + M[4] + M[8];
      double v[9];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
          v[3 * i + j] = (i == j) ? C00 * M[4 * i] + G * (tr - M[4 * i]) : C01 * M[3 * i + j] + G * M[3 * j + i];
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

template <int NN, int NG>
cudaError_t run_warp(Ctx &c, ElemArgs a, int64_t count) {
  if (count <= 0) return cudaSuccess;
  using S = WarpSmem<NN, NG>;
  // warps per CTA: four (a dozen and more warps per SM from several CTAs)
  constexpr int WPC = 4;
  auto kern = elem_warp_kernel<NN, NG, WPC>;
  const int smem = (int)(S::stride * WPC);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, WPC * 32, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  per_sm = elem_per_sm(c, per_sm, a.ctas_per_sm);
  int64_t grid = (int64_t)per_sm * c.sm_count;
  const int64_t need = (count + WPC - 1) / WPC;
  if (grid > need) grid = need;
  a.ne = count;
  kern<<<(unsigned)grid, WPC * 32, smem, c.stream>>>(a);
  c.launches++;
  return cudaGetLastError();
}

}  // namespace

// Whether a bucket has the warp-per-element stiffness kernel (small-strain
// hex8 / hex20 and their Gauss rules)
bool warp_supported(const Bucket &B) {
  if (B.tl) return false;
  if (B.type == FAST_ELEM_HEX8) return B.ng == 1 || B.ng == 8 || B.ng == 27;
  if (B.type == FAST_ELEM_HEX20) return B.ng == 8 || B.ng == 27 || B.ng == 64;
  return false;
}

// One colour of a hex bucket's stiffness, warp per element (a.K the target)
cudaError_t launch_warp_elements(Ctx &c, const Bucket &B, ElemArgs a, int64_t count) {
  if (B.type == FAST_ELEM_HEX8) {
    switch (B.ng) {
      case 1: return run_warp<8, 1>(c, a, count);
      case 8: return run_warp<8, 8>(c, a, count);
      case 27: return run_warp<8, 27>(c, a, count);
      default: break;
    }
  } else if (B.type == FAST_ELEM_HEX20) {
    switch (B.ng) {
      case 8: return run_warp<20, 8>(c, a, count);
      case 27: return run_warp<20, 27>(c, a, count);
      case 64: return run_warp<20, 64>(c, a, count);
      default: break;
    }
  }
  return cudaErrorNotSupported;
}

}  // namespace fastgpu
