// tl_kernels.cu - total-Lagrangian (St. Venant-Kirchhoff) element tangent and
// internal force, and the small-strain internal force (sm_100a).
//
// Computes what cElmParamTL::StiffMat / IntForce (elc/elmparam.cpp:1615-1807)
// compute for an isotropic solid, with the Green strain of
// cElmParamTL::GreenStrain (:1899-1919) and cSolid::BlMatrix / BnlMatrix /
// SMatrix (elc/anmodel.cpp:1451-1568):
//     F = I + H,  H_ij = sum_a u_a,i dN_a/dX_j,   E = (F^T F - I) / 2,
//     S = lambda tr(E) I + 2 mu E                 (C E in Voigt form),
//     K_t = sum_g c_g [(B+Bl)^T C (B+Bl) + Bnl^T S Bnl],   g = sum_g c_g (B+Bl)^T S.
// Written per node pair (a, b) with h_a = F grad N_a, the 3x3 tangent block is
//     K_ab = lambda P + mu P^T + mu Q + s I,
//     P = sum_g c_g h_a h_b^T,  Q = sum_g c_g (grad N_a . grad N_b) F F^T,
//     s = sum_g c_g grad N_a . S grad N_b,
// and the internal force of node a is g_a = sum_g c_g F S grad N_a.  With
// F = I and S = C sym(H) the same kernel gives the small-strain internal force
// of cElmParam::IntForce (elc/elmparam.cpp:449-535).
//
// Scatter: like the stiffness assembly, one launch per colour, so neither the
// tangent blocks nor the nodal forces need atomics; results are bit-identical
// run to run.  Internal forces of DOFs without an equation are not added, so
// the node-space residual f - g is zero there.
#include <cstdint>

#include "elem_common.cuh"
#include "internal.h"

namespace fastgpu {

template <int NN, int NG>
struct TlSmem {
  static constexpr int ND = 3 * NN;
  static constexpr int total = 2 * NN * 3 /*X, U*/ + NG * 9 /*J*/ + NG /*c*/ + 3 * NG * ND /*D, h, S.D*/ +
                               NG * 9 /*F*/ + NG * 9 /*F S*/ + NG * 6 /*F F^T*/ + NG * 2 /*lambda tr, pad*/;
  static constexpr size_t bytes = total * sizeof(double) + 64;
};

template <int NN, int NG, int NT, bool TL, bool WANT_K, bool WANT_G>
__global__ void __launch_bounds__(NT, (NT >= 128 ? 3 : 8)) tl_kernel(ElemArgs A) {
  using S_ = TlSmem<NN, NG>;
  constexpr int ND = S_::ND;
  constexpr int NP = NN * (NN + 1) / 2;
  static_assert(NP <= NT, "one thread per node pair");
  extern __shared__ __align__(16) double sm[];
  double *sX = sm;
  double *sU = sX + NN * 3;
  double *sJ = sU + NN * 3;
  double *sc = sJ + NG * 9;
  double *sD = sc + NG;
  double *sHa = sD + NG * ND;     // h_a = F grad N_a
  double *sSD = sHa + NG * ND;    // S grad N_a
  double *sF = sSD + NG * ND;
  double *sFS = sF + NG * 9;
  double *sFF = sFS + NG * 9;
  uint8_t *sfix = reinterpret_cast<uint8_t *>(sFF + NG * 6 + NG * 2);
  const double *__restrict__ gdN = A.dN;
  const double *__restrict__ gw = A.w;
  const int tid = threadIdx.x;
  int pa = 0, pb = 0;
  if (tid < NP) pair_of(tid, NN, pa, pb);

  if (A.skip && *A.skip) return;
  for (int64_t it = blockIdx.x; it < A.ne; it += gridDim.x) {
    const int64_t e = A.index ? (int64_t)A.index[it] : A.offset + it;
    __syncthreads();
    const int32_t *en = A.conn + e * NN;
    for (int i = tid; i < NN * 3; i += NT) {
      const int32_t n = en[i / 3];
      sX[i] = A.X[3 * (int64_t)n + (i % 3)];
      sU[i] = A.U[4 * (int64_t)n + (i % 3)];
    }
    for (int i = tid; i < NN; i += NT) sfix[i] = A.fix[en[i]];

    double *Kab = nullptr, *Kba = nullptr;
    double oab[9], oba[9];
    if (WANT_K && A.K && tid < NP) {
      Kab = A.K + (int64_t)A.slot[(e * NN + pa) * NN + pb] * 9;
      if (pa != pb) Kba = A.K + (int64_t)A.slot[(e * NN + pb) * NN + pa] * 9;
#pragma unroll
      for (int k = 0; k < 9; k++) oab[k] = Kab[k];
      if (Kba) {
#pragma unroll
        for (int k = 0; k < 9; k++) oba[k] = Kba[k];
      }
    }
    __syncthreads();

    // Jacobians (cShapeSolid::DrvShpXYZ, shp/shpsolid.cpp:58-126)
    for (int t = tid; t < NG * 9; t += NT) {
      const int g = t / 9, pq = t - 9 * g, p = pq / 3, q = pq - 3 * p;
      const double *d = gdN + g * NN * 3 + p;
      double s = 0.0;
#pragma unroll 4
      for (int a = 0; a < NN; a++) s += d[3 * a] * sX[3 * a + q];
      sJ[t] = s;
    }
    __syncthreads();
    for (int g = tid; g < NG; g += NT) {
      double *J = sJ + 9 * g;
      const double j00 = J[0], j01 = J[1], j02 = J[2], j10 = J[3], j11 = J[4], j12 = J[5], j20 = J[6],
                   j21 = J[7], j22 = J[8];
      const double det = j00 * (j11 * j22 - j12 * j21) - j01 * (j10 * j22 - j12 * j20) + j02 * (j10 * j21 - j11 * j20);
      if (!(det > 0.0)) atomicOr(A.status, 1);
      // cofactors times 1/det: one division instead of nine (the reference divides
      // each cofactor; the entries differ by at most an ulp)
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
    // D[g][i*NN + a] = dN_a/dX_i
    for (int t = tid; t < NG * NN; t += NT) {
      const int g = t / NN, a = t - NN * g;
      const double *J = sJ + 9 * g;
      const double *dn = gdN + (g * NN + a) * 3;
      const double d0 = dn[0], d1 = dn[1], d2 = dn[2];
      double *D = sD + g * ND;
      D[a] = J[0] * d0 + J[1] * d1 + J[2] * d2;
      D[NN + a] = J[3] * d0 + J[4] * d1 + J[5] * d2;
      D[2 * NN + a] = J[6] * d0 + J[7] * d1 + J[8] * d2;
    }
    __syncthreads();
    // displacement gradient H_ij = sum_a u_a,i dN_a/dX_j -> F = I + H
    for (int t = tid; t < NG * 9; t += NT) {
      const int g = t / 9, ij = t - 9 * g, i = ij / 3, j = ij - 3 * i;
      const double *D = sD + g * ND + j * NN;
      double s = 0.0;
#pragma unroll 4
      for (int a = 0; a < NN; a++) s += sU[3 * a + i] * D[a];
      sF[t] = s + (i == j ? 1.0 : 0.0);
    }
    __syncthreads();
    // strain, stress (S = lambda tr(E) I + 2 mu E), F S and F F^T per Gauss point
    const double Ey = A.E[e], nu = A.nu[e];
    const double lam = Ey * nu / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = 0.5 * Ey / (1.0 + nu);
    for (int g = tid; g < NG; g += NT) {
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
      double S[9];
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

    if (WANT_K && TL) {
      // h_a = F grad N_a and S grad N_a; S is rebuilt from F with the same
      // arithmetic as above (cheaper than keeping a fourth per-point array)
      for (int t = tid; t < NG * NN; t += NT) {
        const int g = t / NN, a = t - NN * g;
        const double *F = sF + 9 * g;
        const double *D = sD + g * ND;
        const double d0 = D[a], d1 = D[NN + a], d2 = D[2 * NN + a];
        double *H = sHa + g * ND;
        H[a] = F[0] * d0 + F[1] * d1 + F[2] * d2;
        H[NN + a] = F[3] * d0 + F[4] * d1 + F[5] * d2;
        H[2 * NN + a] = F[6] * d0 + F[7] * d1 + F[8] * d2;
        double E[9];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++)
            E[3 * i + j] = 0.5 * (F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j] - (i == j ? 1.0 : 0.0));
        const double tr = E[0] + E[4] + E[8];
        double S[9];
#pragma unroll
        for (int k = 0; k < 9; k++) S[k] = 2.0 * mu * E[k] + ((k % 4 == 0) ? lam * tr : 0.0);
        double *SD = sSD + g * ND;
        SD[a] = S[0] * d0 + S[1] * d1 + S[2] * d2;
        SD[NN + a] = S[3] * d0 + S[4] * d1 + S[5] * d2;
        SD[2 * NN + a] = S[6] * d0 + S[7] * d1 + S[8] * d2;
      }
      __syncthreads();
    }

    if (WANT_K && TL && tid < NP) {
      double P[9], Q[6], sg = 0.0;
#pragma unroll
      for (int k = 0; k < 9; k++) P[k] = 0.0;
#pragma unroll
      for (int k = 0; k < 6; k++) Q[k] = 0.0;
      for (int g = 0; g < NG; g++) {
        const double cg = sc[g];
        const double *H = sHa + g * ND, *D = sD + g * ND, *SD = sSD + g * ND, *FF = sFF + 6 * g;
        const double ha0 = cg * H[pa], ha1 = cg * H[NN + pa], ha2 = cg * H[2 * NN + pa];
        const double hb0 = H[pb], hb1 = H[NN + pb], hb2 = H[2 * NN + pb];
        P[0] = fma(ha0, hb0, P[0]); P[1] = fma(ha0, hb1, P[1]); P[2] = fma(ha0, hb2, P[2]);
        P[3] = fma(ha1, hb0, P[3]); P[4] = fma(ha1, hb1, P[4]); P[5] = fma(ha1, hb2, P[5]);
        P[6] = fma(ha2, hb0, P[6]); P[7] = fma(ha2, hb1, P[7]); P[8] = fma(ha2, hb2, P[8]);
        const double da0 = D[pa], da1 = D[NN + pa], da2 = D[2 * NN + pa];
        const double gg = cg * (da0 * D[pb] + da1 * D[NN + pb] + da2 * D[2 * NN + pb]);
#pragma unroll
        for (int k = 0; k < 6; k++) Q[k] = fma(gg, FF[k], Q[k]);
        sg += cg * (da0 * SD[pb] + da1 * SD[NN + pb] + da2 * SD[2 * NN + pb]);
      }
      const double Qf[9] = {Q[0], Q[1], Q[2], Q[1], Q[3], Q[4], Q[2], Q[4], Q[5]};
      double v[9];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
          v[3 * i + j] = lam * P[3 * i + j] + mu * P[3 * j + i] + mu * Qf[3 * i + j] + (i == j ? sg : 0.0);
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
      if (Kab) {
        const uint8_t fa = sfix[pa], fb = sfix[pb];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++)
            if (!((fa >> i) & 1) && !((fb >> j) & 1)) {
              Kab[3 * i + j] = oab[3 * i + j] + v[3 * i + j];
              if (Kba) Kba[3 * j + i] = oba[3 * j + i] + v[3 * i + j];
            }
      }
    }

    if (WANT_G && tid < NN) {
      // g_a = sum_g c_g (F S) grad N_a
      const int a = tid;
      double g0 = 0.0, g1 = 0.0, g2 = 0.0;
      for (int g = 0; g < NG; g++) {
        const double cg = sc[g];
        const double *FS = sFS + 9 * g, *D = sD + g * ND;
        const double d0 = cg * D[a], d1 = cg * D[NN + a], d2 = cg * D[2 * NN + a];
        g0 += FS[0] * d0 + FS[1] * d1 + FS[2] * d2;
        g1 += FS[3] * d0 + FS[4] * d1 + FS[5] * d2;
        g2 += FS[6] * d0 + FS[7] * d1 + FS[8] * d2;
      }
      if (A.G) {
        const uint8_t f = sfix[a];
        double *Gn = A.G + 4 * (int64_t)en[a];
        if (!(f & 1)) Gn[0] += g0;
        if (!(f & 2)) Gn[1] += g1;
        if (!(f & 4)) Gn[2] += g2;
      }
      if (A.Ke_out && !WANT_K) {
        // internal force requested as the element output: [ne][3NN]
        double *Go = A.Ke_out + it * ND;
        Go[3 * a] = g0;
        Go[3 * a + 1] = g1;
        Go[3 * a + 2] = g2;
      }
    }
  }
}

template <int NN, int NG, int NT, bool TL, bool WK, bool WG>
static cudaError_t run_tl(Ctx &c, ElemArgs a, int64_t count) {
  if (count <= 0) return cudaSuccess;
  using S_ = TlSmem<NN, NG>;
  auto kern = tl_kernel<NN, NG, NT, TL, WK, WG>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S_::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, S_::bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * c.sm_count;
  if (grid > count) grid = count;
  a.ne = count;
  kern<<<(unsigned)grid, NT, S_::bytes, c.stream>>>(a);
  c.launches++;
  return cudaGetLastError();
}

// mode: 0 tangent + internal force, 1 tangent only, 2 internal force only
template <bool TL>
static cudaError_t dispatch_tl(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, int mode) {
  const int ng = B.ng;
#define FASTGPU_TL_CASES(NN, NG, NT)                                                          \
  if (mode == 0) return run_tl<NN, NG, NT, TL, true, true>(c, a, count);                    \
  if (mode == 1) return run_tl<NN, NG, NT, TL, true, false>(c, a, count);                   \
  return run_tl<NN, NG, NT, TL, false, true>(c, a, count);
  if (B.type == FAST_ELEM_HEX8) {
    if (ng == 8) { FASTGPU_TL_CASES(8, 8, 64) }
    if (ng == 27) { FASTGPU_TL_CASES(8, 27, 64) }
    if (ng == 1) { FASTGPU_TL_CASES(8, 1, 64) }
  } else if (B.type == FAST_ELEM_HEX20) {
    if (ng == 27) { FASTGPU_TL_CASES(20, 27, 224) }
    if (ng == 8) { FASTGPU_TL_CASES(20, 8, 224) }
    if (ng == 64) { FASTGPU_TL_CASES(20, 64, 224) }
  }
#undef FASTGPU_TL_CASES
  return cudaErrorInvalidValue;
}

static ElemArgs tl_args(Ctx &c, const Bucket &B, double *K, double *G) {
  ElemArgs a{};
  a.conn = B.d_conn;
  a.E = B.d_E;
  a.nu = B.d_nu;
  a.rho = B.d_rho;
  a.slot = B.d_slot;
  a.X = c.d_X;
  a.fix = c.d_fix;
  a.dN = B.d_dN;
  a.N = B.d_N;
  a.w = B.d_w;
  a.K = K;
  a.status = c.d_status;
  a.U = c.d_disp;
  a.G = G;
  return a;
}

// Total-Lagrangian buckets: tangent into K and/or internal force into G at the
// current displacements.  Small-strain buckets: internal force only (their
// stiffness comes from launch_assemble).
cudaError_t launch_tl(Ctx &c, double *K, double *G, bool want_k, bool want_g) {
  return launch_tl_at(c, K, G, want_k, want_g, c.d_disp, nullptr);
}

// G[n][i] += sum of the node's element entries, in the order of d_ginc, on
// the DOFs without a fixity (the colour scatter's additions, one node per
// thread); nothing when *skip
__global__ void gather_elem_force(int64_t nnode, const int64_t *__restrict__ ptr, const int64_t *__restrict__ inc,
                                  const double *__restrict__ Fe, const uint8_t *__restrict__ fix,
                                  double *__restrict__ G, const int32_t *__restrict__ skip) {
  if (skip && *skip) return;
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  double *Gn = G + 4 * n;
  double g0 = Gn[0], g1 = Gn[1], g2 = Gn[2];
  for (int64_t p = ptr[n]; p < ptr[n + 1]; p++) {
    const double *f = Fe + inc[p];
    g0 += f[0];
    g1 += f[1];
    g2 += f[2];
  }
  const uint8_t fx = fix[n];
  if (!(fx & 1)) Gn[0] = g0;
  if (!(fx & 2)) Gn[1] = g1;
  if (!(fx & 4)) Gn[2] = g2;
}

cudaError_t launch_tl_at(Ctx &c, double *K, double *G, bool want_k, bool want_g, const double *U, const int32_t *skip) {
  if (!want_k && want_g && G && c.force_gather && c.use_force_gather) {
    // every element of a bucket in one launch, its force into its own slot,
    // then one gather over the nodes
    for (size_t b = 0; b < c.buckets.size(); b++) {
      const Bucket &B = c.buckets[b];
      const int64_t cnt = B.color_off.empty() ? 0 : B.color_off.back();
      if (cnt == 0) continue;
      ElemArgs a = tl_args(c, B, nullptr, nullptr);
      a.U = U;
      a.skip = skip;
      a.offset = 0;
      a.Ke_out = c.d_elem_g + c.elem_g_off[b];
      cudaError_t e = B.tl ? dispatch_tl<true>(c, B, a, cnt, 2) : dispatch_tl<false>(c, B, a, cnt, 2);
      if (e != cudaSuccess) return e;
    }
    gather_elem_force<<<(unsigned)((c.nnode + 255) / 256), 256, 0, c.stream>>>(c.nnode, c.d_gptr, c.d_ginc,
                                                                              c.d_elem_g, c.d_fix, G, skip);
    c.launches++;
    return cudaGetLastError();
  }
  for (size_t b = 0; b < c.buckets.size(); b++) {
    const Bucket &B = c.buckets[b];
    int mode;
    if (B.tl) {
      if (!want_k && !want_g) continue;
      mode = want_k && want_g ? 0 : (want_k ? 1 : 2);
    } else {
      if (!want_g) continue;
      mode = 2;
    }
    for (size_t k = 0; k + 1 < B.color_off.size(); k++) {
      ElemArgs a = tl_args(c, B, (B.tl && want_k) ? K : nullptr, want_g ? G : nullptr);
      a.U = U;
      a.skip = skip;
      a.offset = B.color_off[k];
      const int64_t cnt = B.color_off[k + 1] - B.color_off[k];
      cudaError_t e = B.type == FAST_ELEM_BSP_SOLID ? launch_bsp_tl(c, B, a, cnt, mode)
                      : B.tl                         ? dispatch_tl<true>(c, B, a, cnt, mode)
                                                     : dispatch_tl<false>(c, B, a, cnt, mode);
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

// Element tangents (what = 0) or element internal forces (what = 1) of
// selected elements at the current displacements, dense, for inspection.
cudaError_t launch_tl_element(Ctx &c, int what, int bucket, int64_t count, double *d_out_and_index) {
  const Bucket &B = c.buckets[bucket];
  const int nd = 3 * B.nn;
  ElemArgs a = tl_args(c, B, nullptr, nullptr);
  a.Ke_out = d_out_and_index;
  const size_t per = (what == 0) ? (size_t)nd * nd : (size_t)nd;
  a.index = reinterpret_cast<const int32_t *>(d_out_and_index + (size_t)count * per);
  if (B.type == FAST_ELEM_BSP_SOLID) {
    if (what == 0 && !B.tl) return cudaErrorInvalidValue;
    return launch_bsp_tl(c, B, a, count, what == 0 ? 1 : 2);
  }
  if (what == 0) return B.tl ? dispatch_tl<true>(c, B, a, count, 1) : cudaErrorInvalidValue;
  return B.tl ? dispatch_tl<true>(c, B, a, count, 2) : dispatch_tl<false>(c, B, a, count, 2);
}

}  // namespace fastgpu
