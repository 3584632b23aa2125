// elem_kernels.cu - element integration and colour-scheduled scatter (sm_100a).
//
// Computes what cElmParam::StiffMat (elc/elmparam.cpp:539-597) computes for an
// isotropic solid element,
//     K_e = sum_g w_g detJ_g B_g^T C B_g ,
// and adds it into the node-block CSR matrix the way cElement::AddGlobMat
// (elc/element.cpp:2975-3002) adds it into a cSysMatrix.
//
// Arithmetic.  With per-element E and nu, B^T C B factors through the
// Gauss-point contraction
//     H[(i,a),(j,b)] = sum_g c_g dN_a/dx_i(g) dN_b/dx_j(g),   c_g = w_g detJ_g,
// a (3nn x 3nn) symmetric product over the ngp Gauss points, after which the
// (a,b) 3x3 block of K_e is
//     i == j : C00 H_ii(a,b) + G (S(a,b) - H_ii(a,b)),  S = H_xx + H_yy + H_zz
//     i != j : C01 H_ij(a,b) + G H_ji(a,b)
// with C00 = E(1-nu)/d, C01 = E nu/d, G = E/(2(1+nu)), d = (1+nu)(1-2nu)
// (cSolid::QMatrix, elc/anmodel.cpp:1286-1298; Voigt order and engineering
// shear as cSolid::BMatrix, elc/anmodel.cpp:1418-1447).  This is the same
// sum as the reference's zero-skipping MatTripBtCB (mlib/matvec.cpp:372-388)
// in a different association order; FP64 results agree to rounding.
//
// Work per element (hex20, 3x3x3): H is 1830 unique entries x 27 FMAs, about
// 0.1 MFLOP, an order of magnitude below the dense B^T(CB) count, so the
// FP64 kernel is bound by the K read-modify-write, not by arithmetic.
//
// Scatter.  A launch covers one colour of one bucket; elements of a colour
// share no node, hence write disjoint 3x3 blocks: no atomics, and the order
// in which contributions reach an entry is the fixed colour order, so K is
// bit-identical from run to run.
#include <cstdint>

#include "elem_common.cuh"
#include "internal.h"

namespace fastgpu {

template <int NN, int NG, bool MASS>
struct ElemSmem {
  static constexpr int ND = 3 * NN;
  static constexpr int kN = MASS ? NG * NN : 0;   // shape functions (mass only)
  static constexpr int kX = NN * 3;
  static constexpr int kJ = NG * 9;               // Jacobian, then its inverse
  static constexpr int kC = NG;
  static constexpr int kD = MASS ? 0 : NG * ND;   // dN/dx at the Gauss points
  // hex20 and larger stage the scatter through shared memory (coalesced);
  // hex8 (64 blocks per element) keeps per-pair register scatter, measured faster
  static constexpr bool STAGE = NN > 8;
  static constexpr int NP = NN * (NN + 1) / 2;
  static constexpr int kK = STAGE ? NN * NN * 9 : 0;   // current K blocks of the element's node pairs
  static constexpr int kV = STAGE ? NP * 9 : 0;        // the element's 3x3 blocks, a <= b
  static constexpr int total = kN + kX + kJ + kC + kD + kK + kV;
  static constexpr size_t bytes = total * sizeof(double) + (STAGE ? NN * NN : 0) * sizeof(int32_t) + 2 * 256 + 64;
};

// asynchronous 8-byte global -> shared copy
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// One CTA integrates one element at a time (grid-stride over the colour).
// Thread p < NP owns node pair (a, b), a <= b, and forms
//     M_ij = sum_g c_g dN_a/dx_i dN_b/dx_j
// in registers, turns M into the 3x3 stiffness block and adds it to K.  The
// current values of the element's K blocks are read at the start of the
// element, so the read latency overlaps the Jacobian and derivative work:
//   * hex8: each pair thread loads its blocks (a,b) and (b,a) to registers and
//     writes them back itself;
//   * hex20 (STAGE): the CTA copies all NN^2 blocks to shared memory with
//     cp.async, consecutive threads taking consecutive entries of a block, and
//     writes old + new back the same way (block (b, a) is the transpose of
//     (a, b)): coalesced, where per-pair accesses touch one cache line per
//     thread and instruction.
template <int NN, int NG, int NT, bool MASS>
__global__ void __launch_bounds__(NT, (NT >= 128 ? 3 : 8)) elem_kernel(ElemArgs A) {
  using S = ElemSmem<NN, NG, MASS>;
  constexpr int ND = S::ND;
  extern __shared__ __align__(16) double sm[];
  double *sN = sm;
  double *sX = sN + S::kN;
  double *sJ = sX + S::kX;
  double *sc = sJ + S::kJ;
  double *sD = sc + S::kC;
  double *sKo = sD + S::kD;
  double *sV = sKo + S::kK;
  int32_t *sSlot = reinterpret_cast<int32_t *>(sV + S::kV);
  uint8_t *sfix = reinterpret_cast<uint8_t *>(sSlot + (S::STAGE ? NN * NN : 0));
  constexpr int NP = NN * (NN + 1) / 2;
  static_assert(NP <= NT, "one thread per node pair");
  // Gauss-point tables are read through the L1 cache (read-only, shared by all blocks)
  const double *__restrict__ gdN = A.dN;
  const double *__restrict__ gw = A.w;

  const int tid = threadIdx.x;
  if (MASS)
    for (int i = tid; i < S::kN; i += NT) sN[i] = A.N[i];
  int pa = 0, pb = 0;
  if (tid < NP) pair_of(tid, NN, pa, pb);

  for (int64_t it = blockIdx.x; it < A.ne; it += gridDim.x) {
    const int64_t e = A.index ? (int64_t)A.index[it] : A.offset + it;
    __syncthreads();
    const int32_t *en = A.conn + e * NN;
    for (int i = tid; i < NN * 3; i += NT) {
      const int32_t n = en[i / 3];
      sX[i] = A.X[3 * (int64_t)n + (i % 3)];
    }
    for (int i = tid; i < NN; i += NT) sfix[i] = A.fix[en[i]];

    // early scatter loads: slots, then the current block values
    // (a block this element writes first is not read: sSlot holds ~slot for it)
    double *Kab = nullptr, *Kba = nullptr;
    double oab[9], oba[9];
    bool fab = false, fba = false;
    if (S::STAGE && A.K) {
      const int32_t *es = A.slot + e * NN * NN;
      if (BlockWalk<NN, NT>::takes(tid))
        for (BlockWalk<NN, NT> w(tid); w.q < NN * NN; w.next()) {
          const int32_t sl = es[w.q];
          const bool fst = first_touch(A, e, w.q);
          if (w.k == 0) sSlot[w.q] = fst ? ~sl : sl;
          if (!fst) cp_async8(sKo + 9 * w.q + w.k, A.K + (int64_t)sl * 9 + w.k);
        }
      cp_async_commit();
    } else if (A.K && tid < NP) {
      Kab = A.K + (int64_t)A.slot[(e * NN + pa) * NN + pb] * 9;
      if (pa != pb) Kba = A.K + (int64_t)A.slot[(e * NN + pb) * NN + pa] * 9;
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
    __syncthreads();

    // Jacobians J[g][p][q] = sum_a dN_a/dxi_p X_a,q (cShapeSolid::DrvShpXYZ, shp/shpsolid.cpp:58-126)
    for (int t = tid; t < NG * 9; t += NT) {
      const int g = t / 9, pq = t - 9 * g, p = pq / 3, q = pq - 3 * p;
      const double *d = gdN + g * NN * 3 + p;
      double s = 0.0;
#pragma unroll 4
      for (int a = 0; a < NN; a++) s += d[3 * a] * sX[3 * a + q];
      sJ[t] = s;
    }
    __syncthreads();
    // determinant and inverse by cofactors (cShape::ShpMatInv, shp/shape.cpp:360-393)
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

    double v[9];
    if (MASS) {
      // M_ab = rho * sum_g c_g N_a N_b * I3  (cElmParam::MassMat, elc/elmparam.cpp:672-739)
      if (tid < NP) {
        const double rho = A.rho ? A.rho[e] : 0.0;
        double s = 0.0;
        for (int g = 0; g < NG; g++) s += sc[g] * sN[g * NN + pa] * sN[g * NN + pb];
        s *= rho;
#pragma unroll
        for (int k = 0; k < 9; k++) v[k] = (k % 4 == 0) ? s : 0.0;
      }
    } else {
      // D[g][i*NN + a] = sqrt(c_g) dN_a/dx_i at Gauss point g: the weight
      // w_g detJ_g is split between the two factors of every product below
      // (detJ > 0 is required; a non-positive one is reported as EDETJ)
      for (int t = tid; t < NG * NN; t += NT) {
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
      __syncthreads();
      if (tid < NP) {
        // M_ij = sum_g c_g dNa/dx_i dNb/dx_j, then the isotropic block
        //   i == j : C00 M_ii + G (tr M - M_ii);   i != j : C01 M_ij + G M_ji
        // (cSolid::QMatrix elc/anmodel.cpp:1286-1298, BMatrix :1418-1447)
        double M[9];
#pragma unroll
        for (int k = 0; k < 9; k++) M[k] = 0.0;
        for (int g = 0; g < NG; g++) {
          const double *D = sD + g * ND;
          const double a0 = D[pa], a1 = D[NN + pa], a2 = D[2 * NN + pa];
          const double b0 = D[pb], b1 = D[NN + pb], b2 = D[2 * NN + pb];
          M[0] = fma(a0, b0, M[0]); M[1] = fma(a0, b1, M[1]); M[2] = fma(a0, b2, M[2]);
          M[3] = fma(a1, b0, M[3]); M[4] = fma(a1, b1, M[4]); M[5] = fma(a1, b2, M[5]);
          M[6] = fma(a2, b0, M[6]); M[7] = fma(a2, b1, M[7]); M[8] = fma(a2, b2, M[8]);
        }
        const double E = A.E[e], nu = A.nu[e];
        const double dd = (1.0 + nu) * (1.0 - 2.0 * nu);
        const double C00 = E * (1.0 - nu) / dd, C01 = E * nu / dd, G = 0.5 * E / (1.0 + nu);
        const double tr = M[0] + M[4] + M[8];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++)
            v[3 * i + j] = (i == j) ? C00 * M[4 * i] + G * (tr - M[4 * i]) : C01 * M[3 * i + j] + G * M[3 * j + i];
      }
    }

    if (tid < NP) {
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
      if (S::STAGE && A.K) {
#pragma unroll
        for (int k = 0; k < 9; k++) sV[9 * tid + k] = v[k];
      }
      if (Kab) {
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
    if (S::STAGE && A.K) {
      cp_async_wait_all();
      __syncthreads();
      // old + new for every entry whose two DOFs have equations (first
      // writes: new, and the fixed entries too)
      if (BlockWalk<NN, NT>::takes(tid)) {
        BlockWalk<NN, NT> w(tid);
        const int k = w.k, i = k / 3, j = k - 3 * i, kt = 3 * j + i;
        for (; w.q < NN * NN; w.next()) {
          const int32_t s0 = sSlot[w.q];
          const bool fst = s0 < 0;
          const bool fixed = ((sfix[w.a] >> i) & 1) || ((sfix[w.b] >> j) & 1);
          const double add = sV[upper_entry<NN>(w.a, w.b, k, kt)];
          double out;
          if (entry_value(fst, fixed, w.a == w.b && i == j, fst ? 0.0 : sKo[9 * w.q + k], add, out))
            A.K[(int64_t)(fst ? ~s0 : s0) * 9 + k] = out;
        }
      }
    }
  }
}

template <int NN, int NG, int NT, bool MASS>
static cudaError_t run(Ctx &c, ElemArgs a, int64_t count) {
  if (count <= 0) return cudaSuccess;
  using S = ElemSmem<NN, NG, MASS>;
  auto kern = elem_kernel<NN, NG, NT, MASS>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, S::bytes);
  if (e != cudaSuccess) return e;
  per_sm = elem_per_sm(c, per_sm, a.ctas_per_sm);
  int64_t grid = (int64_t)per_sm * c.sm_count;
  if (grid > count) grid = count;
  a.ne = count;
  kern<<<(unsigned)grid, NT, S::bytes, c.stream>>>(a);
  c.launches++;
  return cudaGetLastError();
}

template <bool MASS>
static cudaError_t dispatch(Ctx &c, const Bucket &B, ElemArgs a, int64_t count) {
  const int ng = B.ng;
  if (B.type == FAST_ELEM_BSP_SOLID) return launch_bsp_elements(c, B, a, count, MASS);
  // the warp-per-element kernel, where the autotuner chose it (stiffness into K only)
  if (!MASS && B.tune_kernel == 1 && a.K && !a.Ke_out && warp_supported(B)) return launch_warp_elements(c, B, a, count);
  if (B.type == FAST_ELEM_HEX8) {
    switch (ng) {
      case 1: return run<8, 1, 64, MASS>(c, a, count);
      case 8: return run<8, 8, 64, MASS>(c, a, count);
      case 27: return run<8, 27, 64, MASS>(c, a, count);
      default: break;
    }
  } else if (B.type == FAST_ELEM_HEX20) {
    switch (ng) {
      case 8: return run<20, 8, 224, MASS>(c, a, count);
      case 27: return run<20, 27, 224, MASS>(c, a, count);
      case 64: return run<20, 64, 224, MASS>(c, a, count);
      default: break;
    }
  }
  return cudaErrorInvalidValue;
}

static ElemArgs base_args(Ctx &c, const Bucket &B, double *K) {
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
  a.ctas_per_sm = B.tune_ctas;
  a.split = B.tune_split;
  return a;
}

__global__ void zero_fixed_identity(int64_t nnode, const uint8_t *fix, const int32_t *diag, double *K) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  const uint8_t f = fix[n];
  if (!f) return;
  const int32_t d = diag[n];
  if (d < 0) return;
  for (int i = 0; i < 3; i++)
    if ((f >> i) & 1) K[(int64_t)d * 9 + 4 * i] = 1.0;
}

cudaError_t launch_zero_matrix(Ctx &c, double *K, bool identity_on_fixed) {
  cudaError_t e = cudaMemsetAsync(K, 0, sizeof(double) * 9 * (size_t)c.nnzb, c.stream);
  if (e != cudaSuccess || !identity_on_fixed) return e;
  const int bs = 256;
  zero_fixed_identity<<<(unsigned)((c.nnode + bs - 1) / bs), bs, 0, c.stream>>>(c.nnode, c.d_fix, c.d_diag, K);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_fixed_identity(Ctx &c, double *K) {
  const int bs = 256;
  zero_fixed_identity<<<(unsigned)((c.nnode + bs - 1) / bs), bs, 0, c.stream>>>(c.nnode, c.d_fix, c.d_diag, K);
  c.launches++;
  return cudaGetLastError();
}

cudaError_t launch_tied_element_matrices(Ctx &c) {
  const TiedSet &T = c.tied;
  for (size_t b = 0; b < c.buckets.size(); b++) {
    if (T.bucket_pos[b].empty()) continue;
    const Bucket &B = c.buckets[b];
    ElemArgs a = base_args(c, B, nullptr);
    a.Ke_out = T.d_ke + T.bucket_keoff[b];
    a.index = T.d_bucket_pos[b];
    cudaError_t e = dispatch<false>(c, B, a, (int64_t)T.bucket_pos[b].size());
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_assemble(Ctx &c, int what, double *target) {
  for (size_t b = 0; b < c.buckets.size(); b++) {
    const Bucket &B = c.buckets[b];
    if (what == FAST_ASM_MASS && !B.has_rho) continue;
    if (what == FAST_ASM_STIFFNESS && B.tl) continue;  // tangent: launch_tl
    for (size_t k = 0; k + 1 < B.color_off.size(); k++) {
      ElemArgs a = base_args(c, B, target);
      a.offset = B.color_off[k];
      if (what == FAST_ASM_STIFFNESS && c.use_first_touch()) {
        a.first = B.d_first;
        a.fw = first_words(B.nn);
      }
      const int64_t cnt = B.color_off[k + 1] - B.color_off[k];
      cudaError_t e = (what == FAST_ASM_MASS) ? dispatch<true>(c, B, a, cnt) : dispatch<false>(c, B, a, cnt);
      if (e != cudaSuccess) return e;
    }
  }
  if (what == FAST_ASM_STIFFNESS) return launch_tied_assemble(c, target);
  return cudaSuccess;
}

cudaError_t launch_assemble_bucket(Ctx &c, size_t b, double *target) {
  const Bucket &B = c.buckets[b];
  if (B.tl) return cudaErrorNotSupported;
  for (size_t k = 0; k + 1 < B.color_off.size(); k++) {
    ElemArgs a = base_args(c, B, target);
    a.offset = B.color_off[k];
    if (c.use_first_touch()) {
      a.first = B.d_first;
      a.fw = first_words(B.nn);
    }
    cudaError_t e = dispatch<false>(c, B, a, B.color_off[k + 1] - B.color_off[k]);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_element_matrices(Ctx &c, int what, int bucket, int64_t first_sorted_unused, int64_t count,
                                    double *d_out_and_index) {
  (void)first_sorted_unused;
  // d_out_and_index: caller packs [count] int32 positions at the end of the buffer
  const Bucket &B = c.buckets[bucket];
  const int nd = 3 * B.nn;
  ElemArgs a = base_args(c, B, nullptr);
  a.Ke_out = d_out_and_index;
  a.index = reinterpret_cast<const int32_t *>(d_out_and_index + (size_t)count * nd * nd);
  return (what == FAST_ASM_MASS) ? dispatch<true>(c, B, a, count) : dispatch<false>(c, B, a, count);
}

}  // namespace fastgpu
