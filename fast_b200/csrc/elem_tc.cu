// elem_tc.cu - element stiffness on the tensor cores: tcgen05.mma.kind::tf32
// with the 3xTF32 split, FP32 accumulators in tensor memory (sm_100a).
//
// Computes what cElmParam::StiffMat (elc/elmparam.cpp:539-597) computes for
// an isotropic solid element, K_e = sum_g w_g detJ_g B_g^T C B_g, in the
// factored form used by elem_kernels.cu: with D[(i,a)][g] = sqrt(c_g)
// dN_a/dx_i(g) (c_g = w_g detJ_g, detJ > 0 required), the Gauss-point
// contraction
//     H = D D^T,   H[(i,a),(j,b)] = sum_g c_g dN_a/dx_i dN_b/dx_j ,
// is the one dense product of the element (the MatTripBtCB of
// mlib/matvec.cpp:372-388, regrouped), and the 3x3 block (a, b) of K_e follows
// from H and the isotropic C (cSolid::QMatrix, elc/anmodel.cpp:1286-1298):
//     i == j : C00 H_ii + G (tr - H_ii),   i != j : C01 H_ij + G H_ji .
//
// This kernel serves the mixed-precision path, whose stiffness has to be as
// accurate as its FP32 storage: the iteration's FP32 operator and the FP64
// residual it is corrected by may differ by little more than FP32 rounding,
// or the corrections stall on ill-conditioned systems.  H is formed on the
// tensor cores from TF32 operands split in three, D = D_hi + D_lo + D_mid,
// as the six partial products down to 2^-22 of the product (D_lo D_lo^T,
// D_hi D_mid^T, D_mid D_hi^T, D_hi D_lo^T, D_lo D_hi^T, D_hi D_hi^T, smallest
// first) accumulated in FP32; the dropped terms are below 2^-32 of it.  (The
// two-part "3xTF32" product leaves about 2^-21, some 8x the FP32 rounding of
// the entries, which stalled the corrections on slender and large models.)
// The blocks are added into an FP32 block matrix.  Geometry (Jacobian,
// determinant, inverse, dN/dx) stays in FP64.
//
// Per element (one CTA processes the elements of one colour in turn):
//   1. one thread starts bulk copies (cp.async.bulk, completion on an
//      mbarrier) of the element's incidence row and its NN x NN slot row;
//      the natural-derivative table was brought in the same way once per CTA;
//   2. coordinates are gathered, the element's current FP32 K blocks are
//      requested with cp.async (they arrive while the element is computed);
//   3. Jacobians, inverses and D in FP64; D is split and written as three
//      K-major TF32 operands (rows (i, a), K = Gauss points padded to 8);
//   4. one elected thread issues 6 x KP/8 tcgen05.mma (M = 128 rows, N = the
//      rows rounded up to 16; A and B are operands in shared memory) and
//      commits them to an mbarrier;
//   5. the accumulator is read back with tcgen05.ld (one thread per row),
//      staged as H in shared memory, turned into 3x3 blocks by one thread per
//      node pair and added to the old blocks; the write-back is coalesced and
//      skips DOFs without an equation.
// Elements of a colour share no node, so the scatter needs no atomics and K
// is bit-identical from run to run.  Every mbarrier wait is bounded (1 s): a
// wait that runs out sets status bit 2, the CTA waits once more (bounded) for
// work in flight, frees its tensor memory and returns.
#include <cstdint>

#include "elem_common.cuh"
#include "internal.h"
#include "tc_common.cuh"

namespace fastgpu {

// bsp_tc.cu
bool bsp_tc_supported(const int pd[3], int ngp);
cudaError_t launch_bsp_tc(Ctx &c, const Bucket &B, ElemArgs a, int64_t count, float *K32);

namespace {

constexpr uint64_t kTcWaitNs = 1000000000ull;
constexpr int kTcThreads = 256;

__host__ __device__ constexpr int pow2_cols(int n) { return n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : (n <= 256 ? 256 : 512))); }

template <int NN, int NG>
struct TcHex {
  static constexpr int R = 3 * NN;                 // operand rows (i, a), i-major
  static constexpr int KP = (NG + 7) / 8 * 8;      // Gauss points padded to the MMA K
  static constexpr int N = (R + 15) / 16 * 16;     // accumulator columns (M = 128 needs N % 16 == 0)
  static constexpr int RP = 128;                   // operand rows held (one M tile)
  static constexpr int NP = NN * (NN + 1) / 2;
  static constexpr int OPB = RP * KP * 4;          // bytes of one operand part (hi, lo or mid)
  static constexpr int TCOLS = pow2_cols(N);
  static_assert(R <= 128, "one M tile");
  static_assert(NP <= kTcThreads, "one thread per node pair");
  static_assert((NN * NN * 4) % 16 == 0 && (NN * 4) % 16 == 0 && (NG * NN * 3 * 8) % 16 == 0,
                "bulk-copy sizes are multiples of 16 bytes");
  // shared memory carve-up (bytes, every piece starts on a 16-byte boundary)
  static constexpr int al(int x) { return (x + 15) / 16 * 16; }
  static constexpr int oHi = 0, oLo = oHi + OPB, oMid = oLo + OPB;
  static constexpr int oH = oMid + OPB;                       // float [R][R]
  static constexpr int oKo = oH + al(R * R * 4);              // float [NN*NN][9] old blocks
  static constexpr int oV = oKo + al(NN * NN * 9 * 4);        // float [NP][9] new blocks
  static constexpr int odN = oV + al(NP * 9 * 4);             // double [NG][NN][3] (bulk-copy target)
  static constexpr int ow = odN + al(NG * NN * 3 * 8);        // double [NG]
  static constexpr int oX = ow + al(NG * 8);                  // double [NN][3]
  static constexpr int oJ = oX + al(NN * 3 * 8);              // double [NG][9]
  static constexpr int oc = oJ + al(NG * 9 * 8);              // double [NG]
  static constexpr int oSlot = oc + al(NG * 8);               // int32 [NN][NN] (bulk-copy target)
  static constexpr int oConn = oSlot + al(NN * NN * 4);       // int32 [NN] (bulk-copy target)
  static constexpr int FW = (NN * NN + 127) / 128 * 4;        // first-touch flag words (first_words)
  static constexpr int oFirst = oConn + al(NN * 4);           // uint32 [FW] (bulk-copy target)
  static constexpr int oFix = oFirst + FW * 4;                // uint8 [NN]
  static constexpr int oBar = oFix + al(NN);                  // 2 mbarriers
  static_assert(odN % 16 == 0 && oSlot % 16 == 0 && oConn % 16 == 0 && oFirst % 16 == 0 && oBar % 16 == 0 &&
                    OPB % 16 == 0 && (FW * 4) % 16 == 0,
                "bulk-copy targets and barriers on 16-byte boundaries");
  static constexpr int bytes = oBar + 16 + 1024;                        // + alignment slack
  static_assert(bytes <= 232448, "shared memory of one CTA");
};

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(tc::smem_u32(smem)), "l"(gmem));
}

template <int NN, int NG>
__global__ void __launch_bounds__(kTcThreads, 1) elem_tc_kernel(ElemArgs A, float *__restrict__ K32) {
  using S = TcHex<NN, NG>;
  constexpr int R = S::R, KP = S::KP, N = S::N;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *sm = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t *opHi = sm + S::oHi, *opLo = sm + S::oLo, *opMid = sm + S::oMid;
  float *sH = reinterpret_cast<float *>(sm + S::oH);
  float *sKo = reinterpret_cast<float *>(sm + S::oKo);
  float *sV = reinterpret_cast<float *>(sm + S::oV);
  double *sdN = reinterpret_cast<double *>(sm + S::odN);
  double *sw = reinterpret_cast<double *>(sm + S::ow);
  double *sX = reinterpret_cast<double *>(sm + S::oX);
  double *sJ = reinterpret_cast<double *>(sm + S::oJ);
  double *sc = reinterpret_cast<double *>(sm + S::oc);
  int32_t *sSlot = reinterpret_cast<int32_t *>(sm + S::oSlot);
  int32_t *sConn = reinterpret_cast<int32_t *>(sm + S::oConn);
  uint32_t *sFirst = reinterpret_cast<uint32_t *>(sm + S::oFirst);
  uint8_t *sfix = sm + S::oFix;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sm + S::oBar);  // [0] bulk copies, [1] MMAs
  __shared__ uint32_t tmem_base_sh;
  __shared__ int fail_sh;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     tc::smem_u32(&tmem_base_sh)),
                 "r"(S::TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // operands start as zeros: the K padding (Gauss points NG..KP-1) and rows
  // R..127 stay zero for every element
  for (int i = tid; i < 3 * S::OPB / 16; i += kTcThreads) reinterpret_cast<uint4 *>(opHi)[i] = make_uint4(0, 0, 0, 0);
  if (tid == 0) {
    tc::mbar_init(&bars[0], 1);
    tc::mbar_init(&bars[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fail_sh = 0;
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base_sh;

  // Gauss-point tables, once per CTA (bulk copies on barrier 0, phase 0)
  uint32_t ph_tma = 0, ph_mma = 0;
  if (tid == 0) {
    tc::mbar_arrive_tx(&bars[0], NG * NN * 3 * 8);
    tc::bulk_g2s(sdN, A.dN, NG * NN * 3 * 8, &bars[0]);
  }
  for (int g = tid; g < NG; g += kTcThreads) sw[g] = A.w[g];  // 8 * NG bytes: not a bulk-copy size
  if (!tc::mbar_wait(&bars[0], ph_tma, kTcWaitNs)) fail_sh = 1;
  ph_tma ^= 1;
  int32_t pa = 0, pb = 0;
  if (tid < S::NP) pair_of(tid, NN, pa, pb);
  constexpr uint32_t kLBO = 128, kSBO = (KP / 4) * 128;
  constexpr uint32_t kId = tc::idesc(128, N, tc::kTypeTF32);
  bool mma_pending = false;

  for (int64_t it = blockIdx.x; it < A.ne; it += gridDim.x) {
    __syncthreads();
    if (fail_sh) break;
    const int64_t e = A.index ? (int64_t)A.index[it] : A.offset + it;
    if (tid == 0) {
      tc::mbar_arrive_tx(&bars[0], NN * NN * 4 + NN * 4 + (A.first ? S::FW * 4 : 0));
      tc::bulk_g2s(sSlot, A.slot + e * NN * NN, NN * NN * 4, &bars[0]);
      tc::bulk_g2s(sConn, A.conn + e * NN, NN * 4, &bars[0]);
      if (A.first) tc::bulk_g2s(sFirst, A.first + e * S::FW, S::FW * 4, &bars[0]);
    }
    if (!tc::mbar_wait(&bars[0], ph_tma, kTcWaitNs)) atomicExch(&fail_sh, 1);
    ph_tma ^= 1;
    __syncthreads();
    if (fail_sh) break;
    for (int i = tid; i < NN * 3; i += kTcThreads) sX[i] = A.X[3 * (int64_t)sConn[i / 3] + (i % 3)];
    for (int i = tid; i < NN; i += kTcThreads) sfix[i] = A.fix[sConn[i]];
    if (K32) {
      for (int t = tid; t < NN * NN * 9; t += kTcThreads) {
        const int q = t / 9;
        // a block this element writes first is not read
        if (!(A.first && ((sFirst[q >> 5] >> (q & 31)) & 1u))) cp_async4(sKo + t, K32 + (int64_t)sSlot[q] * 9 + (t - 9 * q));
      }
      asm volatile("cp.async.commit_group;\n" ::);
    }
    __syncthreads();
    // Jacobians J[g][p][q] = sum_a dN_a/dxi_p X_a,q (cShapeSolid::DrvShpXYZ, shp/shpsolid.cpp:58-126)
    for (int t = tid; t < NG * 9; t += kTcThreads) {
      const int g = t / 9, pq = t - 9 * g, p = pq / 3, q = pq - 3 * p;
      const double *d = sdN + g * NN * 3 + p;
      double s = 0.0;
#pragma unroll 4
      for (int a = 0; a < NN; a++) s += d[3 * a] * sX[3 * a + q];
      sJ[t] = s;
    }
    __syncthreads();
    // determinant and inverse by cofactors (cShape::ShpMatInv, shp/shape.cpp:360-393)
    for (int g = tid; g < NG; g += kTcThreads) {
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
      sc[g] = sqrt(fmax(sw[g] * det, 0.0));
    }
    __syncthreads();
    // D[(i,a)][g] = sqrt(c_g) dN_a/dx_i, split into three TF32 operands
    for (int t = tid; t < NG * NN; t += kTcThreads) {
      const int g = t / NN, a = t - NN * g;
      const double *J = sJ + 9 * g;
      const double *dn = sdN + (g * NN + a) * 3;
      const double d0 = dn[0], d1 = dn[1], d2 = dn[2], sq = sc[g];
      const double x[3] = {sq * (J[0] * d0 + J[1] * d1 + J[2] * d2), sq * (J[3] * d0 + J[4] * d1 + J[5] * d2),
                           sq * (J[6] * d0 + J[7] * d1 + J[8] * d2)};
#pragma unroll
      for (int i = 0; i < 3; i++) {
        uint32_t hi, lo, mid;
        tc::split3_tf32(x[i], hi, lo, mid);
        const uint32_t off = tc::kmajor_off4(i * NN + a, g, KP);
        *reinterpret_cast<uint32_t *>(opHi + off) = hi;
        *reinterpret_cast<uint32_t *>(opLo + off) = lo;
        *reinterpret_cast<uint32_t *>(opMid + off) = mid;
      }
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after();
      const uint32_t part[3] = {tc::smem_u32(opHi), tc::smem_u32(opLo), tc::smem_u32(opMid)};
#pragma unroll
      for (int tm = 0; tm < tc::kSplitTerms; tm++) {
        int pa_, pb_;
        tc::split_term(tm, pa_, pb_);
#pragma unroll
        for (int kk = 0; kk < KP / 8; kk++)
          tc::mma_tf32(tmem, tc::smem_desc(part[pa_] + kk * 256, kLBO, kSBO),
                       tc::smem_desc(part[pb_] + kk * 256, kLBO, kSBO), kId, (tm > 0 || kk > 0) ? 1u : 0u);
      }
      tc::commit(&bars[1]);
    }
    mma_pending = true;
    if (!tc::mbar_wait(&bars[1], ph_mma, kTcWaitNs)) atomicExch(&fail_sh, 1);
    ph_mma ^= 1;
    __syncthreads();
    if (fail_sh) break;
    mma_pending = false;
    tc::fence_after();
    // accumulator -> H (lane = row (i, a), column = (j, b))
    if (warp < 4 && warp * 32 < R) {
      const int r = warp * 32 + lane;
      const uint32_t tb = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
      for (int c0 = 0; c0 < N; c0 += 8) {
        float v[8];
        tc::ld_32x32b_x8(tb + c0, v);
        if (r < R) {
#pragma unroll
          for (int j = 0; j < 8; j++)
            if (c0 + j < R) sH[r * R + c0 + j] = v[j];
        }
      }
    }
    tc::fence_before();
    __syncthreads();
    if (tid < S::NP) {
      double M[9];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) M[3 * i + j] = (double)sH[(i * NN + pa) * R + j * NN + pb];
      const double E = A.E[e], nu = A.nu[e];
      const double dd = (1.0 + nu) * (1.0 - 2.0 * nu);
      const double C00 = E * (1.0 - nu) / dd, C01 = E * nu / dd, G = 0.5 * E / (1.0 + nu);
      const double tr = M[0] + M[4] + M[8];
      double v[9];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
          v[3 * i + j] = (i == j) ? C00 * M[4 * i] + G * (tr - M[4 * i]) : C01 * M[3 * i + j] + G * M[3 * j + i];
      if (A.Ke_out) {
        constexpr int ND = 3 * NN;
        double *Ko = A.Ke_out + it * ND * ND;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) {
            Ko[(3 * pa + i) * ND + 3 * pb + j] = v[3 * i + j];
            Ko[(3 * pb + j) * ND + 3 * pa + i] = v[3 * i + j];
          }
      }
#pragma unroll
      for (int k = 0; k < 9; k++) sV[9 * tid + k] = (float)v[k];
    }
    if (K32) {
      asm volatile("cp.async.wait_all;\n" ::: "memory");
      __syncthreads();
      // old + new for every entry whose two DOFs have equations (block (b, a)
      // is the transpose of (a, b)); first writes store new, fixed entries too
      for (int t = tid; t < NN * NN * 9; t += kTcThreads) {
        const int q = t / 9, k = t - 9 * q;
        const int a = q / NN, b = q - NN * a, i = k / 3, j = k - 3 * i;
        const bool fst = A.first && ((sFirst[q >> 5] >> (q & 31)) & 1u);
        const bool fixed = ((sfix[a] >> i) & 1) || ((sfix[b] >> j) & 1);
        const float add = (a <= b) ? sV[9 * (a * NN - a * (a - 1) / 2 + (b - a)) + k]
                                   : sV[9 * (b * NN - b * (b - 1) / 2 + (a - b)) + 3 * j + i];
        float out;
        if (entry_value(fst, fixed, a == b && i == j, fst ? 0.f : sKo[t], add, out)) K32[(int64_t)sSlot[q] * 9 + k] = out;
      }
    }
  }
  __syncthreads();
  if (fail_sh) {
    if (tid == 0) atomicOr(A.status, 4);
    // let work in flight finish before the memory goes away (bounded)
    if (mma_pending) tc::mbar_wait(&bars[1], ph_mma, kTcWaitNs);
    tc::mbar_wait(&bars[0], ph_tma, kTcWaitNs);
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::TCOLS) : "memory");
}

template <int NN, int NG>
cudaError_t run_tc(Ctx &c, ElemArgs a, int64_t count, float *K32) {
  if (count <= 0) return cudaSuccess;
  using S = TcHex<NN, NG>;
  auto kern = elem_tc_kernel<NN, NG>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, S::bytes);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTcThreads, S::bytes);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  // tensor-memory columns of the CTAs resident on one SM stay within its 512
  if (per_sm * S::TCOLS > 512) per_sm = 512 / S::TCOLS;
  per_sm = elem_per_sm(c, per_sm, a.ctas_per_sm);
  int64_t grid = (int64_t)per_sm * c.sm_count;
  if (grid > count) grid = count;
  a.ne = count;
  kern<<<(unsigned)grid, kTcThreads, S::bytes, c.stream>>>(a, K32);
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
